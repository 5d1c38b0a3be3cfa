"""Fixtures restated from the reference's own known-answer tests.

dyadic_activity_fixture: cpp/tests/test_gpu_presolve_kernels.cpp:49-137 -- rows
of lengths {0,1,8,9,31,32,33,1024,1025,4097} over dyadic coefficients and
bounds, so every activity sum is exact in any association order; the expected
values are the test's own CPU loop.
hash_fixture: test_gpu_presolve_kernels.cpp:139-179 -- the exact FNV-1a row
hash values in sequential and XOR-aggregate modes.
"""
from __future__ import annotations

import struct

import numpy as np

INF = np.inf


def dyadic_activity_fixture():
    lengths = [0, 1, 8, 9, 31, 32, 33, 1024, 1025, 4097]
    rows, cols = 2100, 4097
    j = np.arange(cols)
    lower = np.where(j % 113 == 0, -INF, -((j % 7) + 1) * 0.5)
    upper = np.where(j % 127 == 0, INF, ((j % 11) + 1) * 0.5)
    ptr = [0]
    idx, val = [], []
    exp_lo = np.zeros(rows)
    exp_hi = np.zeros(rows)
    exp_ni = np.zeros(rows, np.int32)
    exp_pi = np.zeros(rows, np.int32)
    for i in range(rows):
        L = lengths[i % 10]
        jj = np.arange(L)
        a = np.where(jj % 71 == 0, 0.0, np.where(jj % 2 == 1, -0.5, 2.0))
        idx.extend(jj.tolist())
        val.extend(a.tolist())
        nz = a != 0.0
        lo = np.where(a >= 0, a * lower[:L], a * upper[:L])[nz]
        hi = np.where(a >= 0, a * upper[:L], a * lower[:L])[nz]
        exp_lo[i] = float(np.sum(lo[np.isfinite(lo)]))
        exp_hi[i] = float(np.sum(hi[np.isfinite(hi)]))
        exp_ni[i] = int(np.sum(~np.isfinite(lo)))
        exp_pi[i] = int(np.sum(~np.isfinite(hi)))
        ptr.append(len(idx))
    ptr = np.array(ptr, np.int32)
    idx = np.array(idx, np.int32)
    val = np.array(val, np.float64)
    exp_max = np.array([np.max(np.abs(val[ptr[i]:ptr[i + 1]]), initial=0.0) for i in range(rows)])
    return dict(rows=rows, cols=cols, ptr=ptr, idx=idx, val=val, lower=lower, upper=upper,
                lo=exp_lo, hi=exp_hi, ni=exp_ni, pi=exp_pi, max=exp_max,
                medium_rows=1050, long_rows=420)


FNV_OFFSET = 0xCBF29CE484222325
FNV_PRIME = 0x100000001B3
M64 = (1 << 64) - 1


def _mix(h, x):
    return ((h ^ x) * FNV_PRIME) & M64


def _bits(x):
    return struct.unpack("<Q", struct.pack("<d", x))[0]


def hash_fixture(rows):
    lengths = [0, 1, 8, 9, 31, 32, 33, 1024, 1025, 4097]
    ptr = [0]
    idx, val = [], []
    keep = np.ones(2100, np.uint8)
    keep[7] = 0
    for row in range(2100):
        length = lengths[row] if row < 10 else 1
        for j in range(length):
            idx.append(j)
            val.append(-0.5 if j % 2 else 2.0)
        ptr.append(len(idx))
    ptr = np.array(ptr[:rows + 1], np.int32)
    idx = np.array(idx[:ptr[-1]], np.int32)
    val = np.array(val[:ptr[-1]], np.float64)
    use_xor = ptr[-1] > 32 * rows
    expected = np.zeros(rows, np.uint64)
    for row in range(rows):
        first, last = ptr[row], ptr[row + 1]
        if not keep[row]:
            expected[row] = row
            continue
        if first == last:
            expected[row] = _mix(FNV_OFFSET, row)
            continue
        h = _mix(FNV_OFFSET, int(last - first))
        agg = 0
        for p in range(first, last):
            b = _bits(val[p] / val[first])
            if use_xor:
                agg ^= _mix(_mix(FNV_OFFSET, int(idx[p])), b)
            else:
                h = _mix(_mix(h, int(idx[p])), b)
        expected[row] = _mix(h, agg) if use_xor else h
    return dict(rows=rows, cols=4097, ptr=ptr, idx=idx, val=val, keep=keep[:rows], expected=expected,
                mode=1 if use_xor else 0)
