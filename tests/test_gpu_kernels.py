"""Kernel-level parity on the GPU: the CUDA activity / live-statistics /
column-max / compaction kernels against the oracle, bit for bit."""
import ctypes as C

import numpy as np
import pytest

import fixtures
import pyoracle
from gpp_b200 import capi, lpgen
from gpp_b200.device import _d2h, _raise, ptr, to_device

pytestmark = pytest.mark.gpu


def dev_csr(rows, cols, p, i, v):
    tp, ti, tv = to_device(p, np.int32), to_device(i, np.int32), to_device(v, np.float64)
    return capi.Csr(rows, cols, int(p[-1]), ptr(tp), ptr(ti), ptr(tv)), (tp, ti, tv)


def gpu_activity(rows, cols, p, i, v, l, u, zero_tol, keep_row=None, keep_col=None, live=None):
    import torch
    A, keep = dev_csr(rows, cols, p, i, v)
    dl, du = to_device(l, np.float64), to_device(u, np.float64)
    kr = to_device(keep_row, np.uint8) if keep_row is not None else None
    kc = to_device(keep_col, np.uint8) if keep_col is not None else None
    ld = to_device(live, np.int32) if live is not None else None
    out = [torch.zeros(rows, dtype=torch.float64, device="cuda"), torch.zeros(rows, dtype=torch.float64, device="cuda"),
           torch.zeros(rows, dtype=torch.int32, device="cuda"), torch.zeros(rows, dtype=torch.int32, device="cuda")]
    _raise(capi.load().gpp_row_activity_summary(C.byref(A), ptr(dl), ptr(du), zero_tol, ptr(kr), ptr(kc), ptr(ld),
                                                *(ptr(t) for t in out)))
    return [t.cpu().numpy() for t in out]


def test_dyadic_activity_fixture_exact():
    f = fixtures.dyadic_activity_fixture()
    lo, hi, ni, pi = gpu_activity(f["rows"], f["cols"], f["ptr"], f["idx"], f["val"], f["lower"], f["upper"], 1e-12)
    assert np.array_equal(lo, f["lo"]) and np.array_equal(hi, f["hi"])
    assert np.array_equal(ni, f["ni"]) and np.array_equal(pi, f["pi"])


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_masked_activity_bitwise_vs_oracle(seed):
    rng = np.random.default_rng(seed)
    # rows of lengths spanning all three buckets, random (non-dyadic) data
    lengths = rng.choice([0, 1, 5, 8, 9, 20, 33, 300, 1024, 1025, 3000, 5000], size=600)
    cols = 6000
    p = np.zeros(lengths.size + 1, np.int32)
    p[1:] = np.cumsum(lengths)
    idx = np.concatenate([np.sort(rng.choice(cols, size=k, replace=False)) for k in lengths]).astype(np.int32)
    val = rng.uniform(-10, 10, size=idx.size)
    val[rng.random(idx.size) < 0.01] = 0.0
    l = rng.uniform(-5, 0, size=cols)
    u = rng.uniform(0, 5, size=cols)
    l[rng.random(cols) < 0.05] = -np.inf
    u[rng.random(cols) < 0.05] = np.inf
    keep_r = (rng.random(lengths.size) < 0.9).astype(np.uint8)
    keep_c = (rng.random(cols) < 0.8).astype(np.uint8)
    deg, *_ = pyoracle.live_stats(lengths.size, cols, p, idx, val, keep_r, keep_c)
    ref = pyoracle.row_activity_summary(lengths.size, cols, p, idx, val, l, u, 1e-10, keep_r, keep_c, deg)
    got = gpu_activity(lengths.size, cols, p, idx, val, l, u, 1e-10, keep_r, keep_c, deg)
    for a, b in zip(ref, got):
        assert np.array_equal(a.view(np.uint64) if a.dtype == np.float64 else a,
                              b.view(np.uint64) if b.dtype == np.float64 else b)
    # unmasked, bucketed by stored length
    ref = pyoracle.row_activity_summary(lengths.size, cols, p, idx, val, l, u, 1e-10)
    got = gpu_activity(lengths.size, cols, p, idx, val, l, u, 1e-10)
    for a, b in zip(ref, got):
        assert np.array_equal(a, b)


def test_live_stats_and_col_max_vs_oracle():
    import torch
    rng = np.random.default_rng(7)
    lp = lpgen.random_lp(3000, 7000, seed=7, hub_rows=3)
    keep_r = (rng.random(lp.m) < 0.85).astype(np.uint8)
    keep_c = (rng.random(lp.n) < 0.85).astype(np.uint8)
    for (rows, cols, p, i, v, ko, ki) in [(lp.m, lp.n, lp.row_ptr, lp.col_idx, lp.values, keep_r, keep_c),
                                          (lp.n, lp.m, lp.at_ptr, lp.at_idx, lp.at_val, keep_c, keep_r)]:
        M, keep = dev_csr(rows, cols, p, i, v)
        dko, dki = to_device(ko, np.uint8), to_device(ki, np.uint8)
        deg = torch.zeros(rows, dtype=torch.int32, device="cuda")
        emp = torch.zeros(rows, dtype=torch.uint8, device="cuda")
        sng = torch.zeros(rows, dtype=torch.uint8, device="cuda")
        sup = torch.zeros(rows, dtype=torch.int32, device="cuda")
        coef = torch.zeros(rows, dtype=torch.float64, device="cuda")
        tot = torch.zeros(1, dtype=torch.int64, device="cuda")
        _raise(capi.load().gpp_live_stats(C.byref(M), ptr(dko), ptr(dki), ptr(deg), ptr(emp), ptr(sng), ptr(sup),
                                          ptr(coef), ptr(tot)))
        ref = pyoracle.live_stats(rows, cols, p, i, v, ko, ki)
        for a, b in zip(ref[:5], (deg, emp, sng, sup, coef)):
            assert np.array_equal(a, b.cpu().numpy())
        assert ref[5] == int(tot.item())
    AT, keep = dev_csr(lp.n, lp.m, lp.at_ptr, lp.at_idx, lp.at_val)
    out = torch.zeros(lp.n, dtype=torch.float64, device="cuda")
    dkr = to_device(keep_r, np.uint8)
    _raise(capi.load().gpp_col_max_abs(C.byref(AT), ptr(dkr), ptr(out)))
    assert np.array_equal(out.cpu().numpy(), pyoracle.col_max_abs(lp.n, lp.m, lp.at_ptr, lp.at_idx, lp.at_val, keep_r))


def sparse_rows(m, n, lengths, seed):
    """CSR with the given row lengths, distinct sorted columns per row."""
    rng = np.random.default_rng(seed)
    ptr_ = np.zeros(m + 1, np.int64)
    ptr_[1:] = np.cumsum(lengths)
    idx = np.concatenate([np.sort(rng.choice(n, size=k, replace=False)) for k in lengths if k] or [np.zeros(0, int)])
    val = rng.standard_normal(idx.size)
    return ptr_.astype(np.int32), idx.astype(np.int32), val


def compaction_case(name):
    rng = np.random.default_rng(11)
    if name == "random_hubs":
        lp = lpgen.random_lp(2500, 6000, seed=11, hub_rows=4)
        m, n, p_, i_, v_ = lp.m, lp.n, lp.row_ptr, lp.col_idx, lp.values
        return m, n, p_, i_, v_, (rng.random(m) < 0.7).astype(np.uint8), (rng.random(n) < 0.6).astype(np.uint8)
    if name == "empty_runs":
        # Leading, trailing and long interior runs of empty rows.
        m, n = 60000, 3000
        lengths = np.zeros(m, np.int64)
        lengths[5000:55000:97] = rng.integers(1, 40, size=len(range(5000, 55000, 97)))
        p_, i_, v_ = sparse_rows(m, n, lengths, 12)
        return m, n, p_, i_, v_, (rng.random(m) < 0.8).astype(np.uint8), (rng.random(n) < 0.7).astype(np.uint8)
    if name == "long_rows":
        # Rows of thousands of entries interleaved with short and empty rows.
        m, n = 40, 20000
        lengths = rng.integers(0, 30, size=m)
        lengths[[3, 17, 18, 39]] = [9000, 4500, 12000, 7000]
        p_, i_, v_ = sparse_rows(m, n, lengths, 13)
        keep_r = np.ones(m, np.uint8)
        keep_r[17] = 0
        return m, n, p_, i_, v_, keep_r, (rng.random(n) < 0.5).astype(np.uint8)
    if name == "dense_columns":
        # Five columns in every row (longer than the short-column transpose
        # takes), the rest short: the transpose takes its sorting path.
        m, n = 3000, 500
        lengths = rng.integers(0, 8, size=m)
        p0, i0, _ = sparse_rows(m, n - 5, lengths, 15)
        rows = np.repeat(np.arange(m), np.diff(p0))
        r = np.concatenate([rows, np.repeat(np.arange(m), 5)])
        c = np.concatenate([i0.astype(np.int64) + 5, np.tile(np.arange(5), m)])
        p_, i_, v_ = lpgen.coo_to_csr(m, r.astype(np.int64), c, rng.standard_normal(r.size))
        return m, n, p_, i_, v_, (rng.random(m) < 0.9).astype(np.uint8), (rng.random(n) < 0.8).astype(np.uint8)
    if name == "nothing_left":
        # Kept rows, kept columns, but no kept entry: every new pointer is 0.
        m, n = 3000, 600
        lengths = rng.integers(0, 6, size=m)
        p_, i_, v_ = sparse_rows(m, 500, lengths, 14)   # columns 500.. hold no entry
        keep_c = np.zeros(n, np.uint8)
        keep_c[500:503] = 1
        return m, n, p_, i_, v_, (rng.random(m) < 0.5).astype(np.uint8), keep_c
    raise ValueError(name)


@pytest.mark.parametrize("case", ["random_hubs", "empty_runs", "long_rows", "dense_columns", "nothing_left"])
def test_compaction_and_transpose_vs_numpy(case):
    m, n, row_ptr, col_idx, values, keep_r, keep_c = compaction_case(case)
    A, keep = dev_csr(m, n, row_ptr, col_idx, values)
    Ao, ATo = capi.Csr(), capi.Csr()
    dkr, dkc = to_device(keep_r, np.uint8), to_device(keep_c, np.uint8)   # kept alive across the call
    _raise(capi.load().gpp_compact_and_transpose(C.byref(A), ptr(dkr), ptr(dkc), C.byref(Ao), C.byref(ATo)))
    rmap = np.cumsum(keep_r.astype(np.int64)) - 1
    cmap = np.cumsum(keep_c.astype(np.int64)) - 1
    rows = np.repeat(np.arange(m), np.diff(row_ptr))
    sel = keep_r[rows].astype(bool) & keep_c[col_idx].astype(bool)
    m2, n2 = int(keep_r.sum()), int(keep_c.sum())
    ptr2, idx2, val2 = lpgen.coo_to_csr(m2, rmap[rows[sel]], cmap[col_idx[sel]], values[sel])
    tp, ti, tv = lpgen.csr_transpose(m2, n2, ptr2, idx2, val2)
    assert Ao.rows == m2 and Ao.cols == n2 and Ao.nnz == idx2.size
    assert np.array_equal(_d2h(Ao.rowPtr, m2 + 1, np.int32), ptr2)
    assert np.array_equal(_d2h(Ao.colVal, Ao.nnz, np.int32), idx2)
    assert np.array_equal(_d2h(Ao.nzVal, Ao.nnz, np.float64), val2)
    assert np.array_equal(_d2h(ATo.rowPtr, n2 + 1, np.int32), tp)
    assert np.array_equal(_d2h(ATo.colVal, ATo.nnz, np.int32), ti)
    assert np.array_equal(_d2h(ATo.nzVal, ATo.nnz, np.float64), tv)
    lib = capi.load()
    for p_ in (Ao.rowPtr, Ao.colVal, Ao.nzVal, ATo.rowPtr, ATo.colVal, ATo.nzVal):
        lib.gpp_device_free(p_)


@pytest.mark.parametrize("rows", [10, 2100])
def test_row_hash_fixture_on_gpu(rows):
    import torch
    f = fixtures.hash_fixture(rows)
    A, keep = dev_csr(rows, f["cols"], f["ptr"], f["idx"], f["val"])
    dk = to_device(f["keep"], np.uint8)
    out = torch.zeros(rows, dtype=torch.int64, device="cuda")
    _raise(capi.load().gpp_parallel_row_hashes(C.byref(A), ptr(dk), None, -1, ptr(out)))
    assert np.array_equal(out.cpu().numpy().view(np.uint64), f["expected"])
