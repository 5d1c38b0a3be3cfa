"""ctypes binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, always as the checker, never as the product.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "gpu-preprocessor-ijoc_b200"))
from gpp_b200.capi import Params, Summary  # noqa: E402

_lib = None
vp = C.c_void_p


class OrcLp(C.Structure):
    _fields_ = [("m", C.c_int32), ("n", C.c_int32), ("ptr", vp), ("idx", vp), ("val", vp),
                ("at_ptr", vp), ("at_idx", vp), ("at_val", vp), ("c", vp), ("AL", vp),
                ("AU", vp), ("l", vp), ("u", vp), ("obj", C.c_double)]


def build() -> None:
    subprocess.run(["make", "-s", "-f", os.path.join(HERE, "Makefile")], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        _lib = C.CDLL(LIB)
        _lib.orc_presolve.argtypes = [C.POINTER(OrcLp), C.POINTER(Params), C.POINTER(vp)]
        _lib.orc_free.argtypes = [vp]
        _lib.orc_summary.argtypes = [vp, C.POINTER(Summary)]
        _lib.orc_reduced.argtypes = [vp] + [vp] * 11 + [C.POINTER(C.c_double)]
        _lib.orc_maps.argtypes = [vp, vp, vp]
        _lib.orc_tape_sizes.argtypes = [vp] + [C.POINTER(C.c_int64)] * 4
        _lib.orc_tape.argtypes = [vp] * 8
        _lib.orc_trace_count.argtypes = [vp]
        _lib.orc_trace.argtypes = [vp, C.c_int]
        _lib.orc_trace.restype = C.c_char_p
        _lib.orc_postsolve.argtypes = [vp] * 7
        _lib.orc_fold_map.argtypes = [vp] * 5
        _lib.orc_last_error.restype = C.c_char_p
        _lib.orc_row_activity_summary.argtypes = [C.c_int, C.c_int, vp, vp, vp, vp, vp, C.c_double,
                                                  vp, vp, vp, vp, vp, vp, vp]
        _lib.orc_live_stats.argtypes = [C.c_int, C.c_int] + [vp] * 10
        _lib.orc_col_max_abs.argtypes = [C.c_int, C.c_int] + [vp] * 5
        _lib.orc_row_hash.argtypes = [C.c_int, C.c_int, vp, vp, vp, C.c_int, vp, C.c_int]
        _lib.orc_row_hash.restype = C.c_uint64
        _lib.orc_det_sum.argtypes = [vp, C.c_int64]
        _lib.orc_det_sum.restype = C.c_double
    return _lib


def ptr(a):
    return None if a is None else a.ctypes.data_as(vp)


class OracleResult:
    """Host copies of everything the oracle produced for one presolve call."""

    def __init__(self, handle, lp):
        L = lib()
        self._h = handle
        s = Summary()
        L.orc_summary(handle, C.byref(s))
        self.summary = s
        m, n, nnz = s.reduced_rows, s.reduced_cols, s.reduced_nnz
        self.A_ptr = np.zeros(m + 1, np.int32)
        self.A_idx = np.zeros(nnz, np.int32)
        self.A_val = np.zeros(nnz)
        self.AT_ptr = np.zeros(n + 1, np.int32)
        self.AT_idx = np.zeros(nnz, np.int32)
        self.AT_val = np.zeros(nnz)
        self.c, self.l, self.u = np.zeros(n), np.zeros(n), np.zeros(n)
        self.AL, self.AU = np.zeros(m), np.zeros(m)
        obj = C.c_double()
        L.orc_reduced(handle, *(ptr(a) for a in (self.A_ptr, self.A_idx, self.A_val, self.AT_ptr,
                                                 self.AT_idx, self.AT_val, self.c, self.AL, self.AU,
                                                 self.l, self.u)), C.byref(obj))
        self.obj_constant = obj.value
        self.row_map = np.zeros(m, np.int32)
        self.col_map = np.zeros(n, np.int32)
        L.orc_maps(handle, ptr(self.row_map), ptr(self.col_map))
        r, i, v, f = (C.c_int64() for _ in range(4))
        L.orc_tape_sizes(handle, C.byref(r), C.byref(i), C.byref(v), C.byref(f))
        self.tape_types = np.zeros(r.value, np.int32)
        self.tape_is = np.zeros(r.value + 1, np.int64)
        self.tape_vs = np.zeros(r.value + 1, np.int64)
        self.tape_idx = np.zeros(i.value, np.int32)
        self.tape_val = np.zeros(v.value)
        self.fixed_idx = np.zeros(f.value, np.int32)
        self.fixed_val = np.zeros(f.value)
        L.orc_tape(handle, *(ptr(a) for a in (self.tape_types, self.tape_is, self.tape_vs,
                                              self.tape_idx, self.tape_val, self.fixed_idx,
                                              self.fixed_val)))
        self.trace = [L.orc_trace(handle, k).decode() for k in range(L.orc_trace_count(handle))]
        self.m0, self.n0 = lp.m, lp.n

    def fold_map(self):
        """(row_color, col_color, row_scale, col_scale) when folding applied, else None."""
        s = self.summary
        if not s.folding_applied:
            return None
        rc, cc = np.zeros(self.m0, np.int32), np.zeros(self.n0, np.int32)
        rs, cs = np.zeros(self.m0), np.zeros(self.n0)
        lib().orc_fold_map(self._h, ptr(rc), ptr(cc), ptr(rs), ptr(cs))
        return rc, cc, rs, cs

    def postsolve(self, x_red, y_red, z_red):
        x = np.zeros(self.n0)
        y = np.zeros(self.m0)
        z = np.zeros(self.n0)
        st = lib().orc_postsolve(self._h, ptr(x_red), ptr(y_red), ptr(z_red), ptr(x), ptr(y), ptr(z))
        if st:
            raise RuntimeError(lib().orc_last_error().decode())
        return x, y, z

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_free(self._h)
            self._h = None


def presolve(lp, params) -> OracleResult:
    lp.ensure_transpose()
    arrays = [np.ascontiguousarray(a) for a in (lp.row_ptr, lp.col_idx, lp.values, lp.at_ptr,
                                                lp.at_idx, lp.at_val, lp.c, lp.AL, lp.AU, lp.l, lp.u)]
    h = OrcLp(lp.m, lp.n, *(ptr(a) for a in arrays), lp.obj_constant)
    out = vp()
    st = lib().orc_presolve(C.byref(h), C.byref(params), C.byref(out))
    if st:
        raise RuntimeError(lib().orc_last_error().decode())
    return OracleResult(out, lp)


def row_activity_summary(m, n, ptr_, idx, val, l, u, zero_tol=1e-10, keep_row=None, keep_col=None,
                         live_degrees=None):
    out = [np.zeros(m), np.zeros(m), np.zeros(m, np.int32), np.zeros(m, np.int32)]
    lib().orc_row_activity_summary(m, n, ptr(ptr_), ptr(idx), ptr(val), ptr(l), ptr(u), zero_tol,
                                   ptr(keep_row), ptr(keep_col), ptr(live_degrees), *(ptr(a) for a in out))
    return out


def live_stats(rows, cols, ptr_, idx, val, keep_outer=None, keep_inner=None):
    deg = np.zeros(rows, np.int32)
    empty = np.zeros(rows, np.uint8)
    single = np.zeros(rows, np.uint8)
    sup = np.zeros(rows, np.int32)
    coef = np.zeros(rows)
    total = C.c_int64(0)
    lib().orc_live_stats(rows, cols, ptr(ptr_), ptr(idx), ptr(val), ptr(keep_outer), ptr(keep_inner),
                         ptr(deg), ptr(empty), ptr(single), ptr(sup), ptr(coef),
                         C.cast(C.byref(total), vp))
    return deg, empty, single, sup, coef, total.value


def col_max_abs(rows, cols, ptr_, idx, val, keep_row=None):
    out = np.zeros(rows)
    lib().orc_col_max_abs(rows, cols, ptr(ptr_), ptr(idx), ptr(val), ptr(keep_row), ptr(out))
    return out


def det_sum(v):
    v = np.ascontiguousarray(v, dtype=np.float64)
    return lib().orc_det_sum(ptr(v), v.size)
