"""Host-side mirror of the reference's plain-path API over the C ABI.

``DeviceLp`` uploads a host LP to CUDA memory (torch tensors are used only as
device allocations) and exposes the ``gpp_lp`` view the engine expects.
``preprocess`` / ``postprocess`` / ``free_summary`` mirror
gpu_preprocessor::preprocess/postprocess/free_summary
(cpp/include/gpu_preprocessor/gpu_preprocessor.hpp:22-39); errors surface as
the same Python exception families the reference's C++ exceptions map to.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi

_ERR = {1: RuntimeError, 2: OverflowError, 3: ValueError, 4: RuntimeError, 5: RuntimeError}


def _raise(status: int):
    if status:
        msg = capi.load().gpp_last_error().decode(errors="replace")
        raise _ERR.get(status, RuntimeError)(f"gpp status {status}: {msg}")


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("no CUDA device")
    return torch


def to_device(arr, dtype=None):
    torch = _torch()
    a = np.ascontiguousarray(arr if dtype is None else np.asarray(arr, dtype=dtype))
    return torch.from_numpy(a).to("cuda")


def ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None and t.numel() else C.c_void_p(0)


def f64ptr(t, name="solution vector"):
    """ptr() of a contiguous CUDA float64 tensor (the C ABI reads doubles)."""
    if t is not None and t.numel():
        torch = _torch()
        if t.dtype != torch.float64 or not t.is_cuda or not t.is_contiguous():
            raise TypeError(f"{name} must be a contiguous CUDA float64 tensor, got {t.dtype} on {t.device}")
    return ptr(t)


class DeviceLp:
    """A host LP uploaded to the GPU; keeps the tensors alive."""

    def __init__(self, lp, pinned: bool = False):
        torch = _torch()
        lp.ensure_transpose()
        self.host = lp
        self.m, self.n, self.nnz = lp.m, lp.n, lp.nnz
        arrays = {
            "A_ptr": (lp.row_ptr, np.int32), "A_idx": (lp.col_idx, np.int32), "A_val": (lp.values, np.float64),
            "AT_ptr": (lp.at_ptr, np.int32), "AT_idx": (lp.at_idx, np.int32), "AT_val": (lp.at_val, np.float64),
            "c": (lp.c, np.float64), "AL": (lp.AL, np.float64), "AU": (lp.AU, np.float64),
            "l": (lp.l, np.float64), "u": (lp.u, np.float64),
        }
        self.t = {}
        for k, (a, dt) in arrays.items():
            h = torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=dt)))
            if pinned:
                h = h.pin_memory()
            self.t[k] = h.to("cuda", non_blocking=pinned)
        self.obj_constant = float(lp.obj_constant)

    def load_from_host(self, host) -> None:
        """gpp_lp_from_host: refill this LP's device arrays from host tensors
        or arrays (keys A_ptr, A_idx, A_val, c, AL, AU, l, u, of this LP's
        sizes); AT is rebuilt on the GPU.  Page-locked tensors copy
        asynchronously."""
        def hp(k):
            a = host[k]
            return C.c_void_p(a.data_ptr() if hasattr(a, "data_ptr") else a.ctypes.data)
        h = capi.HostLp(self.m, self.n, self.nnz, hp("A_ptr"), hp("A_idx"), hp("A_val"), hp("c"), hp("AL"),
                        hp("AU"), hp("l"), hp("u"), self.obj_constant)
        dev = self.struct()
        _raise(capi.load().gpp_lp_from_host(C.byref(h), C.byref(dev)))

    def struct(self) -> capi.Lp:
        t = self.t
        A = capi.Csr(self.m, self.n, self.nnz, ptr(t["A_ptr"]), ptr(t["A_idx"]), ptr(t["A_val"]))
        AT = capi.Csr(self.n, self.m, self.nnz, ptr(t["AT_ptr"]), ptr(t["AT_idx"]), ptr(t["AT_val"]))
        return capi.Lp(A, AT, ptr(t["c"]), ptr(t["AL"]), ptr(t["AU"]), ptr(t["l"]), ptr(t["u"]),
                       self.obj_constant, 0, None)


def _d2h(p, count, dtype):
    """Copy `count` elements of a device pointer into a new numpy array."""
    torch = _torch()
    out = np.zeros(count, dtype=dtype)
    if count and p:
        torch.cuda.synchronize()
        cudart = _cudart()
        st = cudart.cudaMemcpy(C.c_void_p(out.ctypes.data), C.c_void_p(p), C.c_size_t(out.nbytes), 2)
        if st:
            raise RuntimeError(f"cudaMemcpy failed ({st})")
    return out


_CUDART = None


def _cudart():
    global _CUDART
    if _CUDART is None:
        import glob
        import os
        import torch
        cands = glob.glob(os.path.join(os.path.dirname(torch.__file__), "lib", "libcudart.so*"))
        cands += glob.glob("/usr/local/cuda/lib64/libcudart.so*")
        for c in cands:
            try:
                _CUDART = C.CDLL(c)
                break
            except OSError:
                continue
        if _CUDART is None:
            _CUDART = C.CDLL("libcudart.so")
        _CUDART.cudaMemcpy.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]
    return _CUDART


class Result:
    """Host copy of a presolve summary and its reduced LP, maps and tape."""

    def __init__(self, summary: capi.Summary, copy_lp: bool = True, copy_tape: bool = True):
        lib = capi.load()
        s = summary
        self.summary = s
        m, n, nnz = s.reduced_rows, s.reduced_cols, s.reduced_nnz
        if copy_lp and s.has_infeasible == 0 and s.has_unbounded == 0:
            L = s.reduced_lp
            self.A_ptr = _d2h(L.A.rowPtr, m + 1, np.int32)
            self.A_idx = _d2h(L.A.colVal, nnz, np.int32)
            self.A_val = _d2h(L.A.nzVal, nnz, np.float64)
            self.AT_ptr = _d2h(L.AT.rowPtr, n + 1, np.int32)
            self.AT_idx = _d2h(L.AT.colVal, nnz, np.int32)
            self.AT_val = _d2h(L.AT.nzVal, nnz, np.float64)
            self.c = _d2h(L.c, n, np.float64)
            self.l = _d2h(L.l, n, np.float64)
            self.u = _d2h(L.u, n, np.float64)
            self.AL = _d2h(L.AL, m, np.float64)
            self.AU = _d2h(L.AU, m, np.float64)
            self.obj_constant = L.obj_constant
        self.row_map = np.zeros(m, np.int32)
        self.col_map = np.zeros(n, np.int32)
        _raise(lib.gpp_export_maps(C.byref(s), self.row_map.ctypes.data_as(C.c_void_p),
                                   self.col_map.ctypes.data_as(C.c_void_p)))
        if copy_tape:
            r, i, v, f = (C.c_int64() for _ in range(4))
            _raise(lib.gpp_tape_sizes(C.byref(s), C.byref(r), C.byref(i), C.byref(v), C.byref(f)))
            self.tape_types = np.zeros(r.value, np.int32)
            self.tape_is = np.zeros(r.value + 1, np.int64)
            self.tape_vs = np.zeros(r.value + 1, np.int64)
            self.tape_idx = np.zeros(i.value, np.int32)
            self.tape_val = np.zeros(v.value)
            self.fixed_idx = np.zeros(f.value, np.int32)
            self.fixed_val = np.zeros(f.value)
            _raise(lib.gpp_export_tape(C.byref(s), *(a.ctypes.data_as(C.c_void_p) for a in (
                self.tape_types, self.tape_is, self.tape_vs, self.tape_idx, self.tape_val, self.fixed_idx,
                self.fixed_val))))
            self.checkpoints, self.absolute_value = export_recoveries(s)
            self.variable_pair = export_variable_pairs(s, self.checkpoints)


def export_variable_pairs(s, checkpoints):
    """The record's variable-pair recoveries as dicts of host arrays."""
    lib = capi.load()
    out = []
    for i in range(sum(1 for k, _, _ in checkpoints if k == 1)):
        n = C.c_int32()
        _raise(lib.gpp_variable_pair_size(C.byref(s), i, C.byref(n)))
        a = {k: np.zeros(n.value, np.int32) for k in ("plus", "minus", "root_plus", "root_minus")}
        a.update({k: np.zeros(n.value) for k in ("plus_shift", "minus_shift")})
        _raise(lib.gpp_export_variable_pair(C.byref(s), i, *(a[k].ctypes.data_as(C.c_void_p) for k in (
            "plus", "minus", "root_plus", "root_minus", "plus_shift", "minus_shift"))))
        out.append(a)
    return out


def export_recoveries(s):
    """The record's primal-recovery checkpoints [(kind, payload, tape
    position)] and its absolute-value recoveries as dicts of host arrays."""
    lib = capi.load()
    k = C.c_int32()
    _raise(lib.gpp_recovery_checkpoints(C.byref(s), C.byref(k), None, None, None))
    kinds, payloads = np.zeros(k.value, np.int32), np.zeros(k.value, np.int32)
    pos = np.zeros(k.value, np.int64)
    _raise(lib.gpp_recovery_checkpoints(C.byref(s), C.byref(k), *(a.ctypes.data_as(C.c_void_p)
                                                                   for a in (kinds, payloads, pos))))
    steps = []
    for i in range(int((kinds == 0).sum())):
        z = np.zeros(6, np.int32)
        _raise(lib.gpp_absolute_value_sizes(C.byref(s), i, z.ctypes.data_as(C.c_void_p)))
        pattern, ns, npairs, nl, ng, ne = (int(v) for v in z)
        a = dict(pattern=pattern, split_t=np.zeros(ns, np.int32), split_e=np.zeros(ns, np.int32),
                 split_rho=np.zeros(ns), pair_bound=np.zeros(npairs, np.int32), pair_free=np.zeros(npairs, np.int32),
                 link_slack=np.zeros(nl, np.int32), link_t=np.zeros(nl, np.int32), link_factor=np.zeros(nl),
                 max_slack=np.zeros(ng, np.int32), max_start=np.zeros(ng + 1, np.int32),
                 max_t=np.zeros(ne, np.int32), max_factor=np.zeros(ne))
        keys = ("split_t", "split_e", "split_rho", "pair_bound", "pair_free", "link_slack", "link_t", "link_factor",
                "max_slack", "max_start", "max_t", "max_factor")
        _raise(lib.gpp_export_absolute_value(C.byref(s), i, *(a[q].ctypes.data_as(C.c_void_p) for q in keys)))
        steps.append(a)
    return list(zip(kinds.tolist(), payloads.tolist(), pos.tolist())), steps


def restore_absolute_value(x, steps, original_l=None):
    """postsolve_restore_piecewise_linear_reformulation_absolute_value_gpu on
    the device vector `x` (torch, float64) with host steps (dicts as
    export_recoveries returns)."""
    lib = capi.load()
    keep = []

    def ptr(v, dt):
        v = np.ascontiguousarray(v, dtype=dt)
        keep.append(v)
        return v.ctypes.data_as(C.c_void_p)

    arr = (capi.AbsoluteValueRecovery * max(1, len(steps)))()
    for i, a in enumerate(steps):
        ng = len(a["max_slack"])
        arr[i] = capi.AbsoluteValueRecovery(
            a["pattern"], len(a["split_t"]), ptr(a["split_t"], np.int32), ptr(a["split_e"], np.int32),
            ptr(a["split_rho"], np.float64), len(a["pair_bound"]), ptr(a["pair_bound"], np.int32),
            ptr(a["pair_free"], np.int32), len(a["link_slack"]), ptr(a["link_slack"], np.int32),
            ptr(a["link_t"], np.int32), ptr(a["link_factor"], np.float64), ng, ptr(a["max_slack"], np.int32),
            ptr(a["max_start"] if ng else np.zeros(1), np.int32), ptr(a["max_t"], np.int32),
            ptr(a["max_factor"], np.float64))
    lp = C.c_void_p(original_l.data_ptr()) if original_l is not None else None
    _raise(lib.gpp_restore_absolute_value(C.c_void_p(x.data_ptr()), arr, len(steps), lp))


def preprocess(dlp: DeviceLp, params=None) -> capi.Summary:
    lib = capi.load()
    params = params or capi.Params.defaults()
    s = capi.Summary()
    lp = dlp.struct()
    _raise(lib.gpp_preprocess(C.byref(lp), C.byref(params), C.byref(s)))
    return s


def postprocess(x_red, y_red, z_red, summary: capi.Summary, original: DeviceLp, out=None):
    """x/y/z_red: torch CUDA float64 tensors in reduced order; returns host x, y, z in original order.

    ``out`` may give the three host arrays (numpy arrays, or CPU torch tensors such as
    page-locked ones, which download faster); otherwise numpy arrays are allocated."""
    lib = capi.load()
    if out is None:
        out = (np.zeros(summary.original_cols), np.zeros(summary.original_rows), np.zeros(summary.original_cols))
    addr = [a.ctypes.data if isinstance(a, np.ndarray) else a.data_ptr() for a in out]
    lp = original.struct()
    _raise(lib.gpp_postprocess(f64ptr(x_red), f64ptr(y_red), f64ptr(z_red), C.byref(summary), C.byref(lp),
                               *(C.c_void_p(v) for v in addr)))
    return out


def free_summary(summary: capi.Summary) -> None:
    capi.load().gpp_free_summary(C.byref(summary))


def postsolve_device(x_red, y_red, z_red, summary: capi.Summary, original: DeviceLp, out=None):
    """presolve::postsolve_gpu: original-space x, y, z as CUDA tensors."""
    torch = _torch()
    if out is None:
        out = (torch.empty(summary.original_cols, dtype=torch.float64, device="cuda"),
               torch.empty(summary.original_rows, dtype=torch.float64, device="cuda"),
               torch.empty(summary.original_cols, dtype=torch.float64, device="cuda"))
    lp = original.struct()
    _raise(capi.load().gpp_postsolve_device(f64ptr(x_red), f64ptr(y_red), f64ptr(z_red), C.byref(summary), C.byref(lp),
                                            *(ptr(t) for t in out)))
    return out


def fold_map(summary: capi.Summary):
    """folding::copy_map_to_host: (row_color, col_color, row_scale, col_scale) or None."""
    if not summary.folding_applied:
        return None
    rc = np.zeros(summary.original_rows, np.int32)
    cc = np.zeros(summary.original_cols, np.int32)
    rs = np.zeros(summary.original_rows)
    cs = np.zeros(summary.original_cols)
    _raise(capi.load().gpp_export_folding_map(C.byref(summary), *(a.ctypes.data_as(C.c_void_p)
                                                                  for a in (rc, cc, rs, cs))))
    return rc, cc, rs, cs


def unfold(x_folded, y_folded, z_folded, summary: capi.Summary):
    """folding::unfold_solution_device_to_host: folded-model CUDA tensors -> original-model host arrays."""
    x = np.zeros(summary.original_cols)
    y = np.zeros(summary.original_rows)
    z = np.zeros(summary.original_cols)
    _raise(capi.load().gpp_unfold_solution(C.byref(summary), ptr(x_folded), ptr(y_folded), ptr(z_folded),
                                           x.ctypes.data_as(C.c_void_p), y.ctypes.data_as(C.c_void_p),
                                           z.ctypes.data_as(C.c_void_p)))
    return x, y, z


def _ptr_array(values):
    arr = (C.c_void_p * max(1, len(values)))()
    for k, v in enumerate(values):
        arr[k] = v
    return arr


def preprocess_batch(dlps, params=None, workers: int = 0):
    """gpp_preprocess_batch: one summary per LP (each as gpp_preprocess gives it) and the per-LP statuses.

    Raises on a failed batch after freeing the summaries it made."""
    lib = capi.load()
    params = params or capi.Params.defaults()
    lps = (capi.Lp * len(dlps))(*[d.struct() for d in dlps])
    out = (capi.Summary * len(dlps))()
    status = np.zeros(len(dlps), np.int32)
    rc = lib.gpp_preprocess_batch(C.cast(lps, C.c_void_p), len(dlps), C.byref(params), workers,
                                  C.cast(out, C.c_void_p), status.ctypes.data_as(C.c_void_p))
    summaries = [out[k] for k in range(len(dlps))]
    if rc != 0:
        for s in summaries:
            free_summary(s)
        _raise(rc)
    return summaries, status


def postprocess_batch(xs, ys, zs, summaries, dlps, workers: int = 0):
    """gpp_postprocess_batch: xs/ys/zs are per-LP CUDA float64 tensors (or None) in reduced order;
    returns per-LP host (x, y, z) in original order."""
    lib = capi.load()
    k = len(summaries)
    outs = [(np.zeros(s.original_cols), np.zeros(s.original_rows), np.zeros(s.original_cols)) for s in summaries]
    sums = (capi.Summary * k)(*summaries)
    lps = (capi.Lp * k)(*[d.struct() for d in dlps])
    dev = [_ptr_array([f64ptr(v[i]) if v is not None and v[i] is not None else None for i in range(k)])
           for v in (xs, ys, zs)]
    host = [_ptr_array([o[j].ctypes.data for o in outs]) for j in range(3)]
    status = np.zeros(k, np.int32)
    _raise(lib.gpp_postprocess_batch(*(C.cast(a, C.c_void_p) for a in dev), C.cast(sums, C.c_void_p),
                                     C.cast(lps, C.c_void_p), k, workers,
                                     *(C.cast(a, C.c_void_p) for a in host), status.ctypes.data_as(C.c_void_p)))
    return outs


def batch_autotune(dlps, params=None, max_workers: int = 32):
    """gpp_batch_autotune: (best worker count, {worker count: sampled LPs/s})."""
    lib = capi.load()
    params = params or capi.Params.defaults()
    lps = (capi.Lp * len(dlps))(*[d.struct() for d in dlps])
    best = C.c_int32(0)
    counts = [1 << k for k in range(max_workers.bit_length()) if (1 << k) <= max_workers]
    rates = np.zeros(len(counts))
    _raise(lib.gpp_batch_autotune(C.cast(lps, C.c_void_p), len(dlps), C.byref(params), max_workers, C.byref(best),
                                  rates.ctypes.data_as(C.c_void_p)))
    return int(best.value), {w: round(float(r), 2) for w, r in zip(counts, rates)}
