"""gpp_lp_from_host: a host CSR and the vectors loaded into device arrays,
with A^T built on the GPU.  The device transpose must equal the stable host
CSC (upload_lp's AT, cpp/tools/gpu_preprocessor_tool_common.hpp:108-141) bit
for bit, and presolve on the loaded LP must equal presolve on the LP
uploaded with its host CSC."""
import numpy as np
import pytest

from gpp_b200 import device, lpgen
from gpp_b200.capi import params_with_rules

pytestmark = pytest.mark.gpu

FULL = ["infeasible_and_fixed_variables", "empty_columns", "empty_rows", "singleton_rows", "singleton_columns",
        "bound_strengthening", "infeasible_and_redundant_rows", "dual_fix", "parallel_rows", "parallel_columns",
        "doubleton_equations"]


def host_arrays(lp, pinned):
    import torch
    arrays = {"A_ptr": (lp.row_ptr, np.int32), "A_idx": (lp.col_idx, np.int32), "A_val": (lp.values, np.float64),
              "c": (lp.c, np.float64), "AL": (lp.AL, np.float64), "AU": (lp.AU, np.float64),
              "l": (lp.l, np.float64), "u": (lp.u, np.float64)}
    out = {}
    for k, (a, dt) in arrays.items():
        t = torch.from_numpy(np.array(a, dtype=dt, copy=True))   # never a view of the LP's own arrays
        out[k] = t.pin_memory() if pinned else t
    return out


def blank_like(dlp):
    """A DeviceLp of the same sizes whose device arrays hold garbage."""
    import torch
    other = device.DeviceLp(dlp.host)
    for t in other.t.values():
        if t.dtype == torch.float64:
            t.fill_(float("nan"))
        else:
            t.fill_(-7)
    return other


def with_empty_rows_and_columns(seed=3):
    """Random LP whose first and last rows and a run of columns hold no entry."""
    lp = lpgen.random_lp(600, 1500, seed)
    dense = np.zeros((lp.m, lp.n))
    rows = np.repeat(np.arange(lp.m), np.diff(lp.row_ptr))
    dense[rows, lp.col_idx] = lp.values
    dense[0, :] = 0.0
    dense[-1, :] = 0.0
    dense[:, 100:140] = 0.0
    nz = dense != 0
    lp.row_ptr = np.concatenate([[0], np.cumsum(nz.sum(axis=1))]).astype(np.int32)
    r, c = np.nonzero(nz)
    lp.col_idx = c.astype(np.int32)
    lp.values = dense[r, c]
    lp.at_ptr = lp.at_idx = lp.at_val = None
    return lp


def with_dense_columns(seed=5):
    """Random LP plus two columns holding an entry in every row: columns far
    longer than 64 entries take the radix-sort transpose."""
    lp = lpgen.random_lp(3000, 2000, seed)
    rows = np.repeat(np.arange(lp.m), np.diff(lp.row_ptr))
    extra = np.arange(lp.m)
    r = np.concatenate([rows, extra, extra])
    c = np.concatenate([lp.col_idx, np.full(lp.m, lp.n), np.full(lp.m, lp.n + 1)])
    v = np.concatenate([lp.values, np.full(lp.m, 1.5), np.full(lp.m, -0.25)])
    lp.row_ptr, lp.col_idx, lp.values = lpgen.coo_to_csr(lp.m, r, c, v)
    lp.n += 2
    lp.c = np.concatenate([lp.c, [1.0, 2.0]])
    lp.l = np.concatenate([lp.l, [0.0, 0.0]])
    lp.u = np.concatenate([lp.u, [10.0, 10.0]])
    lp.at_ptr = lp.at_idx = lp.at_val = None
    return lp


CASES = [
    ("random:2000x5000", 0),
    ("slack:3000x7000", 1),
    ("random:40000x100000", 2),   # past the single-launch scan sizes
    ("qap:6", 0),
    ("dense_columns", 0),         # long columns: the radix-sort transpose
]


@pytest.mark.parametrize("name,seed", CASES)
@pytest.mark.parametrize("pinned", [True, False])
def test_device_transpose_equals_host_csc(name, seed, pinned):
    lp = with_dense_columns() if name == "dense_columns" else lpgen.workload(name, seed)
    ref = device.DeviceLp(lp)
    dlp = blank_like(ref)
    dlp.load_from_host(host_arrays(lp, pinned))
    for k in ref.t:
        a, b = ref.t[k].cpu().numpy(), dlp.t[k].cpu().numpy()
        if a.dtype == np.float64:
            a, b = a.view(np.uint64), b.view(np.uint64)
        assert np.array_equal(a, b), k


def test_empty_rows_and_columns():
    lp = with_empty_rows_and_columns()
    ref = device.DeviceLp(lp)
    dlp = blank_like(ref)
    dlp.load_from_host(host_arrays(lp, True))
    for k in ("AT_ptr", "AT_idx", "AT_val"):
        assert np.array_equal(ref.t[k].cpu().numpy(), dlp.t[k].cpu().numpy()), k


@pytest.mark.parametrize("name", ["random:2000x5000", "slack:3000x7000"])
def test_presolve_on_loaded_lp_equals_uploaded(name):
    lp = lpgen.workload(name, 0)
    ref = device.DeviceLp(lp)
    dlp = blank_like(ref)
    dlp.load_from_host(host_arrays(lp, True))
    params = params_with_rules(FULL, enable_folding=1)
    s0, s1 = device.preprocess(ref, params), device.preprocess(dlp, params)
    try:
        r0, r1 = device.Result(s0), device.Result(s1)
        for f in ("reduced_rows", "reduced_cols", "reduced_nnz", "iterations"):
            assert getattr(s0, f) == getattr(s1, f), f
        for f in ("A_ptr", "A_idx", "A_val", "AT_ptr", "AT_idx", "AT_val", "row_map", "col_map"):
            assert np.array_equal(getattr(r0, f), getattr(r1, f)), f
    finally:
        device.free_summary(s0)
        device.free_summary(s1)


@pytest.mark.parametrize("fault", ["column_out_of_range", "negative_column", "pointer_decreases", "pointer_end"])
def test_invalid_csr_is_rejected_before_the_transpose(fault):
    lp = lpgen.workload("random:500x1200", 4)
    host = host_arrays(lp, False)
    if fault == "column_out_of_range":
        host["A_idx"][17] = lp.n
    elif fault == "negative_column":
        host["A_idx"][3] = -1
    elif fault == "pointer_decreases":
        host["A_ptr"][10] = host["A_ptr"][9] - 1
    else:
        host["A_ptr"][-1] = host["A_ptr"][-1] - 1
    dlp = device.DeviceLp(lp)
    with pytest.raises(ValueError, match="not a valid CSR"):
        dlp.load_from_host(host)
    # The context stays usable: a valid load right after succeeds.
    dlp.load_from_host(host_arrays(lp, False))
    ref = device.DeviceLp(lp)
    assert np.array_equal(ref.t["AT_idx"].cpu().numpy(), dlp.t["AT_idx"].cpu().numpy())
