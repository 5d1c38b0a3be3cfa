"""End-to-end parity on the GPU through the C ABI: preprocess -> reduced LP,
maps, tape and fixed values against the oracle (bitwise), then postprocess
against the oracle's postsolve and the unreduced LP's optimum (HiGHS)."""
import numpy as np
import pytest

import lpsolve
import pyoracle
from gpp_b200 import device, lpgen
from gpp_b200.capi import params_with_rules

pytestmark = pytest.mark.gpu

CLEANUP = ["infeasible_and_fixed_variables", "empty_columns", "empty_rows", "singleton_rows"]
BUILT = CLEANUP + ["bound_strengthening"]
PROPAGATION = BUILT + ["infeasible_and_redundant_rows", "dual_fix"]
PARALLEL = PROPAGATION + ["parallel_rows", "parallel_columns"]
SINGLETON = CLEANUP + ["singleton_columns"]
FULL = PARALLEL + ["singleton_columns"]
ALL = FULL + ["doubleton_equations"]
SMALL_BATCH = dict(doubleton_equations_min_selected_per_batch=1, doubleton_equations_min_selected_ratio=0.0)


def bits(a):
    a = np.asarray(a)
    return a.view(np.uint64) if a.dtype == np.float64 else a


def assert_same(gpu, orc):
    s, o = gpu.summary, orc.summary
    for f in ("reduced_rows", "reduced_cols", "reduced_nnz", "iterations", "has_infeasible", "has_unbounded",
              "has_change", "stopped_at_iteration_limit"):
        assert getattr(s, f) == getattr(o, f), f
    for f in ("A_ptr", "A_idx", "A_val", "AT_ptr", "AT_idx", "AT_val", "c", "l", "u", "AL", "AU", "row_map",
              "col_map", "tape_types", "tape_is", "tape_vs", "tape_idx", "tape_val", "fixed_idx", "fixed_val"):
        assert np.array_equal(bits(getattr(gpu, f)), bits(getattr(orc, f))), f
    assert s.obj_constant_delta == o.obj_constant_delta


@pytest.mark.parametrize("rules", [CLEANUP, BUILT, PROPAGATION, PARALLEL, SINGLETON, FULL])
@pytest.mark.parametrize("workload", ["random:400x1000", "small", "slack:400x1000", "slack:2000x5000"])
def test_presolve_bitwise_vs_oracle(rules, workload):
    lp = lpgen.workload(workload, seed=0)
    params = params_with_rules(rules, enable_folding=0)
    dlp = device.DeviceLp(lp)
    s = device.preprocess(dlp, params)
    try:
        gpu = device.Result(s)
        orc = pyoracle.presolve(lp, params)
        assert_same(gpu, orc)
    finally:
        device.free_summary(s)
        device.free_summary(s)  # idempotent


@pytest.mark.parametrize("workload,extra", [("random:400x1000", SMALL_BATCH), ("slack:2000x5000", SMALL_BATCH),
                                            ("random:20000x50000", {})])
def test_doubleton_bitwise_vs_oracle(workload, extra):
    lp = lpgen.workload(workload, seed=0)
    params = params_with_rules(ALL, enable_folding=0, **extra)
    dlp = device.DeviceLp(lp)
    s = device.preprocess(dlp, params)
    try:
        gpu = device.Result(s)
        orc = pyoracle.presolve(lp, params)
        assert_same(gpu, orc)
        assert 13 in gpu.tape_types.tolist()   # the batch ran
    finally:
        device.free_summary(s)


@pytest.mark.parametrize("workload,extra", [("slack:2000x5000", SMALL_BATCH), ("random:20000x50000", {})])
def test_parallel_replay_matches_serial_oracle(workload, extra):
    """Tapes of >= 1024 records replay as independent record groups on the
    GPU; the result must equal the oracle's one-record-at-a-time replay bit
    for bit, for any reduced point (here a seeded one inside the bounds)."""
    import torch
    lp = lpgen.workload(workload, seed=0)
    params = params_with_rules(ALL, enable_folding=0, **extra)
    dlp = device.DeviceLp(lp)
    s = device.preprocess(dlp, params)
    try:
        gpu = device.Result(s)
        assert len(gpu.tape_types) >= 1024
        rng = np.random.default_rng(1)
        lo = np.where(np.isfinite(gpu.l), gpu.l, -10.0)
        hi = np.where(np.isfinite(gpu.u), gpu.u, lo + 20.0)
        xr = lo + rng.random(s.reduced_cols) * (hi - lo)
        yr = rng.standard_normal(s.reduced_rows)
        zr = rng.standard_normal(s.reduced_cols)
        x, y, z = device.postprocess(torch.from_numpy(xr).cuda(), torch.from_numpy(yr).cuda(),
                                     torch.from_numpy(zr).cuda(), s, dlp)
        orc = pyoracle.presolve(lp, params)
        xo, yo, zo = orc.postsolve(xr, yr, zr)
        assert np.array_equal(bits(x), bits(xo))
        assert np.array_equal(bits(y), bits(yo))
        assert np.array_equal(bits(z), bits(zo))
    finally:
        device.free_summary(s)


@pytest.mark.parametrize("rules", [PROPAGATION, FULL, ALL])
@pytest.mark.parametrize("workload,seed", [("random:400x1000", 0), ("random:400x1000", 3), ("slack:400x1000", 0)])
def test_postprocess_vs_oracle_and_highs(rules, workload, seed):
    import torch
    lp = lpgen.workload(workload, seed=seed)
    params = params_with_rules(rules, enable_folding=0, **SMALL_BATCH)
    dlp = device.DeviceLp(lp)
    s = device.preprocess(dlp, params)
    try:
        gpu = device.Result(s)
        res0, _, _ = lpsolve.solve(lp.m, lp.n, lp.row_ptr, lp.col_idx, lp.values, lp.c, lp.AL, lp.AU, lp.l, lp.u)
        rr, yr, zr = lpsolve.solve(s.reduced_rows, s.reduced_cols, gpu.A_ptr, gpu.A_idx, gpu.A_val, gpu.c, gpu.AL,
                                   gpu.AU, gpu.l, gpu.u)
        xd = torch.from_numpy(rr.x).cuda()
        yd = torch.from_numpy(yr).cuda()
        zd = torch.from_numpy(zr).cuda()
        x, y, z = device.postprocess(xd, yd, zd, s, dlp)
        orc = pyoracle.presolve(lp, params)
        xo, yo, zo = orc.postsolve(rr.x, yr, zr)
        assert np.array_equal(bits(x), bits(xo))
        assert np.array_equal(bits(y), bits(yo))
        assert np.array_equal(bits(z), bits(zo))
        assert abs(lp.c @ x - res0.fun) <= 1e-9 * max(1.0, abs(res0.fun))
    finally:
        device.free_summary(s)


def test_identity_when_presolve_disabled():
    lp = lpgen.random_lp(200, 500, seed=1)
    dlp = device.DeviceLp(lp)
    s = device.preprocess(dlp, params_with_rules(BUILT, enable_folding=0, enable_presolve=0))
    try:
        assert s.owns_reduced_lp == 0 and s.reduced_rows == lp.m and s.reduced_cols == lp.n
        assert s.reduced_lp.A.rowPtr == dlp.t["A_ptr"].data_ptr()
    finally:
        device.free_summary(s)
