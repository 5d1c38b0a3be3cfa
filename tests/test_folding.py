"""Symmetry folding: the reference's known answers (cpp/tests/test_folding.cpp)
on the oracle and the CUDA engine, the skip decision on asymmetric LPs, and
engine-vs-oracle agreement on replicated LPs (identical blocks plus a coupling
row), where folding applies."""
import numpy as np
import pytest

from gpp_b200 import lpgen
from gpp_b200.capi import RULE_FLAGS, params_with_rules
from rule_cases import INF, Run, bits, make_lp

BACKENDS = ["oracle", pytest.param("gpu", marks=pytest.mark.gpu)]
NO_RULES = []
ALL = [f[len("enable_"):] for f in RULE_FLAGS if f not in ("enable_structure_specific_rules", "enable_startup",
                                                             "enable_redundant_variable_bounds")]


def symmetric_2x2(values=(1.0, 1.0, 1.0, 1.0), rhs=4.0, obj=0.0):
    lp = make_lp(2, [[(0, values[0]), (1, values[1])], [(0, values[2]), (1, values[3])]], c=[2.0, 2.0],
                 l=[0.0, 0.0], u=[10.0, 10.0], AL=[rhs, rhs], AU=[rhs, rhs])
    lp.obj_constant = obj
    return lp


@pytest.mark.parametrize("backend", BACKENDS)
def test_run_folding_reduces_identical_rows_and_cols(backend):
    # test_run_folding_reduces_identical_rows_and_cols.
    r = Run(backend, symmetric_2x2(), NO_RULES, enable_folding=1, max_iters=1)
    assert r.s.folding_applied == 1
    assert (r.s.original_rows, r.s.original_cols) == (2, 2)
    assert (r.s.folded_rows, r.s.folded_cols) == (1, 1)
    rc, cc, rs, cs = r.fold
    assert rc.tolist() == [1, 1] and cc.tolist() == [1, 1]
    assert rs.tolist() == [0.5, 0.5] and cs.tolist() == [0.5, 0.5]
    assert (r.s.reduced_rows, r.s.reduced_cols, r.s.reduced_nnz) == (1, 1, 1)
    # Folded entry: the four unit entries each weighted by 1/|R| = 1/2.
    assert r.A_val.tolist() == [2.0] and r.c.tolist() == [4.0]
    assert r.AL.tolist() == [4.0] and r.AU.tolist() == [4.0] and r.l.tolist() == [0.0] and r.u.tolist() == [10.0]


@pytest.mark.gpu
def test_unfold_solution_scales_duals_and_slacks():
    # test_unfold_solution_scales_duals_and_slacks, through gpp_unfold_solution.
    import torch
    from gpp_b200 import device
    dlp = device.DeviceLp(symmetric_2x2())
    s = device.preprocess(dlp, params_with_rules(NO_RULES, enable_folding=1, max_iters=1))
    try:
        t = lambda v: torch.tensor(v, dtype=torch.float64, device="cuda")
        x, y, z = device.unfold(t([4.0]), t([6.0]), t([8.0]), s)
        assert x.tolist() == [4.0, 4.0] and y.tolist() == [3.0, 3.0] and z.tolist() == [4.0, 4.0]
        # test_postsolve_and_unfold_restores_original_dimensions.
        x, y, z = device.postprocess(t([4.0]), t([6.0]), t([8.0]), s, dlp)
        assert x.tolist() == [4.0, 4.0] and np.all(np.isfinite(y)) and np.all(np.isfinite(z))
    finally:
        device.free_summary(s)


def test_unfold_oracle():
    import pyoracle
    lp = symmetric_2x2()
    r = pyoracle.presolve(lp, params_with_rules(NO_RULES, enable_folding=1, max_iters=1))
    x, y, z = r.postsolve(np.array([4.0]), np.array([6.0]), np.array([8.0]))
    assert x.tolist() == [4.0, 4.0] and np.all(np.isfinite(y)) and np.all(np.isfinite(z))


@pytest.mark.parametrize("backend", BACKENDS)
def test_equitable_partition_folded_model(backend):
    # test_equitable_partition_and_original_kkt: rows [1 2] and [2 1], both = 3.
    lp = symmetric_2x2(values=(1.0, 2.0, 2.0, 1.0), rhs=3.0, obj=7.0)
    r = Run(backend, lp, ALL, enable_folding=1, max_iters=0)
    assert r.s.folding_applied == 1
    assert (r.s.original_rows, r.s.original_cols) == (2, 2)
    assert (r.s.reduced_rows, r.s.reduced_cols) == (1, 1)
    assert r.obj_constant == 7.0
    assert abs(r.A_val[0] - 3.0) < 1e-12 and abs(r.c[0] - 4.0) < 1e-12


def test_equitable_partition_original_kkt_oracle():
    import pyoracle
    lp = symmetric_2x2(values=(1.0, 2.0, 2.0, 1.0), rhs=3.0, obj=7.0)
    r = pyoracle.presolve(lp, params_with_rules(ALL, enable_folding=1, max_iters=0))
    x, y, z = r.postsolve(np.array([1.0]), np.array([4.0 / 3.0]), np.array([0.0]))
    vals = [1.0, 2.0, 2.0, 1.0]
    for j in range(2):
        assert abs(x[j] - 1.0) < 1e-12
        aty = vals[j] * y[0] + vals[2 + j] * y[1]
        assert abs(aty + z[j] - 2.0) < 1e-12 and abs(z[j]) < 1e-12
    assert abs(2 * (x[0] + x[1]) + 7 - 11) < 1e-12


@pytest.mark.parametrize("backend", BACKENDS)
def test_asymmetric_lp_is_not_folded(backend):
    # Random costs give nearly every column its own colour: refinement gives up
    # (more than 80% distinct on both sides) and presolve runs on the input.
    lp = lpgen.random_lp(400, 1000, seed=0)
    folded = Run(backend, lp, ALL, enable_folding=1)
    plain = Run(backend, lp, ALL, enable_folding=0)
    assert folded.s.folding_applied == 0 and folded.fold is None
    assert (folded.s.folded_rows, folded.s.folded_cols) == (400, 1000)
    for k in ("A_idx", "A_val", "c", "l", "u", "row_map", "col_map", "tape_types", "tape_idx"):
        assert np.array_equal(getattr(folded, k), getattr(plain, k)), k


@pytest.mark.gpu
@pytest.mark.parametrize("workload", ["replicated:100x250*4", "replicated:400x1000*3", "replicated:2000x5000*2"])
def test_replicated_fold_matches_oracle(workload):
    """Replicated LPs fold; the engine's colours, folded model and the presolve
    of it equal the oracle's."""
    lp = lpgen.workload(workload, seed=0)
    g = Run("gpu", lp, ALL, enable_folding=1)
    o = Run("oracle", lp, ALL, enable_folding=1)
    assert g.s.folding_applied == 1 and o.s.folding_applied == 1
    assert (g.s.folded_rows, g.s.folded_cols) == (o.s.folded_rows, o.s.folded_cols)
    for a, b in zip(g.fold, o.fold):
        assert np.array_equal(a, b)
    for k in ("A_ptr", "A_idx", "A_val", "c", "l", "u", "AL", "AU", "row_map", "col_map", "tape_types", "tape_idx",
              "tape_val"):
        assert np.array_equal(bits(getattr(g, k)) if getattr(g, k).dtype == np.float64 else getattr(g, k),
                              bits(getattr(o, k)) if getattr(o, k).dtype == np.float64 else getattr(o, k)), k


@pytest.mark.parametrize("workload", ["replicated:100x250*4", "replicated:400x1000*3"])
def test_replicated_fold_objective_oracle(workload):
    """Folding + presolve + postsolve + unfold reproduce the unreduced optimum."""
    import lpsolve
    import pyoracle
    lp = lpgen.workload(workload, seed=0)
    res0, _, _ = lpsolve.solve(lp.m, lp.n, lp.row_ptr, lp.col_idx, lp.values, lp.c, lp.AL, lp.AU, lp.l, lp.u)
    r = pyoracle.presolve(lp, params_with_rules(ALL, enable_folding=1))
    s = r.summary
    assert s.folding_applied == 1
    rr, yr, zr = lpsolve.solve(s.reduced_rows, s.reduced_cols, r.A_ptr, r.A_idx, r.A_val, r.c, r.AL, r.AU, r.l, r.u)
    x, y, z = r.postsolve(rr.x, yr, zr)
    assert abs(lp.c @ x - res0.fun) <= 1e-9 * max(1.0, abs(res0.fun))
    assert lpsolve.primal_violation(lp, x) <= 1e-6
