"""CPU tests of the oracle: the reference's known-answer fixtures and the
objective of presolve -> HiGHS -> postsolve against HiGHS on the unreduced LP."""
import numpy as np
import pytest

import fixtures
import lpsolve
import pyoracle
from gpp_b200 import lpgen
from gpp_b200.capi import params_with_rules

CLEANUP = ["infeasible_and_fixed_variables", "empty_columns", "empty_rows", "singleton_rows"]
BUILT = CLEANUP + ["bound_strengthening"]
PROPAGATION = BUILT + ["infeasible_and_redundant_rows", "dual_fix"]
PARALLEL = PROPAGATION + ["parallel_rows", "parallel_columns"]
SINGLETON = CLEANUP + ["singleton_columns"]
FULL = PARALLEL + ["singleton_columns"]
ALL = FULL + ["doubleton_equations"]


def test_dyadic_activity_matches_reference_fixture():
    f = fixtures.dyadic_activity_fixture()
    lo, hi, ni, pi = pyoracle.row_activity_summary(f["rows"], f["cols"], f["ptr"], f["idx"], f["val"],
                                                   f["lower"], f["upper"], 1e-12)
    assert np.array_equal(lo, f["lo"]) and np.array_equal(hi, f["hi"])
    assert np.array_equal(ni, f["ni"]) and np.array_equal(pi, f["pi"])


def test_col_max_matches_reference_fixture():
    f = fixtures.dyadic_activity_fixture()
    out = pyoracle.col_max_abs(f["rows"], f["cols"], f["ptr"], f["idx"], f["val"])
    assert np.array_equal(out, f["max"])


def test_live_stats_masks():
    rng = np.random.default_rng(3)
    lp = lpgen.random_lp(300, 700, seed=3)
    keep_r = (rng.random(lp.m) < 0.8).astype(np.uint8)
    keep_c = (rng.random(lp.n) < 0.7).astype(np.uint8)
    deg, empty, single, sup, coef, total = pyoracle.live_stats(lp.m, lp.n, lp.row_ptr, lp.col_idx, lp.values,
                                                               keep_r, keep_c)
    for i in range(lp.m):
        cols = lp.col_idx[lp.row_ptr[i]:lp.row_ptr[i + 1]]
        vals = lp.values[lp.row_ptr[i]:lp.row_ptr[i + 1]]
        live = keep_c[cols].astype(bool) & bool(keep_r[i])
        assert deg[i] == live.sum()
        assert empty[i] == (keep_r[i] and live.sum() == 0)
        if live.sum() == 1:
            assert sup[i] == cols[live][0] and coef[i] == vals[live][0]
        else:
            assert sup[i] == -1
    assert total == deg.sum()


def test_det_sum_tree():
    v = np.random.default_rng(0).standard_normal(5000) * 1e3
    total = 0.0
    for b in range(0, v.size, 2048):
        chunk = v[b:b + 2048]
        s = [float(np.sum(chunk[t::256][:0])) for t in range(256)]
        for t in range(256):
            acc = 0.0
            for x in chunk[t::256]:
                acc += x
            s[t] = acc
        h = 128
        while h:
            for t in range(h):
                s[t] = s[t] + s[t + h]
            h //= 2
        total += s[0]
    assert pyoracle.det_sum(v) == total


@pytest.mark.parametrize("rules", [CLEANUP, BUILT, PROPAGATION, PARALLEL, SINGLETON, FULL, ALL])
@pytest.mark.parametrize("workload,seed", [("random:400x1000", 0), ("random:400x1000", 1), ("slack:400x1000", 0),
                                           ("slack:400x1000", 1)])
def test_postsolved_objective_matches_unreduced(rules, workload, seed):
    lp = lpgen.workload(workload, seed=seed)
    res0, _, _ = lpsolve.solve(lp.m, lp.n, lp.row_ptr, lp.col_idx, lp.values, lp.c, lp.AL, lp.AU, lp.l, lp.u)
    assert res0.status == 0
    # Small doubleton batches allowed so the rule runs at this size.
    r = pyoracle.presolve(lp, params_with_rules(rules, doubleton_equations_min_selected_per_batch=1,
                                                doubleton_equations_min_selected_ratio=0.0))
    s = r.summary
    assert not s.has_infeasible and not s.has_unbounded
    rr, yr, zr = lpsolve.solve(s.reduced_rows, s.reduced_cols, r.A_ptr, r.A_idx, r.A_val, r.c, r.AL, r.AU, r.l, r.u)
    assert rr.status == 0
    x, y, z = r.postsolve(rr.x, yr, zr)
    obj = float(lp.c @ x)
    assert abs(obj - res0.fun) <= 1e-9 * max(1.0, abs(res0.fun))
    assert abs((rr.fun + r.obj_constant) - res0.fun) <= 1e-9 * max(1.0, abs(res0.fun))
    assert lpsolve.primal_violation(lp, x) <= 1e-6


def test_reduced_structure_consistent():
    lp = lpgen.random_lp(400, 1000, seed=5)
    r = pyoracle.presolve(lp, params_with_rules(BUILT))
    s = r.summary
    # A^T of the reduced LP is the row-sorted transpose of its A.
    t_ptr, t_idx, t_val = lpgen.csr_transpose(s.reduced_rows, s.reduced_cols, r.A_ptr, r.A_idx, r.A_val)
    assert np.array_equal(t_ptr, r.AT_ptr) and np.array_equal(t_idx, r.AT_idx) and np.array_equal(t_val, r.AT_val)
    # Maps are strictly increasing original indices.
    assert np.all(np.diff(r.row_map) > 0) and np.all(np.diff(r.col_map) > 0)
    # Kept entries carry the original coefficients.
    A0 = {}
    for i in range(lp.m):
        for p in range(lp.row_ptr[i], lp.row_ptr[i + 1]):
            A0[(i, lp.col_idx[p])] = lp.values[p]
    for i in range(s.reduced_rows):
        for p in range(r.A_ptr[i], r.A_ptr[i + 1]):
            assert A0[(r.row_map[i], r.col_map[r.A_idx[p]])] == r.A_val[p]


def test_schedule_trace_phase_order():
    lp = lpgen.random_lp(400, 1000, seed=2)
    r = pyoracle.presolve(lp, params_with_rules(BUILT))
    phases = [t for t in r.trace if t.startswith("phase=")]
    assert phases[0] == "phase=cleanup"
    # Propagation is always followed by Cleanup or Aggregation.
    for a, b in zip(phases, phases[1:]):
        if a == "phase=propagation":
            assert b in ("phase=cleanup", "phase=aggregation")
    assert r.summary.iterations >= 1


@pytest.mark.parametrize("rows", [10, 2100])
def test_row_hash_matches_reference_fixture(rows):
    f = fixtures.hash_fixture(rows)
    for i in range(rows):
        if not f["keep"][i]:
            continue
        h = pyoracle.lib().orc_row_hash(rows, f["cols"], pyoracle.ptr(f["ptr"]), pyoracle.ptr(f["idx"]),
                                        pyoracle.ptr(f["val"]), i, None, f["mode"])
        assert h == int(f["expected"][i]), i


def test_parallel_rules_postsolve_objective():
    lp = lpgen.random_lp(600, 1500, seed=4)
    rules = BUILT + ["infeasible_and_redundant_rows", "dual_fix", "parallel_rows", "parallel_columns"]
    res0, _, _ = lpsolve.solve(lp.m, lp.n, lp.row_ptr, lp.col_idx, lp.values, lp.c, lp.AL, lp.AU, lp.l, lp.u)
    r = pyoracle.presolve(lp, params_with_rules(rules))
    s = r.summary
    rr, yr, zr = lpsolve.solve(s.reduced_rows, s.reduced_cols, r.A_ptr, r.A_idx, r.A_val, r.c, r.AL, r.AU, r.l, r.u)
    x, _, _ = r.postsolve(rr.x, yr, zr)
    assert abs(lp.c @ x - res0.fun) <= 1e-9 * max(1.0, abs(res0.fun))
    assert lpsolve.primal_violation(lp, x) <= 1e-6
