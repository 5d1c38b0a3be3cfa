"""Structure-specific Startup rules: column domination on unit set-covering
LPs, and the projected auxiliaries (two-row variable elimination, zero-cost
product variables) that share its plan.

CPU: the oracle on the reference's own known-answer models and fail-closed
variants (cpp/tests/test_rule_column_domination.cpp:62-206,
cpp/tests/test_rule_projected_auxiliaries.cpp:103-400), on generated
set-covering LPs (exactly the columns whose cost exceeds their degree go, and
only past both thresholds), on generated LPs with projected-auxiliary blocks
and decoys, and the postsolved objective of the full pipeline against HiGHS.
GPU: the engine bit-exact against the oracle, the known-answer models through
the C ABI with postsolve, and parity with the reference library itself with
its structure-specific rules on."""
import numpy as np
import pytest

import lpsolve
import pyoracle
from gpp_b200 import capi, lpgen
from gpp_b200.capi import params_with_rules

INF = np.inf
ALL = ["infeasible_and_fixed_variables", "empty_columns", "empty_rows", "singleton_rows", "bound_strengthening",
       "infeasible_and_redundant_rows", "dual_fix", "parallel_rows", "parallel_columns", "singleton_columns",
       "doubleton_equations"]
VARIANTS = ("valid", "non_unit_coefficient", "non_covering_row", "missing_witness", "non_binary_bound")


def covering_lp(variant="valid"):
    """The reference test's 3 x 6 covering model (test_rule_column_domination.cpp:62-104)."""
    ptr = np.array([0, 4, 8, 11], np.int32)
    idx = np.array([0, 3, 4, 5, 1, 3, 4, 5, 2, 4, 5], np.int32)
    val = np.ones(11)
    c = np.array([1.0, 1.0, 1.0, 3.0, 3.0, 4.0])
    AL, AU, u = np.ones(3), np.full(3, INF), np.ones(6)
    if variant == "non_unit_coefficient":
        val[1] = 0.5
    elif variant == "non_covering_row":
        AU[0] = 1.0
    elif variant == "missing_witness":
        c[2] = 2.0
    elif variant == "non_binary_bound":
        u[5] = 2.0
    return lpgen.HostLP(3, 6, ptr, idx, val, c, AL, AU, np.zeros(6), u).ensure_transpose()


def rule_params(**extra):
    """Only the Startup phase, one iteration (test_rule_column_domination.cpp:106-132)."""
    kw = dict(max_iters=1, enable_folding=0, column_domination_min_fixed_cols=1,
              column_domination_min_candidate_ratio=0.20)
    kw.update(extra)
    return params_with_rules([], **kw)


def dims(r):
    return r.summary.reduced_rows, r.summary.reduced_cols, r.summary.reduced_nnz


def test_known_answer_reduction_and_primal_recovery():
    r = pyoracle.presolve(covering_lp(), rule_params())
    assert dims(r) == (3, 4, 6)
    assert sorted(r.fixed_idx.tolist()) == [3, 5] and np.all(r.fixed_val == 0.0)
    assert r.col_map.tolist() == [0, 1, 2, 4]
    x, _, _ = r.postsolve(np.array([1.0, 1.0, 1.0, 0.0]), np.zeros(3), np.zeros(4))
    assert x.tolist() == [1.0, 1.0, 1.0, 0.0, 0.0, 0.0]


def test_rule_is_owned_by_startup():
    assert dims(pyoracle.presolve(covering_lp(), rule_params(enable_startup=0))) == (3, 6, 11)


@pytest.mark.parametrize("variant", VARIANTS[1:])
def test_fail_closed(variant):
    assert dims(pyoracle.presolve(covering_lp(variant), rule_params())) == (3, 6, 11)


def test_master_switch_turns_it_off():
    assert dims(pyoracle.presolve(covering_lp(), rule_params(enable_structure_specific_rules=0))) == (3, 6, 11)
    assert dims(pyoracle.presolve(covering_lp(), rule_params(enable_column_domination=0))) == (3, 6, 11)


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_generated_cover_removes_exactly_the_dominated_columns(seed):
    lp = lpgen.setcover_lp(3000, 20000, seed=seed)
    degree = np.bincount(lp.col_idx, minlength=lp.n)
    dominated = lp.c > degree
    assert dominated.sum() >= 4096 and dominated.mean() >= 0.2
    r = pyoracle.presolve(lp, rule_params(column_domination_min_fixed_cols=4096))
    assert r.col_map.tolist() == np.flatnonzero(~dominated).tolist()
    assert r.summary.reduced_rows == lp.m and r.summary.reduced_nnz == int(degree[~dominated].sum())
    assert sorted(r.fixed_idx.tolist()) == np.flatnonzero(dominated).tolist()


def test_thresholds_and_witness():
    lp = lpgen.setcover_lp(3000, 20000, seed=4)
    count = int((lp.c > np.bincount(lp.col_idx, minlength=lp.n)).sum())
    share = count / lp.n
    assert dims(pyoracle.presolve(lp, rule_params(column_domination_min_fixed_cols=count)))[1] == lp.n - count
    assert dims(pyoracle.presolve(lp, rule_params(column_domination_min_fixed_cols=count + 1)))[1] == lp.n
    assert dims(pyoracle.presolve(lp, rule_params(column_domination_min_candidate_ratio=share)))[1] == lp.n - count
    assert dims(pyoracle.presolve(lp, rule_params(column_domination_min_candidate_ratio=share + 1e-6)))[1] == lp.n
    nowit = lpgen.setcover_lp(3000, 20000, seed=4, witness=False)
    assert dims(pyoracle.presolve(nowit, rule_params()))[1] == lp.n


@pytest.mark.parametrize("seed", [5, 6])
def test_full_pipeline_keeps_the_optimal_objective(seed):
    lp = lpgen.setcover_lp(1500, 8000, seed=seed)
    r = pyoracle.presolve(lp, params_with_rules(ALL, enable_folding=0, column_domination_min_fixed_cols=1000))
    assert r.summary.reduced_cols < lp.n - 1000
    full, _, _ = lpsolve.solve(lp.m, lp.n, lp.row_ptr, lp.col_idx, lp.values, lp.c, lp.AL, lp.AU, lp.l, lp.u)
    red, y, z = lpsolve.solve(r.summary.reduced_rows, r.summary.reduced_cols, r.A_ptr, r.A_idx, r.A_val, r.c, r.AL,
                              r.AU, r.l, r.u)
    assert full.status == 0 and red.status == 0
    assert abs(red.fun + r.obj_constant - full.fun) <= 1e-9 * max(1.0, abs(full.fun))
    x, _, _ = r.postsolve(red.x, y, z)
    assert lpsolve.primal_violation(lp, x) <= 1e-9
    assert abs(lp.c @ x - full.fun) <= 1e-9 * max(1.0, abs(full.fun))


def pair_block_lp(second_rhs=4.0, recourse_cost=0.0):
    """The reference test's 5 x 6 chained two-row / McCormick model
    (test_rule_projected_auxiliaries.cpp:103-127)."""
    ptr = np.array([0, 3, 5, 7, 11, 15], np.int32)
    idx = np.array([0, 1, 4, 0, 4, 1, 4, 2, 3, 4, 5, 2, 3, 4, 5], np.int32)
    val = np.array([-1, -1, 1, -1, 1, -1, 1, 1, -1, 2, -2, -1, 1, 2, 2], float)
    return lpgen.HostLP(5, 6, ptr, idx, val, np.array([-1.0, -2.0, 0.0, 0.0, 0.0, recourse_cost]),
                        np.array([-1.0, -INF, -INF, -INF, -INF]), np.array([INF, 0.0, 0.0, 2.0, second_rhs]),
                        np.zeros(6), np.ones(6)).ensure_transpose()


def mccormick_lp(corrupt_upper_row=False, nonunit_endpoint=False):
    """test_rule_projected_auxiliaries.cpp:128-146."""
    ptr = np.array([0, 3, 5, 7], np.int32)
    idx = np.array([0, 1, 2, 0, 2, 1, 2], np.int32)
    val = np.array([-1.0, -1.0, 1.0, -0.5 if corrupt_upper_row else -1.0, 1.0, -1.0, 1.0])
    u = np.array([1.0, 2.0 if nonunit_endpoint else 1.0, 1.0])
    return lpgen.HostLP(3, 3, ptr, idx, val, np.zeros(3), np.array([-1.0, -INF, -INF]), np.array([INF, 0.0, 0.0]),
                        np.zeros(3), u).ensure_transpose()


def projected_params(**extra):
    """test_rule_projected_auxiliaries.cpp:148-172."""
    kw = dict(max_iters=1, enable_folding=0, enable_column_domination=0,
              enable_piecewise_linear_reformulation_variable_pair=0,
              enable_piecewise_linear_reformulation_absolute_value=0, two_row_variable_elimination_min_candidates=1,
              two_row_variable_elimination_min_candidate_ratio=0.0, zero_cost_product_variables_min_candidates=1,
              zero_cost_product_variables_min_candidate_ratio=0.0)
    kw.update(extra)
    return params_with_rules([], **kw)


PAIR_BLOCK_X = [1.0, 1.0, 0.4, 0.2, 1.0, 0.1]


def test_chained_projection_and_primal_recovery():
    r = pyoracle.presolve(pair_block_lp(), projected_params())
    assert dims(r) == (0, 4, 0)
    assert r.tape_types.tolist() == [14, 14]
    x, _, _ = r.postsolve(np.array([1.0, 1.0, 0.4, 0.2]), np.zeros(0), np.zeros(4))
    assert np.allclose(x, PAIR_BLOCK_X, rtol=0, atol=1e-12)


@pytest.mark.parametrize("rhs,cost", [(3.0, 0.0), (4.0, 0.25)])
def test_bounded_projection_fails_closed(rhs, cost):
    r = pyoracle.presolve(pair_block_lp(rhs, cost), projected_params(enable_zero_cost_product_variables=0))
    assert dims(r) == (5, 6, 15) and len(r.tape_types) == 0


@pytest.mark.parametrize("corrupt,nonunit,removed", [(False, False, True), (True, False, False), (False, True, False)])
def test_mccormick_detector_is_exact_and_fail_closed(corrupt, nonunit, removed):
    r = pyoracle.presolve(mccormick_lp(corrupt, nonunit), projected_params(enable_two_row_variable_elimination=0))
    assert dims(r) == ((0, 2, 0) if removed else (3, 3, 7))


def test_projected_rules_are_startup_only():
    r = pyoracle.presolve(pair_block_lp(), projected_params(enable_startup=0))
    assert dims(r) == (5, 6, 15) and len(r.tape_types) == 0


def test_batch_sees_the_live_columns():
    # test_rule_projected_auxiliaries.cpp:304-345: after the two-row step 5
    # columns are live, so 1/5 passes a 0.19 share where 1/6 would not.
    batch = pyoracle.presolve(pair_block_lp(), projected_params(zero_cost_product_variables_min_candidate_ratio=0.19))
    assert dims(batch) == (0, 4, 0)
    first = pyoracle.presolve(pair_block_lp(), projected_params(enable_zero_cost_product_variables=0))
    assert dims(first)[:2] == (3, 5)


@pytest.mark.parametrize("seed", [1, 2])
def test_generated_auxiliary_blocks(seed):
    lp = lpgen.auxiliary_lp(4000, 10000, seed=seed)
    r = pyoracle.presolve(lp, params_with_rules([], enable_folding=0, max_iters=1))
    recs = int((r.tape_types == 14).sum())
    pairs, products = int(0.02 * 10000), int(0.02 * 10000)
    # Every block but the decoys: one in 16 of each kind conflicts or has no
    # margin / a wrong coefficient, and the chained products drop their outer z.
    decoy_pairs = sum(1 for k in range(pairs) if k % 16 in (5, 11))
    decoy_products = sum(1 for k in range(products) if k % 16 == 3)
    assert recs == (pairs - decoy_pairs) + (products - decoy_products)
    assert r.summary.reduced_cols == lp.n - recs
    off = pyoracle.presolve(lp, params_with_rules([], enable_folding=0, max_iters=1, enable_structure_specific_rules=0))
    assert dims(off) == (lp.m, lp.n, lp.nnz)


@pytest.mark.parametrize("seed", [3, 4])
def test_auxiliary_pipeline_keeps_the_optimal_objective(seed):
    lp = lpgen.auxiliary_lp(1200, 3000, seed=seed, pairs=0.05, products=0.05)
    params = params_with_rules(ALL, enable_folding=0, two_row_variable_elimination_min_candidates=1,
                               zero_cost_product_variables_min_candidates=1)
    r = pyoracle.presolve(lp, params)
    assert (r.tape_types == 14).sum() > 100
    full, _, _ = lpsolve.solve(lp.m, lp.n, lp.row_ptr, lp.col_idx, lp.values, lp.c, lp.AL, lp.AU, lp.l, lp.u)
    red, y, z = lpsolve.solve(r.summary.reduced_rows, r.summary.reduced_cols, r.A_ptr, r.A_idx, r.A_val, r.c, r.AL,
                              r.AU, r.l, r.u)
    assert full.status == 0 and red.status == 0
    assert abs(red.fun + r.obj_constant - full.fun) <= 1e-8 * max(1.0, abs(full.fun))
    x, _, _ = r.postsolve(red.x, y, z)
    assert lpsolve.primal_violation(lp, x) <= 1e-8
    assert abs(lp.c @ x - full.fun) <= 1e-8 * max(1.0, abs(full.fun))


# ---------------------------------------------------------------- GPU


def bits(a):
    return np.asarray(a).view(np.uint8)


@pytest.mark.gpu
@pytest.mark.parametrize("variant", VARIANTS)
def test_gpu_known_answer_and_variants(variant):
    import torch
    from gpp_b200 import device
    lp = covering_lp(variant)
    d = device.DeviceLp(lp)
    s = device.preprocess(d, rule_params())
    try:
        got = (s.reduced_rows, s.reduced_cols, s.reduced_nnz)
        if variant != "valid":
            assert got == (3, 6, 11)
            return
        assert got == (3, 4, 6)
        r = device.Result(s)
        assert sorted(r.fixed_idx.tolist()) == [3, 5]
        x, _, _ = device.postprocess(torch.tensor([1.0, 1.0, 1.0, 0.0], dtype=torch.float64, device="cuda"),
                                     torch.zeros(3, dtype=torch.float64, device="cuda"),
                                     torch.zeros(4, dtype=torch.float64, device="cuda"), s, d)
        assert np.asarray(x).tolist() == [1.0, 1.0, 1.0, 0.0, 0.0, 0.0]
    finally:
        device.free_summary(s)


@pytest.mark.gpu
@pytest.mark.parametrize("m,n,seed", [(3000, 20000, 1), (40000, 200000, 2)])
@pytest.mark.parametrize("rules", [[], ALL])
def test_gpu_matches_oracle_on_set_covering(m, n, seed, rules):
    from gpp_b200 import device
    lp = lpgen.setcover_lp(m, n, seed=seed)
    params = params_with_rules(rules, enable_folding=0)
    orc = pyoracle.presolve(lp, params)
    d = device.DeviceLp(lp)
    s = device.preprocess(d, params)
    try:
        r = device.Result(s)
        assert (s.reduced_rows, s.reduced_cols, s.reduced_nnz, s.iterations) == (
            orc.summary.reduced_rows, orc.summary.reduced_cols, orc.summary.reduced_nnz, orc.summary.iterations)
        assert s.reduced_cols < lp.n - 4096
        for k in ("A_ptr", "A_idx", "A_val", "c", "l", "u", "AL", "AU", "row_map", "col_map", "tape_types",
                  "tape_idx", "tape_val", "fixed_idx", "fixed_val"):
            assert np.array_equal(bits(getattr(r, k)), bits(getattr(orc, k))), k
    finally:
        device.free_summary(s)


@pytest.mark.gpu
@pytest.mark.parametrize("workload", ["setcover:3000x20000", "setcover:40000x200000"])
@pytest.mark.parametrize("others", [0, 1])
def test_gpu_matches_reference_with_structure_rules_on(workload, others):
    """The reference with its structure-specific rules on: column domination
    fires; with ``others`` its remaining structure-specific detectors run too
    and reject these models."""
    import test_reference_parity as trp
    if not trp.DRIVER or not __import__("os").path.exists(trp.DRIVER):
        pytest.skip("reference build (oracle/_ref) not present")
    extra = {"enable_structure_specific_rules": 1, "enable_column_domination": 1}
    if not others:
        extra.update(enable_two_row_variable_elimination=0, enable_zero_cost_product_variables=0,
                     enable_piecewise_linear_reformulation_variable_pair=0,
                     enable_piecewise_linear_reformulation_absolute_value=0)
    lp = lpgen.workload(workload, seed=0)
    got = trp.check_against_reference(lp, trp.ALL, extra)
    assert got.summary.reduced_cols < lp.n - 4096


@pytest.mark.gpu
def test_gpu_chained_projection_and_primal_recovery():
    import torch
    from gpp_b200 import device
    lp = pair_block_lp()
    d = device.DeviceLp(lp)
    s = device.preprocess(d, projected_params())
    try:
        assert (s.reduced_rows, s.reduced_cols, s.reduced_nnz) == (0, 4, 0)
        orc = pyoracle.presolve(lp, projected_params())
        r = device.Result(s)
        for k in ("tape_types", "tape_idx", "tape_val", "col_map"):
            assert np.array_equal(bits(getattr(r, k)), bits(getattr(orc, k))), k
        x, _, _ = device.postprocess(torch.tensor([1.0, 1.0, 0.4, 0.2], dtype=torch.float64, device="cuda"),
                                     torch.zeros(0, dtype=torch.float64, device="cuda"),
                                     torch.zeros(4, dtype=torch.float64, device="cuda"), s, d)
        assert np.allclose(np.asarray(x), PAIR_BLOCK_X, rtol=0, atol=1e-12)
    finally:
        device.free_summary(s)


@pytest.mark.gpu
@pytest.mark.parametrize("corrupt,nonunit", [(False, False), (True, False), (False, True)])
def test_gpu_mccormick_variants(corrupt, nonunit):
    from gpp_b200 import device
    lp = mccormick_lp(corrupt, nonunit)
    params = projected_params(enable_two_row_variable_elimination=0)
    s = device.preprocess(device.DeviceLp(lp), params)
    try:
        assert (s.reduced_rows, s.reduced_cols, s.reduced_nnz) == dims(pyoracle.presolve(lp, params))
    finally:
        device.free_summary(s)


@pytest.mark.gpu
@pytest.mark.parametrize("m,n,seed", [(4000, 10000, 1), (200000, 500000, 2)])
@pytest.mark.parametrize("rules", [[], ALL])
def test_gpu_matches_oracle_on_auxiliary_blocks(m, n, seed, rules):
    from gpp_b200 import device
    lp = lpgen.auxiliary_lp(m, n, seed=seed)
    params = params_with_rules(rules, enable_folding=0)
    orc = pyoracle.presolve(lp, params)
    d = device.DeviceLp(lp)
    s = device.preprocess(d, params)
    try:
        r = device.Result(s)
        assert (s.reduced_rows, s.reduced_cols, s.reduced_nnz, s.iterations) == (
            orc.summary.reduced_rows, orc.summary.reduced_cols, orc.summary.reduced_nnz, orc.summary.iterations)
        assert (r.tape_types == 14).sum() > 0.02 * n
        for k in ("A_ptr", "A_idx", "A_val", "c", "l", "u", "AL", "AU", "row_map", "col_map", "tape_types",
                  "tape_idx", "tape_val", "fixed_idx", "fixed_val"):
            assert np.array_equal(bits(getattr(r, k)), bits(getattr(orc, k))), k
    finally:
        device.free_summary(s)


@pytest.mark.gpu
@pytest.mark.parametrize("workload", ["auxiliary:4000x10000", "auxiliary:200000x500000"])
def test_gpu_auxiliary_matches_reference(workload):
    import test_reference_parity as trp
    if not __import__("os").path.exists(trp.DRIVER):
        pytest.skip("reference build (oracle/_ref) not present")
    lp = lpgen.workload(workload, seed=0)
    got = trp.check_against_reference(lp, trp.ALL, {"enable_structure_specific_rules": 1})
    assert (got.tape_types == 14).sum() > 0
