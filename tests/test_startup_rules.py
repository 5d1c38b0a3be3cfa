"""Structure-specific Startup rule: column domination on unit set-covering LPs.

CPU: the oracle on the reference's own known-answer model and its fail-closed
variants (cpp/tests/test_rule_column_domination.cpp:62-206), on generated
set-covering LPs (exactly the columns whose cost exceeds their degree go, and
only past both thresholds), and the postsolved objective of the full pipeline
against HiGHS.  GPU: the engine bit-exact against the oracle, the known-answer
model through the C ABI with postsolve, and parity with the reference library
itself with its structure-specific rules on."""
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
        x, _, _ = device.postprocess(torch.tensor([1.0, 1.0, 1.0, 0.0], device="cuda"),
                                     torch.zeros(3, dtype=torch.float64, device="cuda"),
                                     torch.zeros(4, dtype=torch.float64, device="cuda"), s, d)
        assert x.cpu().tolist() == [1.0, 1.0, 1.0, 0.0, 0.0, 0.0]
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
