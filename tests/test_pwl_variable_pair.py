"""Variable-pair piecewise-linear reformulation (a Startup rule): epigraph and
shifted antipodal.

Generated models of both layouts (lpgen.epigraph_pair_lp, antipodal_pair_lp)
run on the engine and on the reference library (oracle/_ref/ref_driver, the
reference compiled from its own sources) on the same GPU with the same
settings: Startup alone (max_iters = 1, so the reduced model is the rule's
rewrite) and the whole default pipeline with a postsolved point.  Everything
the reference exports must agree: reduced model, maps, tape, the
primal-recovery checkpoints and the variable-pair payload.  Decoys must be
rejected by both.  HiGHS confirms that the postsolved optimum of the reduced
model is the original optimum.
"""
import numpy as np
import pytest

from gpp_b200 import capi, device, lpgen

import lpsolve
import test_reference_parity as trp

pytestmark = pytest.mark.gpu

SMALL = {"enable_structure_specific_rules": 1,
         "piecewise_linear_reformulation_variable_pair_epigraph_min_pairs": 16,
         "piecewise_linear_reformulation_variable_pair_shifted_antipodal_min_pairs": 16}


def check_variable_pair(got):
    ref = got.ref
    kinds = np.fromfile(f"{ref['dir']}/ckpt_kind", dtype=np.int32)
    pay = np.fromfile(f"{ref['dir']}/ckpt_payload", dtype=np.int32)
    pos = np.fromfile(f"{ref['dir']}/ckpt_position", dtype=np.int64)
    assert got.checkpoints == list(zip(kinds.tolist(), pay.tolist(), pos.tolist()))
    assert len(got.variable_pair) == int(ref["meta"]["variable_pair_steps"])
    for k, a in enumerate(got.variable_pair):
        for key, dt in (("plus", np.int32), ("minus", np.int32), ("root_plus", np.int32), ("root_minus", np.int32),
                        ("plus_shift", np.float64), ("minus_shift", np.float64)):
            want = np.fromfile(f"{ref['dir']}/vp{k}_{key}", dtype=dt)
            assert np.array_equal(a[key], want), key


def run(lp, extra, postsolve=False):
    """Startup-only settings (max_iters 1) also turn every other rule off."""
    rules = [] if extra.get("max_iters") == 1 else trp.ALL
    got = trp.check_against_reference(lp, rules, extra, oracle=False, postsolve=postsolve)
    check_variable_pair(got)
    return got


@trp.needs_reference
@pytest.mark.parametrize("components,size,tails", [(40, 4, 1), (60, 3, 3), (25, 8, 8), (100, 2, 2)])
@pytest.mark.parametrize("seed", [0, 1])
def test_epigraph_startup_matches_reference(components, size, tails, seed):
    lp = lpgen.epigraph_pair_lp(components, size, tails=tails, seed=seed)
    got = run(lp, {**SMALL, "max_iters": 1})
    (vp,) = got.variable_pair
    assert np.all(vp["plus_shift"] == 0.0)
    assert got.summary.reduced_cols < lp.n


@trp.needs_reference
@pytest.mark.parametrize("uniform", [True, False])
@pytest.mark.parametrize("components,size", [(40, 4), (80, 3), (20, 10)])
@pytest.mark.parametrize("seed", [0, 1])
def test_antipodal_startup_matches_reference(components, size, uniform, seed):
    lp = lpgen.antipodal_pair_lp(components, size, seed=seed, uniform_cost=uniform)
    got = run(lp, {**SMALL, "max_iters": 1})
    (vp,) = got.variable_pair
    assert got.summary.reduced_cols == 2 * components
    assert np.any(vp["plus_shift"] != 0.0)


@trp.needs_reference
@pytest.mark.parametrize("maker", [lambda s: lpgen.epigraph_pair_lp(50, 4, seed=s),
                                   lambda s: lpgen.antipodal_pair_lp(50, 4, seed=s)])
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_default_pipeline_and_postsolve_match_reference(maker, seed):
    got = run(maker(seed), SMALL, postsolve=True)
    assert len(got.checkpoints) == 1


@trp.needs_reference
@pytest.mark.parametrize("maker", [lambda: lpgen.epigraph_pair_lp(50, 4, decoy="epigraph_side"),
                                   lambda: lpgen.epigraph_pair_lp(50, 4, decoy="stray"),
                                   lambda: lpgen.antipodal_pair_lp(50, 4, decoy="shift"),
                                   lambda: lpgen.antipodal_pair_lp(50, 4, decoy="cost")])
def test_decoys_rejected_like_the_reference(maker):
    lp = maker()
    got = run(lp, {**SMALL, "max_iters": 1})
    assert got.checkpoints == []
    assert (got.summary.reduced_rows, got.summary.reduced_cols) == (lp.m, lp.n)


@trp.needs_reference
def test_thresholds_at_reference_defaults():
    """With the reference's default minimum (4,096 merge edges) a model of
    6,000 pairs in components of four applies and one of 2,000 does not."""
    big = lpgen.antipodal_pair_lp(1500, 4, seed=5)
    got = run(big, {"enable_structure_specific_rules": 1, "max_iters": 1})
    assert len(got.checkpoints) == 1
    small = lpgen.antipodal_pair_lp(500, 4, seed=5)
    got = run(small, {"enable_structure_specific_rules": 1, "max_iters": 1})
    assert got.checkpoints == []


@pytest.mark.parametrize("maker", [lambda: lpgen.epigraph_pair_lp(30, 4, seed=7),
                                   lambda: lpgen.antipodal_pair_lp(30, 4, seed=7),
                                   lambda: lpgen.antipodal_pair_lp(30, 4, seed=8, uniform_cost=False)])
def test_postsolved_optimum_is_the_original_one(maker):
    import torch
    lp = maker()
    params = capi.params_with_rules(trp.ALL, enable_folding=0, **SMALL)
    dlp = device.DeviceLp(lp)
    s = device.preprocess(dlp, params)
    try:
        got = device.Result(s)
        assert len(got.checkpoints) == 1 and got.checkpoints[0][0] == 1
        res0, _, _ = lpsolve.solve(lp.m, lp.n, lp.row_ptr, lp.col_idx, lp.values, lp.c, lp.AL, lp.AU, lp.l, lp.u)
        rr, yr, zr = lpsolve.solve(s.reduced_rows, s.reduced_cols, got.A_ptr, got.A_idx, got.A_val, got.c, got.AL,
                                   got.AU, got.l, got.u)
        assert res0.status == 0 and rr.status == 0
        x, _, _ = device.postprocess(torch.from_numpy(rr.x).cuda(), torch.from_numpy(yr).cuda(),
                                     torch.from_numpy(zr).cuda(), s, dlp)
        x = np.asarray(x)
        assert abs(lp.c @ x - res0.fun) <= 1e-7 * max(1.0, abs(res0.fun))
        assert lpsolve.primal_violation(lp, x) <= 1e-7
    finally:
        device.free_summary(s)
