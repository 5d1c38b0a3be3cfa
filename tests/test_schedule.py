"""Learned round schedule: the MLP kernels against a float64 numpy
restatement (with a finite-difference check of that restatement on the CPU),
the round traces and labels, and presolve scheduled by a model: a model that
keeps every rule must reproduce the plain run bit for bit, and the shipped
model must keep at least 98% of the plain nnz removal with the same
postsolved objective."""
import os
import re

import numpy as np
import pytest

import lpsolve
import mlp_reference as ref
from gpp_b200 import capi, device, lpgen, schedule

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def random_batch(n, seed):
    rng = np.random.default_rng(seed)
    X = rng.uniform(0.0, 1.0, size=(n, schedule.FEATURES)).astype(np.float32)
    Y = (rng.random((n, schedule.OUTPUTS)) < 0.4).astype(np.float32)
    M = (rng.random((n, schedule.OUTPUTS)) < 0.8).astype(np.float32)
    return X, Y, M


def test_parameter_count_matches_header():
    text = open(os.path.join(ROOT, "include", "gpp.h")).read()
    expr = re.search(r"#define GPP_SCHEDULE_PARAMS \(([^)]*)\)", text).group(1)
    assert eval(expr) == schedule.PARAMS == schedule.init_params().size


def test_reference_gradient_matches_finite_differences():
    X, Y, M = random_batch(20, 1)
    w = schedule.init_params(3).astype(np.float64)
    g = ref.gradients(w, X, Y, M)
    rng = np.random.default_rng(5)
    for i in rng.choice(w.size, size=60, replace=False):
        e = np.zeros_like(w)
        e[i] = 1e-6
        num = (ref.loss(w + e, X, Y, M) - ref.loss(w - e, X, Y, M)) / 2e-6
        assert abs(num - g[i]) <= 1e-6 + 1e-5 * abs(num), i


def test_labels_from_a_trace():
    tr = {"phase": np.array([0, 1, 0, 2]), "ran": np.array([1, 0b110, 1, 0b1000]),
          "changed": np.array([1, 0b010, 0, 0]), "nnz_before": np.array([1000, 700, 500, 495]),
          "nnz_after": np.array([700, 500, 495, 495]), "features": np.zeros((4, 32), np.float32)}
    Y, M = schedule.labels(tr)
    assert M[:, 0].tolist() == [1, 0, 1, 0] and Y[:, 0].tolist() == [1, 0, 0, 0]
    assert M[:, 1].tolist() == [0, 1, 0, 0] and Y[:, 1].tolist() == [0, 1, 0, 0]
    assert M[:, 2].tolist() == [0, 1, 0, 0] and Y[:, 2].tolist() == [0, 0, 0, 0]
    assert M[:, 3].tolist() == [0, 0, 0, 1] and Y[:, 3].tolist() == [0, 0, 0, 0]
    # Total removal 505; stop once at most 1% (5.05) is still to come.
    assert Y[:, 6].tolist() == [0, 0, 1, 1] and M[:, 6].tolist() == [1, 1, 1, 1]


@pytest.mark.gpu
def test_gpu_gradients_and_forward_match_reference():
    X, Y, M = random_batch(300, 2)
    w = schedule.init_params(7)
    g, loss = schedule.gradients(w, X, Y, M)
    want = ref.gradients(w.astype(np.float64), X, Y, M)
    assert np.allclose(g, want, rtol=1e-3, atol=1e-6)
    assert abs(loss - ref.loss(w.astype(np.float64), X, Y, M)) <= 1e-5 * max(1.0, abs(loss))
    p = schedule.forward(w, X)
    z = ref.forward(w.astype(np.float64), X)[2]
    assert np.allclose(p, 1.0 / (1.0 + np.exp(-z)), rtol=1e-5, atol=1e-6)


@pytest.mark.gpu
def test_training_learns_a_rule_of_the_features():
    rng = np.random.default_rng(4)
    X = rng.uniform(0.0, 1.0, size=(2000, schedule.FEATURES)).astype(np.float32)
    Y = np.zeros((2000, schedule.OUTPUTS), np.float32)
    Y[:, 0] = X[:, 5] > 0.5                      # output 0 follows feature 5
    Y[:, 6] = X[:, 22] > 0.7                     # the stop output follows feature 22
    M = np.ones_like(Y)
    w, loss = schedule.train(X, Y, M, epochs=60, batch=128, lr=3e-3, seed=1)
    assert loss[-1] < 0.5 * loss[0]
    p = schedule.forward(w, X)
    assert ((p[:, 0] > 0.5) == (Y[:, 0] > 0.5)).mean() > 0.95
    assert ((p[:, 6] > 0.5) == (Y[:, 6] > 0.5)).mean() > 0.95


def bits(a):
    return np.asarray(a).view(np.uint8)


def same_result(a, b):
    assert (a.summary.reduced_rows, a.summary.reduced_cols, a.summary.reduced_nnz, a.summary.iterations) == (
        b.summary.reduced_rows, b.summary.reduced_cols, b.summary.reduced_nnz, b.summary.iterations)
    for k in ("A_ptr", "A_idx", "A_val", "c", "l", "u", "AL", "AU", "row_map", "col_map", "tape_types", "tape_val",
              "fixed_idx", "fixed_val"):
        assert np.array_equal(bits(getattr(a, k)), bits(getattr(b, k))), k


@pytest.mark.gpu
@pytest.mark.parametrize("m,seed", [(2000, 1), (20000, 2)])
def test_trace_and_keep_all_schedule_reproduce_plain(m, seed):
    lp = lpgen.random_lp(m, int(2.5 * m), seed=seed)
    d = device.DeviceLp(lp)
    params = capi.Params.defaults()
    plain = device.preprocess(d, params)
    traced, tr = schedule.traced_preprocess(d, params)
    with schedule.Model(schedule.keep_all_params(), 0.5) as model:
        kept = schedule.scheduled_preprocess(d, params, model)
    try:
        rp = device.Result(plain)
        same_result(rp, device.Result(traced))
        same_result(rp, device.Result(kept))
        r = len(tr["phase"])
        assert r >= 3 and tr["nnz_before"][0] == lp.nnz and tr["nnz_after"][-1] == plain.reduced_nnz
        assert np.all(tr["nnz_after"] <= tr["nnz_before"]) and np.all(tr["features"][:, :4].sum(1) == 1.0)
    finally:
        for s in (plain, traced, kept):
            device.free_summary(s)


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(schedule.MODEL_FILE), reason="no trained schedule model shipped")
@pytest.mark.parametrize("seed", [9001, 9002, 9003])
def test_shipped_schedule_keeps_98_percent_and_the_objective(seed):
    import torch
    w, skip_below, stop_above = schedule.load_model()
    lp = lpgen.random_lp(1500, 3750, seed=seed)
    d = device.DeviceLp(lp)
    params = capi.Params.defaults()
    plain = device.preprocess(d, params)
    with schedule.Model(w, skip_below, stop_above) as model:
        s = schedule.scheduled_preprocess(d, params, model)
    try:
        removed_plain = lp.nnz - plain.reduced_nnz
        assert lp.nnz - s.reduced_nnz >= 0.98 * removed_plain
        res0, _, _ = lpsolve.solve(lp.m, lp.n, lp.row_ptr, lp.col_idx, lp.values, lp.c, lp.AL, lp.AU, lp.l, lp.u)
        r = device.Result(s)
        rr, yr, zr = lpsolve.solve(s.reduced_rows, s.reduced_cols, r.A_ptr, r.A_idx, r.A_val, r.c, r.AL, r.AU, r.l,
                                   r.u)
        x, _, _ = device.postprocess(torch.from_numpy(rr.x).cuda(), torch.from_numpy(yr).cuda(),
                                     torch.from_numpy(zr).cuda(), s, d)
        assert abs(lp.c @ x + lp.obj_constant - (res0.fun + lp.obj_constant)) <= 1e-9 * max(1.0, abs(res0.fun))
    finally:
        device.free_summary(plain)
        device.free_summary(s)


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(schedule.MODEL_FILE), reason="no trained schedule model shipped")
@pytest.mark.parametrize("m,seed", [(200000, 9101), (400000, 9102)])
def test_shipped_schedule_gains_over_plain(m, seed):
    """What the trained network gains over the plain loop on LPs it was not
    trained on: fewer rounds and less presolve time (means of three warm runs
    each), while keeping at least 98% of the plain run's nnz removal."""
    w, skip_below, stop_above = schedule.load_model()
    lp = lpgen.random_lp(m, int(2.5 * m), seed=seed)
    d = device.DeviceLp(lp)
    params = capi.Params.defaults()

    def timed(fn):
        out = []
        for it in range(4):
            s = fn()
            out.append((s.elapsed_seconds, s.iterations, s.reduced_nnz))
            device.free_summary(s)
        return np.mean([t for t, _, _ in out[1:]]), out[-1][1], out[-1][2]

    t_plain, it_plain, nnz_plain = timed(lambda: device.preprocess(d, params))
    with schedule.Model(w, skip_below, stop_above) as model:
        t_sched, it_sched, nnz_sched = timed(lambda: schedule.scheduled_preprocess(d, params, model))
    assert lp.nnz - nnz_sched >= 0.98 * (lp.nnz - nnz_plain)
    assert it_sched < it_plain
    assert t_sched < t_plain


def test_threshold_search_keeps_the_removal_bar():
    """The held-out threshold search on a synthetic cost model: skipping rule
    2 is free of loss and saves time, skipping rule 0 loses removal; stopping
    early saves time but loses removal below 0.8."""
    from gpp_b200.train_schedule import KEEP_SHARE, choose_thresholds

    def evaluate(skip, stop):
        ratio = 1.0 - 0.3 * (skip[2] > 0) - 0.2 * (skip[0] > 0) - 0.1 * (stop < 1.0)
        kept = 1.0 - (0.05 if skip[0] > 0 else 0.0) - (0.03 if stop < 0.8 else 0.0)
        return ratio, kept

    skip, stop, ratio, table = choose_thresholds(evaluate, 6)
    assert skip[0] == 0.0 and skip[2] > 0.0
    assert 0.8 <= stop < 1.0
    assert abs(ratio - 0.6) < 1e-12
    assert all(t["min_kept"] >= KEEP_SHARE or t["time_ratio"] >= ratio for t in table)
