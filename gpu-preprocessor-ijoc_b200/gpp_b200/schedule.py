"""Learned round schedule: traces of the plain phase machine, labels, the
schedule MLP (trained and run by the library's CUDA kernels) and presolve
scheduled by it.

A round is one step of the phase machine.  Per round the model sees 32
features (see include/gpp.h) and outputs, for each of six gated rules, the
probability that the rule will change the model this round, and the
probability that presolve should stop.  Labels come from traces of the plain
loop: a rule that ran is labelled by whether it changed the model; a round is
a stop point when less than ``STOP_SHARE`` of the run's total nnz removal is
still to come after it (half of the 2% that the 98% bar allows).  The plain
loop stays the default and the yardstick: a scheduled run must keep at least
98% of the plain run's nnz removal.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import capi
from .device import _raise

FEATURES, HIDDEN, OUTPUTS = 32, 64, 7
GATED_RULES = ("singleton_columns", "bound_strengthening", "redundant_rows_dual_fix", "doubleton_equations",
               "parallel_rows", "parallel_columns")
PARAMS = FEATURES * HIDDEN + HIDDEN + HIDDEN * HIDDEN + HIDDEN + HIDDEN * OUTPUTS + OUTPUTS
STOP_SHARE = 0.01
MODEL_FILE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "schedule_model.npz")
MAX_ROUNDS = 4096


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def traced_preprocess(dlp, params):
    """gpp_preprocess_traced: (summary, trace) with trace = dict of per-round arrays."""
    lib = capi.load()
    feats = np.zeros((MAX_ROUNDS, FEATURES), np.float32)
    info = np.zeros((MAX_ROUNDS, 4), np.int32)
    nnz = np.zeros((MAX_ROUNDS, 2), np.int64)
    rounds = C.c_int32(0)
    s = capi.Summary()
    lp = dlp.struct()
    _raise(lib.gpp_preprocess_traced(C.byref(lp), C.byref(params), C.byref(s), _p(feats), _p(info), _p(nnz),
                                     MAX_ROUNDS, C.byref(rounds)))
    r = min(rounds.value, MAX_ROUNDS)
    return s, {"features": feats[:r].copy(), "phase": info[:r, 0].copy(), "iteration": info[:r, 1].copy(),
               "ran": info[:r, 2].copy(), "changed": info[:r, 3].copy(), "nnz_before": nnz[:r, 0].copy(),
               "nnz_after": nnz[:r, 1].copy()}


def labels(trace):
    """(Y, M) per round: rule outputs labelled where the rule ran; the stop output everywhere."""
    r = len(trace["phase"])
    Y = np.zeros((r, OUTPUTS), np.float32)
    M = np.zeros((r, OUTPUTS), np.float32)
    for g in range(len(GATED_RULES)):
        ran = (trace["ran"] >> g) & 1
        M[:, g] = ran
        Y[:, g] = ran & ((trace["changed"] >> g) & 1)
    if r:
        final = trace["nnz_after"][-1]
        total = trace["nnz_before"][0] - final
        to_come = trace["nnz_before"] - final
        Y[:, OUTPUTS - 1] = (to_come <= STOP_SHARE * total) if total > 0 else 1.0
        M[:, OUTPUTS - 1] = 1.0
    return Y, M


def init_params(seed=0):
    """He-initialised weights, zero biases, in the library's flat layout."""
    rng = np.random.default_rng(seed)
    parts = []
    for fan_in, fan_out in ((FEATURES, HIDDEN), (HIDDEN, HIDDEN), (HIDDEN, OUTPUTS)):
        parts.append((rng.standard_normal((fan_in, fan_out)) * np.sqrt(2.0 / fan_in)).ravel())
        parts.append(np.zeros(fan_out))
    w = np.concatenate(parts).astype(np.float32)
    assert w.size == PARAMS
    return w


def train(X, Y, M, params=None, epochs=200, batch=256, lr=3e-3, seed=0):
    """gpp_mlp_train: (trained params, loss per epoch)."""
    w = (init_params(seed) if params is None else np.array(params, np.float32)).copy()
    X, Y, M = (np.ascontiguousarray(a, np.float32) for a in (X, Y, M))
    loss = np.zeros(epochs, np.float32)
    _raise(capi.load().gpp_mlp_train(_p(w), _p(X), _p(Y), _p(M), len(X), epochs, batch, C.c_float(lr), seed,
                                     _p(loss)))
    return w, loss


def forward(params, X):
    """gpp_mlp_forward: sigmoid outputs, n x OUTPUTS."""
    X = np.ascontiguousarray(X, np.float32)
    w = np.ascontiguousarray(params, np.float32)
    out = np.zeros((len(X), OUTPUTS), np.float32)
    _raise(capi.load().gpp_mlp_forward(_p(w), _p(X), len(X), _p(out)))
    return out


def gradients(params, X, Y, M):
    """gpp_mlp_gradients: (gradient of the mean masked loss, the loss)."""
    X, Y, M = (np.ascontiguousarray(a, np.float32) for a in (X, Y, M))
    w = np.ascontiguousarray(params, np.float32)
    g = np.zeros(PARAMS, np.float32)
    loss = C.c_float(0.0)
    _raise(capi.load().gpp_mlp_gradients(_p(w), _p(X), _p(Y), _p(M), len(X), _p(g), C.byref(loss)))
    return g, float(loss.value)


def keep_all_params():
    """Weights whose outputs say "run every rule, never stop" (the plain loop)."""
    w = np.zeros(PARAMS, np.float32)
    b3 = w[PARAMS - OUTPUTS:]
    b3[:len(GATED_RULES)] = 20.0
    b3[-1] = -20.0
    return w


def save_model(path, params, skip_below, stop_above, **info):
    """Parameters, the decision thresholds (skip: one value, or one per gated
    rule) and training notes in one .npz."""
    np.savez(path, params=np.asarray(params, np.float32), skip_below=np.asarray(skip_below, np.float64),
             stop_above=np.float64(stop_above), **{k: np.asarray(v) for k, v in info.items()})


def load_model(path=MODEL_FILE):
    """(parameters, skip_below, stop_above) of a saved schedule model;
    skip_below is a float or a list of one threshold per gated rule."""
    with np.load(path) as z:
        w = z["params"].astype(np.float32)
        sb = np.asarray(z["skip_below"], np.float64)
        skip_below = float(sb) if sb.ndim == 0 else [float(v) for v in sb]
        stop_above = float(z["stop_above"])
    if w.size != PARAMS:
        raise ValueError(f"{path}: {w.size} parameters, expected {PARAMS}")
    return w, skip_below, stop_above


class Model:
    """gpp_schedule_model_create(_per_rule) / gpp_schedule_model_free.
    skip_below: one threshold for every gated rule, or one per rule."""

    def __init__(self, params, skip_below=0.5, stop_above=0.5):
        self.w = np.ascontiguousarray(params, np.float32)
        self.h = C.c_void_p()
        sb = np.ascontiguousarray(np.broadcast_to(np.asarray(skip_below, np.float64), (len(GATED_RULES),)))
        self.skip_below = sb
        _raise(capi.load().gpp_schedule_model_create_per_rule(_p(self.w), _p(sb), float(stop_above),
                                                              C.byref(self.h)))

    def close(self):
        if self.h:
            capi.load().gpp_schedule_model_free(self.h)
            self.h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def scheduled_preprocess(dlp, params, model: Model):
    """gpp_preprocess_scheduled."""
    s = capi.Summary()
    lp = dlp.struct()
    _raise(capi.load().gpp_preprocess_scheduled(C.byref(lp), C.byref(params), model.h, C.byref(s)))
    return s
