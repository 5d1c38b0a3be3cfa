"""Trains the learned round schedule.

    python -m gpp_b200.train_schedule --out schedule_model.npz [--lps 20000] [--seed 0]

1. Draws training LPs from the plain-presolve generator (lpgen.random_lp, the
   generator of the 2,000 x 5,000 case and of the batched workload) with m
   log-uniform in [1,000, 500,000] and n = 2.5 m, generated by spawned
   processes while the GPU traces the ones already made, and records a trace
   of the plain phase machine on each (one trace per LP, one sample per
   round).
2. Trains the schedule MLP on the rounds of all traces (the library's CUDA
   kernels; Adam, masked binary cross-entropy).
3. Chooses the decision thresholds on held-out LPs (skip a gated rule below
   its own probability threshold, stop above another), searching greedily
   for the least total presolve time that keeps at least 98% of the plain
   run's nnz removal on every held-out LP (the plain loop -- skip nothing,
   never stop -- if nothing does).
4. Writes parameters, thresholds and training notes to --out.
"""
from __future__ import annotations

import argparse
import itertools
import json
import multiprocessing as mp
import os
import sys
import time

import numpy as np

KEEP_SHARE = 0.98
SKIP_BELOW = (0.5, 0.3, 0.15, 0.05, 0.0)
STOP_ABOVE = (0.5, 0.8, 0.95, 0.99, 1.0)   # 1.0: never stop


def _draw(job):
    from gpp_b200 import lpgen
    m, seed = job
    lp = lpgen.random_lp(m, int(2.5 * m), seed=seed)
    lp.ensure_transpose()
    return lp


def jobs(count, seed, lo=1000, hi=500000):
    rng = np.random.default_rng(seed)
    ms = np.exp(rng.uniform(np.log(lo), np.log(hi), size=count)).astype(int)
    return [(int(m), int(seed * 100000 + k)) for k, m in enumerate(ms)]


def bounded_imap(pool, fn, items, window):
    """pool.imap with at most `window` results pending: generated LPs wait in
    host memory only until the GPU has traced the ones before them."""
    from collections import deque
    it = iter(items)
    pending = deque(pool.apply_async(fn, (x,)) for x in itertools.islice(it, window))
    while pending:
        r = pending.popleft().get()
        nxt = next(it, None)
        if nxt is not None:
            pending.append(pool.apply_async(fn, (nxt,)))
        yield r


def removal(lp, s):
    return lp.nnz - s.reduced_nnz


def choose_thresholds(evaluate, rules):
    """Decision thresholds on held-out LPs.  `evaluate(skip, stop)` gives
    (time ratio, smallest kept share) for one skip threshold per gated rule.
    First the stop threshold with no rule skipped; then, rule by rule, the
    skip threshold that lowers the time most while every held-out LP keeps at
    least KEEP_SHARE of its plain removal; then the stop threshold again for
    the chosen skips.  Returns (skip per rule, stop, table of every try)."""
    table = []

    def run(skip, stop):
        ratio, kept = evaluate(list(skip), stop)
        table.append({"skip_below": list(skip), "stop_above": stop, "time_ratio": ratio, "min_kept": kept})
        return ratio, kept

    skip = [0.0] * rules
    best_stop, best_ratio = 1.0, run(skip, 1.0)[0]
    for stop in STOP_ABOVE[:-1]:
        ratio, kept = run(skip, stop)
        if kept >= KEEP_SHARE and ratio < best_ratio:
            best_stop, best_ratio = stop, ratio
    for g in range(rules):
        for t in SKIP_BELOW[:-1]:
            trial = list(skip)
            trial[g] = t
            ratio, kept = run(trial, best_stop)
            if kept >= KEEP_SHARE and ratio < best_ratio:
                skip, best_ratio = trial, ratio
    for stop in STOP_ABOVE:
        if stop == best_stop:
            continue
        ratio, kept = run(skip, stop)
        if kept >= KEEP_SHARE and ratio < best_ratio:
            best_stop, best_ratio = stop, ratio
    return skip, best_stop, best_ratio, table


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--lps", type=int, default=20000)
    ap.add_argument("--holdout", type=int, default=40)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--batch", type=int, default=512)
    ap.add_argument("--max-m", type=int, default=500000)
    ap.add_argument("--max-trace-seconds", type=float, default=None,
                    help="stop tracing new LPs after this long (the notes record how many were traced)")
    ap.add_argument("--traces-out", default=None, help="save the traced rounds (compressed .npz)")
    args = ap.parse_args(argv)

    ctx = mp.get_context("spawn")
    workers = max(1, min(48, (os.cpu_count() or 2) - 2))
    X, Y, M = [], [], []
    t0 = time.perf_counter()
    train_nnz = 0
    with ctx.Pool(workers) as pool:
        hold = pool.map_async(_draw, jobs(args.holdout, args.seed + 2, hi=args.max_m), chunksize=1)
        from gpp_b200 import capi, device, schedule
        params = capi.Params.defaults()
        # Traced as they arrive; each LP is dropped once traced.
        traced = 0
        for lp in bounded_imap(pool, _draw, jobs(args.lps, args.seed + 1, hi=args.max_m), 2 * workers):
            if args.max_trace_seconds and time.perf_counter() - t0 > args.max_trace_seconds:
                pool.terminate()
                break
            traced += 1
            d = device.DeviceLp(lp)
            s, tr = schedule.traced_preprocess(d, params)
            device.free_summary(s)
            y, m = schedule.labels(tr)
            X.append(tr["features"]); Y.append(y); M.append(m)
            train_nnz += lp.nnz
            del d, lp
        hold_lps = hold.get() if hold.ready() or traced == args.lps else None
    if hold_lps is None:   # the pool was stopped early: draw the held-out LPs now
        with ctx.Pool(workers) as pool:
            hold_lps = pool.map(_draw, jobs(args.holdout, args.seed + 2, hi=args.max_m), chunksize=1)
    X, Y, M = (np.concatenate(a) for a in (X, Y, M))
    trace_s = time.perf_counter() - t0
    if args.traces_out:
        np.savez_compressed(args.traces_out, X=X, Y=Y, M=M, train_lps=traced, train_nnz=train_nnz)
    t1 = time.perf_counter()
    w, loss = schedule.train(X, Y, M, epochs=args.epochs, batch=args.batch, seed=args.seed)
    train_s = time.perf_counter() - t1

    # Thresholds on held-out LPs, against their plain runs.
    dlps = [device.DeviceLp(lp) for lp in hold_lps]
    plain_t, plain_r = [], []
    for lp, d in zip(hold_lps, dlps):
        s = device.preprocess(d, params)   # warm caches once
        device.free_summary(s)
        s = device.preprocess(d, params)
        plain_t.append(s.preprocessing_seconds)
        plain_r.append(removal(lp, s))
        device.free_summary(s)

    def evaluate(skip, stop):
        times, kept = [], []
        with schedule.Model(w, skip, stop) as model:
            for lp, d, pr in zip(hold_lps, dlps, plain_r):
                s = schedule.scheduled_preprocess(d, params, model)
                times.append(s.preprocessing_seconds)
                kept.append(removal(lp, s) / pr if pr > 0 else 1.0)
                device.free_summary(s)
        return float(np.sum(times) / np.sum(plain_t)), float(np.min(kept))

    skip, stop, ratio, table = choose_thresholds(evaluate, len(schedule.GATED_RULES))
    notes = {"samples": int(len(X)), "train_lps": traced, "train_nnz": int(train_nnz), "holdout_lps": args.holdout,
             "m_range": [1000, args.max_m], "generator_workers": workers, "train_seconds": train_s,
             "epochs": args.epochs, "batch": args.batch, "trace_seconds": trace_s,
             "final_loss": float(loss[-1]) if len(loss) else None, "thresholds": table,
             "chosen": {"skip_below": skip, "stop_above": stop, "time_ratio": ratio},
             "positive_rate": [float(x) for x in (Y * M).sum(0) / np.maximum(M.sum(0), 1)]}
    schedule.save_model(args.out, w, skip, stop, loss=loss, notes=json.dumps(notes))
    print(json.dumps(notes, indent=1))


if __name__ == "__main__":
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    main()
