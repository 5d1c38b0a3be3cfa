"""Parity with the REFERENCE implementation itself, run on the same GPU.

oracle/_ref/ref_driver is the reference GPU-Preprocessor library, compiled from
its own sources by oracle/ref.mk, behind a small exporter (oracle/ref_driver.cpp).
The test runs it and the CUDA engine on identical synthetic LPs with the same
rule set and requires drop-in parity: the removed rows and columns,
the row/column maps and the sparsity pattern bit-exact; coefficients, bounds
and sides within 1e-12 relative.  Skipped when the reference build is absent
(it needs the reference sources at build time).
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import pyoracle
from gpp_b200 import device, lpgen
from gpp_b200.capi import RULE_FLAGS, params_with_rules

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_driver")
CLEANUP = ["infeasible_and_fixed_variables", "empty_columns", "empty_rows", "singleton_rows"]
BUILT = CLEANUP + ["bound_strengthening"]
PROPAGATION = BUILT + ["infeasible_and_redundant_rows", "dual_fix"]
PARALLEL = PROPAGATION + ["parallel_rows", "parallel_columns"]
SINGLETON = CLEANUP + ["singleton_columns"]
FULL = PARALLEL + ["singleton_columns"]
ALL = FULL + ["doubleton_equations"]
SMALL_BATCH = dict(doubleton_equations_min_selected_per_batch=1, doubleton_equations_min_selected_ratio=0.0)


def run_reference(lp, rules, extra=None, point=None):
    """Runs the reference library on `lp` and reads back what it exported.

    `point` = (x, y, z) in reduced order also runs the reference's
    postprocess on that point; its x_org, y_org, z_org are returned."""
    d = tempfile.mkdtemp()
    path = os.path.join(d, "lp.bin")
    lpgen.save_lp(path, lp)
    args = [DRIVER, path, d, "enable_folding=0", "enable_structure_specific_rules=0"]
    for f in RULE_FLAGS:
        args.append(f"{f}={1 if f[len('enable_'):] in rules else 0}")
    args += extra or []
    if point is not None:
        files = []
        for name, v in zip(("x_red", "y_red", "z_red"), point):
            files.append(os.path.join(d, name))
            np.ascontiguousarray(v, dtype=np.float64).tofile(files[-1])
        args += ["--postsolve", *files]
    r = subprocess.run(args, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    meta = {}
    for line in open(os.path.join(d, "meta.txt")):
        k, *v = line.split()
        meta[k] = v[0] if len(v) == 1 else v
    out = {"meta": meta, "dir": d}
    spec = {"A_ptr": np.int32, "A_idx": np.int32, "A_val": np.float64, "AT_ptr": np.int32, "AT_idx": np.int32,
            "AT_val": np.float64, "c": np.float64, "l": np.float64, "u": np.float64, "AL": np.float64,
            "AU": np.float64, "row_map": np.int32, "col_map": np.int32, "fixed_idx": np.int32,
            "fixed_val": np.float64, "tape_types": np.int32, "tape_is": np.int32, "tape_vs": np.int32,
            "tape_idx": np.int32, "tape_val": np.float64, "row_color": np.int32, "col_color": np.int32,
            "row_scale": np.float64, "col_scale": np.float64, "x_org": np.float64, "y_org": np.float64,
            "z_org": np.float64}
    for k, dt in spec.items():
        p = os.path.join(d, k)
        out[k] = np.fromfile(p, dtype=dt) if os.path.exists(p) else None
    return out


def close(a, b, rel=1e-12):
    a, b = np.asarray(a), np.asarray(b)
    if a.shape != b.shape:
        return False
    both_inf = np.isinf(a) & np.isinf(b) & (np.sign(a) == np.sign(b))
    ok = both_inf | (np.abs(a - b) <= rel * np.maximum(1.0, np.maximum(np.abs(a), np.abs(b))))
    return bool(np.all(ok))


needs_reference = pytest.mark.skipif(not os.path.exists(DRIVER), reason="reference build (oracle/_ref) not present")


def reduced_point(got, rows, cols, seed=1):
    """A seeded reduced primal/dual point: x inside the reduced bounds (finite
    boxes of width 20 where a bound is infinite), y and z standard normal."""
    rng = np.random.default_rng(seed)
    lo = np.where(np.isfinite(got.l), got.l, np.where(np.isfinite(got.u), got.u - 20.0, -10.0))
    hi = np.where(np.isfinite(got.u), got.u, lo + 20.0)
    return lo + rng.random(cols) * (hi - lo), rng.standard_normal(rows), rng.standard_normal(cols)


# Recovered solutions are compared at 1e-9 relative (the objective too).  The
# reference is compiled with floating-point contraction on (nvcc's default),
# so its doubleton replay x_elim = beta + alpha * x_keep is one fused rounding
# where this engine (and its oracle) round twice; where the two terms nearly
# cancel the difference grows past 1e-12: on the 29.8M-nnz LP, 2 of 5,000,000
# entries differ by 1.7e-12 and 1.5e-12 relative, with the objective equal.
POSTSOLVE_REL = 1e-9


def check_against_reference(lp, rules, extra=None, oracle=True, postsolve=False):
    """Presolves `lp` with the engine and with the reference library and
    requires drop-in parity.  With `postsolve`, both also postprocess the same
    reduced point, and the recovered x, y, z must agree within POSTSOLVE_REL
    and give the same objective within 1e-9 relative.  `postsolve` is True for
    a seeded point inside the reduced bounds, or a function (result, summary)
    -> (x, y, z) giving the point."""
    import torch
    extra = {"enable_structure_specific_rules": 0, **(extra or {})}
    params = params_with_rules(rules, **{"enable_folding": 0, **extra})
    dlp = device.DeviceLp(lp)
    s = device.preprocess(dlp, params)
    try:
        got = device.Result(s)
        got.fold = device.fold_map(s)
        got.summary = type(s).from_buffer_copy(s)
        point = None
        if callable(postsolve):
            point = postsolve(got, s)
        elif postsolve:
            point = reduced_point(got, s.reduced_rows, s.reduced_cols)
        ref = run_reference(lp, rules, [f"{k}={v}" for k, v in extra.items()], point)
        got.ref = ref
        m = ref["meta"]
        assert (s.reduced_rows, s.reduced_cols, s.reduced_nnz) == (
            int(m["reduced_rows"]), int(m["reduced_cols"]), int(m["reduced_nnz"]))
        assert s.iterations == int(m["iterations"])
        assert np.array_equal(got.row_map, ref["row_map"]) and np.array_equal(got.col_map, ref["col_map"])
        for k in ("A_ptr", "A_idx", "AT_ptr", "AT_idx"):
            assert np.array_equal(getattr(got, k), ref[k]), k
        for k in ("A_val", "AT_val", "c", "l", "u", "AL", "AU"):
            assert close(getattr(got, k), ref[k]), k
        assert np.array_equal(np.sort(got.fixed_idx), np.sort(ref["fixed_idx"]))
        assert np.array_equal(got.tape_types, ref["tape_types"])
        assert np.array_equal(got.tape_idx, ref["tape_idx"])
        assert close(got.tape_val, ref["tape_val"], 1e-9)
        if postsolve:
            x, y, z = device.postprocess(*(torch.from_numpy(v).cuda() for v in point), s, dlp)
            for k, v in (("x_org", x), ("y_org", y), ("z_org", z)):
                assert close(v, ref[k], POSTSOLVE_REL), k
            obj, obj_ref = float(lp.c @ x), float(lp.c @ ref["x_org"])
            assert abs(obj - obj_ref) <= 1e-9 * max(1.0, abs(obj_ref))
            got.solution = (x, y, z)
        if oracle:
            # The oracle agrees with both.
            orc = pyoracle.presolve(lp, params)
            assert np.array_equal(orc.row_map, ref["row_map"]) and np.array_equal(orc.col_map, ref["col_map"])
        return got
    finally:
        device.free_summary(s)


@needs_reference
@pytest.mark.parametrize("rules", [CLEANUP, BUILT, PROPAGATION, PARALLEL, SINGLETON, FULL])
@pytest.mark.parametrize("workload", ["random:400x1000", "small", "slack:400x1000", "slack:2000x5000"])
def test_structure_matches_reference(rules, workload):
    check_against_reference(lpgen.workload(workload, seed=0), rules)


@needs_reference
@pytest.mark.parametrize("workload,extra", [("random:400x1000", SMALL_BATCH), ("slack:2000x5000", SMALL_BATCH),
                                            ("random:20000x50000", {})])
def test_doubleton_structure_matches_reference(workload, extra):
    got = check_against_reference(lpgen.workload(workload, seed=0), ALL, extra)
    assert 13 in got.tape_types.tolist()   # the batch ran


@needs_reference
@pytest.mark.parametrize("workload", ["replicated:100x250*4", "replicated:400x1000*3", "random:400x1000"])
def test_folding_matches_reference(workload):
    """The default pipeline with folding on: the fold decision, folded sizes,
    colour maps and the presolve of the folded model equal the reference's."""
    lp = lpgen.workload(workload, seed=0)
    got = check_against_reference(lp, ALL, {"enable_folding": 1})
    ref = run_reference(lp, ALL, ["enable_folding=1"])
    m = ref["meta"]
    assert got.summary.folding_applied == int(m["folding_applied"])
    assert (got.summary.folded_rows, got.summary.folded_cols) == (int(m["folded_rows"]), int(m["folded_cols"]))
    if got.summary.folding_applied:
        assert np.array_equal(got.fold[0], ref["row_color"]) and np.array_equal(got.fold[1], ref["col_color"])
        assert np.array_equal(got.fold[2], ref["row_scale"]) and np.array_equal(got.fold[3], ref["col_scale"])


@needs_reference
@pytest.mark.parametrize("workload", ["random:400x1000", "small", "slack:2000x5000", "random:20000x50000"])
def test_reference_startup_rules_do_not_fire(workload):
    """On these workloads the reference's own structure-specific detectors
    reject every structure-specific startup rule: its output with the rules on
    equals its output with them off, so the parity tests above (rules off)
    also hold for the reference's default settings."""
    lp = lpgen.workload(workload, seed=0)
    on = run_reference(lp, ALL, ["enable_structure_specific_rules=1"])
    off = run_reference(lp, ALL)
    for k in ("row_map", "col_map", "A_idx", "tape_types"):
        assert np.array_equal(on[k], off[k]), k
    assert on["meta"]["iterations"] == off["meta"]["iterations"]


@needs_reference
@pytest.mark.parametrize("rules", [PROPAGATION, FULL, ALL])
@pytest.mark.parametrize("workload", ["random:400x1000", "slack:2000x5000", "random:20000x50000"])
def test_postsolve_matches_reference(rules, workload):
    """The reference's postprocess and the engine's recover the same original
    x, y, z from one seeded reduced point (tapes up to ~10^4 records, so the
    engine's component-parallel replay is compared with the reference's)."""
    extra = SMALL_BATCH if rules is ALL and workload != "random:20000x50000" else {}
    got = check_against_reference(lpgen.workload(workload, seed=0), rules, extra, oracle=False, postsolve=True)
    if rules is ALL:
        assert 13 in got.tape_types.tolist()


@needs_reference
@pytest.mark.parametrize("workload,seed", [("random:400x1000", 0), ("random:400x1000", 3), ("slack:400x1000", 0)])
def test_postsolve_of_optimum_matches_reference(workload, seed):
    """The reduced LP's optimum (HiGHS) postsolved by the reference and by the
    engine: same x, y, z, and the original objective within 1e-9 relative of
    HiGHS on the unreduced LP."""
    import lpsolve
    lp = lpgen.workload(workload, seed=seed)

    def optimum(got, s):
        rr, yr, zr = lpsolve.solve(s.reduced_rows, s.reduced_cols, got.A_ptr, got.A_idx, got.A_val, got.c, got.AL,
                                   got.AU, got.l, got.u)
        return rr.x, yr, zr

    got = check_against_reference(lp, ALL, SMALL_BATCH, oracle=False, postsolve=optimum)
    res0, _, _ = lpsolve.solve(lp.m, lp.n, lp.row_ptr, lp.col_idx, lp.values, lp.c, lp.AL, lp.AU, lp.l, lp.u)
    for x in (got.solution[0], got.ref["x_org"]):
        assert abs(lp.c @ x - res0.fun) <= 1e-9 * max(1.0, abs(res0.fun))
