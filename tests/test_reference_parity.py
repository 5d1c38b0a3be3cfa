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


def run_reference(lp, rules, extra=None):
    d = tempfile.mkdtemp()
    path = os.path.join(d, "lp.bin")
    lpgen.save_lp(path, lp)
    args = [DRIVER, path, d, "enable_folding=0", "enable_structure_specific_rules=0"]
    for f in RULE_FLAGS:
        args.append(f"{f}={1 if f[len('enable_'):] in rules else 0}")
    args += extra or []
    r = subprocess.run(args, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    meta = {}
    for line in open(os.path.join(d, "meta.txt")):
        k, *v = line.split()
        meta[k] = v[0] if len(v) == 1 else v
    out = {"meta": meta}
    spec = {"A_ptr": np.int32, "A_idx": np.int32, "A_val": np.float64, "AT_ptr": np.int32, "AT_idx": np.int32,
            "AT_val": np.float64, "c": np.float64, "l": np.float64, "u": np.float64, "AL": np.float64,
            "AU": np.float64, "row_map": np.int32, "col_map": np.int32, "fixed_idx": np.int32,
            "fixed_val": np.float64, "tape_types": np.int32, "tape_is": np.int32, "tape_vs": np.int32,
            "tape_idx": np.int32, "tape_val": np.float64, "row_color": np.int32, "col_color": np.int32,
            "row_scale": np.float64, "col_scale": np.float64}
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


def check_against_reference(lp, rules, extra=None):
    extra = {"enable_structure_specific_rules": 0, **(extra or {})}
    ref = run_reference(lp, rules, [f"{k}={v}" for k, v in extra.items()])
    params = params_with_rules(rules, **{"enable_folding": 0, **extra})
    dlp = device.DeviceLp(lp)
    s = device.preprocess(dlp, params)
    try:
        got = device.Result(s)
        got.fold = device.fold_map(s)
        got.summary = type(s).from_buffer_copy(s)
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
    """Of the reference's structure-specific startup rules this engine runs
    column domination only.  On these workloads the reference's own detectors
    reject all of them: its output with the rules on equals its output with
    them off, so the engine's parity holds for the reference's default
    settings too."""
    lp = lpgen.workload(workload, seed=0)
    on = run_reference(lp, ALL, ["enable_structure_specific_rules=1"])
    off = run_reference(lp, ALL)
    for k in ("row_map", "col_map", "A_idx", "tape_types"):
        assert np.array_equal(on[k], off[k]), k
    assert on["meta"]["iterations"] == off["meta"]["iterations"]
