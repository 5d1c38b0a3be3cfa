"""MPS input and reduced-LP export.

CPU: the reference reader's known-answer cases
(cpp/mps_reader/tests/test_mpsreader.cpp:12-135), and bit-exact parity with
the reference reader itself (built from its sources by oracle/mps_ref.mk) on
generated files in free and fixed format and on inputs both must reject.
GPU: the library's upload gives the same presolve as the same LP uploaded
from numpy, the export writes the reduced LP in the reference's format, and
the solver handoff (device and host copies of the reduced LP) returns the
summary's reduced LP with a stable transpose."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import mps_cases
from gpp_b200 import capi, device, mps

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_DRIVER = os.path.join(ROOT, "oracle", "_ref", "mps_ref_driver")
INF = np.inf


def test_known_answer_rows_columns_rhs_bounds():
    # test_mpsreader.cpp:12-50
    m = mps.MpsModel(text=(
        "NAME          toy\nROWS\n N  COST\n E  EQ1\n G  GE1\n L  LE1\nCOLUMNS\n"
        "    X1        COST       3.0   EQ1        2.0\n    X1        GE1        1.0\n"
        "    X2        COST       5.0   LE1       -4.0\n    X2        EQ1        1.0\n"
        "RHS\n    RHS1      EQ1       10.0   GE1        7.0\n    RHS1      LE1       20.0\n"
        "BOUNDS\n LO BND1      X1        -1.0\n UP BND1      X1         6.0\n FR BND1      X2\nENDATA\n"))
    assert (m.name, m.rows, m.cols) == ("toy", 3, 2)
    assert m.c.tolist() == [3.0, 5.0]
    assert m.AL.tolist() == [10.0, 7.0, -INF] and m.AU.tolist() == [10.0, INF, 20.0]
    assert m.l.tolist() == [-1.0, -INF] and m.u.tolist() == [6.0, INF]
    assert m.col_ptr.tolist() == [0, 2, 4] and m.row_idx.tolist() == [0, 1, 0, 2]
    assert m.csc_val.tolist() == [2.0, 1.0, 1.0, -4.0]


def test_known_answer_ranges_binary_bounds_duplicates():
    # test_mpsreader.cpp:52-91
    m = mps.MpsModel(text=(
        "NAME ranged\nROWS\n N OBJ\n E EQ1\n L LE1\n G GE1\nCOLUMNS\n"
        "    MARK0000  'MARKER'                 'INTORG'\n    X1        OBJ        1.0   EQ1        1.0\n"
        "    X1        LE1        2.0   LE1        3.0\n    MARK0001  'MARKER'                 'INTEND'\n"
        "    X2        OBJ        2.0   GE1       -1.0\nRHS\n    RHS1      EQ1       10.0   LE1       20.0\n"
        "    RHS1      GE1        5.0\nRANGES\n    RNG1      EQ1        4.0   LE1        6.0\n"
        "    RNG1      GE1        7.0\nBOUNDS\n BV BND1      X1\n UI BND1      X2         9.0\nENDATA\n"))
    assert (m.name, m.rows, m.cols) == ("ranged", 3, 2)
    assert m.c.tolist() == [1.0, 2.0]
    assert m.AL.tolist() == [10.0, 14.0, 5.0] and m.AU.tolist() == [14.0, 20.0, 12.0]
    assert m.l.tolist() == [0.0, 0.0] and m.u.tolist() == [1.0, 9.0]
    assert m.col_ptr.tolist() == [0, 2, 3] and m.row_idx.tolist() == [0, 1, 2]
    assert m.csc_val.tolist() == [1.0, 5.0, -1.0]


def test_known_answer_decimal_digit_accumulation():
    # test_mpsreader.cpp:93-111: "0.000001" is read by digit accumulation,
    # which lands above the correctly rounded 1e-6.
    m = mps.MpsModel(text=("NAME micro\nROWS\n N OBJ\n L ROW1\nCOLUMNS\n    X1        OBJ        1.0   ROW1       1.0\n"
                           "RHS\n    RHS1      ROW1       1.0\nBOUNDS\n UP BND1      X1         0.000001\nENDATA\n"))
    assert m.u.tolist() == [m.u[0]] and m.u[0] > 1.0e-6


def test_known_answer_fixed_format_fallback():
    # test_mpsreader.cpp:113-135
    m = mps.MpsModel(text=("NAME          fixed\nROWS\n N  COST\n L  ROW00001\nCOLUMNS\n"
                           "    COL00001  COST       1.0   ROW00001   2.0\nRHS\n    RHS00001  ROW00001   3.0\nENDATA\n"))
    assert (m.name, m.rows, m.cols) == ("fixed", 1, 1)
    assert m.c.tolist() == [1.0] and m.AU.tolist() == [3.0] and m.csc_val.tolist() == [2.0]


def reference_read(text):
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "model.mps")
        with open(path, "w") as f:
            f.write(text)
        r = subprocess.run([REF_DRIVER, path, d], capture_output=True, text=True)
        if r.returncode != 0:
            return None
        meta = dict(line.split(" ", 1) for line in open(os.path.join(d, "meta.txt")).read().splitlines())
        arrays = {}
        for name, dt in (("row_ptr", np.int64), ("col_idx", np.int32), ("csr_val", np.float64),
                         ("col_ptr", np.int64), ("row_idx", np.int32), ("csc_val", np.float64), ("c", np.float64),
                         ("AL", np.float64), ("AU", np.float64), ("l", np.float64), ("u", np.float64)):
            arrays[name] = np.fromfile(os.path.join(d, name), dtype=dt)
        return meta, arrays


needs_reference = pytest.mark.skipif(not os.path.exists(REF_DRIVER),
                                     reason="reference MPS reader not built (oracle/mps_ref.mk)")


@needs_reference
@pytest.mark.parametrize("fixed", [False, True])
@pytest.mark.parametrize("seed", range(20))
def test_parity_with_reference_reader(seed, fixed):
    text = mps_cases.write_mps(np.random.default_rng(seed), m=12 + seed, n=20 + 2 * seed, fixed=fixed)
    ref = reference_read(text)
    if ref is None:                      # e.g. a generated lower bound above its upper bound
        with pytest.raises(ValueError):
            mps.MpsModel(text=text)
        return
    got = mps.MpsModel(text=text)
    meta, arrays = ref
    assert got.name == meta["name"] and (got.rows, got.cols, got.nnz) == (int(meta["rows"]), int(meta["cols"]),
                                                                         int(meta["nnz"]))
    assert float(meta["obj_constant"]) == got.obj_constant
    for k, v in arrays.items():
        assert np.array_equal(getattr(got, k).view(np.uint8), v.view(np.uint8)), k


@needs_reference
@pytest.mark.parametrize("case", sorted(mps_cases.BAD))
def test_both_readers_reject(case):
    assert reference_read(mps_cases.BAD[case]) is None
    with pytest.raises(ValueError):        # GPP_ERR_INVALID
        mps.MpsModel(text=mps_cases.BAD[case])


@pytest.mark.gpu
def test_upload_and_export_reduced(tmp_path):
    from gpp_b200 import lpgen
    model = mps.MpsModel(text=mps_cases.lp_to_mps(lpgen.random_lp(300, 700, seed=77)))
    lp_c = model.upload()
    dlp = device.DeviceLp(model.host_lp())
    params = capi.Params.defaults()
    try:
        import ctypes as C
        s1 = capi.Summary()
        device._raise(capi.load().gpp_preprocess(C.byref(lp_c), C.byref(params), C.byref(s1)))
        s2 = device.preprocess(dlp, params)
        assert s1.has_infeasible == 0 and s1.has_unbounded == 0 and s1.reduced_nnz > 0
        r1, r2 = device.Result(s1), device.Result(s2)
        for k in ("A_ptr", "A_idx", "A_val", "c", "l", "u", "AL", "AU", "row_map", "col_map", "tape_val"):
            assert np.array_equal(getattr(r1, k).view(np.uint8), getattr(r2, k).view(np.uint8)), k
        mps.export_reduced(s1, str(tmp_path), model.name)
        meta = dict(line.split(" ", 1) for line in (tmp_path / "meta.txt").read_text().splitlines())
        assert meta["format"] == "gpu_preprocessor_reduced_lp_v1" and meta["model"] == model.name
        assert int(meta["reduced_rows"]) == s1.reduced_rows and int(meta["reduced_nnz"]) == s1.reduced_nnz
        for name, key, dt in (("A_rowPtr_i32.bin", "A_ptr", np.int32), ("A_colVal_i32.bin", "A_idx", np.int32),
                              ("A_nzVal_f64.bin", "A_val", np.float64), ("c_f64.bin", "c", np.float64),
                              ("l_f64.bin", "l", np.float64), ("u_f64.bin", "u", np.float64),
                              ("AL_f64.bin", "AL", np.float64), ("AU_f64.bin", "AU", np.float64)):
            assert np.array_equal(np.fromfile(tmp_path / name, dtype=dt), getattr(r1, key)), name
        device.free_summary(s1)
        device.free_summary(s2)
    finally:
        mps.free_lp(lp_c)


@pytest.mark.gpu
def test_solver_handoff_device_and_host():
    from gpp_b200 import lpgen
    lp = lpgen.random_lp(3000, 7500, seed=5)
    d = device.DeviceLp(lp)
    s = device.preprocess(d, capi.Params.defaults())
    try:
        r = device.Result(s)
        host = mps.reduced_to_host(s)
        for k, key in (("row_ptr", "A_ptr"), ("col_idx", "A_idx"), ("val", "A_val"), ("c", "c"), ("AL", "AL"),
                       ("AU", "AU"), ("l", "l"), ("u", "u")):
            assert np.array_equal(host[k].view(np.uint8), getattr(r, key).view(np.uint8)), k
        assert host["obj_constant"] == r.obj_constant
        copy = mps.reduced_to_device(s)
        try:
            m, n, nnz = s.reduced_rows, s.reduced_cols, s.reduced_nnz
            assert (copy.A.rows, copy.A.cols, copy.A.nnz, copy.AT.rows, copy.AT.cols) == (m, n, nnz, n, m)
            got = {k: device._d2h(p, cnt, dt) for k, p, cnt, dt in (
                ("A_ptr", copy.A.rowPtr, m + 1, np.int32), ("A_idx", copy.A.colVal, nnz, np.int32),
                ("A_val", copy.A.nzVal, nnz, np.float64), ("AT_ptr", copy.AT.rowPtr, n + 1, np.int32),
                ("AT_idx", copy.AT.colVal, nnz, np.int32), ("AT_val", copy.AT.nzVal, nnz, np.float64),
                ("c", copy.c, n, np.float64), ("l", copy.l, n, np.float64), ("u", copy.u, n, np.float64))}
            for k, v in got.items():
                assert np.array_equal(v.view(np.uint8), getattr(r, k).view(np.uint8)), k
            # The transpose is the stable one: rows of A^T list A's rows in ascending order.
            t_ptr, t_idx, t_val = lpgen.csr_transpose(m, n, got["A_ptr"], got["A_idx"], got["A_val"])
            assert np.array_equal(t_ptr, got["AT_ptr"]) and np.array_equal(t_idx, got["AT_idx"])
            assert np.array_equal(t_val, got["AT_val"])
        finally:
            mps.free_lp(copy)
    finally:
        device.free_summary(s)
