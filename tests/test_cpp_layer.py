"""The header-only C++ layer (include/gpu_preprocessor/) that mirrors
GPU-Preprocessor's C++ API (gpu_preprocessor.hpp:8-41, presolve/*.hpp,
folding/*.hpp) over the C ABI.

CPU: the layer compiles warning-free against libgpp_b200.so, its
PresolveParams defaults equal gpp_default_params field by field, and a
consumer asking for the 64-bit offset ABI is stopped at compile time.
GPU: tests/cpp/plain_pipeline.cpp, a user program of the layer, runs the plain
pipeline (preprocess / postprocess / free_summary), the presolve-only path
(run_gpu_presolve_with_reduced_lp / postsolve_gpu) and the record and folding
map exports; everything it writes must equal, bit for bit, what the ctypes
path produces on the same LP and the same reduced solution."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_LIB_DIR = os.path.join(ROOT, "gpu-preprocessor-ijoc_b200", "gpp_b200")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
SOURCE = os.path.join(ROOT, "tests", "cpp", "plain_pipeline.cpp")

pytestmark = pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")


def compile_cmd(out, *extra):
    return ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", *extra, "-I", os.path.join(ROOT, "include"),
            "-I", os.path.join(CUDA_HOME, "include"), SOURCE, "-o", out, "-L", PKG_LIB_DIR, "-lgpp_b200",
            "-L", os.path.join(CUDA_HOME, "lib64"), "-lcudart", f"-Wl,-rpath,{PKG_LIB_DIR}"]


@pytest.fixture(scope="module")
def program(tmp_path_factory):
    from gpp_b200 import capi
    capi.load()  # builds nothing; fails loudly when the library is missing
    out = str(tmp_path_factory.mktemp("cpp") / "plain_pipeline")
    r = subprocess.run(compile_cmd(out), capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


def test_layer_compiles_and_defaults_match(program):
    r = subprocess.run([program, "defaults"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "defaults match" in r.stdout


def test_int64_offset_abi_is_rejected(tmp_path):
    src = tmp_path / "use.cpp"
    src.write_text('#include "gpu_preprocessor/gpu_preprocessor.hpp"\nint main() { return 0; }\n')
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-DGPUPREPROCESSOR_USE_INT64_NNZ=1",
                        "-I", os.path.join(ROOT, "include"), str(src)], capture_output=True, text=True)
    assert r.returncode != 0 and "32-bit offset ABI" in r.stderr


ALL_RULES = ["infeasible_and_fixed_variables", "empty_columns", "empty_rows", "singleton_rows",
             "singleton_columns", "bound_strengthening", "infeasible_and_redundant_rows", "dual_fix",
             "parallel_rows", "parallel_columns", "doubleton_equations"]

CASES = [
    ("slack:400x1000", dict(enable_folding=0)),
    ("slack:400x1000", dict(enable_folding=0, doubleton_equations_min_selected_per_batch=1,
                            doubleton_equations_min_selected_ratio=0.0)),
    ("replicated:100x250*4", dict(enable_folding=1)),
    ("hub:300x800", dict()),  # the reference's defaults
    # The piecewise-linear reformulations through the layer's record export and restore.
    ("l1split:200x12", dict(enable_folding=0)),
    ("graphl1:200x12", dict(enable_folding=0)),
    ("antipodal:40x4", dict(enable_folding=0,
                            piecewise_linear_reformulation_variable_pair_shifted_antipodal_min_pairs=16)),
]


def read(path, dtype):
    return np.fromfile(path, dtype=dtype) if os.path.exists(path) else None


def meta(path):
    out = {}
    with open(path) as f:
        for line in f:
            k, v = line.split()
            out[k] = float(v)
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("workload,extra", CASES)
def test_plain_pipeline_matches_ctypes_path(program, tmp_path, workload, extra):
    import torch
    from gpp_b200 import capi, device, lpgen
    name = workload if workload.split(":")[0] in ("slack", "replicated", "l1split", "graphl1", "antipodal") else None
    lp = lpgen.workload(name, seed=3) if name else lpgen.random_lp(300, 800, seed=3, hub_rows=4)
    lp_path = str(tmp_path / "lp.bin")
    lpgen.save_lp(lp_path, lp)
    args = [f"{k}={v}" for k, v in extra.items()]
    if workload.startswith("slack"):
        args += [f"enable_{f}={int(f in ALL_RULES)}" for f in ALL_RULES]
    out = tmp_path / "out"
    out.mkdir()
    r = subprocess.run([program, "run", lp_path, str(out), *args], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    got = meta(out / "meta.txt")

    kw = dict(extra)
    if workload.startswith("slack"):
        kw.update({f"enable_{f}": int(f in ALL_RULES) for f in ALL_RULES})
    params = capi.Params.defaults(**kw)
    dlp = device.DeviceLp(lp)
    s = device.preprocess(dlp, params)
    try:
        ref = device.Result(s, copy_lp=False)
        assert got["original_rows"] == s.original_rows and got["original_cols"] == s.original_cols
        assert got["folded_rows"] == s.folded_rows and got["folded_cols"] == s.folded_cols
        assert got["presolve_original_rows"] == s.folded_rows and got["presolve_original_cols"] == s.folded_cols
        assert got["folding_applied"] == s.folding_applied
        assert (got["reduced_rows"], got["reduced_cols"], got["reduced_nnz"]) == (
            s.reduced_rows, s.reduced_cols, s.reduced_nnz)
        assert got["iterations"] == s.iterations and got["has_change"] == s.has_change
        assert got["obj_constant_delta"] == s.obj_constant_delta
        assert np.array_equal(read(out / "row_map", np.int32), ref.row_map)
        assert np.array_equal(read(out / "col_map", np.int32), ref.col_map)
        assert np.array_equal(read(out / "tape_types", np.int32), ref.tape_types)
        assert np.array_equal(read(out / "tape_is", np.int32), ref.tape_is.astype(np.int32))
        assert np.array_equal(read(out / "tape_vs", np.int32), ref.tape_vs.astype(np.int32))
        assert np.array_equal(read(out / "tape_idx", np.int32), ref.tape_idx)
        assert np.array_equal(read(out / "tape_val", np.float64).view(np.uint64), ref.tape_val.view(np.uint64))
        assert np.array_equal(read(out / "fixed_idx", np.int32), ref.fixed_idx)
        assert np.array_equal(read(out / "fixed_val", np.float64).view(np.uint64), ref.fixed_val.view(np.uint64))
        ck = list(zip(read(out / "ckpt_kind", np.int32).tolist(), read(out / "ckpt_payload", np.int32).tolist(),
                      read(out / "ckpt_position", np.int64).tolist()))
        assert ck == ref.checkpoints
        if workload.split(":")[0] in ("l1split", "graphl1", "antipodal"):
            assert len(ck) == 1
        splits = [(a["split_t"], a["split_e"], a["split_rho"]) for a in ref.absolute_value]
        if splits:
            assert np.array_equal(read(out / "abs_split_t", np.int32), np.concatenate([t for t, _, _ in splits]))
            assert np.array_equal(read(out / "abs_split_e", np.int32), np.concatenate([e for _, e, _ in splits]))
            assert np.array_equal(read(out / "abs_split_rho", np.float64), np.concatenate([r for _, _, r in splits]))
            xv = torch.tensor(0.5 * (np.arange(lp.n) % 9) - 1.0, dtype=torch.float64, device="cuda")
            device.restore_absolute_value(xv, ref.absolute_value, dlp.t["l"])
            assert np.array_equal(read(out / "restored", np.float64).view(np.uint64),
                                  xv.cpu().numpy().view(np.uint64))
        if ref.variable_pair:
            assert np.array_equal(read(out / "vp_plus", np.int32), np.concatenate([a["plus"] for a in ref.variable_pair]))
            assert np.array_equal(read(out / "vp_root_plus", np.int32),
                                  np.concatenate([a["root_plus"] for a in ref.variable_pair]))
            assert np.array_equal(read(out / "vp_plus_shift", np.float64),
                                  np.concatenate([a["plus_shift"] for a in ref.variable_pair]))
        if s.folding_applied:
            rc, cc, rs, cs = device.fold_map(s)
            assert np.array_equal(read(out / "row_color", np.int32), rc)
            assert np.array_equal(read(out / "col_color", np.int32), cc)
            assert np.array_equal(read(out / "row_scale", np.float64), rs)
            assert np.array_equal(read(out / "col_scale", np.float64), cs)
        assert s.has_infeasible == 0 and s.has_unbounded == 0
        xr, yr, zr = (torch.from_numpy(read(out / k, np.float64)).cuda() for k in ("xr", "yr", "zr"))
        x, y, z = device.postprocess(xr, yr, zr, s, dlp)
        for key, want in (("x", x), ("y", y), ("z", z)):
            assert np.array_equal(read(out / key, np.float64).view(np.uint64), want.view(np.uint64)), key
        if not s.folding_applied:
            # postsolve_gpu on the presolve-only summary recovers the same point.
            for key, want in (("px", x), ("py", y), ("pz", z)):
                assert np.array_equal(read(out / key, np.float64).view(np.uint64), want.view(np.uint64)), key
    finally:
        device.free_summary(s)


@pytest.mark.gpu
@pytest.mark.parametrize("workload", ["replicated:100x250*4", "random:300x800"])
def test_run_folding_matches_the_pipeline_map(program, tmp_path, workload):
    """folding::run_folding / free_folded_lp of the layer: the same fold
    decision, sizes and colour map as the pipeline's folding stage (presolve
    off), a folded model of the folded sizes, and an unfold through the run's
    own map equal to the pipeline's unfold of the same folded point."""
    import torch
    from gpp_b200 import capi, device, lpgen
    lp = lpgen.workload(workload, seed=0)
    lp_path = str(tmp_path / "lp.bin")
    lpgen.save_lp(lp_path, lp)
    out = tmp_path / "out"
    out.mkdir()
    r = subprocess.run([program, "fold", lp_path, str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    got = meta(out / "meta.txt")
    dlp = device.DeviceLp(lp)
    s = device.preprocess(dlp, capi.Params.defaults(enable_folding=1, enable_presolve=0, folding_tolerance=1e-9))
    try:
        assert got["applied"] == s.folding_applied
        assert (got["folded_rows"], got["folded_cols"]) == (s.folded_rows, s.folded_cols)
        assert got["owns_folded_lp"] == s.folding_applied
        if not s.folding_applied:
            return
        rc, cc, rs, cs = device.fold_map(s)
        assert np.array_equal(read(out / "row_color", np.int32), rc)
        assert np.array_equal(read(out / "col_color", np.int32), cc)
        assert np.array_equal(read(out / "row_scale", np.float64), rs)
        assert np.array_equal(read(out / "col_scale", np.float64), cs)
        assert np.array_equal(read(out / "dev_row_color", np.int32), rc)
        assert np.array_equal(read(out / "dev_col_scale", np.float64), cs)
        assert len(read(out / "F_ptr", np.int32)) == s.folded_rows + 1
        assert len(read(out / "F_c", np.float64)) == s.folded_cols
        nf, mf = s.folded_cols, s.folded_rows
        xf = torch.tensor([float(j % 5) for j in range(nf)], dtype=torch.float64).cuda()
        yf = torch.tensor([float(i % 4) - 1.0 for i in range(mf)], dtype=torch.float64).cuda()
        zf = torch.tensor([0.5 * float(j % 3) for j in range(nf)], dtype=torch.float64).cuda()
        ux, uy, uz = device.unfold(xf, yf, zf, s)
        for key, want in (("ux", ux), ("uy", uy), ("uz", uz)):
            assert np.array_equal(read(out / key, np.float64), want), key
    finally:
        device.free_summary(s)
