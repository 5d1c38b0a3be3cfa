"""Batched form: gpp_preprocess_batch / gpp_postprocess_batch / gpp_batch_autotune.

Every LP of a batch must come out exactly as the plain entry points give it:
the same summary, reduced model, maps and tape, bit for bit, and the same
recovered solution.  The batch mixes LP sizes (so workers finish out of
order), a folded LP, and, in one test, an invalid LP whose failure must stay
its own."""
import ctypes as C

import numpy as np
import pytest

from gpp_b200 import capi, device, lpgen

pytestmark = pytest.mark.gpu


def batch_lps():
    lps = [lpgen.random_lp(m, int(2.5 * m), seed=s) for m, s in ((200, 1), (3000, 2), (1000, 3), (12000, 4),
                                                                 (500, 5), (6000, 6), (2500, 7))]
    lps.append(lpgen.workload("slack:400x1000", seed=8))
    lps.append(lpgen.workload("replicated:100x250*4", seed=0))
    return lps


def bits(a):
    return np.asarray(a).view(np.uint8)


def same_result(a, b):
    assert (a.summary.reduced_rows, a.summary.reduced_cols, a.summary.reduced_nnz) == (
        b.summary.reduced_rows, b.summary.reduced_cols, b.summary.reduced_nnz)
    assert (a.summary.iterations, a.summary.has_change, a.summary.folding_applied) == (
        b.summary.iterations, b.summary.has_change, b.summary.folding_applied)
    assert bits([a.summary.obj_constant_delta]).tobytes() == bits([b.summary.obj_constant_delta]).tobytes()
    for k in ("A_ptr", "A_idx", "A_val", "AT_ptr", "AT_idx", "AT_val", "c", "l", "u", "AL", "AU", "row_map",
              "col_map", "tape_types", "tape_is", "tape_vs", "tape_idx", "tape_val", "fixed_idx", "fixed_val"):
        assert np.array_equal(bits(getattr(a, k)), bits(getattr(b, k))), k


@pytest.mark.parametrize("workers", [1, 4])
def test_batch_matches_plain(workers):
    import torch
    lps = batch_lps()
    dlps = [device.DeviceLp(lp) for lp in lps]
    params = capi.Params.defaults()
    plain = [device.preprocess(d, params) for d in dlps]
    batch, status = device.preprocess_batch(dlps, params, workers=workers)
    try:
        assert status.tolist() == [0] * len(lps)
        results = []
        for p, b in zip(plain, batch):
            rp, rb = device.Result(p), device.Result(b)
            same_result(rp, rb)
            results.append(rp)
        # Postsolve: the same reduced point through both paths.
        xs, ys, zs = [], [], []
        for r in results:
            s = r.summary
            xs.append(torch.from_numpy(np.clip(np.linspace(-1.0, 2.0, s.reduced_cols), r.l, r.u)).cuda())
            ys.append(torch.from_numpy(np.linspace(-0.5, 0.5, s.reduced_rows)).cuda())
            zs.append(torch.from_numpy(np.linspace(0.25, -0.25, s.reduced_cols)).cuda())
        got = device.postprocess_batch(xs, ys, zs, batch, dlps, workers=workers)
        for k, (d, p) in enumerate(zip(dlps, plain)):
            want = device.postprocess(xs[k], ys[k], zs[k], p, d)
            for g, w in zip(got[k], want):
                assert np.array_equal(bits(g), bits(w)), k
    finally:
        for s in plain + batch:
            device.free_summary(s)


def test_batch_failure_stays_with_its_lp():
    lps = batch_lps()[:4]
    dlps = [device.DeviceLp(lp) for lp in lps]
    structs = [d.struct() for d in dlps]
    structs[2].AT.nnz = structs[2].A.nnz + 1            # A and AT disagree: invalid input
    arr = (capi.Lp * len(structs))(*structs)
    out = (capi.Summary * len(structs))()
    status = np.zeros(len(structs), np.int32)
    lib = capi.load()
    rc = lib.gpp_preprocess_batch(C.cast(arr, C.c_void_p), len(structs), C.byref(capi.Params.defaults()), 3,
                                  C.cast(out, C.c_void_p), status.ctypes.data_as(C.c_void_p))
    try:
        assert rc == 3 and status.tolist() == [0, 0, 3, 0]     # GPP_ERR_INVALID for LP 2 only
        assert b"LP 2" in lib.gpp_last_error()
        assert out[2].record is None
        for k in (0, 1, 3):
            assert out[k].record is not None and out[k].original_rows == lps[k].m
    finally:
        for k in range(len(structs)):
            lib.gpp_free_summary(C.byref(out[k]))


def test_autotune_picks_a_power_of_two():
    dlps = [device.DeviceLp(lp) for lp in batch_lps()]
    best, curve = device.batch_autotune(dlps, capi.Params.defaults(), max_workers=8)
    assert best in (1, 2, 4, 8) and sorted(curve) == [1, 2, 4, 8] and all(r > 0 for r in curve.values())
