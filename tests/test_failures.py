"""Failure handling, with every failure made on the host.

- An out-of-memory failure faked at the engine's allocator
  (gpp_inject_alloc_failure: the k-th device allocation returns
  cudaErrorMemoryAllocation, no device state is touched) must surface as
  GPP_ERR_CUDA with its message from the call it hit, and leave the library
  usable: the next presolve equals an undisturbed one.  In the batched form
  the LP whose allocation failed fails alone.
- The presolve time limit (max_time, reference gpu_presolve.cu:2134-2141):
  a limit that has already passed stops presolve before its first round, as
  the reference's does; a limit part-way through stops it early with a model
  whose postsolved optimum is still the original one.
- A rank that fails in the sharded batched form: its peer gets an error from
  the gather within the process group's timeout instead of waiting forever
  (gloo, CPU).
"""
import ctypes as C
import datetime
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as tmp

from gpp_b200 import capi, lpgen, shard

GPP_ERR_CUDA = 1


def key(s):
    return (s.reduced_rows, s.reduced_cols, s.reduced_nnz, s.iterations, s.obj_constant_delta)


@pytest.mark.gpu
@pytest.mark.parametrize("after", [0, 3, 40, 400])
def test_allocation_failure_is_reported_and_recoverable(after):
    from gpp_b200 import device
    lib = capi.load()
    lp = lpgen.workload("slack:2000x5000", seed=4)
    dlp = device.DeviceLp(lp)
    params = capi.Params.defaults()
    base = device.preprocess(dlp, params)
    want = key(base)
    device.free_summary(base)
    lib.gpp_inject_alloc_failure(after)
    s = capi.Summary()
    try:
        status = lib.gpp_preprocess(C.byref(dlp.struct()), C.byref(params), C.byref(s))
    finally:
        lib.gpp_inject_alloc_failure(-1)
    assert status == GPP_ERR_CUDA
    assert b"out of memory" in lib.gpp_last_error() or b"cudaMalloc" in lib.gpp_last_error()
    lib.gpp_free_summary(C.byref(s))
    again = device.preprocess(dlp, params)
    try:
        assert key(again) == want
    finally:
        device.free_summary(again)


@pytest.mark.gpu
def test_batch_allocation_failure_fails_one_lp_alone():
    from gpp_b200 import device
    lib = capi.load()
    lps = [lpgen.random_lp(1000 + 300 * k, 2500 + 750 * k, seed=60 + k) for k in range(6)]
    dlps = [device.DeviceLp(lp) for lp in lps]
    params = capi.Params.defaults()
    plain = []
    for d in dlps:
        s = device.preprocess(d, params)
        plain.append(key(s))
        device.free_summary(s)
    lps_c = (capi.Lp * len(dlps))(*[d.struct() for d in dlps])
    out = (capi.Summary * len(dlps))()
    status = np.zeros(len(dlps), np.int32)
    lib.gpp_inject_alloc_failure(50)
    try:
        rc = lib.gpp_preprocess_batch(C.cast(lps_c, C.c_void_p), len(dlps), C.byref(params), 3,
                                      C.cast(out, C.c_void_p), status.ctypes.data_as(C.c_void_p))
    finally:
        lib.gpp_inject_alloc_failure(-1)
    try:
        assert rc == GPP_ERR_CUDA
        assert (status != 0).sum() == 1 and status[status != 0][0] == GPP_ERR_CUDA
        for k in range(len(dlps)):
            if status[k] == 0:
                assert key(out[k]) == plain[k]
    finally:
        for k in range(len(dlps)):
            lib.gpp_free_summary(C.byref(out[k]))


@pytest.mark.gpu
def test_time_limit_already_passed_stops_before_the_first_round():
    from test_reference_parity import ALL, DRIVER, run_reference
    from gpp_b200 import device
    lp = lpgen.workload("random:20000x50000", seed=0)
    dlp = device.DeviceLp(lp)
    s = device.preprocess(dlp, capi.params_with_rules(ALL, enable_folding=0, max_time=1e-12))
    try:
        assert s.iterations == 0
        assert (s.reduced_rows, s.reduced_cols, s.reduced_nnz) == (lp.m, lp.n, lp.nnz)
        if os.path.exists(DRIVER):
            ref = run_reference(lp, ALL, ["max_time=1e-12"])
            assert int(ref["meta"]["iterations"]) == 0
            assert (int(ref["meta"]["reduced_rows"]), int(ref["meta"]["reduced_cols"])) == (lp.m, lp.n)
    finally:
        device.free_summary(s)


@pytest.mark.gpu
def test_time_limit_part_way_keeps_a_valid_model():
    import torch
    import lpsolve
    from gpp_b200 import device
    lp = lpgen.workload("slack:2000x5000", seed=5)
    dlp = device.DeviceLp(lp)
    params = capi.Params.defaults(enable_folding=0)
    full = device.preprocess(dlp, params)
    t_full, it_full, nnz_full = full.elapsed_seconds, full.iterations, full.reduced_nnz
    device.free_summary(full)
    s = device.preprocess(dlp, capi.Params.defaults(enable_folding=0, max_time=0.3 * t_full))
    try:
        assert s.iterations <= it_full and s.reduced_nnz >= nnz_full
        r = device.Result(s)
        res0, _, _ = lpsolve.solve(lp.m, lp.n, lp.row_ptr, lp.col_idx, lp.values, lp.c, lp.AL, lp.AU, lp.l, lp.u)
        rr, yr, zr = lpsolve.solve(s.reduced_rows, s.reduced_cols, r.A_ptr, r.A_idx, r.A_val, r.c, r.AL, r.AU, r.l,
                                   r.u)
        x, _, _ = device.postprocess(torch.from_numpy(rr.x).cuda(), torch.from_numpy(yr).cuda(),
                                     torch.from_numpy(zr).cuda(), s, dlp)
        assert abs(lp.c @ x - res0.fun) <= 1e-9 * max(1.0, abs(res0.fun))
    finally:
        device.free_summary(s)


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    nnz = [5, 4, 3, 2]

    def run_shard(indices):
        if rank == 1:
            raise RuntimeError("rank 1 failed while presolving its share")
        return {k: {"nnz": nnz[k]} for k in indices}

    try:
        shard.run_sharded(nnz, run_shard, rank, world)
        outcome = "finished"
    except Exception as e:  # the failing rank and its waiting peer both end here
        outcome = type(e).__name__
    with open(os.path.join(out_dir, f"rank{rank}"), "w") as f:
        f.write(outcome)
    os._exit(0)   # skip the group teardown, which would wait for the failed peer


def test_failing_rank_ends_its_peers_gather_with_an_error(tmp_path):
    world = 2
    tmp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    assert open(tmp_path / "rank1").read() == "RuntimeError"
    assert open(tmp_path / "rank0").read() != "finished"
