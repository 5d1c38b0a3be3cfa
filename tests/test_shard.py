"""The batched form's multi-GPU sharding, on the CPU: the greedy nnz
partition, and two gloo ranks that each take their share and gather the
per-LP records to rank 0 (the records are computed on the host here; on a
GPU box the same function runs the batched presolve)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as tmp

from gpp_b200 import shard


def test_partition_is_complete_disjoint_and_balanced():
    rng = np.random.default_rng(3)
    nnz = (np.exp(rng.uniform(np.log(5e3), np.log(1e6), size=512))).astype(int)
    for world in (1, 2, 3, 4, 8):
        parts = shard.greedy_nnz_partition(nnz, world)
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(len(nnz)))
        loads = shard.shard_loads(nnz, parts)
        # Greedy largest-first: the spread is at most the largest LP.
        assert max(loads) - min(loads) <= int(nnz.max())
        assert parts == shard.greedy_nnz_partition(list(nnz), world)   # deterministic


def test_partition_edge_cases():
    assert shard.greedy_nnz_partition([], 2) == [[], []]
    assert shard.greedy_nnz_partition([5], 3) == [[0], [], []]
    assert shard.greedy_nnz_partition([4, 4, 4, 4], 2) == [[0, 2], [1, 3]]
    with pytest.raises(ValueError):
        shard.greedy_nnz_partition([1], 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, nnz, out_dir):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ran = []

        def run_shard(indices):
            ran.extend(indices)
            return {k: {"nnz": int(nnz[k]), "rank": rank, "reduced": int(nnz[k]) // 2} for k in indices}

        recs, mine = shard.run_sharded(nnz, run_shard, rank, world)
        assert ran == mine
        if rank == 0:
            np.save(os.path.join(out_dir, "records.npy"),
                    np.array([(r["nnz"], r["rank"], r["reduced"]) for r in recs], dtype=np.int64))
        else:
            assert recs is None
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_gather(tmp_path):
    rng = np.random.default_rng(5)
    nnz = rng.integers(1000, 100000, size=37).tolist()
    world = 2
    tmp.spawn(_rank_main, args=(world, _free_port(), nnz, str(tmp_path)), nprocs=world, join=True)
    rec = np.load(tmp_path / "records.npy")
    assert rec[:, 0].tolist() == nnz                  # every LP once, in index order
    assert rec[:, 2].tolist() == [v // 2 for v in nnz]
    parts = shard.greedy_nnz_partition(nnz, world)
    for r, p in enumerate(parts):
        assert set(np.nonzero(rec[:, 1] == r)[0].tolist()) == set(p)


def test_records_for_foreign_lps_are_refused():
    with pytest.raises(RuntimeError):
        shard.run_sharded([3, 2, 1], lambda idx: {99: {}}, 0, 1)
