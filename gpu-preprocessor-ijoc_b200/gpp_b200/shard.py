"""The batched form across GPUs: independent LPs sharded over ranks.

Every LP of a batch is presolved on its own, so the batch shards with no
exchange at all: one process per GPU takes a share of the LPs, presolves
and postsolves it with the batched entry points on its own device, and the
per-LP results (sizes, iteration counts, latencies) are gathered to rank 0
over a host (gloo) group.  No device collective is on the data path.

The share of each rank comes from a greedy nnz balance: LPs in descending
nnz order (index order among equals), each to the rank with the least nnz so
far (lowest rank among equals).  Every rank computes the same partition from
the same sizes, so no rank has to send it.
"""
from __future__ import annotations


def greedy_nnz_partition(nnz, world):
    """Indices of the LPs each of `world` ranks takes, each list ascending."""
    if world < 1:
        raise ValueError("world must be at least 1")
    order = sorted(range(len(nnz)), key=lambda k: (-int(nnz[k]), k))
    loads = [0] * world
    shards = [[] for _ in range(world)]
    for k in order:
        r = min(range(world), key=lambda q: (loads[q], q))
        shards[r].append(k)
        loads[r] += int(nnz[k])
    return [sorted(s) for s in shards]


def shard_loads(nnz, shards):
    return [sum(int(nnz[k]) for k in s) for s in shards]


def gather_records(records, rank, world, group=None):
    """Gathers each rank's {LP index: record} to rank 0 (host objects over
    `group`, a gloo group when the default group is NCCL).  Rank 0 gets the
    records of all LPs as a list in LP index order; the other ranks get None."""
    if world == 1:
        return [records[k] for k in sorted(records)]
    import torch.distributed as dist
    out = [None] * world if rank == 0 else None
    dist.gather_object(records, out, dst=0, group=group)
    if rank != 0:
        return None
    merged = {}
    for part in out:
        for k, v in part.items():
            if k in merged:
                raise RuntimeError(f"LP {k} was presolved on two ranks")
            merged[k] = v
    return [merged[k] for k in sorted(merged)]


def run_sharded(nnz, run_shard, rank, world, group=None):
    """Partitions the LPs by nnz, runs this rank's share and gathers.

    `run_shard(indices)` presolves the LPs with those indices on this rank's
    device and returns {index: record}.  Returns (all records in index order
    on rank 0, None elsewhere; this rank's indices)."""
    mine = greedy_nnz_partition(nnz, world)[rank]
    records = run_shard(mine) if mine else {}
    if set(records) != set(mine):
        raise RuntimeError("run_shard returned records for other LPs than its own")
    return gather_records(records, rank, world, group), mine
