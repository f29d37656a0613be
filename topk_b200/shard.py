"""Object-sharded queries across processes (one process per GPU).

Each rank holds rows [row_begin, row_end) of the table (or a replica and a row
range) and answers its shard with `Table.query(..., row_begin, row_end)`, which
returns global ids.  The shards' top-k lists are exchanged with one all_gather over
torch.distributed (NCCL between GPUs, gloo on CPU) and merged with the engine's
order: score descending, then lower id; the output is ascending like the
reference's result (cpu/TPAc.h:198-206).
"""
import numpy as np


def score_keys(scores):
    """Order-preserving uint32 keys of float32 scores (NaN -> 0, below every number)."""
    s = np.asarray(scores, np.float32)
    u = s.view(np.uint32)
    k = np.where(u & np.uint32(0x80000000), ~u, u | np.uint32(0x80000000)).astype(np.uint32)
    return np.where(np.isnan(s), np.uint32(0), k)


def merge_topk(parts, k):
    """Merge per-shard (ids, scores) lists into the global top-k.

    Returns (ids uint64, scores float32, threshold) ascending by (score, -id)."""
    ids = np.concatenate([np.asarray(p[0], np.uint64) for p in parts]) if parts else np.zeros(0, np.uint64)
    sc = np.concatenate([np.asarray(p[1], np.float32) for p in parts]) if parts else np.zeros(0, np.float32)
    if len(ids) == 0:
        return ids, sc, 0.0
    comp = (score_keys(sc).astype(np.uint64) << np.uint64(32)) | (np.uint64(0xFFFFFFFF) - ids)
    order = np.argsort(comp, kind="stable")[::-1][:k][::-1]
    return ids[order], sc[order], float(sc[order[0]])


def shard_rows(n, rank, world):
    """Contiguous row range of `rank` out of `world` (sizes differ by at most 1)."""
    base, extra = divmod(n, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def sharded_query(local_topk, k, group=None):
    """Gather every rank's local top-k (ids, scores) and merge them on all ranks.

    local_topk: this rank's (ids, scores) for its rows.  Uses all_gather_object, so
    it works with NCCL and gloo process groups alike."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    mine = (np.asarray(local_topk[0], np.uint64), np.asarray(local_topk[1], np.float32))
    gathered = [None] * world
    dist.all_gather_object(gathered, mine, group=group)
    return merge_topk(gathered, k)
