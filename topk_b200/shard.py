"""Object-sharded queries across processes (one process per GPU).

Each rank holds its own row range of the objects, [row_begin, row_end), and answers
it on its GPU with `Table.query_range_device`, which writes the shard's top-k (global
ids) straight into this rank's exchange record.  One all_gather over
torch.distributed (NCCL between GPUs) brings every rank's record to every rank, and
`topk_merge_lists` (one block on the device, exact radix select in the engine's order:
score descending, then the lower id) keeps the best k of the union, ascending like
the reference's result (cpu/TPAc.h:198-206).  This is the reference's merge of its
per-thread heaps (cpu/TPAc.h:335-346) with GPUs in place of threads.

Exchange record of a rank, for a query with k entries per list (stride s = k rounded up
to even, so that every record of a gathered (world, 12 s) tensor starts 8-byte aligned):
    bytes [0, 8s)     ids, uint64 (the first k valid)
    bytes [8s, 12s)   scores, float32
The number of valid entries of rank r is min(k, rows of r) -- known on every rank
from the row split, so no count is exchanged.
"""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import check


def shard_rows(n, rank, world):
    """Contiguous row range of `rank` out of `world` (sizes differ by at most 1)."""
    base, extra = divmod(n, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def record_stride(k):
    """Entries per list in a record: k rounded up to even (8-byte aligned records)."""
    return (int(k) + 1) // 2 * 2


def record_bytes(k):
    """Bytes of one rank's exchange record for lists of k entries."""
    return 12 * record_stride(k)


def record_views(rec, k):
    """(ids, scores) views of a uint8 torch record tensor of record_bytes(k) bytes; the
    first k entries of each are the list."""
    s = record_stride(k)
    return rec[: 8 * s].view(dtype=_torch().int64), rec[8 * s: 12 * s].view(dtype=_torch().float32)


def list_counts(n, world, k):
    """Valid entries of every rank's list: min(k, rows of the rank)."""
    return np.array([min(int(k), e - b) for b, e in (shard_rows(n, r, world) for r in range(world))], np.uint64)


def exchange(rec, group=None):
    """all_gather of every rank's record (uint8 tensor, same size on all ranks) into one
    (world, bytes) tensor on the record's device: NCCL between GPUs, gloo on CPU."""
    import torch.distributed as dist
    torch = _torch()
    world = dist.get_world_size(group)
    out = torch.empty(world * rec.numel(), dtype=torch.uint8, device=rec.device)
    dist.all_gather_into_tensor(out, rec, group=group)
    return out.view(world, rec.numel())


def merge(records, counts, k, bases=None, stream=0):
    """Best min(k, sum of counts) of the gathered lists on their GPU, by
    topk_merge_lists.  records: (world, 12 * stride) uint8 CUDA tensor; bases: each
    list's first global id (None: ids already global).  Returns (ids int64, scores
    float32, threshold float32) CUDA tensors, ascending."""
    torch = _torch()
    if not records.is_cuda:
        raise ValueError("merge runs on the GPU: the gathered records must be a CUDA tensor")
    world, nbytes = records.shape
    stride = nbytes // 12
    k = int(k)
    dev = records.device
    ids = torch.empty(k, dtype=torch.int64, device=dev)
    sc = torch.empty(k, dtype=torch.float32, device=dev)
    th = torch.empty(1, dtype=torch.float32, device=dev)
    kept = C.c_uint64()
    cnt = np.ascontiguousarray(counts, np.uint64)
    base = np.zeros(world, np.uint64) if bases is None else np.ascontiguousarray(bases, np.uint64)
    check(_lib.load().topk_merge_lists(dev.index, C.c_void_p(records.data_ptr()), world, stride, cnt, base, k,
                                       C.c_void_p(ids.data_ptr()), C.c_void_p(sc.data_ptr()),
                                       C.c_void_p(th.data_ptr()), C.byref(kept), C.c_void_p(stream or None)))
    c = kept.value
    return ids[:c], sc[:c], th


def sharded_query(table, n, k, weights, attr, group=None, stream=0):
    """Exact top-k of an object-sharded table: this rank's `table` holds the global
    table's rows shard_rows(n, rank, world) (or the whole table: only this rank's
    rows are scanned).  Every rank returns the same result (CUDA tensors)."""
    import torch.distributed as dist
    torch = _torch()
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    r0, r1 = shard_rows(n, rank, world)
    local_rows = table.n
    # a shard table holds its rows from 0; a replica holds them at their global place
    off = 0 if local_rows < n else r0
    # the scan, the collective and the merge in order on one stream (a stream of its
    # own unless the caller passes one: handle 0 would name the table's own stream)
    s = torch.cuda.ExternalStream(stream) if stream else torch.cuda.Stream()
    with torch.cuda.stream(s):
        rec = torch.zeros(record_bytes(k), dtype=torch.uint8, device="cuda")
        ids, sc = record_views(rec, k)
        table.query_range_device(off, off + (r1 - r0), k, weights, attr, ids.data_ptr(), sc.data_ptr(), 0,
                                 s.cuda_stream)
        gathered = exchange(rec, group)
        # a shard table numbers its rows from 0: the merge adds each shard's first row
        bases = None if local_rows >= n else [shard_rows(n, r, world)[0] for r in range(world)]
        return merge(gathered, list_counts(n, world, k), k, bases, s.cuda_stream)


def _torch():
    import torch
    return torch
