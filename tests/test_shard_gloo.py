"""CPU, world size 2 (gloo): the exchange step of the object-sharded query.

Each rank fills its exchange record (topk_b200/shard.py layout: ids then scores) with
the exact top-k of its row shard -- the oracle stands in for the per-GPU
`Table.query_range_device` call -- and the ranks run the product's `exchange`
(all_gather_into_tensor of the records).  Every rank must then hold every rank's
record byte for byte, and the best k of the gathered lists (score descending, lower
id first: the merge kernel's order, restated here in numpy) must be the
single-process answer bit for bit, ties included.  The device merge kernel itself
runs in tests/test_gpu_shard.py.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from topk_b200 import shard


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _keys(scores):
    s = np.asarray(scores, np.float32)
    u = s.view(np.uint32)
    k = np.where(u & np.uint32(0x80000000), ~u, u | np.uint32(0x80000000)).astype(np.uint32)
    return np.where(np.isnan(s), np.uint32(0), k)


def merge_reference(records, counts, k, stride=None):
    """The merge kernel's order on the host (test checker): best k by (key, -id)."""
    stride = shard.record_stride(k) if stride is None else stride
    ids, sc = [], []
    for rec, c in zip(records, counts):
        ids.append(rec[: 8 * stride].view(np.uint64)[:c])
        sc.append(rec[8 * stride: 12 * stride].view(np.float32)[:c])
    ids, sc = np.concatenate(ids), np.concatenate(sc)
    comp = (_keys(sc).astype(np.uint64) << np.uint64(32)) | (np.uint64(0xFFFFFFFF) - ids)
    order = np.argsort(comp, kind="stable")[::-1][:k][::-1]
    return ids[order], sc[order]


def _worker(rank, world, port, results):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from oracle import oracle as O
    try:
        n, d = 50021, 6
        t = O.generate(n, d, O.CORRELATED, 3)  # clipped values: many ties
        O.normalize(t)
        w = O.gen_weights(d, 4, 0)
        out = []
        for attr, k in (([0, 1], 100), ([5, 2, 3], 1000), ([4], 7), ([0, 1, 2, 3, 4, 5], 4096)):
            a = np.array(attr, np.uint8)
            r0, r1 = shard.shard_rows(n, rank, world)
            ids, sc, _ = O.topk_numpy(t, k, w, a, row0=r0, row1=r1)  # global ids
            rec = torch.zeros(shard.record_bytes(k), dtype=torch.uint8)
            vi, vs = shard.record_views(rec, k)
            vi[: len(ids)] = torch.from_numpy(ids.astype(np.int64))
            vs[: len(sc)] = torch.from_numpy(sc)
            assert rec.numel() % 8 == 0
            got = shard.exchange(rec).numpy()
            counts = shard.list_counts(n, world, k)
            ok = got.shape == (world, shard.record_bytes(k)) and np.array_equal(got[rank], rec.numpy())
            mids, msc = merge_reference(got, counts, k)
            want = O.topk_numpy(t, k, w, a)
            out.append(bool(ok and np.array_equal(mids, want[0]) and
                            np.array_equal(msc.view(np.uint32), want[1].view(np.uint32))))
        results[rank] = all(out)
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_sharded_exchange_world_size_2():
    world = 2
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    results = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, results)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    assert dict(results) == {0: True, 1: True}


def test_shard_rows_and_record_layout():
    assert [shard.shard_rows(10, r, 3) for r in range(3)] == [(0, 4), (4, 7), (7, 10)]
    assert shard.list_counts(10, 3, 3).tolist() == [3, 3, 3]
    assert shard.list_counts(10, 3, 5).tolist() == [4, 3, 3]
    assert [shard.record_bytes(k) for k in (1, 2, 17)] == [24, 24, 216]  # stride rounded up to even
    rec = torch.zeros(shard.record_bytes(4), dtype=torch.uint8)
    ids, sc = shard.record_views(rec, 4)
    ids[:] = torch.tensor([5, 1, 3, 0])
    sc[:] = torch.tensor([1.0, 2.0, 2.0, 0.5])
    r = rec.numpy()
    assert r[:32].view(np.uint64).tolist() == [5, 1, 3, 0]
    assert r[32:48].view(np.float32).tolist() == [1.0, 2.0, 2.0, 0.5]
    mids, msc = merge_reference([r], [4], 3, stride=4)
    assert mids.tolist() == [5, 3, 1] and msc.tolist() == [1.0, 2.0, 2.0]
