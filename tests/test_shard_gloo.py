"""CPU, world size 2 (gloo): the object-sharded query path.

Each rank computes the exact top-k of its row shard (the oracle stands in for the
per-GPU `Table.query(..., row_begin, row_end)` call, which returns global ids), the
ranks all_gather and merge, and every rank must hold the single-process answer
bit-for-bit, ties included.
"""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from topk_b200 import shard


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


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
            merged = shard.sharded_query((ids, sc), k)
            want = O.topk_numpy(t, k, w, a)
            out.append(bool(np.array_equal(merged[0], want[0]) and
                            np.array_equal(merged[1].view(np.uint32), want[1].view(np.uint32))))
        results[rank] = all(out)
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_sharded_query_world_size_2():
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


def test_merge_and_shard_rows_helpers():
    assert [shard.shard_rows(10, r, 3) for r in range(3)] == [(0, 4), (4, 7), (7, 10)]
    a = (np.array([5, 1], np.uint64), np.array([1.0, 2.0], np.float32))
    b = (np.array([3, 0], np.uint64), np.array([2.0, 0.5], np.float32))
    ids, sc, th = shard.merge_topk([a, b], 3)
    assert ids.tolist() == [5, 3, 1] and sc.tolist() == [1.0, 2.0, 2.0] and th == 1.0
    ids, sc, th = shard.merge_topk([a, b], 10)
    assert ids.tolist() == [0, 5, 3, 1]
