"""GPU: the device merge of an object-sharded query (topk_merge_lists).

One process stands in for the ranks: each shard's top-k goes into its exchange
record by `Table.query_range_device`, either from a replica of the whole table (ids
already global) or from a table holding only the shard's rows (ids from 0, the merge
adds the shard's first row).  The merged result must equal the single query over the
whole table bit for bit, ties to the lower id included.
"""
import numpy as np
import pytest

import topk_b200 as T
from oracle import oracle as O
from topk_b200 import shard
from tests import helpers as H

pytestmark = pytest.mark.gpu


def _records(tables, n, world, k, w, a, replica, torch):
    recs = torch.zeros((world, shard.record_bytes(k)), dtype=torch.uint8, device="cuda")
    for r in range(world):
        r0, r1 = shard.shard_rows(n, r, world)
        ids, sc = shard.record_views(recs[r], k)
        t = tables[0] if replica else tables[r]
        off = r0 if replica else 0
        t.query_range_device(off, off + (r1 - r0), k, w, a, ids.data_ptr(), sc.data_ptr())
    torch.cuda.synchronize()
    return recs


@pytest.mark.parametrize("world", [2, 3, 5])
@pytest.mark.parametrize("dist", [0, 1, 3])
def test_merge_of_shards_equals_whole_table(world, dist):
    torch = pytest.importorskip("torch")
    n, d = (1 << 20) + 13, 8
    rng = np.random.default_rng(world * 10 + dist)
    raw = O.generate(n, d, dist, 5)
    with T.Table(n, d) as whole:
        whole.upload(raw)
        whole.normalize()
        norm = whole.download()
        parts = []
        for r in range(world):
            r0, r1 = shard.shard_rows(n, r, world)
            p = T.Table(r1 - r0, d)
            p.upload(np.ascontiguousarray(norm[:, r0:r1]))
            parts.append(p)
        try:
            for j in range(6):
                w, a = H.random_query(rng, d)
                k = int(rng.choice([1, 17, 256, 1024, 4096]))
                want = whole.query(k, w, a)
                counts = shard.list_counts(n, world, k)
                for replica in (True, False):
                    recs = _records([whole] if replica else parts, n, world, k, w, a, replica, torch)
                    bases = None if replica else [shard.shard_rows(n, r, world)[0] for r in range(world)]
                    ids, sc, th = shard.merge(recs, counts, k, bases)
                    torch.cuda.synchronize()
                    got = (ids.cpu().numpy().astype(np.uint64), sc.cpu().numpy(), float(th.cpu()[0]))
                    H.assert_same_result(got, want)
        finally:
            for p in parts:
                p.close()


def test_merge_of_tied_lists_and_short_shards():
    """Coarse values (many ties across shards) and shards shorter than k."""
    torch = pytest.importorskip("torch")
    n, d, world = 3000, 3, 4
    raw = (np.floor(O.generate(n, d, 1, 2) * 4) / 4).astype(np.float32)
    with T.Table(n, d) as whole:
        whole.upload(raw)
        whole.normalize()
        w = np.array([0.5, 0.25, 0.125], np.float32)
        a = np.array([0, 1, 2], np.uint8)
        for k in (5, 700, 1000, 4096):  # 1000 and 4096 exceed each shard's 750 rows
            want = whole.query(k, w, a)
            recs = _records([whole], n, world, k, w, a, True, torch)
            ids, sc, th = shard.merge(recs, shard.list_counts(n, world, k), k)
            torch.cuda.synchronize()
            H.assert_same_result((ids.cpu().numpy().astype(np.uint64), sc.cpu().numpy(), float(th.cpu()[0])), want)


def test_merge_rejects_bad_arguments():
    torch = pytest.importorskip("torch")
    recs = torch.zeros((2, shard.record_bytes(8)), dtype=torch.uint8, device="cuda")
    with pytest.raises(T.TopKError):
        shard.merge(recs, [9, 1], 8)  # a count above the stride
    with pytest.raises(ValueError):
        shard.merge(recs.cpu(), [1, 1], 8)  # the merge runs on the GPU only
