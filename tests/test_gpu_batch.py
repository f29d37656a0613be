"""GPU: the batched multi-query path (topk_query_batch) against the oracle.

The reference answers many queries with its multi-query loop
(validation/bench_cpu.h:198-232 -> TPAc::findTopKsimdMQ); the batched path scores
each staged table tile for a group of queries.  Every query must match the oracle
bit-exactly, whichever batch method runs.
"""
import numpy as np
import pytest

import topk_b200 as T
from oracle import oracle as O
from tests import helpers as H

pytestmark = pytest.mark.gpu

LOOP, FP32 = 1, 2


def make_batch(rng, nq, d, kmax, qmax=16, ordered=False):
    W = np.zeros((nq, d), np.float32)
    A = np.zeros((nq, max(qmax, 1)), np.uint8)
    qqs = np.zeros(nq, np.uint32)
    ks = rng.integers(1, kmax + 1, size=nq).astype(np.uint64)
    for j in range(nq):
        w, a = H.random_query(rng, d, qmax=min(qmax, d), ordered=ordered)
        W[j] = w
        A[j, : len(a)] = a
        qqs[j] = len(a)
    return ks, W, A, qqs


def check_batch(t, tn, ks, W, A, qqs):
    ids, sc, counts, ths = t.query_batch(ks, W, A, qqs)
    for j in range(len(ks)):
        c = int(counts[j])
        want = O.topk_numpy(tn, int(ks[j]), W[j], A[j, : qqs[j]])
        H.assert_same_result((ids[j, :c], sc[j, :c], ths[j]), want)
    return ids, sc, counts, ths


@pytest.mark.parametrize("n,dist", [((1 << 20) + 77, 1), (300000, 0), (250001, 2), ((1 << 19) + 5, 3)])
def test_batch_fp32_vs_oracle(n, dist):
    d = 16
    rng = np.random.default_rng(n)
    with T.Table(n, d) as t:
        t.generate(dist, 5)
        t.normalize()
        tn = t.download()
        t.set_batch_method(FP32)
        ks, W, A, qqs = make_batch(rng, 150, d, 1024)
        ks[:3] = [1, 1024, 4096]
        check_batch(t, tn, ks, W, A, qqs)
        st = t.last_batch_stats()
        assert st["device_ms"] > 0 and st["fallbacks"] == 0


def test_batch_methods_agree_and_loop_path():
    n, d = 200000, 12
    rng = np.random.default_rng(1)
    with T.Table(n, d) as t:
        t.generate(1, 9)
        t.normalize()
        ks, W, A, qqs = make_batch(rng, 40, d, 700, ordered=True)
        t.set_batch_method(FP32)
        a = t.query_batch(ks, W, A, qqs)
        t.set_batch_method(LOOP)
        b = t.query_batch(ks, W, A, qqs)
        for x, y in zip(a, b):
            assert np.array_equal(np.asarray(x).view(np.uint8), np.asarray(y).view(np.uint8))


def test_batch_small_tables_and_k_above_n():
    rng = np.random.default_rng(2)
    for n in (1, 7, 100, 8191, 8192, 8193):
        d = 4
        with T.Table(n, d) as t:
            t.generate(1, n)
            t.normalize()
            tn = t.download()
            t.set_batch_method(FP32)
            ks, W, A, qqs = make_batch(rng, 9, d, 300, qmax=4)
            ks[0] = min(n + 5, T.MAX_K)
            check_batch(t, tn, ks, W, A, qqs)


def test_batch_overflow_falls_back_exactly():
    """Scores increasing with the id: every chunk beats every earlier object, so the
    candidate regions overflow; those queries are answered by the exact scan."""
    n, d = 400003, 3
    raw = np.tile(np.linspace(0, 1, n, dtype=np.float32), (d, 1))
    tn = raw.copy()
    O.normalize(tn)
    with T.Table(n, d) as t:
        t.upload(raw)
        t.normalize()
        t.set_batch_method(FP32)
        ks = np.array([5, 700, 4096], np.uint64)
        W = np.ones((3, d), np.float32)
        A = np.array([[0, 1, 2], [2, 0, 1], [1, 1, 1]], np.uint8)
        qqs = np.array([3, 3, 3], np.uint32)
        check_batch(t, tn, ks, W, A, qqs)
        assert t.last_batch_stats()["fallbacks"] >= 1


def test_batch_ties_and_wide_queries():
    n, d = 120000, 40
    rng = np.random.default_rng(3)
    raw = (np.floor(O.generate(n, d, 0, 4) * 8) / 8).astype(np.float32)  # coarse: many ties
    tn = raw.copy()
    O.normalize(tn)
    with T.Table(n, d) as t:
        t.upload(raw)
        t.normalize()
        t.set_batch_method(FP32)
        ks, W, A, qqs = make_batch(rng, 30, d, 2000, qmax=32)
        check_batch(t, tn, ks, W, A, qqs)
        # qq above the batched limit (32): the batch runs the per-query scan instead
        W2 = W[:2].copy()
        A2 = np.tile(np.arange(d, dtype=np.uint8), (2, 1))
        check_batch(t, tn, ks[:2], W2, A2, np.array([40, 33], np.uint32))
