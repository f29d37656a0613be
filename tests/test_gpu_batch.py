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


# ---------------------------------------------------------------- BF16 filter
BF16 = 3


def bf16_ran(t):
    """The last batch ran the tensor-core filter, and every rescored candidate's
    filter score was within half of its error bound."""
    st = t.last_batch_stats()
    assert st["method"] == BF16
    assert 0.0 < st["max_err_ratio"] < 0.5, st
    return st


@pytest.mark.parametrize("n,dist,d", [((1 << 20) + 77, 1, 16), (300000, 0, 16), (250001, 2, 16),
                                      ((1 << 19) + 5, 3, 16), (200003, 1, 8), (100000, 1, 3)])
def test_batch_bf16_vs_oracle(n, dist, d):
    rng = np.random.default_rng(n + d)
    with T.Table(n, d) as t:
        t.generate(dist, 7)
        t.normalize()
        tn = t.download()
        t.set_batch_method(BF16)
        ks, W, A, qqs = make_batch(rng, 150, d, 1024, qmax=min(16, d))
        ks[:3] = [1, 1024, 4096]
        ids, sc, counts, _ = check_batch(t, tn, ks, W, A, qqs)
        st = bf16_ran(t)
        if dist == 1:
            # independent values do not tie at the threshold; clipped correlated values
            # do (many objects at exactly 1.0), and such a query may overflow its
            # candidate region and be answered by the exact scan: results identical
            assert st["fallbacks"] == 0
        # FP32 scores against an FP64 evaluation of the same ids (reported, bounded)
        worst = 0.0
        for j in range(0, len(ks), 15):
            c = int(counts[j])
            a = A[j, : qqs[j]]
            s64 = sum(tn[m][ids[j, :c].astype(np.int64)].astype(np.float64) * np.float64(W[j][m]) for m in a)
            worst = max(worst, float(np.max(np.abs(sc[j, :c].astype(np.float64) - s64))))
        print(f"max |score_fp32 - score_fp64| = {worst:.3e}")
        assert worst < 16 * 2.0 ** -24 * 16


def test_batch_bf16_matches_fp32_across_query_groups():
    """2100 queries = 17 query tiles: two CTA query groups, a partial last tile."""
    n, d = (1 << 18) + 3, 16
    rng = np.random.default_rng(11)
    with T.Table(n, d) as t:
        t.generate(3, 2)
        t.normalize()
        tn = t.download()
        ks, W, A, qqs = make_batch(rng, 2100, d, 1024)
        t.set_batch_method(BF16)
        a = t.query_batch(ks, W, A, qqs)
        bf16_ran(t)
        t.set_batch_method(FP32)
        b = t.query_batch(ks, W, A, qqs)
        assert t.last_batch_stats()["method"] == FP32
        for x, y in zip(a, b):
            assert np.array_equal(np.asarray(x).view(np.uint8), np.asarray(y).view(np.uint8))
        for j in rng.choice(len(ks), size=40, replace=False):
            c = int(a[2][j])
            want = O.topk_numpy(tn, int(ks[j]), W[j], A[j, : qqs[j]])
            H.assert_same_result((a[0][j, :c], a[1][j, :c], a[3][j]), want)


def test_batch_bf16_ties_negative_and_repeated_attributes():
    n, d = 150001, 16
    rng = np.random.default_rng(5)
    raw = (np.floor(O.generate(n, d, 1, 8) * 16) / 16).astype(np.float32)  # coarse: many ties
    tn = raw.copy()
    O.normalize(tn)
    with T.Table(n, d) as t:
        t.upload(raw)
        t.normalize()
        t.set_batch_method(BF16)
        nq = 60
        W = rng.uniform(-1, 1, size=(nq, d)).astype(np.float32)
        A = np.zeros((nq, 6), np.uint8)
        qqs = np.zeros(nq, np.uint32)
        for j in range(nq):
            q = int(rng.integers(1, 7))
            A[j, :q] = rng.integers(0, d, size=q)  # repeats allowed, any order
            qqs[j] = q
        ks = rng.integers(1, 2000, size=nq).astype(np.uint64)
        ids, sc, counts, ths = t.query_batch(ks, W, A, qqs)
        bf16_ran(t)
        for j in range(nq):
            c = int(counts[j])
            want = O.topk(tn, int(ks[j]), W[j], A[j, : qqs[j]])
            H.assert_same_result((ids[j, :c], sc[j, :c], ths[j]), want)


def test_batch_bf16_not_applicable_runs_fp32():
    rng = np.random.default_rng(6)
    # wider than 16 attributes
    with T.Table(70000, 20) as t:
        t.generate(1, 3)
        t.normalize()
        tn = t.download()
        t.set_batch_method(BF16)
        ks, W, A, qqs = make_batch(rng, 20, 20, 500)
        check_batch(t, tn, ks, W, A, qqs)
        assert t.last_batch_stats()["method"] == FP32
    # a value above 2^60 in the table, then a weight above 2^60
    n, d = 70000, 8
    raw = O.generate(n, d, 1, 4)
    raw[3, 1234] = np.float32(1e30)
    with T.Table(n, d) as t:
        t.upload(raw)
        t.set_batch_method(0)
        ks, W, A, qqs = make_batch(rng, 20, d, 500, qmax=d)
        check_batch(t, raw, ks, W, A, qqs)
        assert t.last_batch_stats()["method"] == FP32
        t.generate(1, 4)
        tn = t.download()
        check_batch(t, tn, ks, W, A, qqs)
        assert t.last_batch_stats()["method"] == BF16  # the table changed: the split was rebuilt
        W2 = W.copy()
        W2[0, A[0, 0]] = np.float32(1e20)
        check_batch(t, tn, ks, W2, A, qqs)
        assert t.last_batch_stats()["method"] == FP32


def test_batch_bf16_overflow_falls_back_exactly():
    n, d = 400003, 3
    raw = np.tile(np.linspace(0, 1, n, dtype=np.float32), (d, 1))
    tn = raw.copy()
    O.normalize(tn)
    with T.Table(n, d) as t:
        t.upload(raw)
        t.normalize()
        t.set_batch_method(BF16)
        ks = np.array([5, 700, 4096], np.uint64)
        W = np.ones((3, d), np.float32)
        A = np.array([[0, 1, 2], [2, 0, 1], [1, 1, 1]], np.uint8)
        qqs = np.array([3, 3, 3], np.uint32)
        check_batch(t, tn, ks, W, A, qqs)
        st = t.last_batch_stats()
        # dense scores: the filter hands the queries to the exact FP32 scorer
        assert st["method"] == BF16 and st["switched_fp32"] >= 1


def test_batch_bf16_hybrid_redoes_discarded_chunks():
    """Objects just below the top score (inside the filter's error band, below the
    exact threshold) fill the candidate regions under the filter in a middle chunk
    (rows [32768, 65536)) and in the last one; the filter loses candidates there, the
    query moves to the exact FP32 scorer, which answers the discarded chunk again
    (with the next chunk, and after the loop for the last one): exact results."""
    n, d = 100003, 3
    rng = np.random.default_rng(11)
    raw = (rng.integers(0, 1 << 23, size=(d, n)) * 2.0 ** -24).astype(np.float32)  # [0, 0.5)
    raw[:, 0] = 0.0
    raw[:, 100:110] = 1.0  # the top, in the bootstrap rows
    near = np.float32(1.0 - 2.0 ** -20)
    raw[:, 40000:45000] = near
    raw[:, 70000:75000] = near
    tn = raw.copy()
    O.normalize(tn)
    with T.Table(n, d) as t:
        t.upload(raw)
        t.normalize()
        t.set_batch_method(BF16)
        ks = np.array([5, 10, 64, 3000], np.uint64)
        W = np.ones((4, d), np.float32)
        A = np.tile(np.arange(d, dtype=np.uint8), (4, 1))
        qqs = np.full(4, d, np.uint32)
        check_batch(t, tn, ks, W, A, qqs)
        st = t.last_batch_stats()
        assert st["method"] == BF16 and st["switched_fp32"] >= 1


def test_batch_tune_keeps_results():
    """The autotuner tries its tiles on the caller's queries, keeps the fastest in the
    handle and reports it; batches afterwards return the same exact results."""
    rng = np.random.default_rng(21)
    n, d = 300007, 16
    with T.Table(n, d) as t:
        t.generate(1, 5)
        t.normalize()
        tn = t.download()
        t.set_batch_method(BF16)
        ks, W, A, qqs = make_batch(rng, 300, d, 1024, qmax=16)
        rep = t.tune_batch(ks, W, A, qqs)
        assert rep["query_tiles_per_cta"] in (4, 8, 16) and rep["boot_rows"] in (8192, 16384)
        assert 0 < rep["best_ms"] <= rep["default_ms"]
        qt, boot = t.batch_tiles()
        assert (qt or 16) == rep["query_tiles_per_cta"] and boot == rep["boot_rows"]
        check_batch(t, tn, ks, W, A, qqs)
        bf16_ran(t)
        t.set_batch_tiles(8, 16384)
        check_batch(t, tn, ks, W, A, qqs)
        with pytest.raises(T.TopKError):
            t.set_batch_tiles(4, 1000)


def test_batch_bf16_retires_queries_tied_at_the_maximum():
    """Many rows hold the largest possible score (every queried value at its column
    maximum): once k of them are found the k-th score equals the bound over the
    column extremes, so the filter retires the query instead of passing every later
    tied row (which would overflow its candidates).  Results exact, lowest ids."""
    n, d = 300001, 6
    rng = np.random.default_rng(31)
    raw = (rng.integers(0, 1 << 22, size=(d, n)) * 2.0 ** -23).astype(np.float32)  # [0, 0.5)
    raw[:, ::37] = 1.0  # ~8100 rows at the top in every attribute
    raw[0, 5] = 0.0     # one column minimum of 0 (normalisation keeps the range)
    tn = raw.copy()
    O.normalize(tn)
    with T.Table(n, d) as t:
        t.upload(raw)
        t.normalize()
        t.set_batch_method(BF16)
        nq = 300
        ks = rng.integers(1, 1025, size=nq).astype(np.uint64)
        W = ((rng.integers(0, 1 << 24, size=(nq, d)) + 1) * 2.0 ** -24).astype(np.float32)
        A = np.zeros((nq, d), np.uint8)
        qqs = np.zeros(nq, np.uint32)
        for j in range(nq):
            q = int(rng.integers(1, d + 1))
            A[j, :q] = rng.choice(d, size=q, replace=False)
            qqs[j] = q
        check_batch(t, tn, ks, W, A, qqs)
        st = bf16_ran(t)
        assert st["retired"] == nq and st["switched_fp32"] == 0, st


def test_batch_c5_shaped_mixed_table():
    """The full chosen form's shape at 2^22 rows: a table mixed 1/3 each independent,
    correlated and anticorrelated, 2048 queries with 2-16 attributes and k log-uniform
    in [1, 1024].  The clipped correlated rows tie at the maximum for most small
    queries; those retire, and few queries move to the FP32 scorer.  Every method
    returns the plain FP32 batch's results; a sample is checked against the oracle."""
    n, d, nq = 1 << 22, 16, 2048
    rng = np.random.default_rng(55)
    ks = np.exp(rng.uniform(0.0, np.log(1025.0), nq)).astype(np.uint64).clip(1, 1024)
    W = ((rng.integers(0, 1 << 24, size=(nq, d)) + 1) * 2.0 ** -24).astype(np.float32)
    A = np.zeros((nq, 16), np.uint8)
    qqs = np.zeros(nq, np.uint32)
    for j in range(nq):
        q = int(rng.integers(2, 17))
        A[j, :q] = np.sort(rng.choice(d, size=q, replace=False))
        qqs[j] = q
    with T.Table(n, d) as t:
        t.generate(3, 12)
        t.normalize()
        tn = t.download()
        t.set_batch_method(FP32)
        base = t.query_batch(ks, W, A, qqs)
        t.set_batch_method(BF16)
        got = t.query_batch(ks, W, A, qqs)
        st = bf16_ran(t)
        for x, y in zip(base, got):
            assert np.array_equal(np.asarray(x).view(np.uint8), np.asarray(y).view(np.uint8))
        assert st["switched_fp32"] < nq // 4, st
        assert st["retired"] > nq // 4, st
        for j in rng.choice(nq, size=24, replace=False):
            c = int(got[2][j])
            want = O.topk_numpy(tn, int(ks[j]), W[j], A[j, : qqs[j]])
            H.assert_same_result((got[0][j, :c], got[1][j, :c], got[3][j]), want)
