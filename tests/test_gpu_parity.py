"""GPU parity: the CUDA path through the C ABI against the oracle and the
reference's own recorded outputs, on seeded inputs at sizes the oracle handles
in seconds.  Bar: bit-exact ids, scores and thresholds.
"""
import hashlib
import threading

import numpy as np
import pytest

import topk_b200 as T
from oracle import oracle as O
from tests import helpers as H

pytestmark = pytest.mark.gpu

CASES = H.golden()["cases"]


def _table_from(raw):
    d, n = raw.shape
    t = T.Table(n, d)
    t.upload(raw)
    return t


# ----------------------------------------------------------------------------- data
@pytest.mark.parametrize("dist", [0, 1, 2, 3])
@pytest.mark.parametrize("n,d", [(4099, 8), (1000, 13), (1 << 16, 16), (7, 2)])
def test_generator_bit_exact(dist, n, d):
    with T.Table(n, d) as t:
        t.generate(dist, 123 + dist)
        got = t.download()
    want = O.generate(n, d, dist, 123 + dist)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("c", [c for c in CASES if c["n"] <= (1 << 17)][:24] + [CASES[0]],
                         ids=lambda c: c["name"])
def test_normalize_matches_reference(c):
    raw = H.case_table(c)
    with _table_from(raw) as t:
        mins, maxs = t.normalize()
        got = t.download()
    assert hashlib.sha256(got.tobytes()).hexdigest() == c["table_sha256"]
    want = raw.copy()
    omin, omax = O.normalize(want)
    assert np.array_equal(mins.view(np.uint32), omin.view(np.uint32))
    assert np.array_equal(maxs.view(np.uint32), omax.view(np.uint32))


def test_normalize_edge_values():
    """Signed zeros, negatives, infinities, NaN and a constant column."""
    n = 1031
    raw = np.random.default_rng(1).random((6, n)).astype(np.float32)
    raw[0, 5] = -0.0
    raw[0, 9] = 0.0
    raw[0, :] = np.abs(raw[0, :])
    raw[0, 5] = -0.0  # first zero is negative
    raw[1, :] = np.abs(raw[1, :])
    raw[1, 3] = 0.0
    raw[1, 700] = -0.0  # first zero is positive
    raw[2, :] -= 2.0  # all negative: max stays +0
    raw[3, 17] = np.inf
    raw[3, 18] = np.nan
    raw[4, :] = 0.25  # constant: 0/0 -> NaN everywhere
    raw[5, 100] = -np.inf
    with _table_from(raw) as t:
        mins, maxs = t.normalize()
        got = t.download()
    want = raw.copy()
    omin, omax = O.normalize(want)
    assert np.array_equal(mins.view(np.uint32), omin.view(np.uint32))
    assert np.array_equal(maxs.view(np.uint32), omax.view(np.uint32))
    nan_g, nan_w = np.isnan(got), np.isnan(want)
    assert np.array_equal(nan_g, nan_w)  # NaN payload bits may differ between CPU and GPU
    assert np.array_equal(got[~nan_g].view(np.uint32), want[~nan_w].view(np.uint32))


# ----------------------------------------------------------------------------- queries
@pytest.mark.parametrize("c", CASES, ids=[c["name"] for c in CASES])
def test_query_matches_reference_golden(c):
    raw = H.case_table(c)
    tn = raw.copy()
    O.normalize(tn)
    w = H.case_weights(c)
    attr = np.array(c["attr"], np.uint8)
    with _table_from(raw) as t:
        t.normalize()
        got = t.query(c["k"], w, attr)
    # bit-exact against the oracle (same tie rule) ...
    H.assert_same_result(got, O.topk(tn, c["k"], w, attr))
    # ... and against every recorded reference implementation run
    for run in c["runs"].values():
        H.assert_matches_reference(*got, run, tn, w, attr)


@pytest.mark.parametrize("n", [1, 3, 17, 255, 1000, 4097, (1 << 18) + 5, 1 << 20])
def test_query_random_vs_oracle(n):
    rng = np.random.default_rng(n)
    d = 16
    with T.Table(n, d) as t:
        t.generate(int(n % 4), 9)
        t.normalize()
        tn = t.download()
        for j in range(10):
            w, attr = H.random_query(rng, d, ordered=bool(j % 2))
            k = int(rng.choice([1, 2, 5, 16, 64, 100, 256, 1000, 1024, 4096]))
            H.assert_same_result(t.query(k, w, attr), O.topk_numpy(tn, k, w, attr))


def test_query_duplicate_and_many_attributes():
    rng = np.random.default_rng(3)
    n, d = 50000, 40
    with T.Table(n, d) as t:
        t.generate(1, 4)
        t.normalize()
        tn = t.download()
        w = O.gen_weights(d, 5, 0)
        for attr in ([3, 3, 3], [0, 5, 0, 5], list(range(40)) + list(range(24)), [39, 0]):
            a = np.array(attr, np.uint8)
            H.assert_same_result(t.query(77, w, a), O.topk_numpy(tn, 77, w, a))
        for q in (17, 32, 64):
            a = rng.integers(0, d, size=q).astype(np.uint8)
            H.assert_same_result(t.query(300, w, a), O.topk_numpy(tn, 300, w, a))


@pytest.mark.parametrize("r0,r1", [(0, 1), (3, 4097), (100, 100 + 2048), (65535, 1 << 17), (1 << 16, 1 << 16)])
def test_range_queries(r0, r1):
    n, d = 1 << 17, 8
    with T.Table(n, d) as t:
        t.generate(2, 21)
        t.normalize()
        tn = t.download()
        w = O.gen_weights(d, 22, 0)
        a = np.array([1, 4, 6], np.uint8)
        for k in (1, 33, 1024):
            got = t.query(k, w, a, row_begin=r0, row_end=r1)
            if r1 == r0:
                assert len(got[0]) == 0
                continue
            H.assert_same_result(got, O.topk(tn, k, w, a, row0=r0, row1=r1))


def test_adversarial_orders_and_ties():
    """Scores increasing with id (every object improves the top-k), all-equal
    scores (pure tie-breaking), and coarse values with many ties."""
    n, d = 200003, 3
    inc = np.tile(np.linspace(0, 1, n, dtype=np.float32), (d, 1))
    dec = inc[:, ::-1].copy()
    flat = np.full((d, n), 0.5, np.float32)
    flat[:, 0] = 0.0
    flat[:, 1] = 1.0  # keeps the columns non-constant
    coarse = (np.floor(O.generate(n, d, 1, 2) * 4) / 4).astype(np.float32)
    w = np.array([0.5, 0.25, 1.0], np.float32)
    a = np.array([0, 1, 2], np.uint8)
    for raw in (inc, dec, flat, coarse):
        tn = raw.copy()
        O.normalize(tn)
        with _table_from(raw) as t:
            t.normalize()
            for k in (1, 16, 1000, 4096):
                H.assert_same_result(t.query(k, w, a), O.topk_numpy(tn, k, w, a))


def test_queries_after_high_scoring_ones_stay_exact():
    """A query with low scores right after queries with high ones, few tiles per CTA:
    every CTA's threshold copies must start from this query's own bounds (a slot left
    unset once held the previous kernel's shared-memory contents, a threshold far
    above this query's k-th score)."""
    n, d = 1 << 20, 8
    rng = np.random.default_rng(21)
    with T.Table(n, d) as t:
        t.generate(1, 4)
        t.normalize()
        tn = t.download()
        w = (0.1 * np.arange(1, d + 1)).astype(np.float32)
        for rep in range(3):
            for k in (16, 64, 256, 1024):
                for q in (8, 6, 2, 1, 2):
                    a = np.arange(d - q, d, dtype=np.uint8)
                    if rep == 2:
                        a = np.sort(rng.choice(d, q, replace=False)).astype(np.uint8)
                    H.assert_same_result(t.query(k, w, a)[:3], O.topk_numpy(tn, k, w, a))


def test_nan_scores_rank_last():
    n, d = 5000, 2
    raw = O.generate(n, d, 1, 8)
    raw[1, :] = 0.75  # constant column -> NaN after normalisation
    tn = raw.copy()
    O.normalize(tn)
    with _table_from(raw) as t:
        t.normalize()
        w = np.ones(2, np.float32)
        got = t.query(10, w, np.array([0, 1], np.uint8))
        assert np.isnan(got[1]).all()
        assert got[0].tolist() == list(range(9, -1, -1))  # NaN ties: lowest ids, listed ascending
        got2 = t.query(10, w, np.array([0], np.uint8))
        H.assert_same_result(got2, O.topk(tn, 10, w, np.array([0], np.uint8)))


def test_argument_errors():
    with T.Table(1000, 4) as t:
        w = np.ones(4, np.float32)
        with pytest.raises(T.TopKError) as e:
            t.query(5, w, [0, 1])
        assert e.value.status == 6  # no data yet
        t.generate(1, 1)
        t.normalize()
        for k, a, st in ((0, [0], 1), (T.MAX_K + 1, [0], 5), (5, [4], 1), (5, [], 1)):
            with pytest.raises(T.TopKError) as e:
                t.query(k, w, a)
            assert e.value.status == st
        with pytest.raises(ValueError):
            t.query(5, np.ones(2, np.float32), [0])
        ids, sc, th = t.query(5, w, [0])  # still usable
        assert len(ids) == 5


def test_k_larger_than_n():
    with T.Table(10, 2) as t:
        t.generate(1, 3)
        t.normalize()
        tn = t.download()
        w = np.ones(2, np.float32)
        a = np.array([0, 1], np.uint8)
        got = t.query(100, w, a)
        assert len(got[0]) == 10
        H.assert_same_result(got, O.topk(tn, 100, w, a))


# ----------------------------------------------------------------------------- API surfaces
def test_tpac_mirror_on_config_c1():
    """The reference harness call sequence (validation/bench_cpu.h:155-195) on C1."""
    c = CASES[0]
    assert c["name"] == "C1"
    raw = H.case_table(c)
    tp = T.TPAc(c["n"], c["d"])
    tp.get_cdata()[...] = raw
    tp.init()
    w = H.case_weights(c)
    for fn in (tp.findTopKscalar, tp.findTopKsimd, tp.findTopKthreads):
        fn(c["k"], len(c["attr"]), w, np.array(c["attr"], np.uint8))
        ids = np.array([r[0] for r in tp.get_res()], np.uint64)
        sc = np.array([r[1] for r in tp.get_res()], np.float32)
        for run in c["runs"].values():
            tn = raw.copy()
            O.normalize(tn)
            H.assert_matches_reference(ids, sc, tp.get_thres(), run, tn, w, np.array(c["attr"], np.uint8))
    tp.close()


def test_concurrent_mq_callers():
    """findTopKsimdMQ from many threads at once on one object (bench_cpu.h:204-212)."""
    n, d = 1 << 18, 8
    tp = T.TPAc(n, d)
    tp.init_generated(1, 31)
    tn = tp.table.download()
    rng = np.random.default_rng(0)
    queries = [H.random_query(rng, d) + (int(rng.integers(1, 500)),) for _ in range(32)]
    errors = []

    def worker(tid):
        try:
            for j in range(tid, len(queries), 8):
                w, a, k = queries[j]
                tp.findTopKsimdMQ(k, len(a), w, a, tid)
                got = tp.get_mq_res(tid)
                H.assert_same_result(got, O.topk_numpy(tn, k, w, a))
        except Exception as e:  # pragma: no cover - reported below
            errors.append(e)

    th = [threading.Thread(target=worker, args=(i,)) for i in range(8)]
    for x in th:
        x.start()
    for x in th:
        x.join()
    tp.close()
    assert not errors, errors[0]


def test_batch_api_vs_oracle():
    n, d = 1 << 17, 16
    rng = np.random.default_rng(4)
    with T.Table(n, d) as t:
        t.generate(3, 5)
        t.normalize()
        tn = t.download()
        nq = 12
        W = np.zeros((nq, d), np.float32)
        A = np.zeros((nq, d), np.uint8)
        qqs = np.zeros(nq, np.uint32)
        ks = rng.integers(1, 1025, size=nq).astype(np.uint64)
        for j in range(nq):
            w, a = H.random_query(rng, d)
            W[j] = w
            A[j, : len(a)] = a
            qqs[j] = len(a)
        ids, sc, counts, ths = t.query_batch(ks, W, A, qqs)
        for j in range(nq):
            c = int(counts[j])
            want = O.topk_numpy(tn, int(ks[j]), W[j], A[j, : qqs[j]])
            H.assert_same_result((ids[j, :c], sc[j, :c], ths[j]), want)


def test_device_api_with_torch_buffers():
    torch = pytest.importorskip("torch")
    n, d = 1 << 16, 8
    with T.Table(n, d) as t:
        t.generate(0, 6)
        t.normalize()
        tn = t.download()
        w = O.gen_weights(d, 7, 0)
        a = np.array([7, 2, 5], np.uint8)
        k = 300
        ids = torch.empty(k, dtype=torch.int64, device="cuda")
        sc = torch.empty(k, dtype=torch.float32, device="cuda")
        th = torch.empty(1, dtype=torch.float32, device="cuda")
        s = torch.cuda.current_stream()
        t.query_device(k, w, a, ids.data_ptr(), sc.data_ptr(), th.data_ptr(), s.cuda_stream)
        s.synchronize()
        got = (ids.cpu().numpy().astype(np.uint64), sc.cpu().numpy(), float(th.cpu()[0]))
        H.assert_same_result(got, O.topk_numpy(tn, k, w, a))


def test_bounded_wait_timeout_is_reported_and_recoverable():
    """Host-side fault injection: the scan waits on a barrier nothing completes;
    the bounded wait runs out, the call returns TOPK_ERR_TIMEOUT, and the same
    handle answers correctly afterwards."""
    n, d = 1 << 16, 4
    with T.Table(n, d) as t:
        t.generate(1, 2)
        t.normalize()
        tn = t.download()
        w = np.ones(4, np.float32)
        a = np.array([0, 1], np.uint8)
        t.set_wait_limit(2000)
        t.set_fault_injection(1)
        with pytest.raises(T.TopKError) as e:
            t.query(10, w, a)
        assert e.value.status == 4
        t.set_fault_injection(0)
        t.set_wait_limit(0)
        H.assert_same_result(t.query(10, w, a), O.topk(tn, 10, w, a))


def test_scan_stats_reported():
    with T.Table(1 << 18, 4) as t:
        t.generate(1, 3)
        t.normalize()
        t.query(64, np.ones(4, np.float32), [0, 1, 2, 3])
        cands, reds = t.last_stats()
        assert 64 <= cands <= 148 * 4 * 4096
        assert reds >= 0


def test_scan_tuning_does_not_change_results():
    """The CTAs-per-SM cap (grid size, merge-tree shape) is a performance knob only."""
    n, d = (1 << 20) + 12, 16
    rng = np.random.default_rng(9)
    with T.Table(n, d) as t:
        t.generate(3, 12)
        t.normalize()
        tn = t.download()
        w, a = H.random_query(rng, d)
        want = O.topk_numpy(tn, 200, w, a)
        for ctas in (1, 2, 3, 8, 0):
            t.set_scan_tuning(ctas)
            for q in (1, 2, 5, 12, 16, 17):
                aq = (np.arange(q) % d).astype(np.uint8)  # q = 17 repeats attribute 0
                H.assert_same_result(t.query(77, w, aq), O.topk_numpy(tn, 77, w, aq))
            H.assert_same_result(t.query(200, w, a), want)
            H.assert_same_result(t.query(4096, w, a), O.topk_numpy(tn, 4096, w, a))
        with pytest.raises(T.TopKError):
            t.set_scan_tuning(9)
