"""GPU: the partitioned copy and pruned exact queries against the oracle.

The reference prunes with per-block bounds and stops once the k-th score reaches
the bound of the rest (cpu/VTA.h:210-216, cpu/PTA.h:337-340); here whole
partitions are skipped by the same rule.  Results must equal the plain exact
top-k bit for bit, with or without a predicted cut.
"""
import numpy as np
import pytest

import topk_b200 as T
from oracle import oracle as O
from tests import helpers as H

pytestmark = pytest.mark.gpu


def part_table(n, d, dist, seed, rows):
    t = T.Table(n, d)
    t.generate(dist, seed)
    t.normalize()
    t.build_partitions(rows)
    return t


def test_partition_stats_cover_the_table():
    n, d = 300001, 8
    with part_table(n, d, 2, 3, 4096) as t:
        tn = t.download()
        R, mins, maxs, means = t.partition_info()
        assert R == 4096 and mins.shape == ((n + R - 1) // R, d)
        assert np.all(mins <= means) and np.all(means <= maxs)
        # every row lies in exactly one partition: extremes and sums agree with the table
        assert np.array_equal(mins.min(axis=0), tn.min(axis=1))
        assert np.array_equal(maxs.max(axis=0), tn.max(axis=1))
        counts = np.full(len(means), R, np.float64)
        counts[-1] = n - R * (len(means) - 1)
        sums = (means.astype(np.float64) * counts[:, None]).sum(axis=0)
        assert np.allclose(sums, tn.astype(np.float64).sum(axis=1), rtol=1e-5)


@pytest.mark.parametrize("dist", [2, 1, 0, 3])
def test_pruned_matches_oracle(dist):
    n, d = (1 << 20) + 333, 8
    rng = np.random.default_rng(dist)
    with part_table(n, d, dist, 7, 8192) as t:
        tn = t.download()
        scanned = []
        for j in range(24):
            w, a = H.random_query(rng, d)
            k = int(rng.choice([1, 16, 100, 1024, 4096]))
            ids, sc, th, st = t.query_pruned(k, w, a)
            H.assert_same_result((ids, sc, th), O.topk_numpy(tn, k, w, a))
            assert st[1] == (n + 8191) // 8192 and st[2] == 0
            scanned.append(st[0] / st[1])
        print(f"dist {dist}: mean fraction of partitions scanned {np.mean(scanned):.3f}")
        if dist == 2:  # the Morton order localises anticorrelated data: most partitions are skipped
            assert np.mean(scanned) < 0.6


def test_pruned_with_cut_accepts_or_falls_back_exactly():
    n, d = 400000, 8
    rng = np.random.default_rng(9)
    with part_table(n, d, 2, 1, 4096) as t:
        tn = t.download()
        for j in range(12):
            w, a = H.random_query(rng, d)
            k = int(rng.integers(1, 1025))
            want = O.topk_numpy(tn, k, w, a)
            kth = float(want[2])
            # a cut at or below the k-th score is accepted: one scan, fewer partitions
            ids, sc, th, st = t.query_pruned(k, w, a, cut=np.nextafter(np.float32(kth), np.float32(-np.inf)))
            H.assert_same_result((ids, sc, th), want)
            assert st[2] == 1 and st[3] == 1
            ids, sc, th, st = t.query_pruned(k, w, a, cut=kth)  # exactly the k-th: still enough objects
            H.assert_same_result((ids, sc, th), want)
            assert st[2] == 1
            # a cut above the k-th score leaves fewer than k objects: the plain method answers
            ids, sc, th, st = t.query_pruned(k, w, a, cut=kth + 0.05)
            H.assert_same_result((ids, sc, th), want)
            assert st[2] == 0


def test_pruned_negative_weights_ties_and_small_tables():
    rng = np.random.default_rng(4)
    n, d = 150000, 6
    raw = (np.floor(O.generate(n, d, 2, 5) * 8) / 8).astype(np.float32)  # coarse: many ties
    tn = raw.copy()
    O.normalize(tn)
    with T.Table(n, d) as t:
        t.upload(raw)
        t.normalize()
        t.build_partitions(2048)
        for j in range(16):
            w = rng.uniform(-1, 1, size=d).astype(np.float32)
            q = int(rng.integers(1, 7))
            a = rng.integers(0, d, size=q).astype(np.uint8)  # repeats allowed
            k = int(rng.integers(1, 3000))
            ids, sc, th, st = t.query_pruned(k, w, a)
            H.assert_same_result((ids, sc, th), O.topk(tn, k, w, a))
    for n in (1, 1000, 1025, 5000):
        with part_table(n, 3, 1, n, 1024) as t:
            tn = t.download()
            w, a = H.random_query(rng, 3)
            for k in (1, 7, min(n + 5, T.MAX_K)):
                ids, sc, th, st = t.query_pruned(k, w, a)
                H.assert_same_result((ids, sc, th), O.topk_numpy(tn, k, w, a))


def test_pruned_needs_current_partitions():
    with T.Table(5000, 4) as t:
        t.generate(1, 1)
        with pytest.raises(T.TopKError):
            t.query_pruned(5, np.ones(4, np.float32), np.array([0, 1], np.uint8))
        t.build_partitions(1024)
        t.query_pruned(5, np.ones(4, np.float32), np.array([0, 1], np.uint8))
        t.normalize()  # the table changed: the partitions are stale
        with pytest.raises(T.TopKError):
            t.query_pruned(5, np.ones(4, np.float32), np.array([0, 1], np.uint8))
        with pytest.raises(T.TopKError):
            t.build_partitions(1000)  # not a power of two


def test_pruned_ties_in_reordered_rows_go_to_the_lower_original_id():
    """Few distinct values: many objects tie at the k-th score, and the partitioned
    copy holds them out of id order; the lower original ids must win every tie,
    with or without a cut placed exactly at the k-th score."""
    n, d = (1 << 20) + 3, 3
    rng = np.random.default_rng(12)
    raw = (np.floor(O.generate(n, d, 1, 21) * 4) / 4).astype(np.float32)
    tn = raw.copy()
    O.normalize(tn)
    with T.Table(n, d) as t:
        t.upload(raw)
        t.normalize()
        t.build_partitions(1024)
        for k in (1, 37, 500, 1024, 4096):
            for a in (np.array([0, 1], np.uint8), np.array([2, 0, 1], np.uint8), np.array([1], np.uint8)):
                w = np.array([0.5, 0.25, 0.125], np.float32)
                want = O.topk_numpy(tn, k, w, a)
                got = t.query_pruned(k, w, a)
                H.assert_same_result(got[:3], want)
                got = t.query_pruned(k, w, a, cut=float(want[2]))
                H.assert_same_result(got[:3], want)
                assert got[3][2] == 1


@pytest.mark.parametrize("order", ["vta", "vta16", "pta", "kd"])
@pytest.mark.parametrize("n,d,dist,ties", [(200003, 6, 0, False), (200003, 6, 1, False), (200003, 6, 2, False),
                                          (200003, 6, 3, False), (200003, 6, 0, True), (65536, 1, 0, False),
                                          (70001, 2, 2, False), (50001, 20, 0, False)])
def test_index_order_matches_oracle(order, n, d, dist, ties):
    """The device VTA / PTA orders (stable radix sorts) equal the restatements of
    VTA::init (one row range, or 16 as its threaded build) and PTA::polar +
    create_partitions, ties by the lower id; the partitioned copy holds the rows in
    that order and its block bounds are those rows' maxima."""
    from oracle.vta_oracle import kd_order, pta_order, vta_order
    codes = {"vta": T.ORDER_VTA, "vta16": T.ORDER_VTA_THREADS, "pta": T.ORDER_PTA, "kd": T.ORDER_KD}
    want = {"vta": lambda x: vta_order(x), "vta16": lambda x: vta_order(x, 16), "pta": pta_order,
            "kd": lambda x: kd_order(x, 1024)}
    with T.Table(n, d) as t:
        t.generate(dist, 11 + dist)
        t.normalize()
        if ties:  # few distinct values per attribute: long runs of equal keys
            t.upload(np.round(t.download() * 8) / 8)
        tn = t.download()
        t.build_partitions(1024, order=codes[order])
        perm = t.partition_ids()
        assert np.array_equal(perm, want[order](tn))
        R, mins, maxs, means = t.partition_info()
        pad = (-n) % R
        blocks = np.pad(tn[:, perm], ((0, 0), (0, pad)), constant_values=-np.inf).reshape(d, -1, R)
        assert np.array_equal(maxs, blocks.max(axis=2).T)


@pytest.mark.parametrize("order", [1, 2, 3, 5])
@pytest.mark.parametrize("dist", [2, 0])
def test_pruned_on_vta_pta_partitions_matches_oracle(dist, order):
    n, d = (1 << 19) + 77, 8
    rng = np.random.default_rng(40 + dist)
    with T.Table(n, d) as t:
        t.generate(dist, 5)
        t.normalize()
        tn = t.download()
        t.build_partitions(4096, order=order)
        scanned = []
        for j in range(16):
            w, a = H.random_query(rng, d)
            k = int(rng.choice([1, 10, 256, 1024]))
            ids, sc, th, st = t.query_pruned(k, w, a)
            H.assert_same_result((ids, sc, th), O.topk_numpy(tn, k, w, a))
            scanned.append(st[0] / st[1])
        print(f"order {order} dist {dist}: mean fraction of partitions scanned {np.mean(scanned):.3f}")
        # the Morton copy is replaced: a rebuild in Morton order still answers exactly
        t.build_partitions(4096)
        w, a = H.random_query(rng, d)
        H.assert_same_result(t.query_pruned(64, w, a)[:3], O.topk_numpy(tn, 64, w, a))


def test_kd_order_with_nan_and_constant_columns_matches_oracle():
    """The kd order on a table with NaN values, a constant column and infinities: the
    spread rule leaves NaN out and counts a NaN or missing spread as 0; the device
    permutation equals the restatement and pruned queries stay exact."""
    from oracle.vta_oracle import kd_order
    n, d = 150001, 5
    rng = np.random.default_rng(8)
    x = rng.random((d, n), dtype=np.float32)
    x[1] = 0.25  # constant column: spread 0 in every node
    x[2, rng.integers(0, n, 500)] = np.nan
    x[3, rng.integers(0, n, 50)] = np.inf
    x[4, :4096] = np.nan  # a long run of NaN values in one attribute
    with T.Table(n, d) as t:
        t.upload(x)
        t.build_partitions(1024, order=T.ORDER_KD)
        assert np.array_equal(t.partition_ids(), kd_order(x, 1024))
        for k in (1, 100, 1000):
            w, a = H.random_query(rng, d)
            a = np.array([0, 1, 3], np.uint8)
            H.assert_same_result(t.query_pruned(k, w, a)[:3], O.topk_numpy(x, k, w, a))


def test_kd_order_prunes_more_than_morton_on_anticorrelated_data():
    """The kd order's partition boxes follow the attributes that vary most, so on
    anticorrelated data a query scans fewer partitions than over the Morton order."""
    n, d = 1 << 22, 8
    rng = np.random.default_rng(77)
    fr = {}
    with T.Table(n, d) as t:
        t.generate(2, 9)
        t.normalize()
        tn = t.download()
        qs = []
        for j in range(40):
            w, a = H.random_query(rng, d)
            qs.append((int(rng.choice([16, 100, 1000])), w, a))
        for order in (T.ORDER_MORTON, T.ORDER_KD):
            t.build_partitions(4096, order=order)
            sc = []
            for k, w, a in qs:
                ids, s_, th, st = t.query_pruned(k, w, a)
                if len(sc) < 5:
                    H.assert_same_result((ids, s_, th), O.topk_numpy(tn, k, w, a))
                sc.append(st[0] / st[1])
            fr[order] = float(np.mean(sc))
    print(f"fraction of partitions scanned: Morton {fr[T.ORDER_MORTON]:.3f}, kd {fr[T.ORDER_KD]:.3f}")
    assert fr[T.ORDER_KD] < fr[T.ORDER_MORTON]


def test_partition_order_errors():
    with T.Table(5000, 4) as t:
        t.generate(0, 1)
        with pytest.raises(T.TopKError):
            t.partition_ids()  # nothing built yet
        with pytest.raises(T.TopKError):
            t.build_partitions(1024, order=7)
    with T.Table(5000, 33) as t:
        t.generate(0, 1)
        with pytest.raises(T.TopKError):
            t.build_partitions(1024, order=T.ORDER_PTA)  # 2^32 groups
