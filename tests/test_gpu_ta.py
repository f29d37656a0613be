"""GPU: the device threshold algorithm (cpu/TA.h) against the oracle.

The sorted lists must be TA::init's lists (value descending; ties, which the
reference's parallel sort leaves open, by the lower id).  Every query must equal the
exact top-k bit for bit (ids, scores, threshold), for any weights, ties at the k-th
score going to the lower id: the walk stops only when the k-th score is strictly
above the bound of every object not yet met.
"""
import numpy as np
import pytest

import topk_b200 as T
from oracle import oracle as O
from oracle.vta_oracle import f2key
from tests import helpers as H

pytestmark = pytest.mark.gpu


def ta_table(n, d, dist, seed, coarse=False):
    t = T.Table(n, d)
    if coarse:
        raw = (np.floor(O.generate(n, d, dist, seed) * 8) / 8).astype(np.float32)
        t.upload(raw)
    else:
        t.generate(dist, seed)
    t.normalize()
    t.build_lists()
    return t


def test_lists_are_the_reference_lists():
    n, d = 100003, 5
    with ta_table(n, d, 1, 3, coarse=True) as t:
        tn = t.download()
        for m in range(d):
            ids, vals = t.read_list(m)
            want = np.lexsort((np.arange(n), -f2key(tn[m]).astype(np.int64)))
            assert np.array_equal(ids, want.astype(np.uint32))
            assert np.array_equal(H.bits(vals), H.bits(tn[m][want]))


@pytest.mark.parametrize("dist,coarse", [(0, False), (1, False), (2, False), (3, False), (1, True), (0, True)])
def test_ta_matches_oracle(dist, coarse):
    n, d = (1 << 19) + 7, 8
    rng = np.random.default_rng(dist * 2 + coarse)
    with ta_table(n, d, dist, 11, coarse) as t:
        tn = t.download()
        depths = []
        for j in range(16):
            w, a = H.random_query(rng, d, ordered=bool(j % 2))
            if j % 4 == 3:
                w = rng.uniform(-1, 1, size=d).astype(np.float32)  # negative weights: min bounds
            if j % 5 == 4:
                a = np.array([a[0]] * 2 + list(a), np.uint8)[:8]  # repeated attributes
            k = int(rng.choice([1, 16, 100, 1024, 4096]))
            ids, sc, th, st = t.query_ta(k, w, a)
            H.assert_same_result((ids, sc, th), O.topk_numpy(tn, k, w, a))
            assert st[0] <= n and st[1] <= n
            depths.append(st[0] / n)
        print(f"dist {dist} coarse {coarse}: mean depth walked {np.mean(depths):.3f}")
        if dist == 0 and not coarse:  # correlated data: TA stops early
            assert np.median(depths) < 0.5


def test_ta_small_tables_and_errors():
    for n in (1, 5, 1000):
        with ta_table(n, 3, 1, n) as t:
            tn = t.download()
            w = np.array([0.5, 0.25, 1.0], np.float32)
            a = np.array([2, 0], np.uint8)
            for k in (1, 3, n + 4):
                H.assert_same_result(t.query_ta(k, w, a)[:3], O.topk_numpy(tn, k, w, a))
    with T.Table(5000, 4) as t:
        t.generate(1, 1)
        with pytest.raises(T.TopKError):
            t.query_ta(5, np.ones(4, np.float32), np.array([0], np.uint8))  # no lists
        t.build_lists()
        t.query_ta(5, np.ones(4, np.float32), np.array([0], np.uint8))
        t.normalize()  # the table changed: the lists are stale
        with pytest.raises(T.TopKError):
            t.query_ta(5, np.ones(4, np.float32), np.array([0], np.uint8))


def test_ta_mirror_row_major():
    n, d = 200000, 6
    cols = O.generate(n, d, 0, 5)
    ta = T.TA(n, d)
    ta.set_cdata(np.ascontiguousarray(cols.T))
    ta.init()
    tn = cols.copy()
    O.normalize(tn)
    rng = np.random.default_rng(2)
    for j in range(6):
        w, a = H.random_query(rng, d)
        k = int(rng.integers(1, 2000))
        ta.findTopK(k, len(a), w, a)
        H.assert_same_result((ta.res_ids, ta.res_scores, ta.get_thres()), O.topk_numpy(tn, k, w, a))
    ta.close()
