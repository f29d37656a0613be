"""GPU: row-major tables (the reference's TPAr layout, cpu/TPAr.h) through the device
transpose, and the TPAr mirror.

The rows go up in blocks and are transposed on the device into the column-major
table; download transposes back.  TPAr's normalize (common/common.h:63-92) is the
same arithmetic per attribute as TPAc's, so the normalised table and every query
must equal the oracle's on the transposed table, bit for bit.
"""
import numpy as np
import pytest

import topk_b200 as T
from oracle import oracle as O
from tests import helpers as H

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,d,stride", [(100003, 8, 8), (70000, 17, 20), (4097, 1, 1), (33, 40, 41),
                                        ((1 << 22) + 5, 16, 16)])
def test_rowmajor_round_trip(n, d, stride):
    rng = np.random.default_rng(n + d)
    rows = rng.standard_normal((n, stride)).astype(np.float32)
    with T.Table(n, d) as t:
        t.upload_rowmajor(rows)
        assert np.array_equal(H.bits(t.download()), H.bits(np.ascontiguousarray(rows[:, :d].T)))
        assert np.array_equal(H.bits(t.download_rowmajor()), H.bits(np.ascontiguousarray(rows[:, :d])))


@pytest.mark.parametrize("n,d,dist", [((1 << 20) + 3, 8, 1), (300000, 16, 2), (5000, 3, 0)])
def test_tpar_mirror_matches_oracle(n, d, dist):
    cols = O.generate(n, d, dist, 90 + d)
    tp = T.TPAr(n, d)
    tp.set_cdata(np.ascontiguousarray(cols.T))
    tp.init()
    tn = cols.copy()
    O.normalize(tn)
    assert np.array_equal(H.bits(tp.table.download_rowmajor()), H.bits(np.ascontiguousarray(tn.T)))
    rng = np.random.default_rng(d)
    for j in range(12):
        w, attr = H.random_query(rng, d, ordered=bool(j % 2))
        k = int(rng.choice([1, 16, 100, 1024, 4096]))
        [tp.findTopKscalar, tp.findTopKsimd, tp.findTopKthreads][j % 3](k, len(attr), w, attr)
        want = O.topk_numpy(tn, k, w, attr)
        H.assert_same_result((tp.res_ids, tp.res_scores, tp.get_thres()), want)
    tp.close()


def test_rowmajor_arguments():
    with T.Table(100, 4) as t:
        with pytest.raises(ValueError):
            t.upload_rowmajor(np.zeros((100, 3), np.float32))
        with pytest.raises(T.TopKError):  # no data yet
            t.query(1, np.ones(4, np.float32), np.array([0], np.uint8))
        t.upload_rowmajor(np.ones((100, 4), np.float32))
        ids, sc, th = t.query(3, np.ones(4, np.float32), np.array([0, 1], np.uint8))
        assert list(ids) == [2, 1, 0] and th == 2.0
