"""CPU: the reference's row-major TPAr against the oracle.

TPAr (cpu/TPAr.h) keeps the table row-major and normalises it with normalize
(common/common.h:63-92); its scores accumulate in attr order like TPAc's.  So the
oracle's column-major normalisation and top-k, applied to the transposed table, must
reproduce TPAr exactly: the normalised rows bit for bit and every query of its three
entries (ties at the k-th score compared tie-aware, as for TPAc).  The reference's
loops step 8 or 16 objects with no tail, so n is a multiple of 256 here.

The reference's findTopKsimd and findTopKthreads label each score with the wrong id:
_mm256_set_ps takes its arguments from the highest lane down (cpu/TPAr.h:140-158),
so lane j holds object base + 7 - j but is pushed as base + j.  Their scores and
thresholds are right; their ids are the true ids mirrored within each group of 8.
The scalar entry's ids, the oracle's and the GPU's are the true ids.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests import helpers as H


@pytest.mark.parametrize("n,d,dist", [(1 << 14, 8, 1), (1 << 13, 16, 2), (4096, 5, 0), (1 << 14, 3, 3)])
def test_reference_tpar_matches_oracle(n, d, dist):
    if not O.RefTPAc.available():
        pytest.skip("reference library not built in this environment")
    cols = O.generate(n, d, dist, 70 + d)
    ref = O.RefTPAr(np.ascontiguousarray(cols.T))
    ref.init()
    tn = cols.copy()
    O.normalize(tn)
    assert np.array_equal(H.bits(ref.data()), H.bits(np.ascontiguousarray(tn.T)))
    rng = np.random.default_rng(n + d)
    for j in range(9):
        w, attr = H.random_query(rng, d, ordered=bool(j % 2))
        k = int(rng.integers(1, 700))
        ids, sc, th = O.topk(tn, k, w, attr)
        impl = j % 3
        r_ids, r_sc, r_th, _ = ref.query(impl, k, w, attr)
        if impl:  # undo the lane mirror of the vector entries
            r_ids = (r_ids // 8) * 8 + 7 - r_ids % 8
        run = dict(ids=r_ids.tolist(), score_bits=H.bits(r_sc).tolist(),
                   threshold_bits=int(H.bits(np.float32(r_th))))
        H.assert_matches_reference(ids, sc, th, run, tn, w, attr)
    ref.close()
