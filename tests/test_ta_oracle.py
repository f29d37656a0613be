"""CPU: the reference's TA against the oracle.

TA::findTopK (cpu/TA.h:61-96) scores every attribute of an object with the weight of
the list the object was found in (the inner loop at :83 reuses the outer `weight`),
so its scores are the exact weighted sums only when all queried weights are equal.
With equal weights its result must be the exact top-k (ties at the k-th score
compared tie-aware: its heap and its non-strict stop leave them open).  The device TA
uses each attribute's own weight and is checked against the oracle for any weights
(tests/test_gpu_ta.py).
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests import helpers as H


@pytest.mark.parametrize("n,d,dist", [(20000, 6, 1), (30011, 4, 0), (15000, 8, 2)])
def test_reference_ta_matches_oracle_with_equal_weights(n, d, dist):
    if not O.RefTPAc.available():
        pytest.skip("reference library not built in this environment")
    cols = O.generate(n, d, dist, 40 + d)
    ref = O.RefTA(np.ascontiguousarray(cols.T))
    ref.init()
    tn = cols.copy()
    O.normalize(tn)
    rng = np.random.default_rng(d)
    for j in range(8):
        q = int(rng.integers(1, d + 1))
        attr = rng.choice(d, size=q, replace=False).astype(np.uint8)
        w = np.full(d, np.float32(0.25 + 0.125 * j), np.float32)
        k = int(rng.integers(1, 300))
        ids, sc, th = O.topk(tn, k, w, attr)
        r_ids, r_sc, r_th, _ = ref.query(k, w, attr)
        run = dict(ids=r_ids.tolist(), score_bits=H.bits(r_sc).tolist(),
                   threshold_bits=int(H.bits(np.float32(r_th))))
        H.assert_matches_reference(ids, sc, th, run, tn, w, attr)
    ref.close()
