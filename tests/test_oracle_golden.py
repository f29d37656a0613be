"""CPU: pin the oracle against the golden outputs of the reference itself.

The fixtures (tests/golden/tpac_golden.json) were produced by running the
reference's TPAc (cpu/TPAc.h) compiled strict; see tests/golden/make_golden.py.
"""
import hashlib

import numpy as np
import pytest

from oracle import oracle as O
from tests import helpers as H

CASES = H.golden()["cases"]


def test_generator_pinned():
    """Generator checksums recorded with the fixtures (same definition on the GPU)."""
    for key, sha in H.golden()["generator_sha256"].items():
        dist, d = map(int, key.split("_"))
        t = O.generate(1024, d, dist, 123)
        assert hashlib.sha256(t.tobytes()).hexdigest() == sha, key


@pytest.mark.parametrize("c", CASES, ids=[c["name"] for c in CASES])
def test_oracle_matches_reference(c):
    t = H.case_table(c)
    O.normalize(t)
    # normalize_transpose (common/common.h:30-61) bit-exact
    assert hashlib.sha256(t.tobytes()).hexdigest() == c["table_sha256"]
    w = H.case_weights(c)
    attr = np.array(c["attr"], np.uint8)
    ids, sc, th = O.topk(t, c["k"], w, attr)
    for impl, run in c["runs"].items():
        H.assert_matches_reference(ids, sc, th, run, t, w, attr)
    # ascending, and ties broken lower-id-first (so higher id first in the ascending list)
    comp = [(int(O.lib().orc_key(float(s))), -int(i)) for i, s in zip(ids, sc)]
    assert comp == sorted(comp)


def test_numpy_and_c_oracles_agree():
    rng = np.random.default_rng(5)
    for dist in (0, 1, 2, 3):
        t = O.generate(1 << 14, 12, dist, 77)
        O.normalize(t)
        for _ in range(4):
            w, attr = H.random_query(rng, 12, ordered=False)
            k = int(rng.integers(1, 300))
            H.assert_same_result(O.topk(t, k, w, attr), O.topk_numpy(t, k, w, attr))


def test_f64_oracle_close():
    t = O.generate(1 << 12, 8, 1, 3)
    O.normalize(t)
    w = O.gen_weights(8, 4, 0)
    attr = np.arange(8, dtype=np.uint8)
    ids, sc, _ = O.topk(t, 32, w, attr)
    ids64, sc64 = O.topk_f64(t, 32, w, attr)
    assert np.max(np.abs(np.sort(sc).astype(np.float64) - np.sort(sc64))) < 1e-5


def test_oracle_live_reference_when_built():
    """When oracle/_ref is present, recheck a few fresh random cases live."""
    if not O.RefTPAc.available():
        pytest.skip("reference library not built in this environment")
    rng = np.random.default_rng(11)
    for j in range(6):
        n, d = 1 << 15, 16
        t = O.generate(n, d, j % 4, 500 + j)
        ref = O.RefTPAc(t)
        ref.init()
        tn = ref.data()
        w, attr = H.random_query(rng, d, ordered=bool(j % 2))
        k = int(rng.integers(1, 600))
        ids, sc, th = O.topk(tn, k, w, attr)
        r_ids, r_sc, r_th, _ = ref.query(1, k, w, attr)
        run = dict(ids=r_ids.tolist(), score_bits=H.bits(r_sc).tolist(),
                   threshold_bits=int(H.bits(np.float32(r_th))))
        H.assert_matches_reference(ids, sc, th, run, tn, w, attr)
        ref.close()
