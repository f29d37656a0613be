"""Shared test helpers: golden fixtures and tie-aware result comparison."""
import json
import os

import numpy as np

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "tpac_golden.json")

_golden = None


def golden():
    global _golden
    if _golden is None:
        with open(GOLDEN) as f:
            _golden = json.load(f)
    return _golden


def case_table(c):
    """Raw (un-normalised) table of a golden case, regenerated from its recipe."""
    t = O.generate(c["n"], c["d"], c["dist"], c["seed"])
    if c.get("quant"):
        t = (np.floor(t * c["quant"]) / c["quant"]).astype(np.float32)
    return t


def case_weights(c):
    return np.array(c["weights_bits"], np.uint32).view(np.float32)


def bits(a):
    return np.asarray(a, np.float32).view(np.uint32)


def assert_matches_reference(ids, scores, threshold, run, table_norm, weights, attr):
    """Compare a result with a recorded reference run.

    The reference's tie order at the k-boundary depends on its heap, so: the score
    multisets must be bit-equal, the ids strictly above the threshold must be the
    same set, and every id at the threshold must really score the threshold.
    """
    r_ids = np.array(run["ids"], np.uint64)
    r_sc = np.array(run["score_bits"], np.uint32)
    assert len(ids) == len(r_ids), (len(ids), len(r_ids))
    assert np.array_equal(np.sort(bits(scores)), np.sort(r_sc)), "score multiset differs"
    th_bits = run["threshold_bits"]
    assert int(bits(np.float32(threshold))) == th_bits, (threshold, th_bits)
    th = np.uint32(th_bits).view(np.float32)
    above_mine = set(int(i) for i, s in zip(ids, scores) if s > th)
    above_ref = set(int(i) for i, s in zip(r_ids, r_sc.view(np.float32)) if s > th)
    assert above_mine == above_ref
    tied = [int(i) for i, s in zip(ids, scores) if s == th]
    if tied:
        recomputed = O.scores(table_norm, weights, attr, ids=np.array(tied, np.int64))
        assert np.all(recomputed == th)


def assert_same_result(a, b):
    """Bit-exact equality of two (ids, scores, threshold) results."""
    ia, sa, ta = a
    ib, sb, tb = b
    assert np.array_equal(np.asarray(ia, np.uint64), np.asarray(ib, np.uint64)), "ids differ"
    sa, sb = np.asarray(sa, np.float32), np.asarray(sb, np.float32)
    # NaN payload bits differ between CPU and GPU (0/0 is 0xFFC00000 on x86, 0x7FFFFFFF
    # on the GPU); NaN positions must match and every other score bit-exactly.
    assert np.array_equal(np.isnan(sa), np.isnan(sb)), "NaN positions differ"
    ok = ~np.isnan(sa)
    assert np.array_equal(bits(sa[ok]), bits(sb[ok])), "scores differ"
    ta, tb = np.float32(ta), np.float32(tb)
    assert (np.isnan(ta) and np.isnan(tb)) or bits(ta) == bits(tb), "threshold differs"


def random_query(rng, d, qmax=None, ordered=True):
    qmax = d if qmax is None else qmax
    q = int(rng.integers(1, qmax + 1))
    attr = rng.choice(d, size=q, replace=False)
    if ordered:
        attr = np.sort(attr)
    w = np.zeros(d, np.float32)
    w[:] = ((rng.integers(0, 1 << 24, size=d) + 1) * 2.0 ** -24).astype(np.float32)
    return w, attr.astype(np.uint8)
