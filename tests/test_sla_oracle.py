"""CPU: the SLA restatement against the reference's own SLA (cpu/SLA.h with its
vendored skyline library, compiled into oracle/_ref by oracle/build.py).

The layer peeling must give every row the reference's layer; the depth formulation
(rows in coordinate-sum order, depth = 1 + deepest dominator, then the stop rule) must
give the same layers; and the index order must match the reference's up to the ties
it leaves open (same layer and same minimum position at every place).
"""
import numpy as np
import pytest

from oracle import oracle as O
from oracle import sla_oracle as S
from oracle import vta_oracle as V


def raw_table(n, d, dist, seed, quant=None, distinct=False):
    if distinct:
        rng = np.random.default_rng(seed)
        return np.stack([rng.permutation(n).astype(np.float32) / np.float32(n) for _ in range(d)])
    t = O.generate(n, d, dist, seed)
    if quant:
        t = (np.floor(t * quant) / quant).astype(np.float32)
    return t


@pytest.mark.parametrize("n,d,dist,quant", [(3000, 4, 1, None), (4000, 4, 2, None), (3000, 4, 0, None),
                                           (2500, 4, 1, 8), (2000, 6, 1, None), (1500, 6, 2, 4), (90, 4, 1, None)])
def test_layers_match_reference(n, d, dist, quant):
    raw = raw_table(n, d, dist, 17 + n, quant)
    want = S.ref_sla_layers(raw)
    if want is None:
        pytest.skip("reference SLA library not built for this d")
    tn = raw.copy()
    O.normalize(tn)
    assert np.array_equal(S.skyline_layers(tn), want)


@pytest.mark.parametrize("n,d,dist,quant", [(1500, 4, 1, None), (1200, 4, 0, None), (1000, 6, 2, 4), (150, 3, 1, 2)])
def test_depth_formulation_equals_peeling(n, d, dist, quant):
    tn = raw_table(n, d, dist, 5 + n, quant)
    O.normalize(tn)
    assert np.array_equal(S.layer_depths(tn), S.skyline_layers(tn))


@pytest.mark.parametrize("n,d", [(3000, 4), (2000, 6)])
def test_index_order_matches_reference(n, d):
    raw = raw_table(n, d, 0, 3 + d, distinct=True)
    rows = S.ref_sla_rows(raw)
    if rows is None:
        pytest.skip("reference SLA library not built for this d")
    tn = raw.copy()
    O.normalize(tn)
    layers = S.skyline_layers(tn)
    ref_perm = V.rows_to_ids(tn, rows)
    assert V.same_order_up_to_ties(tn, layers, ref_perm, S.sla_order(tn, layers))


def test_depth_order_puts_dominators_first_at_equal_sums():
    """Rows whose FP32 sums round to the same value while one dominates the other: the
    lexicographic tie-break keeps the dominator first."""
    # table values t, sky values 1 - t: row 0 -> (1, 2^-24), row 1 -> (1, 0); row 1
    # dominates row 0, and both sums are 1.0 in FP32 (1 + 2^-24 rounds to even)
    t_small = np.float32(1.0) - np.float32(2.0 ** -24)
    tn = np.array([[0.0, 0.0], [t_small, 1.0]], np.float32)  # (d, n)
    x = S.sky_values(tn)
    assert x[0, 1] == np.float32(2.0 ** -24) and x[1, 1] == 0.0
    assert np.float32(x[0, 0] + x[0, 1]) == np.float32(x[1, 0] + x[1, 1])
    assert list(S.skyline_layers(tn, stop=0)) == [1, 0]
    assert np.array_equal(S.layer_depths(tn, stop=0), S.skyline_layers(tn, stop=0))
