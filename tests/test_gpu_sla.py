"""GPU: SLA's skyline layers and index order built on the device (cpu/SLA.h).

The device computes each row's depth (1 + deepest dominator, rows in coordinate-sum
order) and applies the reference's stop rule; the layers must equal the oracle's
layer peeling (pinned against the reference's own SLA on the CPU), and the SLA order
(VTA's order inside each layer) must equal the oracle's bit for bit, ties by the
lower id.  Pruned queries over those partitions stay exact.
"""
import numpy as np
import pytest

import topk_b200 as T
from oracle import oracle as O
from oracle import sla_oracle as S
from tests import helpers as H

pytestmark = pytest.mark.gpu


def sla_table(n, d, dist, seed, quant=None):
    raw = O.generate(n, d, dist, seed)
    if quant:
        raw = (np.floor(raw * quant) / quant).astype(np.float32)
    t = T.Table(n, d)
    t.upload(raw)
    t.normalize()
    return t


@pytest.mark.parametrize("n,d,dist,quant", [(3000, 4, 1, None), (5000, 4, 2, None), (1200, 3, 0, None),
                                           (2500, 4, 1, 8), (2000, 6, 1, None), (90, 4, 1, None),
                                           (300, 1, 1, None), (3001, 5, 2, 4)])
def test_skyline_layers_match_oracle(n, d, dist, quant):
    with sla_table(n, d, dist, 31 + n, quant) as t:
        tn = t.download()
        layers, nl = t.skyline_layers()
        want = S.skyline_layers(tn)
        assert np.array_equal(layers.astype(np.int64), want)
        assert nl == int(want.max()) + 1


@pytest.mark.parametrize("n,d,dist", [(4000, 4, 1), (3000, 6, 2), (1200, 3, 0)])
def test_sla_order_and_pruned_queries(n, d, dist):
    rng = np.random.default_rng(n)
    with sla_table(n, d, dist, 7 + d) as t:
        tn = t.download()
        t.build_partitions(1024, order=T.ORDER_SLA)
        assert np.array_equal(t.partition_ids(), S.sla_order(tn))
        for j in range(8):
            w, a = H.random_query(rng, d)
            k = int(rng.choice([1, 10, 100, 1000]))
            H.assert_same_result(t.query_pruned(k, w, a)[:3], O.topk_numpy(tn, k, w, a))


def test_sla_limits():
    with T.Table(5000, 33) as t:
        t.generate(1, 1)
        with pytest.raises(T.TopKError):
            t.skyline_layers()
        with pytest.raises(T.TopKError):
            t.build_partitions(1024, order=T.ORDER_SLA)
    # the O(n^2 d) build refuses tables above 2^22 rows before any device work
    with T.Table((1 << 22) + 1, 1) as t:
        t.generate(1, 1)
        with pytest.raises(T.TopKError, match="2\\^22"):
            t.skyline_layers()
        with pytest.raises(T.TopKError, match="2\\^22"):
            t.build_partitions(1024, order=T.ORDER_SLA)
