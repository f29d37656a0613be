"""CPU: the numpy VTA and PTA orders against loop-level restatements of VTA::init and
PTA::polar / PTA::create_partitions.

The loop version walks the reference's steps one by one (cpu/VTA.h:121-135) with
Python's stable sort and the reference's comparators (cmp_vta_pair: score greater,
cpu/VTA.h:49; cmp_vta_pos: position smaller, cpu/VTA.h:46).  A stable sort over lists
built in id order breaks ties by the lower id, the rule of the device order.
"""
import numpy as np
import pytest

import math

from oracle.vta_oracle import pta_angle_keys, pta_order, vta_order


def vta_order_loops(table):
    d, n = table.shape
    pos = [n] * n
    for m in range(d):
        lst = sorted(range(n), key=lambda j: -float(table[m, j]))  # stable: ties by id
        for j, i in enumerate(lst):
            pos[i] = min(pos[i], j)
    return np.array(sorted(range(n), key=lambda i: pos[i]), np.uint32)


@pytest.mark.parametrize("seed", range(6))
def test_vta_order_matches_loops(seed):
    rng = np.random.default_rng(seed)
    d, n = int(rng.integers(1, 6)), int(rng.integers(1, 400))
    if seed % 2:  # heavy ties: a few distinct values per attribute
        table = rng.integers(0, 4, size=(d, n)).astype(np.float32) / 4
    else:
        table = rng.random((d, n), dtype=np.float32)
    assert np.array_equal(vta_order(table), vta_order_loops(table))


def test_vta_blocks_bound_the_rest():
    """Every row after a block lies below the block's threshold tuple (the reference's
    tarray, cpu/VTA.h:145-146): the max of the next block never exceeds it."""
    rng = np.random.default_rng(9)
    d, n, B = 4, 20000, 1024
    table = rng.random((d, n), dtype=np.float32)
    perm = vta_order(table)
    lists = [np.sort(table[m])[::-1] for m in range(d)]
    pos = np.full(n, n, np.int64)
    for m in range(d):
        order = np.lexsort((np.arange(n), -table[m].astype(np.float64)))
        p = np.empty(n, np.int64)
        p[order] = np.arange(n)
        pos = np.minimum(pos, p)
    for b in range(0, n - B, B):
        last = pos[perm[b + B - 1]]
        tarray = np.array([lists[m][last] for m in range(d)])
        nxt = table[:, perm[b + B:]]
        assert np.all(nxt.max(axis=1) <= tarray)


def pta_order_loops(table):
    """PTA's steps one by one (cpu/PTA.h:88-167, 203-236) with FP32 scalar arithmetic,
    Python's stable sorts and the reference's comparators (cmp_pta_pair_asc for the
    angles, cmp_pta_pos for partitions and positions, cmp_pta_pair for the lists)."""
    d, n = table.shape
    one = np.float32(1.1)
    absf = [[0.0] * n for _ in range(d - 1)]
    for i in range(n):
        curr, s = table[d - 1, i] - one, np.float32(0)
        for m in range(d - 1, 0, -1):
            nxt = table[m - 1, i] - one
            s = np.float32(s + np.float32(curr * curr))
            absf[m - 1][i] = float(abs(np.float32(np.sqrt(s) / nxt)))
            curr = nxt
    part, mul, mod = [0] * n, 1, n // 2
    for c in range(d - 1):
        lst = sorted(range(n), key=lambda i: absf[c][i])
        # the reference sorts by |atan(f)| * 180/pi: monotone in |f|, so this order is one of its orders
        ang = [abs(math.atan(absf[c][i])) for i in lst]
        assert all(a <= b for a, b in zip(ang, ang[1:]))
        for r, i in enumerate(lst):
            part[i] += mul * (r // mod)
        mul *= 2
    part = [min(p, (1 << (d - 1)) - 1) for p in part]
    ppos = sorted(range(n), key=lambda i: part[i])
    out = []
    for p in sorted(set(part)):
        rows = [i for i in ppos if part[i] == p]
        pos = [len(rows)] * len(rows)
        for m in range(d):
            lst = sorted(range(len(rows)), key=lambda j: -float(table[m, rows[j]]))
            for r, j in enumerate(lst):
                pos[j] = min(pos[j], r)
        out += [rows[j] for j in sorted(range(len(rows)), key=lambda j: pos[j])]
    return np.array(out, np.uint32)


@pytest.mark.parametrize("seed", range(6))
def test_pta_order_matches_loops(seed):
    rng = np.random.default_rng(100 + seed)
    d, n = int(rng.integers(1, 6)), int(rng.integers(2, 300))
    if seed % 2:
        table = rng.integers(0, 4, size=(d, n)).astype(np.float32) / 4
    else:
        table = rng.random((d, n), dtype=np.float32)
    assert np.array_equal(pta_order(table), pta_order_loops(table))


def test_pta_single_attribute_is_vta():
    table = np.random.default_rng(3).random((1, 500), dtype=np.float32)
    assert pta_angle_keys(table).shape == (0, 500)
    assert np.array_equal(pta_order(table), vta_order(table))


def distinct_table(rng, d, n):
    """Every column a permutation of distinct values: no value ties, distinct rows."""
    return np.stack([rng.permutation(n).astype(np.float32) / n for _ in range(d)])


@pytest.mark.parametrize("d,imp", [(4, 2), (4, 1), (8, 2), (8, 1)])
@pytest.mark.parametrize("n", [5000, 100001])
def test_orders_pinned_to_reference(d, imp, n):
    """The restated VTA and PTA orders against the reference's own index builds
    (cpu/VTA.h, cpu/PTA.h compiled into oracle/_ref): the same group and the same
    minimum position at every place; only rows the reference's unstable sorts leave
    unordered may differ."""
    from oracle import build as B
    from oracle import oracle as O
    from oracle.vta_oracle import (min_positions, pta_part_ids, ref_index_rows, rows_to_ids,
                                   same_order_up_to_ties, vta_groups)
    B.build_ref_index()
    rng = np.random.default_rng(n + d + imp)
    raw = distinct_table(rng, d, n)
    tn = raw.copy()
    O.normalize(tn)
    got = ref_index_rows("vta", raw, imp)
    if got is None:
        pytest.skip("reference index library not built (reference sources absent)")
    slices = 16 if imp == 2 else 1
    ref_perm = rows_to_ids(tn, got[0])
    ours = vta_order(tn, slices)
    assert same_order_up_to_ties(tn, vta_groups(n, slices), ref_perm, ours)
    # ties are real: the orders differ only inside runs of equal minimum position
    mp = min_positions(tn, vta_groups(n, slices))
    assert np.all(np.diff(mp[ref_perm]) >= 0)
    if imp == 2:  # PTA does not depend on IMP
        ref_perm = rows_to_ids(tn, ref_index_rows("pta", raw, imp)[0])
        assert same_order_up_to_ties(tn, pta_part_ids(tn), ref_perm, pta_order(tn))


def kd_order_loops(table, part_rows):
    """The kd order node by node with Python's stable sort: a node is a range of whole
    partitions [lo, hi) of the order, split at lo + ceil((hi - lo) / 2) after its rows
    are sorted by the attribute of widest spread (FP32 max - min over non-NaN values,
    the lower attribute on a tie)."""
    d, n = table.shape
    P = (n + part_rows - 1) // part_rows
    order = list(range(n))

    def split(lo, hi):
        if hi - lo <= 1:
            return
        a, b = lo * part_rows, min(n, hi * part_rows)
        rows = order[a:b]
        best, bs = 0, np.float32(0)
        for m in range(d):
            v = [table[m, r] for r in rows if not np.isnan(table[m, r])]
            s = np.float32(max(v)) - np.float32(min(v)) if v else np.float32(0)
            if np.isnan(s):
                s = np.float32(0)
            if m == 0 or s > bs:
                best, bs = m, s
        key = lambda r: (0, 0.0) if np.isnan(table[best, r]) else (1, float(table[best, r]))
        order[a:b] = sorted(rows, key=key)
        mid = lo + (hi - lo + 1) // 2
        split(lo, mid)
        split(mid, hi)

    split(0, P)
    return np.array(order, np.uint32)


@pytest.mark.parametrize("seed", range(6))
def test_kd_order_matches_node_by_node_loops(seed):
    """The level-by-level numpy kd order puts the same rows in every partition as the
    node-by-node recursion (stable sorts: equal values keep the order of the level
    before).  Inside a partition the orders may differ: the level form sorts a node
    that is already a single partition again at the later levels."""
    from oracle.vta_oracle import kd_order
    rng = np.random.default_rng(100 + seed)
    d, n, R = int(rng.integers(1, 6)), int(rng.integers(1, 3000)), int(2 ** rng.integers(4, 8))
    if seed % 2:
        table = rng.integers(0, 4, size=(d, n)).astype(np.float32) / 4
    else:
        table = rng.random((d, n), dtype=np.float32)
    if seed % 3 == 0 and n > 10:
        table[0, rng.integers(0, n, n // 10)] = np.nan
    a, b = kd_order(table, R), kd_order_loops(table, R)
    for p0 in range(0, n, R):
        assert np.array_equal(np.sort(a[p0:p0 + R]), np.sort(b[p0:p0 + R]))
