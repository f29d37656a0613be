"""Test infrastructure only: numpy restatement of SLA's skyline layers and index order.

SLA::init (cpu/SLA.h:259-282) normalises the table, turns every value into 1 - x
(sky_data, :87-100: the skyline of the largest values is the minimum skyline of
1 - x), then peels layers (build_layers, :102-139): while more than 100 rows remain,
the skyline of the remaining rows (the rows no other remaining row dominates; p
dominates q when p <= q in every attribute and p < q in one) is the next layer; the
last <= 100 rows form the final layer.  create_lists (:199-251) then orders each layer
as VTA orders a table (lists by value descending, minimum position) and cuts it into
blocks of 1024 rows.

`skyline_layers` restates the peeling.  `layer_depths` computes the same layers the way
a parallel build would: a row's depth is 1 + the largest depth of the rows that
dominate it (0 for the skyline), every dominator of a row has a coordinate sum no
larger (computed in FP32 with one rounding per addition, monotone) and, at an equal
sum, comes first in the lexicographic order of its values, so rows processed in that
order see their dominators first; the stop rule then merges every depth
from the first one with at most 100 rows at or beyond it.  `sla_order` is the index
order with ties by the lower id (the reference's unstable sorts and its skyline
library's output order leave them open).  Pinned against the reference itself
(`ref_sla_layers`, `ref_sla_rows`: oracle/_ref/libref_sla_d{d}.so, built by
oracle/build.py) in tests/test_sla_oracle.py.
"""
import ctypes as C
import os

import numpy as np

from .vta_oracle import min_positions

STOP_ROWS = 100  # cpu/SLA.h:110 `while(last > 100)`


def sky_values(table):
    """(n, d) float32 rows of 1 - x (cpu/SLA.h:96)."""
    return (np.float32(1.0) - np.asarray(table, np.float32)).T.copy()


def _dominated(points, cands, block=256):
    """For each row of cands: does any row of points dominate it?"""
    out = np.zeros(len(cands), bool)
    for a in range(0, len(cands), block):
        c = cands[a:a + block]
        le = np.all(points[None, :, :] <= c[:, None, :], axis=2)
        lt = np.any(points[None, :, :] < c[:, None, :], axis=2)
        out[a:a + block] = np.any(le & lt, axis=1)
    return out


def skyline_layers(table, stop=STOP_ROWS):
    """Layer number of every row (0 = the first skyline), by peeling."""
    x = sky_values(table)
    n = x.shape[0]
    rem = np.arange(n)
    layer = np.full(n, -1, np.int64)
    lv = 0
    while len(rem) > stop:
        dom = _dominated(x[rem], x[rem])
        layer[rem[~dom]] = lv
        rem = rem[dom]
        lv += 1
    if len(rem):
        layer[rem] = lv
    return layer


def layer_depths(table, stop=STOP_ROWS):
    """The same layers by depth: rows in ascending FP32 coordinate-sum order (ties by
    the values, lexicographically), depth = 1 + max depth of the dominators (all earlier
    in that order), then the stop rule."""
    x = sky_values(table)
    n, d = x.shape
    s = np.zeros(n, np.float32)
    for m in range(d):
        s = (s + x[:, m]).astype(np.float32)
    # rounding can give a dominator the same FP32 sum as the row it dominates; among
    # equal sums the lexicographic order of the values still puts the dominator first
    order = np.lexsort(tuple(x[:, m] for m in range(d - 1, -1, -1)) + (s,))
    depth = np.zeros(n, np.int64)
    xs = x[order]
    for j in range(n):
        if j == 0:
            continue
        prev = xs[:j]
        dom = np.all(prev <= xs[j], axis=1) & np.any(prev < xs[j], axis=1)
        if dom.any():
            depth[order[j]] = depth[order[:j]][dom].max() + 1
    # stop rule: the first depth l with at most `stop` rows at depth >= l takes them all
    counts = np.bincount(depth)
    beyond = np.cumsum(counts[::-1])[::-1]  # rows at depth >= l
    lstop = next((l for l in range(len(counts)) if beyond[l] <= stop), len(counts))
    return np.minimum(depth, lstop)


def sla_order(table, layers=None):
    """Rows by layer, inside each layer in VTA's order (ties by the lower id)."""
    if layers is None:
        layers = skyline_layers(table)
    mp = min_positions(table, layers)
    return np.lexsort((np.arange(len(mp)), mp)).astype(np.uint32)


def _lib(d):
    from . import build as B
    path = B.ref_sla_so(d)
    if not os.path.exists(path):
        return None
    L = C.CDLL(path)
    fp = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
    L.ref_sla_layers.argtypes = [fp, C.c_uint64, C.c_uint64, np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")]
    L.ref_sla_layers.restype = C.c_uint64
    L.ref_sla_rows.argtypes = [fp, C.c_uint64, C.c_uint64, fp]
    L.ref_sla_rows.restype = C.c_uint64
    return L


def ref_sla_layers(raw):
    """The reference's layers for a raw (d, n) table, or None when its library is not
    built for this d."""
    d, n = raw.shape
    L = _lib(d)
    if L is None:
        return None
    out = np.zeros(n, np.uint32)
    if L.ref_sla_layers(np.ascontiguousarray(raw, np.float32).reshape(-1).copy(), n, d, out) == 0:
        raise RuntimeError("reference SLA failed")
    return out.astype(np.int64)


def ref_sla_rows(raw):
    """The reference's index rows (n, d), normalised, in its order, or None."""
    d, n = raw.shape
    L = _lib(d)
    if L is None:
        return None
    out = np.zeros((n, d), np.float32)
    got = L.ref_sla_rows(np.ascontiguousarray(raw, np.float32).reshape(-1).copy(), n, d, out.reshape(-1))
    if got != n:
        raise RuntimeError(f"reference SLA index returned {got} of {n} rows")
    return out
