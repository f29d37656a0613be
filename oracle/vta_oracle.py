"""Test infrastructure only: numpy restatement of the VTA and PTA index orders.

VTA::init (cpu/VTA.h:121-135): for every attribute m the list of (id, value) sorted by
value, descending (:121-127); every tuple's minimum position over the lists
(:130-133); tuples sorted by that position (:135) — inside each of VPARTITIONS row
ranges (1, or THREADS = 16 in the threaded build, cpu/VTA.h:13).  PTA::init
(cpu/PTA.h:88-167, 203-236): groups by median splits of hyperspherical angles, then
the same order inside each group.  The reference sorts with __gnu_parallel::sort,
which is not stable: rows sharing a minimum position (frequent: up to d rows share
each) and equal values come in an unspecified order.  This restatement and the
device order both break those ties by the lower id.  Values compare through the
order-preserving 32-bit image of FP32 used throughout this library (NaN lowest).

Pinned against the reference itself: `ref_index_rows` runs the reference's own VTA
and PTA builds (compiled by oracle/build.py) and `same_order_up_to_ties` checks that
an order matches the reference's up to those ties (tests/test_vta_oracle.py).
"""
import numpy as np


def f2key(x):
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    k = np.where(u & 0x80000000, (~u) & 0xFFFFFFFF, u | 0x80000000)
    return np.where(np.isnan(np.asarray(x, np.float32)), 0, k).astype(np.uint64)


def min_positions(table, groups):
    """Every row's minimum position over the attribute lists, each list sorted by
    (group, value descending, lower id): VTA's step inside each group
    (cpu/VTA.h:121-133, cpu/PTA.h:218-234).  A group's rows hold one range of positions
    in every list, so sorting by this position orders rows by group and, inside one,
    by the group-local minimum position."""
    d, n = table.shape
    ids = np.arange(n, dtype=np.int64)
    minpos = np.full(n, n, dtype=np.int64)
    for m in range(d):
        lst = np.lexsort((ids, -f2key(table[m]).astype(np.int64), groups))
        pos = np.empty(n, np.int64)
        pos[lst] = ids
        minpos = np.minimum(minpos, pos)
    return minpos


def vta_groups(n, slices=1):
    """slices > 1: the reference's threaded build (IMP 2) splits the rows into
    VPARTITIONS = THREADS ranges of ceil(n / slices) rows, each ordered on its own
    (cpu/VTA.h:13,78-85)."""
    ids = np.arange(n, dtype=np.int64)
    return ids // ((n - 1) // slices + 1) if n else ids


def vta_order(table, slices=1):
    """table: (d, n) column-major values.  Returns the row permutation (uint32)."""
    d, n = table.shape
    minpos = min_positions(table, vta_groups(n, slices))
    return np.lexsort((np.arange(n), minpos)).astype(np.uint32)


def pta_angle_keys(table):
    """The d-1 hyperspherical angle coordinates of PTA::polar (cpu/PTA.h:88-151) as
    sort magnitudes |f_c|, f_c = sqrt(sum_{j>c} (x_j - 1.1f)^2) / (x_c - 1.1f), in FP32
    with every operation rounded on its own (the AVX path, cpu/PTA.h:108-134).  The
    reference stores |atan(f_c)| * 180/pi; atan and the scaling are monotone, so that
    angle orders the rows as |f_c| does, up to ties the reference's sort leaves
    unspecified.  Returns a (d-1, n) float32 array."""
    x = np.ascontiguousarray(table, np.float32)
    d, n = x.shape
    one = np.float32(1.1)
    out = np.empty((max(d - 1, 0), n), np.float32)
    s = np.zeros(n, np.float32)
    curr = x[d - 1] - one
    for m in range(d - 1, 0, -1):
        nxt = x[m - 1] - one
        s = s + curr * curr
        out[m - 1] = np.abs(np.sqrt(s) / nxt)
        curr = nxt
    return out


def pta_part_ids(table):
    """PTA's partition of every row (cpu/PTA.h:152-167): for each angle coordinate c,
    the rows ascending by angle (ties: lower id), part += 2^c * (rank // (n // 2)),
    then part = min(part, 2^(d-1) - 1).  Needs n >= 2."""
    d, n = table.shape
    ids = np.arange(n, dtype=np.int64)
    part = np.zeros(n, np.int64)
    mod = n // 2
    for c, f in enumerate(pta_angle_keys(table)):
        order = np.lexsort((ids, f2key(f).astype(np.int64)))
        rank = np.empty(n, np.int64)
        rank[order] = ids
        part += (1 << c) * (rank // mod)
    return np.minimum(part, (1 << (d - 1)) - 1)


def pta_order(table):
    """PTA's index order (cpu/PTA.h:203-236): rows grouped by partition (ascending
    id), inside each the VTA order of the partition's rows (lists by value descending,
    minimum position, ties by the lower id).  Returns the row permutation (uint32)."""
    d, n = table.shape
    minpos = min_positions(table, pta_part_ids(table))
    return np.lexsort((np.arange(n), minpos)).astype(np.uint32)


def key2f(k):
    k = np.asarray(k, np.uint64)
    u = np.where(k & 0x80000000, k & 0x7FFFFFFF, (~k) & 0xFFFFFFFF).astype(np.uint32)
    return u.view(np.float32)


def kd_nodes(parts, P, level):
    """Node id at `level` of every partition number in `parts`: the path from the root
    over [0, P), each node [lo, hi) split at lo + ceil((hi - lo) / 2), left 0, right 1."""
    parts = np.asarray(parts, np.int64)
    lo = np.zeros_like(parts)
    hi = np.full_like(parts, P)
    node = np.zeros_like(parts)
    for _ in range(level):
        mid = lo + (hi - lo + 1) // 2
        right = parts >= mid
        node = 2 * node + right
        lo = np.where(right, mid, lo)
        hi = np.where(right, hi, mid)
    return node


def kd_order(table, part_rows):
    """The kd order of this library's partitioned copy (no reference counterpart; the
    device build is topk_b200/csrc/partition.cu): level by level, every node's rows are
    sorted stably by the attribute whose values spread widest in the node (FP32 max -
    min over the non-NaN values, 0 for a node without any; the lower attribute on a
    tie), the node's range splitting at its middle partition boundary.  Returns the row
    permutation (uint32)."""
    d, n = table.shape
    lg = int(part_rows).bit_length() - 1
    P = (n + part_rows - 1) // part_rows
    levels = max(0, (P - 1).bit_length())
    perm = np.arange(n, dtype=np.int64)
    parts = np.arange(n, dtype=np.int64) >> lg
    for level in range(levels):
        nodes = 1 << level
        node = kd_nodes(parts, P, level)
        vals = table[:, perm]
        keys = f2key(vals)
        nan = np.isnan(vals)
        spread = np.zeros((nodes, d), np.float32)
        # nodes are ranges of positions in node order: reduce over each range
        present, starts = np.unique(node, return_index=True)
        for m in range(d):
            kmax = np.zeros(nodes, np.uint64)
            kmin = np.full(nodes, 0xFFFFFFFF, np.uint64)
            kmax[present] = np.maximum.reduceat(np.where(nan[m], 0, keys[m]), starts)
            kmin[present] = np.minimum.reduceat(np.where(nan[m], 0xFFFFFFFF, keys[m]).astype(np.uint64), starts)
            has = kmax != 0
            sp = np.zeros(nodes, np.float32)
            sp[has] = key2f(kmax[has]) - key2f(kmin[has])
            sp[np.isnan(sp)] = 0.0
            spread[:, m] = sp
        attr = np.argmax(spread, axis=1)  # first of equal maxima
        k = (node.astype(np.uint64) << np.uint64(32)) | keys[attr[node], np.arange(n)]
        perm = perm[np.argsort(k, kind="stable")]
    return perm.astype(np.uint32)


def same_order_up_to_ties(table, groups, perm_a, perm_b):
    """True when two row orders agree up to the ties the reference leaves unspecified:
    the same group and the same minimum position at every place (rows sharing both
    may come in any order)."""
    mp = min_positions(table, groups)
    return (np.array_equal(np.sort(perm_a), np.arange(len(mp))) and
            np.array_equal(groups[perm_a], groups[perm_b]) and np.array_equal(mp[perm_a], mp[perm_b]))


def ref_index_rows(kind, raw, imp=2):
    """The reference's own index build (oracle/_ref/libref_index_d{d}_imp{imp}.so, built
    from cpu/VTA.h and cpu/PTA.h by oracle/build.py) on the raw (d, n) table: kind "vta"
    or "pta".  Returns (rows (n, d) normalised, in the reference's index order, the
    reference's init time in ms), or None when that library is not built."""
    import ctypes as C
    import os

    from . import build as B
    d, n = raw.shape
    path = B.ref_index_so(d, imp)
    if not os.path.exists(path):
        return None
    L = C.CDLL(path)
    fp = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
    fn = L.ref_vta_rows if kind == "vta" else L.ref_pta_rows
    fn.argtypes = [fp, C.c_uint64, C.c_uint64, fp, C.POINTER(C.c_double)]
    fn.restype = C.c_uint64
    out = np.zeros((n, d), np.float32)
    ms = C.c_double()
    got = fn(np.ascontiguousarray(raw, np.float32).reshape(-1).copy(), n, d, out.reshape(-1), C.byref(ms))
    if got != n:
        raise RuntimeError(f"reference {kind} index returned {got} of {n} rows")
    return out, ms.value


def rows_to_ids(table, rows):
    """Row ids of the (n, d) rows in a table whose rows are distinct."""
    lookup = {r.tobytes(): i for i, r in enumerate(np.ascontiguousarray(table.T))}
    return np.array([lookup[r.tobytes()] for r in np.ascontiguousarray(rows)], np.int64)
