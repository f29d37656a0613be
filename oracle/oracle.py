"""ctypes view of the CPU checker (TEST INFRASTRUCTURE ONLY).

Imported only by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
reference legs.  The product package never imports this module.

  Oracle  - the C restatement in topk_oracle.c (cites the reference per function).
  RefTPAc - the reference's own TPAc<float,uint64_t> (cpu/TPAc.h) compiled strict
            into oracle/_ref/libref_tpac.so by oracle/build.py.
  RefTPAr - the reference's row-major TPAr<float,uint64_t> (cpu/TPAr.h), same library.
  RefTA   - the reference's TA<float,uint64_t> (cpu/TA.h), same library.
"""
import ctypes as C
import os

import numpy as np

from . import build as _build

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")

CORRELATED, INDEPENDENT, ANTICORRELATED, MIXED = 0, 1, 2, 3

_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        path = _build.ORACLE_SO
        if not os.path.exists(path):
            path = _build.build_oracle()
        L = C.CDLL(path)
        L.orc_generate.argtypes = [_f32p, C.c_uint64, C.c_uint32, C.c_uint64, C.c_uint64, C.c_int, C.c_uint64]
        L.orc_gen_weights.argtypes = [_f32p, C.c_uint32, C.c_uint64, C.c_uint64]
        L.orc_normalize.argtypes = [_f32p, C.c_uint64, C.c_uint64, C.c_uint32, C.c_void_p, C.c_void_p]
        L.orc_score.argtypes = [_f32p, C.c_uint64, C.c_uint64, C.c_uint32, _f32p, _u8p]
        L.orc_score.restype = C.c_float
        L.orc_topk.argtypes = [_f32p, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint32, _f32p, _u8p,
                               C.c_uint64, _u64p, _f32p, C.POINTER(C.c_float)]
        L.orc_topk.restype = C.c_uint64
        L.orc_topk_f64.argtypes = [_f32p, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint32, _f32p, _u8p,
                                   C.c_uint64, _u64p, _f64p]
        L.orc_topk_f64.restype = C.c_uint64
        L.orc_key.argtypes = [C.c_float]
        L.orc_key.restype = C.c_uint32
        _lib = L
    return _lib


def generate(n, d, dist, seed, ld=None, row0=0, rows=None):
    """Column-major (d, ld) float32 table; rows [row0, row0+rows) filled."""
    ld = n if ld is None else ld
    rows = n - row0 if rows is None else rows
    t = np.zeros((d, ld), np.float32)
    lib().orc_generate(t.reshape(-1), ld, d, row0, rows, dist, seed)
    return t


def gen_weights(count, seed, stream):
    w = np.empty(count, np.float32)
    lib().orc_gen_weights(w, count, seed, stream)
    return w


def normalize(table, n=None):
    """In-place normalize_transpose on a (d, ld) table; returns (mins, maxs)."""
    d, ld = table.shape
    n = ld if n is None else n
    mins = np.empty(d, np.float32)
    maxs = np.empty(d, np.float32)
    lib().orc_normalize(table.reshape(-1), n, ld, d, mins.ctypes.data, maxs.ctypes.data)
    return mins, maxs


def _q(weights, attr):
    return np.ascontiguousarray(weights, np.float32), np.ascontiguousarray(attr, np.uint8)


def topk(table, k, weights, attr, row0=0, row1=None):
    """Exact top-k, ascending by (score, -id). Returns (ids, scores, threshold)."""
    d, ld = table.shape
    row1 = ld if row1 is None else row1
    w, a = _q(weights, attr)
    cap = max(1, min(k, row1 - row0))
    ids = np.zeros(cap, np.uint64)
    sc = np.zeros(cap, np.float32)
    th = C.c_float(0)
    c = lib().orc_topk(table.reshape(-1), ld, row0, row1, len(a), w, a, k, ids, sc, C.byref(th))
    return ids[:c], sc[:c], th.value


def topk_f64(table, k, weights, attr, row0=0, row1=None):
    d, ld = table.shape
    row1 = ld if row1 is None else row1
    w, a = _q(weights, attr)
    cap = max(1, min(k, row1 - row0))
    ids = np.zeros(cap, np.uint64)
    sc = np.zeros(cap, np.float64)
    c = lib().orc_topk_f64(table.reshape(-1), ld, row0, row1, len(a), w, a, k, ids, sc)
    return ids[:c], sc[:c]


def scores(table, weights, attr, ids=None):
    """Vectorised exact FP32 scores in the reference order (numpy, same roundings)."""
    w, a = _q(weights, attr)
    s = None
    for m in a:
        col = table[m] if ids is None else table[m][ids]
        p = (col * w[m]).astype(np.float32)
        # the first term is 0 + p, not p: a -0 product (negative weight) becomes +0
        s = (np.float32(0) + p).astype(np.float32) if s is None else (s + p).astype(np.float32)
    if s is None:
        n = table.shape[1] if ids is None else len(ids)
        s = np.zeros(n, np.float32)
    return s


def key(s):
    """Order-preserving uint32 keys of float32 scores (NaN -> 0)."""
    s = np.asarray(s, np.float32)
    u = s.view(np.uint32)
    k = np.where(u & np.uint32(0x80000000), ~u, u | np.uint32(0x80000000)).astype(np.uint32)
    return np.where(np.isnan(s), np.uint32(0), k)


def topk_numpy(table, k, weights, attr, row0=0, row1=None):
    """Vectorised equivalent of topk() for larger tables (same tie rule)."""
    d, ld = table.shape
    row1 = ld if row1 is None else row1
    s = scores(table[:, row0:row1], weights, attr)
    kk = key(s).astype(np.uint64)
    ids = np.arange(row0, row1, dtype=np.uint64)
    comp = (kk << np.uint64(32)) | (np.uint64(0xFFFFFFFF) - (ids - np.uint64(row0)))
    c = min(k, row1 - row0)
    if c == 0:
        return ids[:0], s[:0], 0.0
    part = np.argpartition(comp, len(comp) - c)[len(comp) - c:]
    order = part[np.argsort(comp[part])]
    return ids[order], s[order], float(s[order[0]])


class RefTPAc:
    """The reference TPAc<float,uint64_t> through oracle/_ref/libref_tpac.so."""

    _L = None

    @classmethod
    def available(cls):
        return os.path.exists(_build.REF_SO) or _build.build_ref() is not None

    @classmethod
    def lib(cls):
        if cls._L is None:
            path = _build.REF_SO if os.path.exists(_build.REF_SO) else _build.build_ref()
            if path is None or not os.path.exists(path):
                raise RuntimeError("reference TPAc library not built (oracle/_ref/libref_tpac.so)")
            L = C.CDLL(path)
            L.ref_tpac_create.argtypes = [C.c_uint64, C.c_uint64]
            L.ref_tpac_create.restype = C.c_void_p
            L.ref_tpac_destroy.argtypes = [C.c_void_p]
            L.ref_tpac_load.argtypes = [C.c_void_p, _f32p, C.c_uint64, C.c_uint64]
            L.ref_tpac_init.argtypes = [C.c_void_p]
            L.ref_tpac_get_data.argtypes = [C.c_void_p, _f32p, C.c_uint64, C.c_uint64]
            L.ref_tpac_query.argtypes = [C.c_void_p, C.c_int, C.c_uint64, C.c_uint8, _f32p, _u8p, _u64p, _f32p,
                                         C.c_uint64, C.POINTER(C.c_float), C.POINTER(C.c_double)]
            L.ref_tpac_query.restype = C.c_uint64
            L.ref_tpac_mq.argtypes = [C.c_void_p, C.c_uint64, _u64p, _u8p, _f32p, _u8p, C.c_uint64, C.c_int]
            L.ref_tpac_mq.restype = C.c_double
            L.ref_normalize_transpose.argtypes = [_f32p, C.c_uint64, C.c_uint64]
            L.ref_threads_constant.restype = C.c_int
            cls._L = L
        return cls._L

    def __init__(self, table):
        """table: (d, n) float32 column-major; copied into reference-owned memory."""
        self.d, self.n = table.shape
        L = self.lib()
        self.h = L.ref_tpac_create(self.n, self.d)
        if L.ref_tpac_load(self.h, np.ascontiguousarray(table, np.float32).reshape(-1), self.n, self.d):
            raise MemoryError("reference table allocation failed")

    def init(self):
        self.lib().ref_tpac_init(self.h)

    def data(self):
        out = np.empty((self.d, self.n), np.float32)
        self.lib().ref_tpac_get_data(self.h, out.reshape(-1), self.n, self.d)
        return out

    def query(self, impl, k, weights, attr):
        """impl 0 scalar, 1 simd, 2 threads. Returns (ids, scores, threshold, ms)."""
        w = np.zeros(max(self.d, len(weights)), np.float32)
        w[: len(weights)] = weights
        a = np.ascontiguousarray(attr, np.uint8)
        cap = max(1, min(k, self.n))
        ids = np.zeros(cap, np.uint64)
        sc = np.zeros(cap, np.float32)
        th = C.c_float(0)
        ms = C.c_double(0)
        c = self.lib().ref_tpac_query(self.h, impl, k, len(a), w, a, ids, sc, cap, C.byref(th), C.byref(ms))
        c = min(c, cap)
        return ids[:c], sc[:c], th.value, ms.value

    def mq(self, ks, qqs, weights, attrs, threads):
        """findTopKsimdMQ loop; weights/attrs are (nq, stride) arrays. Returns ms."""
        ks = np.ascontiguousarray(ks, np.uint64)
        qqs = np.ascontiguousarray(qqs, np.uint8)
        w = np.ascontiguousarray(weights, np.float32)
        a = np.ascontiguousarray(attrs, np.uint8)
        assert w.shape == a.shape
        return self.lib().ref_tpac_mq(self.h, len(ks), ks, qqs, w.reshape(-1), a.reshape(-1), w.shape[1], threads)

    def close(self):
        if self.h:
            self.lib().ref_tpac_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RefTPAr:
    """The reference TPAr<float,uint64_t> (cpu/TPAr.h, the row-major variant) through
    oracle/_ref/libref_tpac.so.  Its query loops step 8 or 16 objects with no tail, so
    n must be a multiple of 16 * THREADS (256)."""

    _L = None

    @classmethod
    def lib(cls):
        if cls._L is None:
            L = RefTPAc.lib()
            L.ref_tpar_create.argtypes = [C.c_uint64, C.c_uint64]
            L.ref_tpar_create.restype = C.c_void_p
            L.ref_tpar_destroy.argtypes = [C.c_void_p]
            L.ref_tpar_load.argtypes = [C.c_void_p, _f32p, C.c_uint64, C.c_uint64]
            L.ref_tpar_init.argtypes = [C.c_void_p]
            L.ref_tpar_get_data.argtypes = [C.c_void_p, _f32p, C.c_uint64, C.c_uint64]
            L.ref_tpar_query.argtypes = [C.c_void_p, C.c_int, C.c_uint64, C.c_uint8, _f32p, _u8p, _u64p, _f32p,
                                         C.c_uint64, C.POINTER(C.c_float), C.POINTER(C.c_double)]
            L.ref_tpar_query.restype = C.c_uint64
            cls._L = L
        return cls._L

    def __init__(self, rows):
        """rows: (n, d) float32 row-major; copied into reference-owned memory."""
        self.n, self.d = rows.shape
        if self.n % 256:
            raise ValueError("the reference TPAr needs n to be a multiple of 256")
        L = self.lib()
        self.h = L.ref_tpar_create(self.n, self.d)
        if L.ref_tpar_load(self.h, np.ascontiguousarray(rows, np.float32).reshape(-1), self.n, self.d):
            raise MemoryError("reference table allocation failed")

    def init(self):
        self.lib().ref_tpar_init(self.h)

    def data(self):
        out = np.empty((self.n, self.d), np.float32)
        self.lib().ref_tpar_get_data(self.h, out.reshape(-1), self.n, self.d)
        return out

    def query(self, impl, k, weights, attr):
        """impl 0 scalar, 1 simd, 2 threads. Returns (ids, scores, threshold, ms)."""
        w = np.zeros(max(self.d, len(weights)), np.float32)
        w[: len(weights)] = weights
        a = np.ascontiguousarray(attr, np.uint8)
        cap = max(1, min(k, self.n))
        ids = np.zeros(cap, np.uint64)
        sc = np.zeros(cap, np.float32)
        th = C.c_float(0)
        ms = C.c_double(0)
        c = self.lib().ref_tpar_query(self.h, impl, k, len(a), w, a, ids, sc, cap, C.byref(th), C.byref(ms))
        c = min(c, cap)
        return ids[:c], sc[:c], th.value, ms.value

    def close(self):
        if self.h:
            self.lib().ref_tpar_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RefTA:
    """The reference TA<float,uint64_t> (cpu/TA.h) through oracle/_ref/libref_tpac.so:
    sorted lists over a row-major table, findTopK."""

    _L = None

    @classmethod
    def lib(cls):
        if cls._L is None:
            L = RefTPAc.lib()
            L.ref_ta_create.argtypes = [C.c_uint64, C.c_uint64]
            L.ref_ta_create.restype = C.c_void_p
            L.ref_ta_destroy.argtypes = [C.c_void_p]
            L.ref_ta_load.argtypes = [C.c_void_p, _f32p, C.c_uint64, C.c_uint64]
            L.ref_ta_init.argtypes = [C.c_void_p]
            L.ref_ta_query.argtypes = [C.c_void_p, C.c_uint64, C.c_uint8, _f32p, _u8p, _u64p, _f32p, C.c_uint64,
                                       C.POINTER(C.c_float), C.POINTER(C.c_double)]
            L.ref_ta_query.restype = C.c_uint64
            cls._L = L
        return cls._L

    def __init__(self, rows):
        self.n, self.d = rows.shape
        L = self.lib()
        self.h = L.ref_ta_create(self.n, self.d)
        if L.ref_ta_load(self.h, np.ascontiguousarray(rows, np.float32).reshape(-1), self.n, self.d):
            raise MemoryError("reference table allocation failed")

    def init(self):
        self.lib().ref_ta_init(self.h)

    def query(self, k, weights, attr):
        """Returns (ids, scores, threshold, ms)."""
        w = np.zeros(max(self.d, len(weights)), np.float32)
        w[: len(weights)] = weights
        a = np.ascontiguousarray(attr, np.uint8)
        cap = max(1, min(k, self.n))
        ids = np.zeros(cap, np.uint64)
        sc = np.zeros(cap, np.float32)
        th = C.c_float(0)
        ms = C.c_double(0)
        c = self.lib().ref_ta_query(self.h, k, len(a), w, a, ids, sc, cap, C.byref(th), C.byref(ms))
        c = min(c, cap)
        return ids[:c], sc[:c], th.value, ms.value

    def close(self):
        if self.h:
            self.lib().ref_ta_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
