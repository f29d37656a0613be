"""Python handle over the C ABI: one n x d FP32 table resident on one GPU."""
import ctypes as C
import os
import threading

import numpy as np

from . import _lib
from ._lib import check


def _weights(w, d):
    w = np.ascontiguousarray(w, np.float32).reshape(-1)
    if len(w) < d:
        raise ValueError(f"weights are indexed by attribute id and need length >= d={d}, got {len(w)}")
    return w


def _attr(a):
    return np.ascontiguousarray(a, np.uint8).reshape(-1)


class _CallBlock:
    """One host thread's argument and result buffers for the per-query calls, at
    fixed addresses: ids (MAX_K u64), scores (MAX_K f32), weights (MAX_D f32),
    attributes (MAX_Q u8), stats (4 u64), count (u64), threshold and cut (f32).
    A call copies its weights and attributes in and its results out, so the
    buffers are free again when the method returns."""

    _IDS, _SC = 0, 8 * _lib.MAX_K
    _W = _SC + 4 * _lib.MAX_K
    _A = _W + 4 * 256
    _ST = _A + _lib.MAX_Q
    _CNT = _ST + 32
    _TH = _CNT + 8
    _CUT = _TH + 4
    _BYTES = _CUT + 4

    def __init__(self):
        b = np.zeros(self._BYTES, np.uint8)
        self.buf = b
        base = b.ctypes.data
        self.ids = b[self._IDS:self._SC].view(np.uint64)
        self.sc = b[self._SC:self._W].view(np.float32)
        self.w = b[self._W:self._A].view(np.float32)
        self.a = b[self._A:self._ST]
        self.st = b[self._ST:self._CNT].view(np.uint64)
        self.cnt = b[self._CNT:self._TH].view(np.uint64)
        self.f = b[self._TH:self._BYTES].view(np.float32)  # threshold, cut
        self.p_ids, self.p_sc, self.p_w, self.p_a = (base + self._IDS, base + self._SC, base + self._W,
                                                     base + self._A)
        self.p_st, self.p_cnt, self.p_th, self.p_cut = (base + self._ST, base + self._CNT, base + self._TH,
                                                        base + self._CUT)

    def args_in(self, w, a, d):
        """Copy a query's weights (the first d) and attributes into the block; False
        when they do not fit (the caller then takes the checked bindings, whose C
        call reports the error)."""
        if len(a) > _lib.MAX_Q or d > 256:
            return False
        self.w[:d] = w[:d]
        self.a[:len(a)] = a
        return True

    def results(self):
        c = int(self.cnt[0])
        return self.ids[:c].copy(), self.sc[:c].copy(), float(self.f[0])


_tls = threading.local()


def _call_block():
    b = getattr(_tls, "blk", None)
    if b is None:
        b = _tls.blk = _CallBlock()
    return b


class Table:
    """Device-resident column-major table (the device copy of AA::cdata).

    Entry points map one-to-one onto include/topk_b200.h.
    """

    def __init__(self, n, d, device=0):
        L = _lib.load()
        h = C.c_void_p()
        check(L.topk_create(int(n), int(d), int(device), C.byref(h)))
        self._h = h
        self.n, self.d, self.device = int(n), int(d), int(device)
        ld = C.c_uint64()
        check(L.topk_shape(self._h, None, None, C.byref(ld)))
        self.ld = ld.value

    # -- data ---------------------------------------------------------------
    def upload(self, table):
        """table: (d, ld_host) float32, column m in row m (column-major host layout)."""
        t = np.ascontiguousarray(table, np.float32)
        if t.ndim != 2 or t.shape[0] != self.d or t.shape[1] < self.n:
            raise ValueError(f"expected a ({self.d}, >= {self.n}) array, got {t.shape}")
        check(_lib.load().topk_upload_colmajor(self._h, t.reshape(-1), t.shape[1]))

    def upload_rowmajor(self, rows):
        """rows: (n, row_stride >= d) float32, object i in row i (TPAr's layout)."""
        r = np.ascontiguousarray(rows, np.float32)
        if r.ndim != 2 or r.shape[0] != self.n or r.shape[1] < self.d:
            raise ValueError(f"expected a ({self.n}, >= {self.d}) array, got {r.shape}")
        check(_lib.load().topk_upload_rowmajor(self._h, r.reshape(-1), r.shape[1]))

    def download_rowmajor(self):
        out = np.empty((self.n, self.d), np.float32)
        check(_lib.load().topk_download_rowmajor(self._h, out.reshape(-1), self.d))
        return out

    def load_csv(self, path, chunk_bytes=0):
        """The first n rows of a comma-separated file, parsed on the device (File<float>::load
        with transpose, input/File.h:233-265).  Returns the loader's counters."""
        st = np.zeros(4, np.uint64)
        check(_lib.load().topk_load_csv(self._h, os.fsencode(path), int(chunk_bytes), st))
        return {"bytes": int(st[0]), "rows": int(st[1]), "host_converted": int(st[2]), "chunks": int(st[3])}

    def save_csv(self, path):
        """One line per object, "%f" fields separated by ',' (File<float>::store)."""
        check(_lib.load().topk_save_csv(self._h, os.fsencode(path)))

    def load_binary(self, path):
        check(_lib.load().topk_load_binary(self._h, os.fsencode(path)))

    def save_binary(self, path):
        check(_lib.load().topk_save_binary(self._h, os.fsencode(path)))

    @classmethod
    def from_csv(cls, path, device=0, chunk_bytes=0):
        """A table of the file's shape as File<T>::count reads it (n = newlines), loaded
        on the device.  Blank lines count in n but hold no row, so a file with blank
        lines needs Table(rows, d).load_csv(path) instead."""
        n, d = csv_shape(path)
        t = cls(n, d, device)
        t.load_csv(path, chunk_bytes)
        return t

    @classmethod
    def from_binary(cls, path, device=0):
        n, d = binary_shape(path)
        t = cls(n, d, device)
        t.load_binary(path)
        return t

    def generate(self, dist, seed):
        check(_lib.load().topk_generate(self._h, int(dist), int(seed)))

    def normalize(self):
        mins = np.empty(self.d, np.float32)
        maxs = np.empty(self.d, np.float32)
        check(_lib.load().topk_normalize(self._h, mins.ctypes.data, maxs.ctypes.data))
        return mins, maxs

    def download(self):
        out = np.empty((self.d, self.n), np.float32)
        check(_lib.load().topk_download_colmajor(self._h, out.reshape(-1), self.n))
        return out

    def gather_rows(self, ids):
        ids = np.ascontiguousarray(ids, np.uint64)
        out = np.empty((len(ids), self.d), np.float32)
        check(_lib.load().topk_gather_rows(self._h, ids, len(ids), out.reshape(-1)))
        return out

    # -- queries ------------------------------------------------------------
    def query(self, k, weights, attr, row_begin=None, row_end=None):
        """Exact top-k; returns (ids uint64, scores float32, threshold) ascending by score."""
        w, a = _weights(weights, self.d), _attr(attr)
        r0 = 0 if row_begin is None else int(row_begin)
        r1 = self.n if row_end is None else int(row_end)
        cap = max(1, min(int(k), max(r1 - r0, 0)))
        b = _call_block()
        if cap <= _lib.MAX_K and b.args_in(w, a, self.d):
            F = _lib.lean()
            if row_begin is None and row_end is None:
                check(F.topk_query(self._h, int(k), len(a), b.p_w, b.p_a, b.p_ids, b.p_sc, b.p_cnt, b.p_th))
            else:
                check(F.topk_query_range(self._h, r0, r1, int(k), len(a), b.p_w, b.p_a, b.p_ids, b.p_sc, b.p_cnt,
                                         b.p_th))
            return b.results()
        L = _lib.load()
        ids = np.empty(cap, np.uint64)
        sc = np.empty(cap, np.float32)
        cnt = C.c_uint64()
        th = C.c_float()
        if row_begin is None and row_end is None:
            check(L.topk_query(self._h, int(k), len(a), w, a, ids, sc, C.byref(cnt), C.byref(th)))
        else:
            check(L.topk_query_range(self._h, r0, r1, int(k), len(a), w, a, ids, sc, C.byref(cnt), C.byref(th)))
        c = cnt.value
        return ids[:c], sc[:c], th.value

    # -- threshold algorithm over sorted lists -----------------------------
    def build_lists(self):
        """TA::init's sorted lists (cpu/TA.h:40-58), built on the device."""
        check(_lib.load().topk_build_lists(self._h))

    def read_list(self, m):
        """(ids uint32, values float32) of attribute m's list, value descending."""
        ids = np.empty(self.n, np.uint32)
        vals = np.empty(self.n, np.float32)
        check(_lib.load().topk_read_list(self._h, int(m), ids, vals))
        return ids, vals

    def query_ta(self, k, weights, attr):
        """Exact top-k by the threshold algorithm (cpu/TA.h:61-96); returns (ids, scores,
        threshold, stats) with stats = (depth walked, objects scored, blocks)."""
        w, a = _weights(weights, self.d), _attr(attr)
        cap = max(1, min(int(k), self.n))
        ids = np.empty(cap, np.uint64)
        sc = np.empty(cap, np.float32)
        cnt = C.c_uint64()
        th = C.c_float()
        st = np.zeros(3, np.uint64)
        check(_lib.load().topk_query_ta(self._h, int(k), len(a), w, a, ids, sc, C.byref(cnt), C.byref(th), st))
        c = cnt.value
        return ids[:c], sc[:c], th.value, tuple(int(x) for x in st)

    def query_device(self, k, weights, attr, d_ids, d_scores, d_threshold=0, stream=0):
        """Asynchronous query writing into device pointers (ints) on a stream (int handle)."""
        w, a = _weights(weights, self.d), _attr(attr)
        check(_lib.load().topk_query_device(self._h, int(k), len(a), w, a, C.c_void_p(d_ids), C.c_void_p(d_scores),
                                            C.c_void_p(d_threshold or None), C.c_void_p(stream or None)))

    def query_range_device(self, row_begin, row_end, k, weights, attr, d_ids, d_scores, d_threshold=0, stream=0):
        """query_device over rows [row_begin, row_end) only; global ids."""
        w, a = _weights(weights, self.d), _attr(attr)
        check(_lib.load().topk_query_range_device(self._h, int(row_begin), int(row_end), int(k), len(a), w, a,
                                                  C.c_void_p(d_ids), C.c_void_p(d_scores),
                                                  C.c_void_p(d_threshold or None), C.c_void_p(stream or None)))

    def query_batch(self, ks, weights, attrs, qqs=None, out=None):
        """ks: (nq,), weights: (nq, >=d), attrs: (nq, astride) with qqs[j] valid ids each.
        Returns (ids, scores, counts, thresholds); row j of ids and scores holds
        counts[j] entries, the rest of the row is zero.

        out: optional (ids, scores, counts, thresholds) arrays to write into, of dtypes
        uint64, float32, uint64, float32 and shapes (nq, kstride), (nq, kstride), (nq,),
        (nq,) with kstride = min(max(ks), n), C-contiguous.  A caller that answers
        batches of one shape in a loop keeps them across calls instead of taking fresh
        zeroed arrays each time (whose first-touch page faults cost more than the copy
        of the results into them); then only the first counts[j] entries of row j are
        written, the rest of the row keeps what was there.  Returns the same arrays."""
        L = _lib.load()
        ks = np.ascontiguousarray(ks, np.uint64)
        nq = len(ks)
        W = np.ascontiguousarray(weights, np.float32).reshape(nq, -1)
        A = np.ascontiguousarray(attrs, np.uint8).reshape(nq, -1)
        qqs = np.full(nq, A.shape[1], np.uint32) if qqs is None else np.ascontiguousarray(qqs, np.uint32)
        kstride = int(max(1, min(int(ks.max()) if nq else 1, self.n)))
        if out is None:
            ids = np.zeros((nq, kstride), np.uint64)
            sc = np.zeros((nq, kstride), np.float32)
            counts = np.zeros(nq, np.uint64)
            ths = np.zeros(nq, np.float32)
        else:
            ids, sc, counts, ths = out
            for x, dt, shape, name in ((ids, np.uint64, (nq, kstride), "ids"), (sc, np.float32, (nq, kstride), "scores"),
                                       (counts, np.uint64, (nq,), "counts"), (ths, np.float32, (nq,), "thresholds")):
                if (not isinstance(x, np.ndarray) or x.dtype != dt or x.shape != shape or not x.flags.c_contiguous
                        or not x.flags.writeable):
                    raise ValueError(f"out {name}: need a writeable C-contiguous {np.dtype(dt).name} array of shape "
                                     f"{shape}")
        check(L.topk_query_batch(self._h, nq, ks, qqs, W.reshape(-1), W.shape[1], A.reshape(-1), A.shape[1],
                                 ids.reshape(-1), sc.reshape(-1), kstride, counts.ctypes.data, ths.ctypes.data))
        return ids, sc, counts, ths

    def set_batch_tiles(self, qt_per_cta=0, boot_rows=8192):
        check(_lib.load().topk_set_batch_tiles(self._h, int(qt_per_cta), int(boot_rows)))

    def batch_tiles(self):
        qt, boot = C.c_uint32(), C.c_uint32()
        check(_lib.load().topk_get_batch_tiles(self._h, C.byref(qt), C.byref(boot)))
        return qt.value, boot.value

    def tune_batch(self, ks, weights, attrs, qqs=None):
        """Autotune the batched path's tiles on these queries (see topk_tune_batch);
        returns {query_tiles_per_cta, boot_rows, best_ms, default_ms}."""
        ks = np.ascontiguousarray(ks, np.uint64)
        nq = len(ks)
        W = np.ascontiguousarray(weights, np.float32).reshape(nq, -1)
        A = np.ascontiguousarray(attrs, np.uint8).reshape(nq, -1)
        qqs = np.full(nq, A.shape[1], np.uint32) if qqs is None else np.ascontiguousarray(qqs, np.uint32)
        rep = np.zeros(4, np.float64)
        check(_lib.load().topk_tune_batch(self._h, nq, ks, qqs, W.reshape(-1), W.shape[1], A.reshape(-1), A.shape[1],
                                          rep))
        return {"query_tiles_per_cta": int(rep[0]), "boot_rows": int(rep[1]), "best_ms": float(rep[2]),
                "default_ms": float(rep[3])}

    # -- partitions and pruned queries -------------------------------------
    def build_partitions(self, part_rows=1 << 16, order=0):
        """order: ORDER_MORTON (0), ORDER_VTA (1), ORDER_PTA (2), ORDER_VTA_THREADS (3),
        ORDER_SLA (4) or ORDER_KD (5), see topk_build_partitions_ordered."""
        check(_lib.load().topk_build_partitions_ordered(self._h, int(part_rows), int(order)))

    def skyline_layers(self):
        """(layer of every row, number of layers): SLA's skyline layers (cpu/SLA.h:102-139)."""
        out = np.empty(self.n, np.uint32)
        nl = C.c_uint64()
        check(_lib.load().topk_skyline_layers(self._h, out, C.byref(nl)))
        return out, nl.value

    def partition_ids(self):
        """Row ids of the partitioned copy (row i of the copy is table row ids[i])."""
        out = np.empty(self.n, np.uint32)
        check(_lib.load().topk_partition_ids(self._h, out))
        return out

    def partition_info(self):
        """(part_rows, mins, maxs, means) with arrays of shape (num_parts, d)."""
        L = _lib.load()
        P, R = C.c_uint32(), C.c_uint32()
        check(L.topk_partition_info(self._h, C.byref(P), C.byref(R), None, None, None))
        mins = np.empty((P.value, self.d), np.float32)
        maxs = np.empty_like(mins)
        means = np.empty_like(mins)
        check(L.topk_partition_info(self._h, None, None, mins.ctypes.data, maxs.ctypes.data, means.ctypes.data))
        return R.value, mins, maxs, means

    def query_pruned(self, k, weights, attr, cut=float("nan")):
        """Exact top-k scanning only partitions that can reach the threshold;
        returns (ids, scores, threshold, stats) with stats = (partitions scanned,
        partitions, cut accepted, scans)."""
        w, a = _weights(weights, self.d), _attr(attr)
        cap = max(1, min(int(k), self.n))
        b = _call_block()
        if cap <= _lib.MAX_K and b.args_in(w, a, self.d):
            check(_lib.lean().topk_query_pruned(self._h, int(k), len(a), b.p_w, b.p_a, float(cut), b.p_ids, b.p_sc,
                                                b.p_cnt, b.p_th, b.p_st))
            return b.results() + (tuple(b.st.tolist()),)
        ids = np.empty(cap, np.uint64)
        sc = np.empty(cap, np.float32)
        st = np.zeros(4, np.uint64)
        cnt = C.c_uint64()
        th = C.c_float()
        check(_lib.load().topk_query_pruned(self._h, int(k), len(a), w, a, float(cut), ids, sc, C.byref(cnt),
                                            C.byref(th), st))
        c = cnt.value
        return ids[:c], sc[:c], th.value, tuple(int(x) for x in st)

    # -- learned k-th-score model ------------------------------------------
    def query_features(self, ks, weights, attrs, qqs=None):
        """(X, S): 2d + 18 features per query from the current partitions, and S."""
        ks = np.ascontiguousarray(ks, np.uint64)
        nq = len(ks)
        W = np.ascontiguousarray(weights, np.float32).reshape(nq, -1)
        A = np.ascontiguousarray(attrs, np.uint8).reshape(nq, -1)
        qqs = np.full(nq, A.shape[1], np.uint32) if qqs is None else np.ascontiguousarray(qqs, np.uint32)
        X = np.zeros((nq, 2 * self.d + 18), np.float32)
        S = np.zeros(nq, np.float32)
        check(_lib.load().topk_query_features(self._h, nq, ks, qqs, W.reshape(-1), W.shape[1], A.reshape(-1),
                                              A.shape[1], X.reshape(-1), S.ctypes.data))
        return X, S

    def set_learned_model(self, params, margin):
        p = None if params is None else np.ascontiguousarray(params, np.float32)
        check(_lib.load().topk_set_learned_model(self._h, None if p is None else p.ctypes.data, float(margin)))

    def get_learned_model(self):
        from . import learned
        p = np.empty(learned.param_count(2 * self.d + 18), np.float32)
        m = C.c_float()
        check(_lib.load().topk_get_learned_model(self._h, p.ctypes.data, C.byref(m)))
        return p, m.value

    def learned_fit(self, n_train, n_val, kmin=16, kmax=1024, qmin=2, qmax=None, epochs=20, miss_rate=0.01, seed=0):
        """Fit the handle's model (see topk_learned_fit); returns its report."""
        qmax = self.d if qmax is None else qmax
        rep = np.zeros(6, np.float64)
        check(_lib.load().topk_learned_fit(self._h, int(n_train), int(n_val), int(kmin), int(kmax), int(qmin),
                                           int(qmax), int(epochs), float(miss_rate), int(seed), rep.ctypes.data))
        keys = ("train_loss", "val_rmse", "margin", "val_miss_rate", "label_s", "train_s")
        return dict(zip(keys, rep.tolist()))

    def query_learned(self, k, weights, attr):
        """Exact top-k through the model; returns (ids, scores, threshold, stats, cut)."""
        w, a = _weights(weights, self.d), _attr(attr)
        cap = max(1, min(int(k), self.n))
        b = _call_block()
        if cap <= _lib.MAX_K and b.args_in(w, a, self.d):
            check(_lib.lean().topk_query_learned(self._h, int(k), len(a), b.p_w, b.p_a, b.p_ids, b.p_sc, b.p_cnt,
                                                 b.p_th, b.p_st, b.p_cut))
            return b.results() + (tuple(b.st.tolist()), float(b.f[1]))
        ids = np.empty(cap, np.uint64)
        sc = np.empty(cap, np.float32)
        st = np.zeros(4, np.uint64)
        cnt, th, cut = C.c_uint64(), C.c_float(), C.c_float()
        check(_lib.load().topk_query_learned(self._h, int(k), len(a), w, a, ids, sc, C.byref(cnt), C.byref(th), st,
                                             C.byref(cut)))
        c = cnt.value
        return ids[:c], sc[:c], th.value, tuple(int(x) for x in st), cut.value

    def count_ge(self, weights, attr, thr, row_begin=0, row_end=None):
        w, a = _weights(weights, self.d), _attr(attr)
        r1 = self.n if row_end is None else int(row_end)
        ge, gt = C.c_uint64(), C.c_uint64()
        check(_lib.load().topk_count_ge(self._h, int(row_begin), r1, len(a), w, a, float(thr), C.byref(ge),
                                        C.byref(gt)))
        return ge.value, gt.value

    def set_batch_method(self, method):
        """0 auto, 1 loop of single-query scans, 2 batched FP32, 3 BF16 tensor-core
        filter with exact rescoring, 4 BF16 with the learned start (see
        include/topk_b200.h)."""
        check(_lib.load().topk_set_batch_method(self._h, int(method)))

    def last_batch_stats(self):
        L = _lib.load()
        ms, fb, cand = C.c_double(), C.c_uint64(), C.c_uint64()
        check(L.topk_last_batch_stats(self._h, C.byref(ms), C.byref(fb), C.byref(cand)))
        method, ratio, miss = C.c_int(), C.c_double(), C.c_uint64()
        check(L.topk_last_batch_info(self._h, C.byref(method), C.byref(ratio), C.byref(miss)))
        sw, ret, fl = C.c_uint64(), C.c_uint64(), C.c_double()
        check(L.topk_last_batch_switched(self._h, C.byref(sw)))
        check(L.topk_last_batch_retired(self._h, C.byref(ret)))
        check(L.topk_last_batch_filter_flops(self._h, C.byref(fl)))
        return {"device_ms": ms.value, "fallbacks": fb.value, "candidates": cand.value, "method": method.value,
                "max_err_ratio": ratio.value, "learned_misses": miss.value, "switched_fp32": sw.value,
                "retired": ret.value, "filter_flops": fl.value}

    def set_scan_tuning(self, max_ctas_per_sm=0):
        check(_lib.load().topk_set_scan_tuning(self._h, int(max_ctas_per_sm)))

    def set_fault_injection(self, mode):
        check(_lib.load().topk_set_fault_injection(self._h, int(mode)))

    def last_stats(self):
        c, r = C.c_uint64(), C.c_uint64()
        check(_lib.load().topk_last_stats(self._h, C.byref(c), C.byref(r)))
        return c.value, r.value

    def set_wait_limit(self, iterations):
        check(_lib.load().topk_set_wait_limit(self._h, int(iterations)))

    # -- lifetime -----------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            _lib.load().topk_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def csv_shape(path):
    """(n, d) of a comma-separated table file as File<T>::count reads it."""
    n, d = C.c_uint64(), C.c_uint64()
    check(_lib.load().topk_csv_shape(os.fsencode(path), C.byref(n), C.byref(d)))
    return n.value, d.value


def binary_shape(path):
    """(n, d) of a TOPKCOL1 binary table file."""
    n, d = C.c_uint64(), C.c_uint64()
    check(_lib.load().topk_binary_shape(os.fsencode(path), C.byref(n), C.byref(d)))
    return n.value, d.value
