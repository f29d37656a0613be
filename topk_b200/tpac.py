"""Python mirror of the reference's algorithm-class API for the TPAc path.

Reference: class AA<T,Z> (cpu/AA.h:63-122) and TPAc<T,Z> (cpu/TPAc.h:6-25).
Same method names, argument meaning and call order as the harness uses them
(validation/bench_cpu.h:155-237):

    t = TPAc(n, d)
    t.get_cdata()[...] = table        # or t.set_cdata(table); (d, n) column-major
    t.init()                          # normalize_transpose, on the GPU
    t.findTopKsimd(k, qq, weights, attr)
    t.get_res(), t.get_thres()
    t.benchmark()

Differences, all deliberate:
  * compute runs on the GPU through libtopk_b200.so; findTopKscalar, findTopKsimd and
    findTopKthreads all run the same exact kernel (the reference's three are
    bit-identical when built strictly, except findTopKscalar's use of attr[0]+m for
    column offsets, cpu/TPAc.h:53-81, which is only right for contiguous ascending
    attribute sets: here every entry uses attr[m], like findTopKsimd);
  * findTopKsimdMQ keeps its result per thread id instead of racing on res
    (cpu/TPAc.h:215) and stores real object ids, not lane ids (:247);
  * errors raise TopKError instead of printing and calling exit(1).
"""
import threading
import time

import numpy as np

from .table import Table

QATTR = 1  # cpu/AA.h:11


def FIRST(d, qq):
    """First attribute of the harness's default query (cpu/AA.h:12)."""
    return 0 if QATTR == 0 else d - qq


def LAST(d, qq):
    return qq if QATTR == 0 else d


class AA:
    """Base class: results, timers and statistics (cpu/AA.h:63-122)."""

    def __init__(self, n, d, device=0, mqthreads=256):
        self.n, self.d = int(n), int(d)
        self.algo = ""
        self.res = []          # list of (tid, score), ascending by score
        self.threshold = 0.0
        self.cdata = None      # host (d, n) float32 column-major, like AA::cdata
        self.tt_init = 0.0
        self.tt_processing = 0.0
        self.iter = 1
        self.tuple_count = 0
        self.mqthreads = mqthreads
        self.tt_array = [0.0] * mqthreads
        self.workload = 0
        self.initp = False
        self.topkp = False
        self.device = device

    def get_res(self):
        return list(self.res)

    def get_algo(self):
        return self.algo

    def get_thres(self):
        return self.threshold

    def get_cdata(self):
        if self.cdata is None:
            self.cdata = np.zeros((self.d, self.n), np.float32)
        return self.cdata

    def set_cdata(self, cdata):
        c = np.ascontiguousarray(cdata, np.float32)
        if c.shape != (self.d, self.n):
            raise ValueError(f"cdata must be ({self.d}, {self.n}) column-major, got {c.shape}")
        self.cdata = c

    def set_iter(self, it):
        self.iter = int(it)

    def reset_clocks(self):
        self.tt_processing = 0.0
        self.tt_array = [0.0] * self.mqthreads

    def benchmark(self, multi_query=False):
        """Print the reference's benchmark lines (cpu/AA.h:194-223) and return them."""
        lines = [f"< Benchmark for {self.algo} algorithm >", f"tt_init: {self.tt_init:.8f}"]
        if not multi_query:
            lines.append(f"tt_procesing: {self.tt_processing / self.iter:.8f}")
        else:
            tt = max(self.tt_array) / self.iter
            lines.append(f"tt_procesing: {tt:.8f}")
            if tt > 0:
                lines.append(f"tuples_per_second: {self.workload / (tt / 1000):.8f}")
        for ln in lines:
            print(ln)
        return lines


class TPAc(AA):
    """Column-major full-table evaluation on the GPU (cpu/TPAc.h)."""

    def __init__(self, n, d, device=0, mqthreads=256):
        super().__init__(n, d, device, mqthreads)
        self.algo = "TPAc"
        self._table = Table(n, d, device)
        self._mq_res = {}
        self._lock = threading.Lock()

    @property
    def table(self):
        return self._table

    def init(self):
        """Upload cdata (if the caller filled it) and normalise on the device
        (TPAc::init -> normalize_transpose, cpu/TPAc.h:28-32)."""
        if self.cdata is not None:
            self._table.upload(self.cdata)
        self._table.normalize()
        self.tt_init = 0.0

    def init_generated(self, dist, seed):
        """Generate a seeded synthetic table directly on the device (File::gen,
        input/File.h:335-354) and normalise it."""
        self._table.generate(dist, seed)
        self._table.normalize()

    def _query(self, k, qq, weights, attr):
        a = np.ascontiguousarray(attr, np.uint8)[: int(qq)]
        t0 = time.perf_counter()
        ids, sc, th = self._table.query(int(k), weights, a)
        dt = (time.perf_counter() - t0) * 1e3
        return ids, sc, th, dt

    def _store(self, ids, sc, th, dt):
        self.res = list(zip(ids.tolist(), sc.tolist()))
        self.res_ids, self.res_scores = ids, sc
        self.threshold = th
        self.tt_processing += dt
        self.tuple_count = self.n

    def findTopKscalar(self, k, qq, weights, attr):
        self._store(*self._query(k, qq, weights, attr))

    def findTopKsimd(self, k, qq, weights, attr):
        self._store(*self._query(k, qq, weights, attr))

    def findTopKthreads(self, k, qq, weights, attr):
        self._store(*self._query(k, qq, weights, attr))

    def findTopKsimdMQ(self, k, qq, weights, attr, tid):
        """Thread-safe multi-query entry (cpu/TPAc.h:210-254): concurrent callers
        each get a device context; the result is kept per tid."""
        ids, sc, th, dt = self._query(k, qq, weights, attr)
        with self._lock:
            self.tt_array[tid] += dt
            self._mq_res[tid] = (ids, sc, th)

    def get_mq_res(self, tid):
        return self._mq_res.get(tid)

    def findTopKbatch(self, ks, weights, attrs, qqs=None):
        """Many queries in one call (extension; results for every query)."""
        return self._table.query_batch(ks, weights, attrs, qqs)

    def close(self):
        self._table.close()


class TPAr(TPAc):
    """Row-major full-table evaluation (cpu/TPAr.h:6-33): cdata holds the table
    row-major, (n, d) with object i in row i, and init() normalises it
    (common/common.h:63-92, the same arithmetic per attribute as TPAc's).  On the GPU
    the rows are transposed into the column-major table on upload, so the queries are
    TPAc's exact kernel; results equal the reference TPAr's."""

    def __init__(self, n, d, device=0, mqthreads=256):
        super().__init__(n, d, device, mqthreads)
        self.algo = "TPAr"

    def get_cdata(self):
        if self.cdata is None:
            self.cdata = np.zeros((self.n, self.d), np.float32)
        return self.cdata

    def set_cdata(self, cdata):
        c = np.ascontiguousarray(cdata, np.float32)
        if c.shape != (self.n, self.d):
            raise ValueError(f"cdata must be ({self.n}, {self.d}) row-major, got {c.shape}")
        self.cdata = c

    def init(self):
        """Upload cdata (if the caller filled it) row-major, transposed on the device,
        and normalise there (TPAr::init -> normalize, cpu/TPAr.h:28-33)."""
        if self.cdata is not None:
            self._table.upload_rowmajor(self.cdata)
        self._table.normalize()
        self.tt_init = 0.0


class TA(AA):
    """The threshold algorithm over sorted lists (cpu/TA.h:10-96).  Like the reference,
    cdata holds the table row-major, (n, d); init() normalises it
    (common/common.h:63-92) and builds the sorted lists, on the device; findTopK walks
    them there.  Results are the exact top-k (each attribute scored with its own
    weight; the reference reuses the weight of the list an object was found in,
    cpu/TA.h:83)."""

    def __init__(self, n, d, device=0, mqthreads=256):
        super().__init__(n, d, device, mqthreads)
        self.algo = "TA"
        self._table = Table(n, d, device)
        self.last_stats = None

    @property
    def table(self):
        return self._table

    def get_cdata(self):
        if self.cdata is None:
            self.cdata = np.zeros((self.n, self.d), np.float32)
        return self.cdata

    def set_cdata(self, cdata):
        c = np.ascontiguousarray(cdata, np.float32)
        if c.shape != (self.n, self.d):
            raise ValueError(f"cdata must be ({self.n}, {self.d}) row-major, got {c.shape}")
        self.cdata = c

    def init(self):
        t0 = time.perf_counter()
        if self.cdata is not None:
            self._table.upload_rowmajor(self.cdata)
        self._table.normalize()
        self._table.build_lists()
        self.tt_init = (time.perf_counter() - t0) * 1e3

    def findTopK(self, k, qq, weights, attr):
        a = np.ascontiguousarray(attr, np.uint8)[: int(qq)]
        t0 = time.perf_counter()
        ids, sc, th, st = self._table.query_ta(int(k), weights, a)
        self.tt_processing += (time.perf_counter() - t0) * 1e3
        self.res = list(zip(ids.tolist(), sc.tolist()))
        self.res_ids, self.res_scores = ids, sc
        self.threshold = th
        self.last_stats = st
        self.tuple_count = st[1]

    def close(self):
        self._table.close()
