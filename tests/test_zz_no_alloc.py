"""GPU: topk_query_noalloc, the entry point for callers that must not allocate.

Some callers cannot let a library call cudaMalloc: host applications that own
the whole GPU memory budget and hand it out through their own pool, or paths
that cannot afford the device-wide synchronisation of cudaMalloc/cudaFree.
topk_query_noalloc serves them: the caller brings the table and the output
buffers, and the scan's scratch is a fixed array inside the library.

This test calls it through the C ABI on buffers the test owns (allocated here
with torch, before the call) and checks its results bit-for-bit against the
regular entry point (topk_query) on the same data, on two calls in a row (the
shared scratch keeps the first call's contents), plus its size limit.  It lives
in its own file named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

import topk_b200 as T
from oracle import oracle as O
from topk_b200 import _lib
from tests import helpers as H

pytestmark = pytest.mark.gpu


def _noalloc(L, dt, n, ld, d, k, w, a, ids, sc, th, stream):
    return L.topk_query_noalloc(C.c_void_p(dt.data_ptr()), n, ld, d, k, len(a), w, a, C.c_void_p(ids.data_ptr()),
                                C.c_void_p(sc.data_ptr()), C.c_void_p(th.data_ptr()), C.c_void_p(stream))


def test_noalloc_matches_regular_entry_point_twice():
    torch = pytest.importorskip("torch")
    L = T.load()
    n, d = (1 << 20) + 37, 16
    ld = (n + 63) // 64 * 64
    raw = O.generate(n, d, O.MIXED, 77)
    with T.Table(n, d) as t:
        t.upload(raw)
        t.normalize()
        norm = t.download()
        # the caller's own device table (column-major, stride ld) and outputs
        host = np.zeros((d, ld), np.float32)
        host[:, :n] = norm
        dt = torch.from_numpy(host).cuda()
        ids = torch.empty(1024, dtype=torch.int64, device="cuda")
        sc = torch.empty(1024, dtype=torch.float32, device="cuda")
        th = torch.empty(1, dtype=torch.float32, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        rng = np.random.default_rng(123)
        for call, k in enumerate((1000, 64)):  # two calls in a row on the shared scratch
            w, a = H.random_query(rng, d)
            st = _noalloc(L, dt, n, ld, d, k, w, a, ids, sc, th, stream)
            assert st == _lib.OK, L.topk_last_error()
            torch.cuda.synchronize()
            got = (ids[:k].cpu().numpy().astype(np.uint64), sc[:k].cpu().numpy(), float(th.cpu()[0]))
            H.assert_same_result(got, t.query(k, w, a))


def test_noalloc_large_table_large_k_matches_regular_entry_point():
    """2^26 rows: large enough that a large-k query first runs the threshold pass
    over a tile sample (from k = 128 at two attributes, from k = 512 at four), in
    this entry point as in topk_query; mixed-sign weights and a repeated attribute."""
    torch = pytest.importorskip("torch")
    L = T.load()
    n, d = (1 << 26) + 333, 4
    ld = (n + 63) // 64 * 64
    raw = O.generate(n, d, O.ANTICORRELATED, 41)
    with T.Table(n, d) as t:
        t.upload(raw)
        t.normalize()
        host = np.zeros((d, ld), np.float32)
        host[:, :n] = t.download()
        dt = torch.from_numpy(host).cuda()
        del host
        ids = torch.empty(1024, dtype=torch.int64, device="cuda")
        sc = torch.empty(1024, dtype=torch.float32, device="cuda")
        th = torch.empty(1, dtype=torch.float32, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        rng = np.random.default_rng(9)
        for k in (128, 1024):
            for w in (rng.uniform(-1, 1, d), rng.uniform(0, 1, d)):
                w = w.astype(np.float32)
                for a in (np.array([2, 0], np.uint8), np.array([3, 0, 3, 1], np.uint8)):
                    st = _noalloc(L, dt, n, ld, d, k, w, a, ids, sc, th, stream)
                    assert st == _lib.OK, L.topk_last_error()
                    torch.cuda.synchronize()
                    got = (ids[:k].cpu().numpy().astype(np.uint64), sc[:k].cpu().numpy(), float(th.cpu()[0]))
                    H.assert_same_result(got, t.query(k, w, a))


def test_noalloc_k_above_n_matches_regular_entry_point():
    torch = pytest.importorskip("torch")
    L = T.load()
    n, d = 300, 5  # k > n: min(k, n) objects, like topk_query
    raw = O.generate(n, d, O.INDEPENDENT, 5)
    with T.Table(n, d) as t:
        t.upload(raw)
        t.normalize()
        dt = torch.from_numpy(np.ascontiguousarray(t.download())).cuda()
        ids = torch.full((1024,), -1, dtype=torch.int64, device="cuda")
        sc = torch.empty(1024, dtype=torch.float32, device="cuda")
        th = torch.empty(1, dtype=torch.float32, device="cuda")
        w = np.linspace(0.2, 1.0, d).astype(np.float32)
        a = np.array([4, 1, 2], np.uint8)
        st = _noalloc(L, dt, n, n, d, 1000, w, a, ids, sc, th, torch.cuda.current_stream().cuda_stream)
        assert st == _lib.OK, L.topk_last_error()
        torch.cuda.synchronize()
        got = (ids[:n].cpu().numpy().astype(np.uint64), sc[:n].cpu().numpy(), float(th.cpu()[0]))
        H.assert_same_result(got, t.query(1000, w, a))
        assert int(ids[n].cpu()) == -1  # nothing written past min(k, n)


def test_noalloc_rejects_k_above_its_limit():
    torch = pytest.importorskip("torch")
    L = T.load()
    n, d = 4096, 4
    dt = torch.zeros((d, n), dtype=torch.float32, device="cuda")
    ids = torch.empty(2048, dtype=torch.int64, device="cuda")
    sc = torch.empty(2048, dtype=torch.float32, device="cuda")
    th = torch.empty(1, dtype=torch.float32, device="cuda")
    w = np.ones(d, np.float32)
    a = np.array([0, 1], np.uint8)
    st = _noalloc(L, dt, n, n, d, 1025, w, a, ids, sc, th, 0)
    assert st == _lib.ERR_UNSUPPORTED
    assert b"1024" in L.topk_last_error()
    st = _noalloc(L, dt, n, n, d, 16, w, a, ids, sc, th, 0)  # still usable afterwards
    assert st == _lib.OK, L.topk_last_error()
    torch.cuda.synchronize()
