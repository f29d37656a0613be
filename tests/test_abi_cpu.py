"""CPU: the C-ABI library loads, exports every declared symbol, fails cleanly.

No compute is attempted here (there is no GPU on this machine).
"""
import ctypes as C
import os
import re

import pytest

import topk_b200 as T
from topk_b200 import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "topk_b200.h")


def declared_symbols():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|uint64_t|const char \*)\s*(topk_\w+)\s*\(", src, re.M)))


def test_header_declares_expected_entries():
    syms = declared_symbols()
    for s in ("topk_create", "topk_destroy", "topk_upload_colmajor", "topk_normalize", "topk_query",
              "topk_query_batch", "topk_query_device", "topk_generate"):
        assert s in syms
    # the Python binding types every declared entry
    assert sorted(n for n, _, _ in _lib.SIGNATURES) == syms


def test_library_exports_every_declared_symbol():
    L = T.load()
    for s in declared_symbols():
        assert hasattr(L, s), s
    assert L.topk_version().startswith(b"topk_b200")


def test_status_names():
    assert _lib.status_name(0) == "TOPK_OK"
    assert _lib.status_name(4) == "TOPK_ERR_TIMEOUT"
    assert _lib.status_name(99) == "TOPK_ERR_UNKNOWN"


def test_create_argument_errors_without_gpu():
    L = T.load()
    h = C.c_void_p()
    assert L.topk_create(0, 8, 0, C.byref(h)) == _lib.ERR_ARG
    assert L.topk_create(16, 0, 0, C.byref(h)) == _lib.ERR_ARG
    assert L.topk_create(16, 300, 0, C.byref(h)) == _lib.ERR_ARG
    assert L.topk_create(1 << 33, 4, 0, C.byref(h)) == _lib.ERR_UNSUPPORTED
    assert b"n and d" in L.topk_last_error() or L.topk_last_error()


def test_null_handle_calls_fail_cleanly():
    L = T.load()
    import numpy as np
    w = np.ones(4, np.float32)
    a = np.zeros(2, np.uint8)
    ids = np.zeros(4, np.uint64)
    sc = np.zeros(4, np.float32)
    assert L.topk_query(None, 4, 2, w, a, ids, sc, None, None) == _lib.ERR_ARG
    assert L.topk_destroy(None) == _lib.OK
    assert L.topk_shape(None, None, None, None) == _lib.ERR_ARG


@pytest.mark.skipif(os.environ.get("CUDA_VISIBLE_DEVICES") == "__never__", reason="")
def test_create_without_gpu_reports_cuda_error(gpu_available):
    if gpu_available:
        pytest.skip("a GPU is present")
    with pytest.raises(T.TopKError) as ei:
        T.Table(1024, 4)
    assert ei.value.status == _lib.ERR_CUDA


def test_null_handle_calls_of_the_file_index_and_ta_entries():
    """The table-file, row-major, index-order and TA entries reject a null handle (or
    null arguments) before any device work."""
    import numpy as np
    L = T.load()
    w = np.ones(4, np.float32)
    a = np.zeros(2, np.uint8)
    ids = np.zeros(4, np.uint64)
    sc = np.zeros(4, np.float32)
    st = np.zeros(4, np.uint64)
    rows = np.zeros(16, np.float32)
    u32 = np.zeros(4, np.uint32)
    assert L.topk_load_csv(None, b"/nonexistent.csv", 0, st) == _lib.ERR_ARG
    assert L.topk_save_csv(None, b"x.csv") == _lib.ERR_ARG
    assert L.topk_load_binary(None, b"x.bin") == _lib.ERR_ARG
    assert L.topk_save_binary(None, b"x.bin") == _lib.ERR_ARG
    assert L.topk_upload_rowmajor(None, rows, 4) == _lib.ERR_ARG
    assert L.topk_download_rowmajor(None, rows, 4) == _lib.ERR_ARG
    assert L.topk_build_partitions_ordered(None, 1024, 1) == _lib.ERR_ARG
    assert L.topk_build_partitions_ordered(None, 1024, 9) == _lib.ERR_ARG  # unknown order
    assert L.topk_partition_ids(None, u32) == _lib.ERR_ARG
    assert L.topk_build_lists(None) == _lib.ERR_ARG
    assert L.topk_read_list(None, 0, u32, np.zeros(4, np.float32)) == _lib.ERR_ARG
    assert L.topk_query_ta(None, 4, 2, w, a, ids, sc, None, None, st) == _lib.ERR_ARG
    n, d = C.c_uint64(), C.c_uint64()
    assert L.topk_csv_shape(None, C.byref(n), C.byref(d)) == _lib.ERR_ARG
    assert L.topk_binary_shape(b"/nonexistent.bin", C.byref(n), C.byref(d)) == _lib.ERR_ARG


def test_lean_bindings_match_the_checked_ones():
    """The per-query Table methods call lean bindings (plain addresses); each has the
    checked binding's argument count and returns the same status on a null handle."""
    import numpy as np
    from topk_b200.table import _call_block
    L, F = T.load(), _lib.lean()
    checked = {name: args for name, _, args in _lib.SIGNATURES}
    for name, res, args in _lib.LEAN_SIGNATURES:
        assert len(args) == len(checked[name]), name
    b = _call_block()
    assert b is _call_block()  # one block per thread, reused
    assert b.buf.ctypes.data % 16 == 0 and b.p_st % 8 == 0 and b.p_cnt % 8 == 0
    assert len(b.ids) == _lib.MAX_K and len(b.sc) == _lib.MAX_K and len(b.w) >= _lib.MAX_D
    assert F.topk_query(None, 4, 2, b.p_w, b.p_a, b.p_ids, b.p_sc, b.p_cnt, b.p_th) == _lib.ERR_ARG
    assert F.topk_query_range(None, 0, 4, 4, 2, b.p_w, b.p_a, b.p_ids, b.p_sc, b.p_cnt, b.p_th) == _lib.ERR_ARG
    assert F.topk_query_pruned(None, 4, 2, b.p_w, b.p_a, 0.0, b.p_ids, b.p_sc, b.p_cnt, b.p_th,
                               b.p_st) == _lib.ERR_ARG
    assert F.topk_query_learned(None, 4, 2, b.p_w, b.p_a, b.p_ids, b.p_sc, b.p_cnt, b.p_th, b.p_st,
                                b.p_cut) == _lib.ERR_ARG
    # arguments that do not fit the block go to the checked bindings
    assert not b.args_in(np.ones(8, np.float32), np.zeros(_lib.MAX_Q + 1, np.uint8), 8)
    w = np.arange(1, 9, dtype=np.float32)
    assert b.args_in(w, np.array([7, 2], np.uint8), 8)
    assert b.w[:8].tobytes() == w.tobytes() and list(b.a[:2]) == [7, 2]
    # results come out as copies
    b.cnt[0] = 2
    b.ids[:2] = [5, 9]
    b.sc[:2] = [0.25, 0.5]
    b.f[0] = 0.25
    ids, sc, th = b.results()
    b.ids[:2] = 0
    assert list(ids) == [5, 9] and list(sc) == [0.25, 0.5] and th == 0.25
    assert ids.dtype == np.uint64 and sc.dtype == np.float32


def test_query_batch_writes_into_kept_arrays(monkeypatch):
    """Table.query_batch(out=...) hands the caller's arrays to topk_query_batch and
    returns them; shapes and dtypes are checked before the call.  The C call is
    replaced by a stand-in that writes counts[j] entries per row, as the library
    does, so this runs without a GPU."""
    import numpy as np
    from topk_b200 import table as TB

    calls = []

    class FakeLib:
        def topk_query_batch(self, h, nq, ks, qqs, W, wstride, A, astride, ids, sc, kstride, pcnt, pth):
            calls.append((nq, kstride))
            cnt = np.ctypeslib.as_array(C.cast(pcnt, C.POINTER(C.c_uint64)), (nq,))
            th = np.ctypeslib.as_array(C.cast(pth, C.POINTER(C.c_float)), (nq,))
            ids2, sc2 = ids.reshape(nq, kstride), sc.reshape(nq, kstride)
            for j in range(nq):
                c = int(min(ks[j], kstride))
                ids2[j, :c] = np.arange(c) + 100 * j
                sc2[j, :c] = np.linspace(1.0, 0.5, c, dtype=np.float32)
                cnt[j] = c
                th[j] = sc2[j, c - 1]
            return _lib.OK

    monkeypatch.setattr(_lib, "load", lambda: FakeLib())
    t = TB.Table.__new__(TB.Table)
    t._h, t.n, t.d = None, 1000, 4
    ks = np.array([3, 5, 1], np.uint64)
    W = np.ones((3, 4), np.float32)
    A = np.array([[0, 1], [2, 3], [1, 2]], np.uint8)
    fresh = t.query_batch(ks, W, A)
    bufs = (np.full((3, 5), 7, np.uint64), np.full((3, 5), 9, np.float32), np.zeros(3, np.uint64),
            np.zeros(3, np.float32))
    got = t.query_batch(ks, W, A, out=bufs)
    assert all(g is b for g, b in zip(got, bufs))
    assert calls == [(3, 5), (3, 5)]
    for j in range(3):
        c = int(fresh[2][j])
        assert int(bufs[2][j]) == c
        assert np.array_equal(bufs[0][j, :c], fresh[0][j, :c]) and np.array_equal(bufs[1][j, :c], fresh[1][j, :c])
        assert np.all(fresh[0][j, c:] == 0) and np.all(bufs[0][j, c:] == 7)  # kept rows keep their tail
    assert np.array_equal(bufs[3], fresh[3])
    # wrong shape, dtype or layout: refused before the call
    for bad in ((np.zeros((3, 4), np.uint64),) + bufs[1:], (bufs[0].astype(np.int64),) + bufs[1:],
                bufs[:1] + (np.zeros((5, 3), np.float32).T,) + bufs[2:], bufs[:2] + (np.zeros(3, np.uint32),) + bufs[3:]):
        with pytest.raises(ValueError):
            t.query_batch(ks, W, A, out=bad)
    assert len(calls) == 2
