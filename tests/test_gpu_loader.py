"""GPU: the device CSV loader and the binary table files.

Every loaded table must equal, bit for bit, what the reference's File<float>::load
(input/File.h:233-265, 306-330) reads: fscanf("%f") per field, which rounds as strtof
does.  The oracle (oracle/csv_oracle.py, pinned against that loader on the CPU)
converts each field with strtof.  Small load chunks move the chunk boundaries through
the rows; several files route values to the host conversion (long mantissas, inf,
nan, hex) or through the device's midpoint correction (16-digit decimals of float
midpoints).
"""
import os

import numpy as np
import pytest

import topk_b200 as T
from oracle import csv_oracle as CO
from tests.test_csv_oracle import CASES, sample_table, write_lines

pytestmark = pytest.mark.gpu


def load(path, n, d, chunk=0):
    with T.Table(n, d) as t:
        st = t.load_csv(path, chunk)
        return t.download(), st


def same_bits(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32), np.asarray(b, np.float32).view(np.uint32))


@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("chunk", [0, 4096, 70001])
def test_load_csv_matches_oracle(case, chunk, tmp_path):
    t = sample_table(len(case))
    lines = CASES[case](t)
    p = str(tmp_path / "t.csv")
    write_lines(p, lines, eol="\r\n" if case == "spaced" else "\n")
    n, d = len(lines), t.shape[0]
    got, st = load(p, n, d, chunk)
    assert same_bits(got, CO.load_csv(p, n, d))
    assert st["rows"] == n and st["bytes"] == os.path.getsize(p)
    if case in ("digits25", "special"):
        assert st["host_converted"] > 0
    if case in ("printf_f", "repr9", "exp"):
        assert st["host_converted"] == 0


def test_midpoints_and_exact_ties(tmp_path):
    """Decimals at or within a double ulp of the point halfway between two floats:
    the double rounding lands on the midpoint and the exact remainder decides."""
    rng = np.random.default_rng(5)
    f = (rng.random(40000) * 10.0 ** rng.integers(-3, 12, 40000)).astype(np.float32)
    up = np.nextafter(f, np.float32(np.inf))
    mid = (f.astype(np.float64) + up.astype(np.float64)) / 2  # exact in double
    toks = ["%.16g" % x for x in mid] + ["%.15g" % x for x in mid[:5000]] + ["%.17g" % x for x in mid[:5000]]
    toks += ["16777217", "16777217.000001", "16777216.999999", "33554433", "33554435", "0.5", "1e22", "1e-22"]
    d = 1
    p = str(tmp_path / "m.csv")
    write_lines(p, toks)
    got, st = load(p, len(toks), d)
    want = CO.load_csv(p, len(toks), d)
    bad = np.nonzero(got.view(np.uint32) != want.view(np.uint32))[1]
    assert bad.size == 0, [toks[i] for i in bad[:5]]


def test_large_multi_chunk_round_trip(tmp_path):
    """%.9g round-trips FP32 exactly, so the table written is the table read."""
    n, d = (1 << 19) + 17, 8
    with T.Table(n, d) as t:
        t.generate(T.DIST_INDEPENDENT, 3)
        t.normalize()
        src = t.download()
    src[:, ::7] *= -3.5e-4
    p = str(tmp_path / "big.csv")
    with open(p, "w") as f:
        for i0 in range(0, n, 65536):
            blk = src[:, i0:i0 + 65536].T
            f.write("\n".join(",".join("%.9g" % x for x in row) for row in blk) + "\n")
    got, st = load(p, n, d, 4 << 20)
    assert same_bits(got, src)
    assert st["chunks"] > 4 and st["host_converted"] == 0


def test_blank_lines_crlf_and_no_final_newline(tmp_path):
    t = sample_table(11, d=3, n=3000)
    lines = [",".join("%.6g" % x for x in row) for row in t.T]
    body = lines[:100] + ["", "  \t"] + lines[100:2000] + [""] * 3 + lines[2000:]
    p = str(tmp_path / "b.csv")
    write_lines(p, body, eol="\r\n", final=False)
    for chunk in (0, 1024, 5000):
        got, st = load(p, 3000, 3, chunk)
        assert same_bits(got, CO.load_csv(p, 3000, 3))
    # fewer rows wanted than the file holds: the first n are read
    got, _ = load(p, 1234, 3, 1024)
    assert same_bits(got, CO.load_csv(p, 1234, 3))


@pytest.mark.parametrize("lines,msg", [
    (["1,2,3", "4,5", "7,8,9"], "row 2: fewer than 3 fields"),
    (["1,2,3", "4,5,6", "7,8,9,10"], "row 3: more than 3 fields"),
    (["1,2,3", "4,abc,6", "7,8,9"], "row 2"),
    (["1,2,3", "4,,6", "7,8,9"], "row 2"),
    (["1,2,3", "4,5,6"], "holds 2 rows"),
])
def test_load_csv_errors(lines, msg, tmp_path):
    p = str(tmp_path / "e.csv")
    write_lines(p, lines)
    with T.Table(3, 3) as t:
        with pytest.raises(T.TopKError) as ei:
            t.load_csv(p)
        assert msg in str(ei.value)
        with pytest.raises(T.TopKError):  # a failed load leaves no table data
            t.query(1, np.ones(3, np.float32), np.array([0], np.uint8))


def test_line_longer_than_chunk(tmp_path):
    p = str(tmp_path / "l.csv")
    write_lines(p, [",".join(["1.250000"] * 255)] * 3)  # 2295-byte lines
    with T.Table(3, 255) as t:
        with pytest.raises(T.TopKError):
            t.load_csv(p, 1024)
        t.load_csv(p, 4096)
        assert np.all(t.download() == np.float32(1.25))


def test_save_csv_is_the_reference_format_and_loads_back(tmp_path):
    n, d = 5000, 5
    with T.Table(n, d) as t:
        t.generate(T.DIST_ANTICORRELATED, 9)
        t.normalize()
        src = t.download()
        p = str(tmp_path / "s.csv")
        t.save_csv(p)
    q = str(tmp_path / "ref.csv")
    CO.write_table(q, src, "%f")
    assert open(p, "rb").read() == open(q, "rb").read()
    assert T.csv_shape(p) == (n, d)
    with T.Table.from_csv(p) as t2:
        assert same_bits(t2.download(), CO.load_csv(p, n, d))


def test_binary_round_trip_and_queries(tmp_path):
    n, d = (1 << 20) + 5, 6
    p = str(tmp_path / "t.bin")
    with T.Table(n, d) as t:
        t.generate(T.DIST_CORRELATED, 4)
        t.normalize()
        src = t.download()
        t.save_binary(p)
        w = np.linspace(0.1, 1, d).astype(np.float32)
        a = np.array([0, 2, 5], np.uint8)
        want = t.query(100, w, a)
    assert os.path.getsize(p) == 64 + 4 * n * d
    assert T.binary_shape(p) == (n, d)
    with T.Table.from_binary(p) as t2:
        assert same_bits(t2.download(), src)
        got = t2.query(100, w, a)
        assert all(np.array_equal(x, y) for x, y in zip(got, want))
    with T.Table(n - 1, d) as t3:
        with pytest.raises(T.TopKError):
            t3.load_binary(p)


def test_short_rows_beyond_row_capacity(tmp_path):
    """Rows far shorter than d fields overflow the row array sized for d fields:
    reported as short rows, never written out of bounds."""
    p = str(tmp_path / "s.csv")
    write_lines(p, ["1"] * 5000)
    with T.Table(5000, 8) as t:
        for chunk in (0, 4096):
            with pytest.raises(T.TopKError) as ei:
                t.load_csv(p, chunk)
            assert "fewer than 8 fields" in str(ei.value)


def test_one_handle_reloads(tmp_path):
    """The handle keeps the pipeline buffers: loads with other chunk sizes, CSV then
    binary then CSV, each give the file's table."""
    t0 = sample_table(21, d=4, n=20000)
    p, pb = str(tmp_path / "a.csv"), str(tmp_path / "a.bin")
    write_lines(p, CASES["repr9"](t0))
    want = CO.load_csv(p, 20000, 4)
    with T.Table(20000, 4) as t:
        for chunk in (0, 8192, 0, 1 << 20):
            t.upload(np.zeros((4, 20000), np.float32))
            t.load_csv(p, chunk)
            assert same_bits(t.download(), want)
        t.save_binary(pb)
        t.upload(np.zeros((4, 20000), np.float32))
        t.load_binary(pb)
        assert same_bits(t.download(), want)
        t.load_csv(p)
        assert same_bits(t.download(), want)
