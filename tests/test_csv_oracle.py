"""CPU: the CSV restatement against the reference's own loader, and the library's
host-side file functions (shape counting, binary headers), which need no GPU.

The reference reads tables with File<float>::load (input/File.h:233-265, 306-330):
fscanf("%f,...,%f") per object into column-major memory; the restatement converts
each field with strtof, as "%f" does.  oracle/_ref/libref_file.so is that loader
compiled from input/File.h (oracle/build.py).
"""
import os
import struct

import numpy as np
import pytest

from oracle import csv_oracle as CO


def sample_table(seed, d=6, n=2000):
    rng = np.random.default_rng(seed)
    t = (rng.random((d, n)) * 2 - 1) * 10.0 ** rng.integers(-7, 7, size=(d, n))
    return t.astype(np.float32)


def write_lines(path, lines, eol="\n", final=True):
    with open(path, "w", newline="") as f:
        f.write(eol.join(lines) + (eol if final else ""))


CASES = {
    "printf_f": lambda t: [",".join("%f" % x for x in row) for row in t.T],
    "repr9": lambda t: [",".join("%.9g" % x for x in row) for row in t.T],
    "digits16": lambda t: [",".join("%.16g" % x for x in row) for row in t.T],
    "digits25": lambda t: [",".join("%.25g" % x for x in row) for row in t.T],
    "exp": lambda t: [",".join("%.4E" % x for x in row) for row in t.T],
    "spaced": lambda t: ["  " + ", ".join("%.7g" % x for x in row) for row in t.T],
    "special": lambda t: [",".join(["inf", "-inf", "nan", "0x1.8p1", "-0.0", "+7"][m % 6] if i % 97 == 0 else
                                   "%.8g" % t[m, i] for m in range(t.shape[0])) for i in range(t.shape[1])],
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_oracle_matches_reference_loader(case, tmp_path):
    t = sample_table(len(case))
    lines = CASES[case](t)
    p = str(tmp_path / "t.csv")
    write_lines(p, lines, eol="\r\n" if case == "spaced" else "\n")
    n, d = len(lines), t.shape[0]
    want = CO.ref_load(p, n, d)
    if want is None:
        pytest.skip("reference loader not built (reference sources absent)")
    assert CO.ref_shape(p) == (n, d) == CO.csv_shape(p)
    got = CO.load_csv(p, n, d)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_oracle_blank_lines_and_missing_final_newline(tmp_path):
    t = sample_table(3, d=3, n=50)
    lines = [",".join("%.6g" % x for x in row) for row in t.T]
    body = lines[:10] + ["", "   "] + lines[10:]
    p = str(tmp_path / "b.csv")
    write_lines(p, body, final=False)
    want = CO.ref_load(p, 50, 3)
    if want is None:
        pytest.skip("reference loader not built")
    got = CO.load_csv(p, 50, 3)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_library_csv_shape_matches_reference(tmp_path):
    import topk_b200 as T
    p = str(tmp_path / "s.csv")
    for lines, final in ((["1,2,3", "4,5,6"], True), (["1,2", "3,4", "5,6"], False), (["7"], True)):
        write_lines(p, lines, final=final)
        want = CO.ref_shape(p) or CO.csv_shape(p)
        assert T.csv_shape(p) == want == CO.csv_shape(p)
    with pytest.raises(T.TopKError):
        T.csv_shape(str(tmp_path / "missing.csv"))


def test_library_binary_header(tmp_path):
    import topk_b200 as T
    p = str(tmp_path / "t.bin")
    n, d = 1000, 3
    with open(p, "wb") as f:
        f.write(b"TOPKCOL1" + struct.pack("<IIQQ32x", 1, 4, n, d))
        f.write(np.zeros(n * d, np.float32).tobytes())
    assert T.binary_shape(p) == (n, d)
    with open(p, "r+b") as f:  # truncated data
        f.truncate(64 + 4 * n * d - 4)
    with pytest.raises(T.TopKError):
        T.binary_shape(p)
    with open(p, "wb") as f:
        f.write(b"NOTATABL" + bytes(56))
    with pytest.raises(T.TopKError):
        T.binary_shape(p)
