"""Test infrastructure only: restatement of the reference's table loader.

File<float>::count (input/File.h:108-132): d = 1 + the commas of the first line, n =
the newlines of the file.  File<float>::load with transpose (input/File.h:233-265,
306-330): fscanf("%f,...,%f") per object, stored column-major.  fscanf's "%f" rounds
as strtof does (correctly rounded), so this restatement converts every field with the
C library's strtof; fscanf skips white space (blank lines included) before each
number.  Pinned against the reference itself through `ref_load` (oracle/_ref/
libref_file.so, compiled from input/File.h by oracle/build.py).
"""
import ctypes as C
import ctypes.util
import os

import numpy as np

_libc = C.CDLL(ctypes.util.find_library("c"))
_libc.strtof.restype = C.c_float
_libc.strtof.argtypes = [C.c_char_p, C.POINTER(C.c_char_p)]


def strtof(tok):
    """One field converted by the C library (bytes in, float32 out); ValueError when
    the field is not entirely a number."""
    end = C.c_char_p()
    buf = C.create_string_buffer(tok)
    v = _libc.strtof(buf, C.byref(end))
    used = C.cast(end, C.c_void_p).value - C.cast(buf, C.c_void_p).value
    if used != len(tok) or not tok:
        raise ValueError(f"not a number: {tok!r}")
    return np.float32(v)


def csv_shape(path):
    with open(path, "rb") as f:
        data = f.read()
    first = data.split(b"\n", 1)[0]
    return data.count(b"\n"), first.count(b",") + 1


def load_csv(path, n, d):
    """(d, n) float32: the first n non-blank lines, d fields each."""
    out = np.empty((d, n), np.float32)
    r = 0
    with open(path, "rb") as f:
        for line in f:
            if r == n:
                break
            line = line.rstrip(b"\n")
            if not line.strip(b" \t\r"):
                continue
            fields = line.split(b",")
            if len(fields) != d:
                raise ValueError(f"row {r + 1}: {len(fields)} fields")
            for m, tok in enumerate(fields):
                out[m, r] = strtof(tok.strip(b" \t\r"))
            r += 1
    if r < n:
        raise ValueError(f"{r} rows, {n} wanted")
    return out


def ref_load(path, n, d):
    """The reference's own File<float>::load (transpose) on the file, or None when
    oracle/_ref/libref_file.so is not built."""
    from . import build as B
    if not os.path.exists(B.REF_FILE_SO):
        return None
    L = C.CDLL(B.REF_FILE_SO)
    L.ref_file_load.argtypes = [C.c_char_p, C.c_uint64, C.c_uint64,
                                np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")]
    out = np.zeros((d, n), np.float32)
    L.ref_file_load(os.fsencode(path), n, d, out.reshape(-1))
    return out


def ref_shape(path):
    from . import build as B
    if not os.path.exists(B.REF_FILE_SO):
        return None
    L = C.CDLL(B.REF_FILE_SO)
    L.ref_file_count.argtypes = [C.c_char_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
    n, d = C.c_uint64(), C.c_uint64()
    L.ref_file_count(os.fsencode(path), C.byref(n), C.byref(d))
    return n.value, d.value


def write_table(path, table, fmt="%f", sep=",", eol="\n"):
    """Writes a (d, n) table as text, one object per line (fmt per value)."""
    d, n = table.shape
    with open(path, "w") as f:
        for i in range(n):
            f.write(sep.join(fmt % float(table[m, i]) for m in range(d)) + eol)
