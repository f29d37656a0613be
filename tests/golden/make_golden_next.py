"""Generate tests/golden/next_golden.json by running the reference itself: its table
loader, its VTA and PTA index builds, its row-major TPAr and its TA.

Run in a container that has the reference tree (oracle/build.py compiles it into
oracle/_ref/):
    python tests/golden/make_golden_next.py
Tests read only the JSON (tests/test_golden_next.py), so the fixtures also pin the
restatements where the reference is absent.

  loader  File<float>::load with transpose (input/File.h:233-265, 306-330) on small
          comma-separated texts of several styles: the text itself and the FP32 bits
          of the column-major table the reference read.
  index   VTA::init (IMP 1 and 2) and PTA::init (cpu/VTA.h:74-158, cpu/PTA.h:88-267)
          on tables whose columns are seeded permutations (distinct values): the
          reference's row order, as table row ids, and a SHA-256 of the table.
  tpar    TPAr (cpu/TPAr.h) queries through all three entries: ids, score bits and
          threshold bits as the reference returns them.
  ta      TA (cpu/TA.h) queries with equal weights (its scores are right only then).
"""
import hashlib
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import build as B  # noqa: E402
from oracle import csv_oracle as CO  # noqa: E402
from oracle import oracle as O  # noqa: E402
from oracle import vta_oracle as V  # noqa: E402


def perm_table(d, n, seed):
    """(d, n) float32, each column a seeded permutation of k/n: distinct values."""
    rng = np.random.default_rng(seed)
    return np.stack([rng.permutation(n).astype(np.float32) / np.float32(n) for _ in range(d)])


def loader_texts():
    rng = np.random.default_rng(7)
    t = ((rng.random((4, 300)) * 2 - 1) * 10.0 ** rng.integers(-6, 6, size=(4, 300))).astype(np.float32)
    rows = t.T
    out = {
        "printf_f": "\n".join(",".join("%f" % x for x in r) for r in rows) + "\n",
        "repr9": "\n".join(",".join("%.9g" % x for x in r) for r in rows) + "\n",
        "digits17": "\n".join(",".join("%.17g" % x for x in r) for r in rows) + "\n",
        "exp_spaced_crlf": "\r\n".join("  " + ", ".join("%.5E" % x for x in r) for r in rows) + "\r\n",
        "special": "\n".join(",".join(("inf", "-inf", "nan", "0x1.8p1")[m] if i % 50 == 0 else "%.7g" % r[m]
                                      for m in range(4)) for i, r in enumerate(rows)) + "\n",
    }
    return out


def main():
    if not (O.RefTPAc.available() and B.build_ref_file() and B.build_ref_index()):
        raise SystemExit("reference libraries unavailable: build them with oracle/build.py first")
    doc = {"about": "Outputs of the reference (File<float>::load, VTA/PTA init, TPAr, TA) built from its sources "
                    "by oracle/build.py; made by tests/golden/make_golden_next.py"}
    # loader
    loader = []
    with tempfile.TemporaryDirectory() as td:
        for name, text in loader_texts().items():
            p = os.path.join(td, name + ".csv")
            with open(p, "w", newline="") as f:
                f.write(text)
            n, d = CO.ref_shape(p)
            got = CO.ref_load(p, n, d)
            loader.append(dict(name=name, text=text, n=n, d=d, bits=[int(x) for x in got.view(np.uint32).ravel()]))
    doc["loader"] = loader
    # index orders
    index = []
    for d, n, seed in ((4, 4096, 1), (8, 3001, 2)):
        t = perm_table(d, n, seed)
        tn = t.copy()
        O.normalize(tn)
        rec = dict(d=d, n=n, seed=seed, table_sha256=hashlib.sha256(t.tobytes()).hexdigest(), orders={})
        for kind, imp in (("vta", 1), ("vta", 2), ("pta", 2)):
            rows, _ = V.ref_index_rows(kind, t, imp)
            rec["orders"][f"{kind}_imp{imp}"] = [int(x) for x in V.rows_to_ids(tn, rows)]
        index.append(rec)
    doc["index"] = index
    # TPAr and TA
    tpar, ta = [], []
    rng = np.random.default_rng(11)
    for n, d, dist, seed in ((1 << 13, 8, 1, 3), (4096, 5, 2, 4)):
        cols = O.generate(n, d, dist, seed)
        ref = O.RefTPAr(np.ascontiguousarray(cols.T))
        ref.init()
        rta = O.RefTA(np.ascontiguousarray(cols.T))
        rta.init()
        runs_p, runs_t = [], []
        for j in range(6):
            q = int(rng.integers(1, d + 1))
            attr = [int(x) for x in rng.choice(d, size=q, replace=False)]
            k = int(rng.choice([1, 10, 100, 500]))
            w = O.gen_weights(d, 500 + j, 0)
            a = np.array(attr, np.uint8)
            entries = {}
            for impl in (0, 1, 2):
                ids, sc, th, _ = ref.query(impl, k, w, a)
                entries[str(impl)] = dict(ids=[int(x) for x in ids], score_bits=[int(x) for x in sc.view(np.uint32)],
                                          threshold_bits=int(np.float32(th).view(np.uint32)))
            runs_p.append(dict(k=k, attr=attr, weights_bits=[int(x) for x in w.view(np.uint32)], entries=entries))
            we = np.full(d, np.float32(0.5 + 0.125 * j), np.float32)
            ids, sc, th, _ = rta.query(k, we, a)
            runs_t.append(dict(k=k, attr=attr, weight=float(we[0]), ids=[int(x) for x in ids],
                               score_bits=[int(x) for x in sc.view(np.uint32)],
                               threshold_bits=int(np.float32(th).view(np.uint32))))
        ref.close()
        rta.close()
        tpar.append(dict(n=n, d=d, dist=dist, seed=seed, runs=runs_p))
        ta.append(dict(n=n, d=d, dist=dist, seed=seed, runs=runs_t))
    doc["tpar"] = tpar
    doc["ta"] = ta
    with open(os.path.join(HERE, "next_golden.json"), "w") as f:
        json.dump(doc, f, separators=(",", ":"))
    print("wrote", os.path.join(HERE, "next_golden.json"))


if __name__ == "__main__":
    main()
