"""Generate the golden fixtures in tests/golden/ by running the reference itself.

The reference has no tests or golden vectors of its own (its validators
AA::compare / AA::compare_t, cpu/AA.h:155-189, are never called), so parity is
pinned by executing the reference's TPAc (cpu/TPAc.h) compiled strict into
oracle/_ref/libref_tpac.so (see oracle/build.py) on seeded synthetic tables and
recording what it returns.

Run in a container that has the reference tree:
    python tests/golden/make_golden.py
Writes tests/golden/tpac_golden.json.  The GPU box does not need the reference:
tests read only the JSON.

Each case records the table recipe (n, d, distribution, seed), a SHA-256 of the
table after the reference's own normalize_transpose (common/common.h:30-61), the
query, and for each reference implementation run (0 scalar, 1 simd, 2 threads)
the ids and score bits in the reference's own output order (ascending min-heap
drain) plus get_thres().
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402


def last_q(d, q):
    """The reference harness's QM=0 attribute tables: the last q attributes in
    ascending order (validation/bench_cpu.h:25-45)."""
    return list(range(d - q, d))


def random_subset(rng, d, q, ordered=True):
    a = rng.choice(d, size=q, replace=False)
    return sorted(a.tolist()) if ordered else a.tolist()


def table_for(n, d, dist, seed, quant=None):
    t = O.generate(n, d, dist, seed)
    if quant:
        # coarse values so that many objects tie on score
        t = (np.floor(t * quant) / quant).astype(np.float32)
    return t


def make_cases():
    rng = np.random.default_rng(20261203)
    cases = []
    # C1: the reference's CPU-runnable configuration.
    cases.append(dict(name="C1", n=1 << 20, d=8, dist=1, seed=0, wseed=1, k=16, attr=[4, 5, 6, 7], impls=[0, 1, 2]))
    # harness-shaped sweeps: last-q attribute sets, all three implementations
    for dist in (0, 1, 2, 3):
        for d, q in ((8, 2), (8, 8), (16, 4), (16, 16)):
            for k in (1, 16, 256):
                cases.append(dict(name=f"lastq_d{dist}_{d}_{q}_{k}", n=1 << 16, d=d, dist=dist, seed=10 + dist,
                                  wseed=100 + len(cases), k=k, attr=last_q(d, q), impls=[0, 1, 2]))
    # arbitrary attribute subsets and orders (scalar path is only right for contiguous
    # ascending sets, cpu/TPAc.h:53-81, so simd and threads only)
    for j in range(12):
        d = 16
        q = int(rng.integers(2, 17))
        attr = random_subset(rng, d, q, ordered=(j % 2 == 0))
        k = int(rng.choice([1, 7, 16, 64, 100, 1024]))
        cases.append(dict(name=f"subset_{j}", n=1 << 17, d=d, dist=int(j % 4), seed=40 + j, wseed=200 + j,
                          k=k, attr=attr, impls=[1, 2]))
    # edges: k >= n, k == n, tiny tables, heavy ties
    cases.append(dict(name="k_gt_n", n=64, d=4, dist=1, seed=5, wseed=300, k=100, attr=[0, 1, 2, 3], impls=[0, 1]))
    cases.append(dict(name="k_eq_n", n=256, d=4, dist=0, seed=6, wseed=301, k=256, attr=[2, 3], impls=[0, 1, 2]))
    cases.append(dict(name="tiny", n=16, d=2, dist=2, seed=7, wseed=302, k=3, attr=[0, 1], impls=[0, 1]))
    cases.append(dict(name="ties", n=1 << 14, d=4, dist=1, seed=8, wseed=303, k=64, attr=[1, 2, 3], impls=[0, 1, 2],
                      quant=8))
    cases.append(dict(name="ties_eqw", n=1 << 14, d=4, dist=1, seed=9, wseed=-1, k=200, attr=[0, 1, 2, 3],
                      impls=[0, 1, 2], quant=4))
    return cases


def weights_for(c):
    if c["wseed"] < 0:
        return np.ones(c["d"], np.float32)  # bench_cpu.h:19 uses all-ones weights
    return O.gen_weights(c["d"], c["wseed"], 0)


def main():
    if not O.RefTPAc.available():
        raise SystemExit("reference library unavailable: build it with oracle/build.py first")
    out = []
    for c in make_cases():
        t = table_for(c["n"], c["d"], c["dist"], c["seed"], c.get("quant"))
        w = weights_for(c)
        ref = O.RefTPAc(t)
        ref.init()
        tn = ref.data()
        rec = dict(c)
        rec["table_sha256"] = hashlib.sha256(tn.tobytes()).hexdigest()
        rec["weights_bits"] = [int(x) for x in w.view(np.uint32)]
        rec["runs"] = {}
        for impl in c["impls"]:
            ids, sc, th, _ = ref.query(impl, c["k"], w, np.array(c["attr"], np.uint8))
            rec["runs"][str(impl)] = dict(ids=[int(x) for x in ids], score_bits=[int(x) for x in sc.view(np.uint32)],
                                          threshold_bits=int(np.float32(th).view(np.uint32)))
        ref.close()
        out.append(rec)
        print(c["name"], "ok", flush=True)
    gen = {}
    for dist in (0, 1, 2, 3):
        for d in (2, 8, 16):
            t = O.generate(1024, d, dist, 123)
            gen[f"{dist}_{d}"] = hashlib.sha256(t.tobytes()).hexdigest()
    doc = dict(
        about="Outputs of the reference TPAc (cpu/TPAc.h) built strict, on seeded synthetic tables; "
              "made by tests/golden/make_golden.py",
        generator_sha256=gen,
        cases=out,
    )
    with open(os.path.join(HERE, "tpac_golden.json"), "w") as f:
        json.dump(doc, f, separators=(",", ":"))
    print("wrote", len(out), "cases")


if __name__ == "__main__":
    main()
