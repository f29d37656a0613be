"""CPU: the restatements against fixtures the reference itself produced
(tests/golden/next_golden.json, made by tests/golden/make_golden_next.py): its table
loader, its VTA/PTA index orders, its row-major TPAr and its TA.  The GPU tests check
the device against these restatements, so the device is pinned to the reference's
recorded outputs even where the reference tree is absent.
"""
import hashlib
import json
import os

import numpy as np
import pytest

from oracle import csv_oracle as CO
from oracle import oracle as O
from oracle import vta_oracle as V
from tests import helpers as H

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "next_golden.json")


@pytest.fixture(scope="module")
def golden():
    with open(GOLDEN) as f:
        return json.load(f)


def perm_table(d, n, seed):
    rng = np.random.default_rng(seed)
    return np.stack([rng.permutation(n).astype(np.float32) / np.float32(n) for _ in range(d)])


def test_loader_fixtures(golden, tmp_path):
    import topk_b200 as T
    for case in golden["loader"]:
        p = str(tmp_path / (case["name"] + ".csv"))
        with open(p, "w", newline="") as f:
            f.write(case["text"])
        assert T.csv_shape(p) == (case["n"], case["d"]) == CO.csv_shape(p)
        got = CO.load_csv(p, case["n"], case["d"])
        want = np.array(case["bits"], np.uint32).reshape(case["d"], case["n"])
        assert np.array_equal(got.view(np.uint32), want), case["name"]


def test_index_order_fixtures(golden):
    for rec in golden["index"]:
        d, n = rec["d"], rec["n"]
        t = perm_table(d, n, rec["seed"])
        assert hashlib.sha256(t.tobytes()).hexdigest() == rec["table_sha256"]
        tn = t.copy()
        O.normalize(tn)
        for name, ref_perm in rec["orders"].items():
            ref_perm = np.array(ref_perm, np.int64)
            if name.startswith("vta"):
                slices = 16 if name.endswith("imp2") else 1
                groups, ours = V.vta_groups(n, slices), V.vta_order(tn, slices)
            else:
                groups, ours = V.pta_part_ids(tn), V.pta_order(tn)
            assert V.same_order_up_to_ties(tn, groups, ref_perm, ours), name


def check_run(tn, k, w, attr, run, mirror=False):
    ids, sc, th = O.topk(tn, k, w, np.array(attr, np.uint8))
    r_ids = np.array(run["ids"], np.uint64)
    if mirror:  # TPAr's vector entries push lane j as base + j; it holds base + 7 - j
        r_ids = (r_ids // 8) * 8 + 7 - r_ids % 8
    H.assert_matches_reference(ids, sc, th, dict(run, ids=r_ids.tolist()), tn, w, np.array(attr, np.uint8))


def test_tpar_fixtures(golden):
    for rec in golden["tpar"]:
        tn = O.generate(rec["n"], rec["d"], rec["dist"], rec["seed"])
        O.normalize(tn)
        for run in rec["runs"]:
            w = np.array(run["weights_bits"], np.uint32).view(np.float32)
            for impl, e in run["entries"].items():
                check_run(tn, run["k"], w, run["attr"], e, mirror=impl != "0")


def test_ta_fixtures(golden):
    for rec in golden["ta"]:
        tn = O.generate(rec["n"], rec["d"], rec["dist"], rec["seed"])
        O.normalize(tn)
        for run in rec["runs"]:
            w = np.full(rec["d"], np.float32(run["weight"]), np.float32)
            check_run(tn, run["k"], w, run["attr"], run)
