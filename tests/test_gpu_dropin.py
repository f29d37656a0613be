"""GPU: the C++ drop-in TPAcGPU against the reference's own TPAc in one process.

tests/dropin/tpac_dropin_demo.cpp loads one table into both classes through
get_cdata(), runs init() and the harness's query sweep, and reports whether every
answer agrees (normalised tables bit-identical; same k-th score, score multiset and
ids above it).  The binary is built from the reference headers by
tests/dropin/build_demo.py; where it was not built the test skips.
"""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

BIN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "dropin", "_build", "tpac_dropin_demo")
BIN_TPAR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "dropin", "_build", "tpar_dropin_demo")
BIN_TA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "dropin", "_build", "ta_dropin_demo")


@pytest.mark.parametrize("n,d,seed", [(1 << 20, 8, 1), ((1 << 18) + 48, 16, 7)])
def test_tpacgpu_agrees_with_reference_tpac(n, d, seed):
    if not os.path.exists(BIN):
        pytest.skip("drop-in demo not built (needs the reference headers at build time)")
    r = subprocess.run([BIN, str(n), str(d), str(seed)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "normalize ok" in r.stdout
    assert r.stdout.strip().endswith("PASS"), r.stdout


@pytest.mark.parametrize("n,d,seed", [(1 << 20, 8, 3), ((1 << 18) + 256, 16, 9)])
def test_tpargpu_agrees_with_reference_tpar(n, d, seed):
    """TPArGPU (row-major cdata, include/topk_b200/TPArGPU.h) against the reference's
    TPAr, all three of its query entries."""
    if not os.path.exists(BIN_TPAR):
        pytest.skip("drop-in demo not built (needs the reference headers at build time)")
    r = subprocess.run([BIN_TPAR, str(n), str(d), str(seed)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "normalize ok" in r.stdout
    assert r.stdout.strip().endswith("PASS"), r.stdout


@pytest.mark.parametrize("n,d,seed", [(1 << 20, 8, 5), ((1 << 18) + 5, 6, 2)])
def test_tagpu_agrees_with_reference_ta(n, d, seed):
    """TAGPU (include/topk_b200/TAGPU.h) against the reference's TA with equal weights
    (the reference scores right only then, cpu/TA.h:83)."""
    if not os.path.exists(BIN_TA):
        pytest.skip("drop-in demo not built (needs the reference headers at build time)")
    r = subprocess.run([BIN_TA, str(n), str(d), str(seed)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "normalize ok" in r.stdout
    assert r.stdout.strip().endswith("PASS"), r.stdout
