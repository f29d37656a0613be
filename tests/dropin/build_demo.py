"""Build tests/dropin/_build/tpac_dropin_demo, tpar_dropin_demo and ta_dropin_demo (need
the reference tree for cpu/AA.h, cpu/TPAc.h, cpu/TPAr.h, cpu/TA.h and time/Time.h,
located by the oracle's build recipe, oracle.build.reference_root()).  The binary
then travels with the working tree; without the reference tree nothing is built and
the GPU test that runs it skips."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle.build import reference_root  # noqa: E402

OUT = os.path.join(HERE, "_build", "tpac_dropin_demo")


def _build_one(name, header, ref, verbose):
    out = os.path.join(HERE, "_build", name)
    src = os.path.join(HERE, name + ".cpp")
    hdrs = [os.path.join(ROOT, "include", "topk_b200", h) for h in header]
    lib = os.path.join(ROOT, "topk_b200", "_lib", "libtopk_b200.so")
    if os.path.exists(out) and os.path.getmtime(out) > max(os.path.getmtime(p) for p in [src, lib] + hdrs):
        return out
    os.makedirs(os.path.dirname(out), exist_ok=True)
    cmd = ["g++", "-std=c++14", "-O2", "-march=x86-64-v3", "-ffp-contract=off", "-fopenmp", "-w",
           "-I", ref, "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "oracle", "stub"),
           src, "-o", out, "-L", os.path.dirname(lib), "-ltopk_b200",
           "-Wl,-rpath,$ORIGIN/../../../topk_b200/_lib"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return out


def build(verbose=False):
    """Builds the demos (TPAc, TPAr, TA); returns the TPAc demo's path."""
    ref = reference_root()
    if not os.path.exists(os.path.join(ref, "cpu", "TPAc.h")):
        return OUT if os.path.exists(OUT) else None
    _build_one("tpar_dropin_demo", ["TPAcGPU.h", "TPArGPU.h"], ref, verbose)
    _build_one("ta_dropin_demo", ["TPAcGPU.h", "TAGPU.h"], ref, verbose)
    return _build_one("tpac_dropin_demo", ["TPAcGPU.h"], ref, verbose)


if __name__ == "__main__":
    print(build(verbose=True))
    sys.exit(0)
