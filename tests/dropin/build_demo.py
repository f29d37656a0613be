"""Build tests/dropin/_build/tpac_dropin_demo (needs the reference tree for cpu/AA.h,
cpu/TPAc.h and time/Time.h; TOPK_REFERENCE, default /root/reference).  The binary
then travels with the working tree; without the reference tree nothing is built and
the GPU test that runs it skips."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "_build", "tpac_dropin_demo")


def build(verbose=False):
    ref = os.environ.get("TOPK_REFERENCE", "/root/reference")
    if not os.path.exists(os.path.join(ref, "cpu", "TPAc.h")):
        return OUT if os.path.exists(OUT) else None
    src = os.path.join(HERE, "tpac_dropin_demo.cpp")
    hdr = os.path.join(ROOT, "include", "topk_b200", "TPAcGPU.h")
    lib = os.path.join(ROOT, "topk_b200", "_lib", "libtopk_b200.so")
    if os.path.exists(OUT) and os.path.getmtime(OUT) > max(os.path.getmtime(src), os.path.getmtime(hdr),
                                                             os.path.getmtime(lib)):
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    cmd = ["g++", "-std=c++14", "-O2", "-march=x86-64-v3", "-ffp-contract=off", "-fopenmp", "-w",
           "-I", ref, "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "oracle", "stub"),
           src, "-o", OUT, "-L", os.path.dirname(lib), "-ltopk_b200",
           "-Wl,-rpath,$ORIGIN/../../../topk_b200/_lib"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(verbose=True))
    sys.exit(0)
