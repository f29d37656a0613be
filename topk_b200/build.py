"""Build libtopk_b200.so in-tree with nvcc for sm_100a.

    python -m topk_b200.build [-v] [-f]

Sources: topk_b200/csrc/*.cu and *.cpp.  Output: topk_b200/_lib/libtopk_b200.so
(git-ignored, but it travels with the working tree).  Flags: -O3, -lineinfo,
-gencode arch=compute_100a,code=sm_100a, and no --use_fast_math: the exact path
needs IEEE division and separately rounded multiplies and adds (the kernels also
spell them with __fmul_rn / __fadd_rn / __fdiv_rn so no contraction can happen).
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
OBJDIR = os.path.join(HERE, "_build")
LIB = os.path.join(LIBDIR, "libtopk_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off", "-I", CSRC,
          "-I", INCLUDE]


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build failed: " + " ".join(cmd))
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stdout + r.stderr)


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def headers():
    return sorted(glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) +
                  glob.glob(os.path.join(INCLUDE, "*.h")))


def build(verbose=False, force=False, ptxas_verbose=False, check=False):
    """check=True builds libtopk_b200_check.so with -DTOPK_BOUNDS_CHECK (kernels record
    the first failed bounds/alignment/phase check in their scratch and skip the access)."""
    lib = LIB.replace(".so", "_check.so") if check else LIB
    objdir = OBJDIR + ("_check" if check else "")
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(objdir, exist_ok=True)
    hdr_t = max((os.path.getmtime(h) for h in headers()), default=0)
    objs = []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        objs.append(obj)
        stale = force or not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(src), hdr_t)
        if not stale:
            continue
        cmd = [NVCC] + COMMON + ARCH + (["-DTOPK_BOUNDS_CHECK"] if check else []) + ["-c", src, "-o", obj]
        if src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"] if ptxas_verbose else []
        _run(cmd, verbose or ptxas_verbose)
    if force or not os.path.exists(lib) or any(os.path.getmtime(o) > os.path.getmtime(lib) for o in objs):
        _run([NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", lib] + objs + ["-lpthread", "-ldl", "-lrt"], verbose)
    return lib


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv, ptxas_verbose="--ptxas" in sys.argv,
                check="--check" in sys.argv))
