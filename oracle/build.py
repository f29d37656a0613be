"""Build recipe for the CPU checker (TEST INFRASTRUCTURE ONLY).

Products:
  * oracle/_build/liboracle.so  - the C restatement (topk_oracle.c), strict FP flags.
  * oracle/_ref/libref_tpac.so  - the reference's own TPAc (cpu/TPAc.h, cpu/AA.h,
    common/common.h, time/Time.h) compiled from where its sources lie, through the
    forwarding shim ref_tpac_shim.cpp.  Built only when the reference tree is present
    (see reference_root()); the .so then travels with the repo.
  * oracle/_ref/libref_index_d{D}_imp{I}.so - the reference's VTA and PTA index
    builds (cpu/VTA.h, cpu/PTA.h) through ref_index_shim.cpp, likewise.
  * oracle/_ref/libref_file.so - the reference's table loader (input/File.h) through
    ref_file_shim.cpp, likewise.
  * oracle/_ref/libref_sla_d{D}.so - the reference's SLA layer build (cpu/SLA.h and
    its vendored skyline library) through ref_sla_shim.cpp, likewise.

Strict flags for both: -O3 -ffp-contract=off, never -ffast-math.  The reference's
own Makefile:60 adds -ffast-math, which changes the normalised table and the
scores; the strict build is the one whose scalar/SIMD/threads paths agree.
-march=x86-64-v3 (AVX2) keeps the .so runnable on any AVX2 host.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REF_OUT = os.path.join(HERE, "_ref")
ORACLE_SO = os.path.join(BUILD, "liboracle.so")
REF_SO = os.path.join(REF_OUT, "libref_tpac.so")


# Where the build container mounts the reference tree (read-only).  This recipe is
# the one place that names it; set TOPK_REFERENCE to build from another checkout.
CONTAINER_REFERENCE = "/root/reference"


def reference_root():
    """The reference tree this recipe compiles from: $TOPK_REFERENCE when set, else the
    build container's mount.  Callers check that it exists (it does not on GPU boxes,
    which use the prebuilt libraries under oracle/_ref)."""
    return os.environ.get("TOPK_REFERENCE") or CONTAINER_REFERENCE


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _stale(out, srcs):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(s) > t for s in srcs if os.path.exists(s))


def build_oracle(verbose=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    srcs = [os.path.join(HERE, "topk_oracle.c"), os.path.join(HERE, "topk_oracle.h")]
    if force or _stale(ORACLE_SO, srcs):
        _run(["gcc", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC", "-shared",
              "-std=c11", srcs[0], "-o", ORACLE_SO, "-lm"], verbose)
    return ORACLE_SO


def build_ref(verbose=False, force=False):
    """Compile the reference TPAc through the shim. Returns the .so path or None."""
    root = reference_root()
    hdrs = [os.path.join(root, p) for p in ("cpu/TPAc.h", "cpu/TPAr.h", "cpu/TA.h", "cpu/AA.h",
                                            "common/common.h", "time/Time.h")]
    if not all(os.path.exists(h) for h in hdrs):
        return REF_SO if os.path.exists(REF_SO) else None
    os.makedirs(REF_OUT, exist_ok=True)
    shim = os.path.join(HERE, "ref_tpac_shim.cpp")
    if force or _stale(REF_SO, [shim] + hdrs):
        _run(["g++", "-std=c++14", "-O3", "-march=x86-64-v3", "-ffp-contract=off", "-fno-fast-math",
              "-fopenmp", "-fPIC", "-shared", "-w",
              "-I", root, "-I", os.path.join(HERE, "stub"), shim, "-o", REF_SO], verbose)
    return REF_SO


# (NUM_DIMS, IMP) of the reference index builds compiled for the tests and the
# benchmark: the reference fixes both at compile time (Makefile:22-23,60).
INDEX_CONFIGS = ((4, 2), (4, 1), (8, 2), (8, 1))


def ref_index_so(num_dims, imp):
    return os.path.join(REF_OUT, f"libref_index_d{num_dims}_imp{imp}.so")


def build_ref_index(verbose=False, force=False):
    """Compile the reference VTA / PTA index builds through ref_index_shim.cpp, one
    library per (NUM_DIMS, IMP).  Returns the list of built paths (those present when
    the reference tree is absent)."""
    root = reference_root()
    hdrs = [os.path.join(root, p) for p in ("cpu/VTA.h", "cpu/PTA.h", "cpu/AA.h", "common/common.h",
                                            "time/Time.h")]
    outs = [ref_index_so(dd, imp) for dd, imp in INDEX_CONFIGS]
    if not all(os.path.exists(h) for h in hdrs):
        return [o for o in outs if os.path.exists(o)]
    os.makedirs(REF_OUT, exist_ok=True)
    shim = os.path.join(HERE, "ref_index_shim.cpp")
    for (dd, imp), out in zip(INDEX_CONFIGS, outs):
        if force or _stale(out, [shim] + hdrs):
            _run(["g++", "-std=c++14", "-O3", "-march=x86-64-v3", "-ffp-contract=off", "-fno-fast-math",
                  "-fopenmp", "-fPIC", "-shared", "-w", f"-DNUM_DIMS={dd}", f"-DIMP={imp}",
                  "-I", root, "-I", os.path.join(HERE, "stub"), shim, "-o", out], verbose)
    return outs


SLA_DIMS = (4, 6)


def ref_sla_so(num_dims):
    return os.path.join(REF_OUT, f"libref_sla_d{num_dims}.so")


def build_ref_sla(verbose=False, force=False):
    """Compile the reference SLA layer build (cpu/SLA.h with the skyline library it
    vendors under skyline/) through ref_sla_shim.cpp, one library per NUM_DIMS.
    Returns the list of built paths (those present when the reference is absent)."""
    root = reference_root()
    srcs = [os.path.join(root, p) for p in ("skyline/hybrid/hybrid.cpp", "skyline/common/common.cpp",
                                            "skyline/common/skyline_i.cpp", "skyline/util/timing.cpp")]
    hdrs = [os.path.join(root, p) for p in ("cpu/SLA.h", "cpu/VTA.h", "cpu/AA.h", "common/common.h",
                                            "skyline/hybrid/hybrid.h", "time/Time.h")]
    outs = [ref_sla_so(dd) for dd in SLA_DIMS]
    if not all(os.path.exists(f) for f in srcs + hdrs):
        return [o for o in outs if os.path.exists(o)]
    os.makedirs(REF_OUT, exist_ok=True)
    shim = os.path.join(HERE, "ref_sla_shim.cpp")
    for dd, out in zip(SLA_DIMS, outs):
        if force or _stale(out, [shim] + srcs + hdrs):
            _run(["g++", "-std=c++14", "-O2", "-march=x86-64-v3", "-ffp-contract=off", "-fno-fast-math",
                  "-fopenmp", "-fPIC", "-shared", "-w", f"-DNUM_DIMS={dd}", "-I", root,
                  "-I", os.path.join(HERE, "stub"), "-I", os.path.join(root, "skyline"), shim] + srcs + ["-o", out],
                 verbose)
    return outs


REF_FILE_SO = os.path.join(REF_OUT, "libref_file.so")


def build_ref_file(verbose=False, force=False):
    """Compile the reference table loader (input/File.h) through ref_file_shim.cpp.
    Returns the .so path or None."""
    root = reference_root()
    hdrs = [os.path.join(root, p) for p in ("input/File.h", "time/Time.h",
                                            "input/randdataset-1.1.0/src/randdataset.h")]
    if not all(os.path.exists(h) for h in hdrs):
        return REF_FILE_SO if os.path.exists(REF_FILE_SO) else None
    os.makedirs(REF_OUT, exist_ok=True)
    shim = os.path.join(HERE, "ref_file_shim.cpp")
    if force or _stale(REF_FILE_SO, [shim] + hdrs):
        _run(["g++", "-std=c++14", "-O3", "-march=x86-64-v3", "-fPIC", "-shared", "-w",
              "-I", root, shim, "-o", REF_FILE_SO], verbose)
    return REF_FILE_SO


if __name__ == "__main__":
    v = "-v" in sys.argv
    print(build_oracle(v, force="-f" in sys.argv))
    print(build_ref(v, force="-f" in sys.argv))
    print(build_ref_index(v, force="-f" in sys.argv))
    print(build_ref_file(v, force="-f" in sys.argv))
    print(build_ref_sla(v, force="-f" in sys.argv))
