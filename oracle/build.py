"""Build recipe for the CPU oracle (oracle/_build/liboracle.so) and, where
the reference sources are mounted, for the reference's own baryon
contraction functions compiled as host code (oracle/_ref/libplegma_ref.so).

The oracle is test infrastructure: only tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg load these libraries.

    python oracle/build.py [--ref /path/to/PLEGMA]
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REF_OUT = os.path.join(HERE, "_ref")
DEFAULT_REF = "/root/reference"


def _run(cmd):
    subprocess.run(cmd, check=True)


def _stale(out, srcs):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(s) > t for s in srcs)


def build_oracle(force=False):
    os.makedirs(BUILD, exist_ok=True)
    out = os.path.join(BUILD, "liboracle.so")
    srcs = [os.path.join(HERE, "oracle.cpp"),
            os.path.join(HERE, "..", "plegma_b200", "csrc", "spin_tables.h")]
    if force or _stale(out, srcs):
        _run(["g++", "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared", "-std=c++17",
              "-o", out, srcs[0]])
    return out


def build_ref(ref_root=DEFAULT_REF, force=False):
    """Compile the reference's PLEGMA_baryons_NtoN.cu and PLEGMA_baryons_deltas.cu
    (read in place, never copied) with the small type shim in ref_shim/.
    Returns the library path, or None when the sources are not present."""
    kern = os.path.join(ref_root, "lib", "kernels")
    srcs = [os.path.join(kern, f) for f in ("PLEGMA_baryons_NtoN.cu", "PLEGMA_baryons_NtoR.cu", "PLEGMA_baryons_RtoN.cu",
                                           "PLEGMA_baryons_RtoR.cu", "PLEGMA_baryons_deltas.cu")]
    if not all(os.path.exists(s) for s in srcs):
        return None
    os.makedirs(REF_OUT, exist_ok=True)
    out = os.path.join(REF_OUT, "libplegma_ref.so")
    deps = srcs + [os.path.join(HERE, "ref_wrap.cpp"), os.path.join(HERE, "ref_shim", "PLEGMA_kernel_utils.cuh")]
    if force or _stale(out, deps):
        cmd = ["g++", "-O2", "-fPIC", "-shared", "-std=c++14", "-D__device__=",
               "-I", os.path.join(HERE, "ref_shim"), "-o", out,
               os.path.join(HERE, "ref_wrap.cpp"), "-x", "c++"] + srcs
        _run(cmd)
    return out


if __name__ == "__main__":
    ref = DEFAULT_REF
    if "--ref" in sys.argv:
        ref = sys.argv[sys.argv.index("--ref") + 1]
    print(build_oracle(force=True))
    print(build_ref(ref, force=True))
