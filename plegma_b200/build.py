"""Build recipe for the CUDA library (sm_100a) and the C++ drop-in test driver.

    python -m plegma_b200.build [--force]

Produces plegma_b200/lib/libplegma2pt.so in the source tree (it travels with
the repository to the GPU machine; nothing is JIT-compiled at run time).
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libplegma2pt.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
GENDIR = os.path.join(LIBDIR, "gen")  # headers generated at build time (not committed)
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fopenmp", "--expt-relaxed-constexpr",
                     "-I" + os.path.join(ROOT, "include"), "-I" + GENDIR]


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _deps():
    return _sources() + sorted(glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))) + \
        [os.path.join(ROOT, "include", "plegma2pt.h"), os.path.join(GENDIR, "udsc_tables.h")]


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, jobs=None):
    os.makedirs(LIBDIR, exist_ok=True)
    objdir = os.path.join(LIBDIR, "obj")
    os.makedirs(objdir, exist_ok=True)
    from . import spin, udsc
    spin.emit_header(os.path.join(CSRC, "spin_tables.h"))
    os.makedirs(GENDIR, exist_ok=True)
    udsc.emit_header(os.path.join(GENDIR, "udsc_tables.h"))
    headers = [d for d in _deps() if not d.endswith(".cu")]
    objs = []
    procs = []
    for src in _sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            cmd = [NVCC] + NVCC_FLAGS + ["-c", src, "-o", obj]
            if verbose:
                cmd += ["-Xptxas", "-v"]
            procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0 or verbose:
            sys.stderr.write(out.decode())
        if p.returncode != 0:
            failed.append(src)
    if failed:
        raise RuntimeError("nvcc failed for: " + ", ".join(failed))
    if force or _stale(LIB, objs):
        subprocess.run([NVCC] + ARCH + ["-shared", "-Xcompiler", "-fopenmp", "-o", LIB] + objs + ["-lgomp"],
                       check=True)
    return LIB


def build_cxx_driver(force=False):
    """The C++ drop-in test driver (tests/cxx/calc_2pt.cpp) linked against the library."""
    src = os.path.join(ROOT, "tests", "cxx", "calc_2pt.cpp")
    out_dir = os.path.join(ROOT, "tests", "cxx", "_build")
    os.makedirs(out_dir, exist_ok=True)
    exe = os.path.join(out_dir, "calc_2pt")
    deps = [src, os.path.join(ROOT, "include", "plegma", "PLEGMA_2pt.h"), os.path.join(ROOT, "include", "plegma2pt.h"),
            LIB]
    if force or _stale(exe, deps):
        subprocess.run(["g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"), "-o", exe, src,
                        "-L" + LIBDIR, "-lplegma2pt", "-Wl,-rpath," + LIBDIR], check=True)
    return exe


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
    print(build_cxx_driver(force="--force" in sys.argv))
