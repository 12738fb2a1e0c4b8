"""Build the in-tree shared library ``nebula_b200/libnebula_b200.so``.

CUDA sources are compiled for sm_100a only (``-gencode
arch=compute_100a,code=sm_100a``); host C++ with g++ without FMA
contraction, so host-side float arithmetic (octree bounds, triangle normals,
table transforms) rounds exactly like the reference's CPU build.  The CUDA
runtime is linked statically, so the library does not depend on the runtime
version of whichever framework loads it.

Usage: ``python -m nebula_b200.build`` (or ``build()`` from Python).  The
build is incremental: objects are rebuilt when a source or header is newer.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libnebula_b200.so")
# the command-line driver (a drop-in for the reference's GPU executable)
DRIVER_SRC = os.path.join(CSRC, "driver", "nebula_gpu_main.cpp")
DRIVER = os.path.join(HERE, "nebula_b200_gpu")
# the same source as the energy-deposit executable
DRIVER_EDEP = os.path.join(HERE, "nebula_b200_edep")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
              "--expt-relaxed-constexpr", "-I" + INCLUDE] + ARCH
CXX_FLAGS = ["-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-Wall", "-Wno-unused-function",
             "-I" + os.path.join(CUDA_HOME, "include"), "-I" + INCLUDE]


def _headers():
    return (glob.glob(os.path.join(CSRC, "**", "*.h"), recursive=True)
            + glob.glob(os.path.join(CSRC, "**", "*.hpp"), recursive=True)
            + glob.glob(os.path.join(CSRC, "**", "*.cuh"), recursive=True)
            + glob.glob(os.path.join(INCLUDE, "*.h")))


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n%s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    return r


def sources():
    cu = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    cpp = sorted(glob.glob(os.path.join(CSRC, "host", "*.cpp")))
    return cu, cpp


def build(verbose=False, force=False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = _headers()
    cu, cpp = sources()
    objs = []
    for src in cu:
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        if force or _stale(obj, [src] + headers):
            _run([NVCC] + NVCC_FLAGS + ["-c", src, "-o", obj], verbose)
        objs.append(obj)
    for src in cpp:
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        if force or _stale(obj, [src] + headers):
            _run(["g++"] + CXX_FLAGS + ["-c", src, "-o", obj], verbose)
        objs.append(obj)
    if force or _stale(LIB, objs):
        _run(["g++", "-shared", "-o", LIB] + objs
             + ["-L" + os.path.join(CUDA_HOME, "lib64"), "-lcudart_static", "-lpthread", "-ldl", "-lrt"], verbose)
    for exe, defs in ((DRIVER, []), (DRIVER_EDEP, ["-DNBL_DRIVER_EDEP"])):
        if force or _stale(exe, [DRIVER_SRC, LIB] + glob.glob(os.path.join(INCLUDE, "*.h"))):
            _run(["g++", "-std=c++17", "-O2", "-Wall", "-I" + INCLUDE] + defs + [DRIVER_SRC, "-o", exe, "-L" + HERE,
                  "-lnebula_b200", "-Wl,-rpath,$ORIGIN", "-pthread"], verbose)
    return LIB


def ptxas_report(src="transport.cu"):
    """Registers / spills / shared memory per kernel (nvcc -Xptxas -v)."""
    r = _run([NVCC] + NVCC_FLAGS + ["-Xptxas", "-v", "-c", os.path.join(CSRC, src), "-o", os.devnull], False)
    return r.stderr


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
