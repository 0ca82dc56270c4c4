"""Build libfold3dpmm.so in-tree (sm_100a only).

CUDA sources are compiled with ``--fmad=false`` (no multiply-add
contraction) and host sources with ``-ffp-contract=off``, so that every
floating-point operation rounds on its own exactly as the reference's host
build does; CUDA's double division and square root are IEEE correctly
rounded by default.  Fast-math is never enabled.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libfold3dpmm.so")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3", "-std=c++17", *ARCH, "-lineinfo", "--fmad=false",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-O2,-fvisibility=hidden", "-I", INCLUDE, "-I", CSRC,
]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall",
             "-fvisibility=hidden",
             "-I", INCLUDE, "-I", CSRC, "-I", "/usr/local/cuda/include"]

CU_SOURCES = ["fold3d_kernels.cu", "fold3d_api.cu", "fold3d_noalloc.cu", "fold3d_wavefront.cu", "fold3d_adjoint.cu",
              "fold3d_init_dev.cu"]
CXX_SOURCES = ["fold3d_init.cpp", "fold3d_tables.cpp", "fold3d_io.cpp"]
HEADERS = ["fold3d_internal.h", "fold3d_solver.cuh", "fold3d_fast.cuh", "fold3d_ellip.cuh", "fold3d_sync.cuh",
           "fold3d_seed.h"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: %s\n%s\n%s" % (" ".join(cmd), r.stdout, r.stderr))
    return r


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, build_dir: str | None = None, lib: str | None = None,
          defines=()) -> str:
    """Compile into build_dir and link lib (defaults: _build/, libfold3dpmm.so);
    defines: extra -D flags for every source."""
    BUILD = build_dir or globals()["BUILD"]
    LIB = lib or globals()["LIB"]
    extra = ["-D%s" % d for d in defines]
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, h) for h in ("fold3dpmm.h", "fold3d_acc.h")] + [__file__]
    objs = []
    for src in CU_SOURCES + CXX_SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if force or _stale(obj, [path] + hdrs):
            if src.endswith(".cu"):
                cmd = [NVCC, *NVCC_FLAGS, *extra, "-c", path, "-o", obj]
                if verbose:
                    cmd.insert(1, "-Xptxas=-v")
            else:
                cmd = ["g++", *CXX_FLAGS, *extra, "-c", path, "-o", obj]
            r = _run(cmd)
            if verbose:
                sys.stdout.write(r.stdout + r.stderr)
    if force or _stale(LIB, objs):
        _run([NVCC, "-shared", *ARCH, "-o", LIB, *objs, "-lpthread"])
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
