"""Build the in-tree shared library ``ddg_b200/lib/libddg_sipg.so``.

nvcc cross-compiles for sm_100a only (``-gencode arch=compute_100a,
code=sm_100a``); no GPU is needed to build.  Usage::

    python -m ddg_b200.build [--verbose]      # -Xptxas -v with --verbose
"""

from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libddg_sipg.so")

CU_SOURCES = ["sipg_kernels.cu", "sipg_mg.cu", "sipg_capi.cu", "sipg_pool.cu", "noalloc.cu"]
CXX_SOURCES = ["mesh_connect.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _sources():
    return [os.path.join(CSRC, s) for s in CU_SOURCES + CXX_SOURCES]


def _deps():
    out = _sources()
    for f in os.listdir(CSRC):
        if f.endswith((".h", ".cuh")):
            out.append(os.path.join(CSRC, f))
    out.append(os.path.join(HERE, "..", "include", "ddg_sipg.h"))
    return out


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(p) <= t for p in _deps() if os.path.exists(p))


def build(verbose: bool = False, force: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    cmd = [_nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC,-O2",
           "--expt-relaxed-constexpr", "-o", LIB + ".tmp", *_sources()]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed building libddg_sipg.so")
    if verbose:
        sys.stderr.write(r.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv, force=True))
