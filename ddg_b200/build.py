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

CU_SOURCES = ["sipg_kernels.cu", "sipg_curved.cu", "sipg_mg.cu", "sipg_capi.cu", "sipg_curved_capi.cu",
              "sipg_pool.cu", "noalloc.cu"]
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
    """Compile every translation unit to an object (in parallel: the kernel
    units take minutes each), then link the shared library."""
    if not force and up_to_date():
        return LIB
    from concurrent.futures import ThreadPoolExecutor
    os.makedirs(LIBDIR, exist_ok=True)
    objdir = os.path.join(LIBDIR, "obj")
    os.makedirs(objdir, exist_ok=True)
    flags = [*ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2", "--expt-relaxed-constexpr"]
    if verbose:
        flags.insert(0, "-Xptxas=-v")

    def compile_one(src):
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        r = subprocess.run([_nvcc(), *flags, "-c", src, "-o", obj], capture_output=True, text=True)
        return src, obj, r

    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        results = list(ex.map(compile_one, _sources()))
    for src, _, r in results:
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"nvcc failed on {os.path.basename(src)}")
        if verbose:
            sys.stderr.write(r.stderr)
    r = subprocess.run([_nvcc(), *ARCH, "-shared", "-o", LIB + ".tmp", *[o for _, o, _ in results]],
                       capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed linking libddg_sipg.so")
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv, force=True))
