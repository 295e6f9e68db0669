"""Oracle: build and call the C + OpenMP float64 restatement of the SIPG
apply (``oracle/c/sipg_apply.c``).  Test infrastructure and CPU baseline
only (see ``oracle/__init__.py``); the GPU product never loads it.

``time_apply`` is the ``cpu_baseline`` / ``--impl reference`` leg of
``bench.py``: the apply on the host's cores over the same mesh, bounded in
wall time.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "c", "sipg_apply.c")
LIB = os.path.join(HERE, "lib", "liboracle_sipg.so")


class _Mesh(C.Structure):
    _fields_ = [("N", C.c_int), ("Np", C.c_int), ("Nfp", C.c_int), ("K", C.c_int),
                ("Dr", C.c_void_p), ("Ds", C.c_void_p), ("M", C.c_void_p), ("m1d", C.c_void_p),
                ("Fmask", C.c_void_p),
                ("rx", C.c_void_p), ("sx", C.c_void_p), ("ry", C.c_void_p), ("sy", C.c_void_p),
                ("J", C.c_void_p),
                ("nx", C.c_void_p), ("ny", C.c_void_p), ("sJ", C.c_void_p), ("Fscale", C.c_void_p),
                ("vmapM", C.c_void_p), ("vmapP", C.c_void_p), ("EToE", C.c_void_p), ("EToF", C.c_void_p),
                ("bc", C.c_void_p), ("tau_scale", C.c_double), ("alpha", C.c_double)]


def build(force: bool = False) -> str:
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    cmd = ["gcc", "-O3", "-march=x86-64-v3", "-fopenmp", "-shared", "-fPIC", "-o", LIB + ".tmp", SRC, "-lm"]
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(LIB)
        _lib.oracle_sipg_apply.argtypes = [C.POINTER(_Mesh), C.c_void_p, C.c_void_p, C.c_int]
        _lib.oracle_sipg_apply.restype = None
    return _lib


class CApply:
    """Float64 apply ``alpha J M u + A u`` on an oracle ``Mesh2D``."""

    def __init__(self, mesh, bc_types, tau_scale=200.0, alpha=0.0):
        ref = mesh.ref
        c = lambda a, dt=np.float64: np.ascontiguousarray(a, dtype=dt)  # noqa: E731
        self._keep = [c(ref.Dr), c(ref.Ds), c(ref.M), c(ref.m1d), c(ref.Fmask, np.int64),
                      c(mesh.rx), c(mesh.sx), c(mesh.ry), c(mesh.sy), c(mesh.J),
                      c(mesh.nx), c(mesh.ny), c(mesh.sJ), c(mesh.Fscale),
                      c(mesh.vmapM, np.int64), c(mesh.vmapP, np.int64), c(mesh.EToE, np.int64),
                      c(mesh.EToF, np.int64), c(bc_types, np.int32)]
        self.m = _Mesh(mesh.N, mesh.Np, mesh.Nfp, mesh.K, *[a.ctypes.data for a in self._keep],
                       float(tau_scale), float(alpha))
        self.n = mesh.Np * mesh.K

    def __call__(self, u_flat, threads=None, out=None):
        u = np.ascontiguousarray(u_flat, dtype=np.float64)
        y = np.empty_like(u) if out is None else out
        nt = threads or len(os.sched_getaffinity(0))
        lib().oracle_sipg_apply(C.byref(self.m), u.ctypes.data, y.ctypes.data, nt)
        return y


_CACHE = {}


def _bench_mesh(Kx, Ky, N, tau_scale, alpha):
    key = (Kx, Ky, N, tau_scale, alpha)
    if key not in _CACHE:
        from .mesh import build_mesh_2d, uniform_rectangle_mesh_2d
        m = build_mesh_2d(*uniform_rectangle_mesh_2d(0.0, 1.0, 0.0, 1.0, Kx, Ky), N)
        isb = m.EToE == np.arange(m.K)[:, None]
        nxf = m.nx.reshape((m.Nfp, 3, m.K), order="F")[0].T
        bc = np.where(isb, np.where(np.abs(nxf) > 0.5, 1, 2), 0).astype(np.int32)
        _CACHE[key] = CApply(m, bc, tau_scale, alpha)
    return _CACHE[key]


def apply_stepper(Kx, Ky, N, tau_scale, alpha):
    """One timed float64 apply per call on all host cores (the reference arm
    of the benchmark); returns (step() -> seconds, DOFs, threads)."""
    op = _bench_mesh(Kx, Ky, N, tau_scale, alpha)
    u = np.random.default_rng(1).standard_normal(op.n)
    y = np.zeros_like(u)                         # output pages touched once, outside the timing
    nt = len(os.sched_getaffinity(0))

    def step():
        t0 = time.perf_counter()
        op(u, nt, out=y)
        return time.perf_counter() - t0
    return step, op.n, nt


def time_apply(Kx, Ky, N, tau_scale, alpha, budget_s=15.0, reps=None):
    """Median time of the C+OpenMP float64 apply on all host cores."""
    op = _bench_mesh(Kx, Ky, N, tau_scale, alpha)
    u = np.random.default_rng(1).standard_normal(op.n)
    y = np.zeros_like(u)                         # output pages touched once, outside the timing
    nt = len(os.sched_getaffinity(0))
    op(u, nt, out=y)                             # warm-up
    times = []
    t_start = time.perf_counter()
    while True:
        t0 = time.perf_counter()
        op(u, nt, out=y)
        times.append(time.perf_counter() - t0)
        if reps is not None and len(times) >= reps:
            break
        if reps is None and (time.perf_counter() - t_start > budget_s or len(times) >= 200):
            break
    t = float(np.median(times))
    return {"value": op.n / t / 1e9, "unit": "GDOF/s", "cores": nt, "kind": "port",
            "sample": f"{len(times)} float64 applies of the full {2 * Kx * Ky}-element N={N} mesh "
                      f"(C+OpenMP restatement of the reference operator; median), {t * 1e3:.2f} ms each",
            "median_ms": t * 1e3}
