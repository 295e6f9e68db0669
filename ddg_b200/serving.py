"""Continuous-batching serving of SIPG solves on one GPU.

Requests (a mesh, a polynomial degree, a Helmholtz coefficient, a source and
a tolerance) arrive over time.  Each degree has a device pool
(``ddg_pool_*`` in ``libddg_sipg.so``) that packs the elements of many
requests into one array; every pool launch (a captured CUDA graph of
block-Jacobi PCG iterations) advances all of its active requests at once,
with per-request CG scalars, so a request's iterates are identical alone and
in any mix.  The scheduler admits arrivals whenever a slot and an element
range are free (ranges are sized against an HBM budget), keeps iterating the
others meanwhile, and retires each request as soon as it converges.

Extension: the reference solves one mesh per call and has no serving layer.
"""

from __future__ import annotations

import ctypes as C
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .autotune import Tile, TileAutotuner
from .dg2d.mesh import build_mesh_2d, uniform_rectangle_mesh_2d
from .dg2d.reference import ref_element


@dataclass
class Request:
    rid: int
    arrival: float          # seconds after the stream start
    n: int                  # n x n quads -> 2 n^2 triangles on [0,1]^2
    N: int                  # polynomial degree
    alpha: float            # Helmholtz coefficient k^2
    tol: float
    modes: tuple            # (amplitudes, kx, ky) of the 8-mode source
    # filled by the engine
    admitted: float = -1.0
    done: float = -1.0
    iterations: int = 0
    status: str = ""
    precision: str = ""     # "fp32" or "fp64": the pool that served it
    x: np.ndarray | None = field(default=None, repr=False)

    @property
    def latency(self) -> float:
        return self.done - self.arrival


def make_requests(count=4096, rate=None, seed=0, n_range=(8, 96), degrees=(2, 3, 4), k2_range=(0.0, 10.0),
                  tols=(1e-6, 1e-9)):
    """Seeded request stream: n ~ U{8..96}, N ~ U{2,3,4}, k^2 ~ U[0,10], tol in
    {1e-6, 1e-9}, RHS = sum of 8 modes a sin(pi i x) sin(pi j y) with
    i, j ~ U{1..6}, a ~ N(0,1); Poisson arrivals with ``rate`` per second
    (all at t = 0 when rate is None)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(count):
        if rate is not None:
            t += rng.exponential(1.0 / rate)
        modes = (rng.standard_normal(8), rng.integers(1, 7, 8), rng.integers(1, 7, 8))
        out.append(Request(rid=i, arrival=t if rate is not None else 0.0,
                           n=int(rng.integers(n_range[0], n_range[1] + 1)), N=int(rng.choice(degrees)),
                           alpha=float(rng.uniform(*k2_range)), tol=float(rng.choice(tols)), modes=modes))
    return out


class _MeshCache:
    """Host mesh data per (n, N): built once, reused by every request."""

    def __init__(self):
        self._c = {}

    def get(self, n, N):
        key = (n, N)
        if key not in self._c:
            m = build_mesh_2d(*uniform_rectangle_mesh_2d(0.0, 1.0, 0.0, 1.0, n, n), N)
            isb = m.EToE == np.arange(m.K)[:, None]
            bc = np.where(isb, 1, 0).astype(np.int32)                        # Dirichlet walls
            ref = ref_element(N)
            arrays = dict(Dr=np.ascontiguousarray(ref.Dr), Ds=np.ascontiguousarray(ref.Ds),
                          M=np.ascontiguousarray(ref.M), m1d=np.ascontiguousarray(ref.m1d),
                          Fmask=np.ascontiguousarray(ref.Fmask, dtype=np.int64),
                          rot=np.ascontiguousarray(ref.rot_perm, dtype=np.int64),
                          geo=np.ascontiguousarray(m.element_geometry()),
                          EToE=np.ascontiguousarray(m.EToE), EToF=np.ascontiguousarray(m.EToF),
                          vmapM=np.ascontiguousarray(m.vmapM), vmapP=np.ascontiguousarray(m.vmapP), bc=bc)
            self._c[key] = (m, arrays)
        return self._c[key]


def _desc(m, a, tau_scale, device):
    dp = lambda x: x.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
    ip = lambda x: x.ctypes.data_as(C.POINTER(C.c_int64))   # noqa: E731
    return _lib.MeshDesc(N=m.N, K=m.K, device=device, reserved=0, tau_scale=tau_scale,
                         Dr=dp(a["Dr"]), Ds=dp(a["Ds"]), M=dp(a["M"]), m1d=dp(a["m1d"]),
                         Fmask=ip(a["Fmask"]), rot_perm=ip(a["rot"]), geo=dp(a["geo"]),
                         EToE=ip(a["EToE"]), EToF=ip(a["EToF"]), vmapM=ip(a["vmapM"]), vmapP=ip(a["vmapP"]),
                         bc_types=a["bc"].ctypes.data_as(C.POINTER(C.c_int32)))


def source_nodal(m, modes):
    amp, kx, ky = modes
    return sum(a * np.sin(np.pi * i * m.x) * np.sin(np.pi * j * m.y) for a, i, j in zip(amp, kx, ky))


def bytes_per_element(N: int, fp32: bool = False) -> int:
    """Device bytes a pool element needs (geometry, words, inverses, vectors;
    a float32 pool adds float32 copies of the geometry and inverses and keeps
    its iteration vectors in float32)."""
    Np = (N + 1) * (N + 2) // 2
    nS = Np * (Np + 1) // 2
    base = 14 * 8 + 12 + 4 + 8 + nS * 8 + Np * 8 + 16            # geometry, words, seg, alpha, binv, b
    if fp32:
        return base + 14 * 4 + nS * 4 + 6 * Np * 4
    return base + 6 * Np * 8


class SolvePool:
    """One ``ddg_pool`` (one polynomial degree and vector precision)."""

    def __init__(self, N, capacity, max_requests, max_request_K, tau_scale, device=0, fp32=False):
        self.N = N
        self.fp32 = fp32
        self.tau_scale = tau_scale
        self.device = device
        self.max_requests = max_requests
        h = C.c_void_p()
        _lib.check(_lib.lib().ddg_pool_create_ex(N, capacity, max_requests, max_request_K, tau_scale,
                                                 _lib.DDG_FP32 if fp32 else _lib.DDG_FP64, device, C.byref(h)),
                   "ddg_pool_create_ex")
        self._h = h
        self.slot_req = {}
        self.elements = 0           # elements of the requests admitted and not retired
        self._tile = None
        self._act = np.zeros(max_requests, dtype=np.int32)
        self._its = np.zeros(max_requests, dtype=np.int32)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.lib().ddg_pool_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def admit(self, req, mesh, arrays, stream, maxiter=100000):
        f = np.ascontiguousarray(source_nodal(mesh, req.modes).T)         # (K, Np) element-major
        slot = C.c_int(-1)
        rc = _lib.lib().ddg_pool_admit(self._h, C.byref(_desc(mesh, arrays, self.tau_scale, self.device)),
                                       req.alpha, req.tol, 0.0, maxiter, f.ctypes.data, stream, C.byref(slot))
        if rc == 4:          # DDG_ERR_NOMEM: no slot / range free right now
            return False
        _lib.check(rc, "ddg_pool_admit")
        self.slot_req[slot.value] = (req, mesh)
        self.elements += mesh.K
        req.precision = "fp32" if self.fp32 else "fp64"
        return True

    def set_tile(self, tile: Tile):
        if tile != self._tile:
            _lib.check(_lib.lib().ddg_pool_set_tile(self._h, tile.threads, tile.persistent), "ddg_pool_set_tile")
            self._tile = tile

    def iterate(self, pairs, stream):
        _lib.check(_lib.lib().ddg_pool_iterate(self._h, pairs, stream), "ddg_pool_iterate")

    def finished(self, stream):
        _lib.check(_lib.lib().ddg_pool_poll(self._h, self._act.ctypes.data, self._its.ctypes.data, stream),
                   "ddg_pool_poll")
        return [s for s in self.slot_req if self._act[s] == 0]

    def retire(self, slot, stream):
        req, mesh = self.slot_req.pop(slot)
        self.elements -= mesh.K
        x = np.empty((mesh.K, mesh.Np))
        info = _lib.SolveInfo()
        _lib.check(_lib.lib().ddg_pool_retire(self._h, slot, x.ctypes.data, stream, C.byref(info)),
                   "ddg_pool_retire")
        req.x = x.T.copy()
        req.iterations = info.iterations
        req.status = _lib.SOLVE_STATUS.get(info.status, str(info.status))
        return req

    @property
    def active(self):
        return len(self.slot_req)


class ServingEngine:
    """Continuous-batching scheduler over one pool per polynomial degree.

    ``autotune`` (default on): the tile shape of every pool launch (threads
    per block, persistent grid, iterations per graph) comes from a
    :class:`~ddg_b200.autotune.TileAutotuner` keyed on (degree, active
    element count); pass a tuner to share or preload one.  With
    ``autotune=False`` every launch uses 128 threads, one thread per element
    and ``pairs``.

    ``fp32_tol`` (default 1e-6): requests whose tolerance is at least this
    run in a float32 pool of their degree (float32 vectors, geometry and
    inverses; float64 reductions), the others in the float64 pool; None
    keeps every request in float64."""

    def __init__(self, degrees=(2, 3, 4), hbm_budget_bytes=120e9, tau_scale=0.5, max_requests=4096,
                 max_request_K=2 * 96 * 96, capacity=None, pairs=4, device=0, autotune=True, fp32_tol=1e-6):
        import torch
        torch.cuda.set_device(device)
        self.device = device
        self.tau_scale = tau_scale
        self.pairs = pairs
        if autotune is True:
            self.tuner = TileAutotuner()
        elif autotune:
            self.tuner = autotune
        else:
            self.tuner = None
        self.meshes = _MeshCache()
        self.fp32_tol = fp32_tol
        self.pools = {}
        kinds = (False, True) if fp32_tol is not None else (False,)
        share = hbm_budget_bytes / (len(degrees) * len(kinds))
        for N in degrees:
            for f32 in kinds:
                cap = (int(min(share // bytes_per_element(N, f32), 32_000_000)) if capacity is None
                       else int(capacity))
                self.pools[(N, f32)] = SolvePool(N, cap, max_requests, max_request_K, tau_scale, device, fp32=f32)
        self.stream = torch.cuda.Stream(device=device)
        self._torch = torch

    def close(self):
        for p in self.pools.values():
            p.close()

    def run(self, requests, realtime=True):
        """Serve ``requests`` (arrival times relative to the start).  Returns
        the finished requests with latency, iterations and solution."""
        s = self.stream.cuda_stream
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        waiting = {key: deque() for key in self.pools}
        done = []
        t0 = time.perf_counter()
        while len(done) < len(requests):
            now = time.perf_counter() - t0
            while pending and (pending[0].arrival <= now or not realtime):
                r = pending.popleft()
                waiting[(r.N, self.fp32_tol is not None and r.tol >= self.fp32_tol)].append(r)
            for key, q in waiting.items():            # admit while slots / ranges are free
                pool = self.pools[key]
                while q:
                    m, arrays = self.meshes.get(q[0].n, pool.N)
                    if not pool.admit(q[0], m, arrays, s):
                        break
                    q.popleft().admitted = time.perf_counter() - t0
            busy = [p for p in self.pools.values() if p.active]
            timed = []
            for p in busy:
                tkey = f"N{p.N}-fp32" if p.fp32 else f"N{p.N}"
                tile = self.tuner.choose(tkey, p.elements) if self.tuner else Tile(128, 0, self.pairs)
                p.set_tile(tile)
                if self.tuner:
                    ev = (self._torch.cuda.Event(enable_timing=True), self._torch.cuda.Event(enable_timing=True))
                    ev[0].record(self.stream)
                    p.iterate(tile.pairs, s)
                    ev[1].record(self.stream)
                    timed.append((tkey, p.elements, tile, ev))
                else:
                    p.iterate(tile.pairs, s)
            for p in busy:
                for slot in p.finished(s):
                    r = p.retire(slot, s)
                    r.done = time.perf_counter() - t0
                    done.append(r)
            for tkey, el, tile, ev in timed:   # finished() synchronised the stream
                self.tuner.record(tkey, el, tile, ev[0].elapsed_time(ev[1]) * 1e-3 / (2 * tile.pairs))
            if not busy and pending and realtime:
                time.sleep(max(0.0, min(0.002, pending[0].arrival - (time.perf_counter() - t0))))
        self.elapsed = time.perf_counter() - t0
        return done


def summarize(done, elapsed):
    lat = np.array([r.latency for r in done])
    return {"requests": len(done), "elapsed_s": elapsed, "solves_per_s": len(done) / elapsed,
            "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "mean_iterations": float(np.mean([r.iterations for r in done])),
            "converged": int(sum(r.status == "converged" for r in done)),
            "fp32_requests": int(sum(r.precision == "fp32" for r in done))}


def solve_one_at_a_time(requests, tau_scale=0.5):
    """Baseline: each request alone through the float64 block-Jacobi PCG of
    ``solve_sipg_helmholtz_2d`` (device operator per mesh, cached)."""
    from .dg2d import sipg as ps
    cache = _MeshCache()
    out = []
    t0 = time.perf_counter()
    for r in requests:
        m, arrays = cache.get(r.n, r.N)
        pc = ps.make_helmholtz_block_jacobi_preconditioner(m, alpha=r.alpha, nu=1.0, bc_types=arrays["bc"],
                                                           tau_scale=tau_scale)
        u, info = ps.solve_sipg_helmholtz_2d(m, source_nodal(m, r.modes), alpha=r.alpha, nu=1.0,
                                             bc_types=arrays["bc"], tau_scale=tau_scale, preconditioner=pc,
                                             iterative=ps.IterativeConfig(tol=r.tol, maxiter=100000),
                                             return_info=True)
        out.append((u, info))
    return out, time.perf_counter() - t0
