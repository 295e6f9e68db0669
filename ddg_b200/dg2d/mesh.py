"""2D triangle mesh (host setup) with the field names of ddg's ``Mesh2D``.

Mirrors ``src/ddg/dg2d/mesh.py``: ``uniform_rectangle_mesh_2d`` (:125-156)
and ``build_mesh_2d`` (:691-760) produce the same arrays (volume fields
``(Np, K)``, face fields ``(3 Nfp, K)``, ``vmapM``/``vmapP`` into the
element-major flat vector).  The topological connectivity (``EToE``,
``EToF``) and the node maps are computed by the C++ routines
``ddg_mesh_connect`` / ``ddg_mesh_maps`` of ``libddg_sipg.so``, bit-exact
with the reference's Python loops.  Geometry is float64 numpy.

A ``Mesh2D`` also caches the device-resident SIPG operators built on it
(see :meth:`Mesh2D.device_operator`).
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .. import _lib
from .reference import RefElement, ref_element


def uniform_rectangle_mesh_2d(xmin, xmax, ymin, ymax, Kx: int, Ky: int):
    """``2 Kx Ky`` triangles; each cell (i, j) gives (v00, v10, v11) and
    (v00, v11, v01) with vertex id ``j (Kx+1) + i``
    (``src/ddg/dg2d/mesh.py:125-156``).  Returns numpy ``(VX, VY, EToV)``."""
    xs = np.linspace(xmin, xmax, Kx + 1)
    ys = np.linspace(ymin, ymax, Ky + 1)
    VX = np.tile(xs, Ky + 1)
    VY = np.repeat(ys, Kx + 1)
    j, i = np.meshgrid(np.arange(Ky), np.arange(Kx), indexing="ij")
    v00 = (j * (Kx + 1) + i).reshape(-1)
    v10, v01 = v00 + 1, v00 + Kx + 1
    v11 = v01 + 1
    lower = np.stack([v00, v10, v11], axis=1)
    upper = np.stack([v00, v11, v01], axis=1)
    EToV = np.stack([lower, upper], axis=1).reshape(-1, 3).astype(np.int64)
    return VX, VY, EToV


@dataclass(eq=False)
class Mesh2D:
    """Operators and connectivity of a nodal-DG triangle mesh (the reference's
    ``Mesh2D`` fields, numpy arrays)."""
    N: int
    Np: int
    K: int
    Nfp: int
    Nfaces: int
    VX: np.ndarray
    VY: np.ndarray
    EToV: np.ndarray
    r: np.ndarray
    s: np.ndarray
    V: np.ndarray
    invV: np.ndarray
    Dr: np.ndarray
    Ds: np.ndarray
    LIFT: np.ndarray
    Fmask: np.ndarray
    x: np.ndarray
    y: np.ndarray
    rx: np.ndarray
    sx: np.ndarray
    ry: np.ndarray
    sy: np.ndarray
    J: np.ndarray
    nx: np.ndarray
    ny: np.ndarray
    sJ: np.ndarray
    Fscale: np.ndarray
    EToE: np.ndarray
    EToF: np.ndarray
    vmapM: np.ndarray
    vmapP: np.ndarray
    vmapB: np.ndarray
    mapB: np.ndarray
    _ops: dict = field(default_factory=dict, repr=False)

    @property
    def ref(self) -> RefElement:
        return ref_element(self.N)

    def element_geometry(self) -> np.ndarray:
        """(K, 14) per-element affine geometry: rx sx ry sy J, then nx ny sJ
        of faces 0, 1, 2 (first node of the element / of each face, the nodes
        ``sipg.py:261-263`` reads sJ and Fscale at)."""
        g = np.empty((self.K, 14))
        g[:, 0], g[:, 1] = self.rx[0], self.sx[0]
        g[:, 2], g[:, 3] = self.ry[0], self.sy[0]
        g[:, 4] = self.J[0]
        for f in range(3):
            row = f * self.Nfp
            g[:, 5 + 3 * f] = self.nx[row]
            g[:, 6 + 3 * f] = self.ny[row]
            g[:, 7 + 3 * f] = self.sJ[row]
        return g

    def device_operator(self, bc_types, tau_scale: float = 200.0, device: int | None = None):
        """The device-resident SIPG operator for these BC tags and penalty,
        cached per (tau_scale, device, BC tags); a few BC sets are kept."""
        from .operator import SipgOperator
        import torch
        dev = torch.cuda.current_device() if device is None else int(device)
        bc = np.ascontiguousarray(np.asarray(bc_types), dtype=np.int32)
        if bc.shape != (self.K, 3):
            raise ValueError(f"bc_types must have shape (K, 3) = ({self.K}, 3), got {bc.shape}")
        key = (float(tau_scale), dev, bc.tobytes())
        op = self._ops.pop(key, None)
        if op is None:
            op = SipgOperator(self, bc, tau_scale=tau_scale, device=dev)
            while len(self._ops) >= 4:
                # drop only the cache's reference: a preconditioner or caller
                # may still hold the operator; its handle is freed with the
                # last reference
                self._ops.pop(next(iter(self._ops)))
        self._ops[key] = op            # most recently used last
        return op


def _connect(EToV: np.ndarray):
    L = _lib.lib()
    K = EToV.shape[0]
    EToV = np.ascontiguousarray(EToV, dtype=np.int64)
    EToE = np.empty((K, 3), dtype=np.int64)
    EToF = np.empty((K, 3), dtype=np.int64)
    _lib.check(L.ddg_mesh_connect(K, _lib.ptr(EToV), _lib.ptr(EToE), _lib.ptr(EToF)), "ddg_mesh_connect")
    return EToE, EToF


def _maps(N, Fmask, x, y, EToE, EToF, EToV, VX, VY, node_tol=1e-10):
    L = _lib.lib()
    K = EToV.shape[0]
    Nfp = N + 1
    vmapM = np.empty(3 * Nfp * K, dtype=np.int64)
    vmapP = np.empty(3 * Nfp * K, dtype=np.int64)
    arrs = [np.ascontiguousarray(a) for a in (Fmask.astype(np.int64), x, y, EToE, EToF,
                                               EToV.astype(np.int64), VX, VY)]
    _lib.check(L.ddg_mesh_maps(K, N, *[_lib.ptr(a) for a in arrs], node_tol,
                               _lib.ptr(vmapM), _lib.ptr(vmapP)), "ddg_mesh_maps")
    return vmapM, vmapP


def build_mesh_2d(VX, VY, EToV, N: int) -> Mesh2D:
    """StartUp2D: ``src/ddg/dg2d/mesh.py:691-760``."""
    EToV = np.asarray(EToV, dtype=np.int64)
    VX = np.asarray(VX, dtype=np.float64)
    VY = np.asarray(VY, dtype=np.float64)
    K = EToV.shape[0]
    ref = ref_element(N)
    Np, Nfp = ref.Np, ref.Nfp
    r, s = ref.r, ref.s
    va, vb, vc = EToV[:, 0], EToV[:, 1], EToV[:, 2]
    x = 0.5 * (np.outer(-(r + s), VX[va]) + np.outer(1.0 + r, VX[vb]) + np.outer(1.0 + s, VX[vc]))
    y = 0.5 * (np.outer(-(r + s), VY[va]) + np.outer(1.0 + r, VY[vb]) + np.outer(1.0 + s, VY[vc]))
    xr, xs, yr, ys = ref.Dr @ x, ref.Ds @ x, ref.Dr @ y, ref.Ds @ y
    J = xr * ys - xs * yr
    rx, sx, ry, sy = ys / J, -yr / J, -xs / J, xr / J
    ff = ref.Fmask.flatten(order="F")
    fxr, fxs, fyr, fys = xr[ff], xs[ff], yr[ff], ys[ff]
    nx = np.empty((3 * Nfp, K))
    ny = np.empty((3 * Nfp, K))
    a, b, c = slice(0, Nfp), slice(Nfp, 2 * Nfp), slice(2 * Nfp, 3 * Nfp)
    nx[a], ny[a] = fyr[a], -fxr[a]
    nx[b], ny[b] = fys[b] - fyr[b], fxr[b] - fxs[b]
    nx[c], ny[c] = -fys[c], fxs[c]
    sJ = np.sqrt(nx * nx + ny * ny)
    nx, ny = nx / sJ, ny / sJ
    Fscale = sJ / J[ff, :]
    EToE, EToF = _connect(EToV)
    vmapM, vmapP = _maps(N, ref.Fmask, x, y, EToE, EToF, EToV, VX, VY)
    mapB = np.flatnonzero(vmapP == vmapM)
    return Mesh2D(N=N, Np=Np, K=K, Nfp=Nfp, Nfaces=3, VX=VX, VY=VY, EToV=EToV,
                  r=r, s=s, V=ref.V, invV=ref.invV, Dr=ref.Dr, Ds=ref.Ds, LIFT=ref.LIFT,
                  Fmask=ref.Fmask, x=x, y=y, rx=rx, sx=sx, ry=ry, sy=sy, J=J,
                  nx=nx, ny=ny, sJ=sJ, Fscale=Fscale, EToE=EToE, EToF=EToF,
                  vmapM=vmapM, vmapP=vmapP, vmapB=vmapM[mapB], mapB=mapB)
