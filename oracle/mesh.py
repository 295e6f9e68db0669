"""Oracle: 2D triangle mesh, geometric factors and connectivity maps.

Test infrastructure only (see ``oracle/__init__.py``).

Restates ``src/ddg/dg2d/mesh.py``: ``uniform_rectangle_mesh_2d`` (:125-156),
``_ti_connect_2d`` (:520-571), ``_build_maps_2d`` (:574-627),
``_geometric_factors_2d`` (:634-644), ``_normals_2d`` (:647-684) and
``build_mesh_2d`` (:691-760).  Layout is the reference's: volume fields
(Np, K), face fields (3 Nfp, K), ``vmapM``/``vmapP`` index the column-major
flat (element-major) vector ``u.T.reshape(-1)``.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .refelem import RefElement


def uniform_rectangle_mesh_2d(xmin, xmax, ymin, ymax, Kx, Ky):
    """``src/ddg/dg2d/mesh.py:125-156``: two triangles per cell,
    (v00, v10, v11) then (v00, v11, v01), vid = j (Kx+1) + i."""
    xs = np.linspace(xmin, xmax, Kx + 1)
    ys = np.linspace(ymin, ymax, Ky + 1)
    VX = np.tile(xs, Ky + 1)
    VY = np.repeat(ys, Kx + 1)
    tris = []
    for j in range(Ky):
        for i in range(Kx):
            v00 = j * (Kx + 1) + i
            v10 = v00 + 1
            v01 = v00 + (Kx + 1)
            v11 = v01 + 1
            tris.append((v00, v10, v11))
            tris.append((v00, v11, v01))
    return VX, VY, np.array(tris, dtype=np.int64)


def ti_connect_2d(EToV):
    """``src/ddg/dg2d/mesh.py:520-571``: face keys v_min*n_nodes+v_max,
    stable argsort, adjacent equal keys pair up; boundary faces self-point."""
    K = EToV.shape[0]
    nn = int(EToV.max()) + 1
    fn = np.vstack([EToV[:, [0, 1]], EToV[:, [1, 2]], EToV[:, [2, 0]]])
    fn = np.sort(fn, axis=1)
    EToE = np.tile(np.arange(K).reshape(-1, 1), (1, 3))
    EToF = np.tile(np.arange(3).reshape(1, -1), (K, 1))
    fid = fn[:, 0] * nn + fn[:, 1]
    elem = np.tile(np.arange(K), 3)
    face = np.repeat(np.arange(3), K)
    order = np.argsort(fid, kind="stable")
    fs, es, ffs = fid[order], elem[order], face[order]
    for i in np.where(fs[:-1] == fs[1:])[0]:
        k1, f1, k2, f2 = es[i], ffs[i], es[i + 1], ffs[i + 1]
        EToE[k1, f1] = k2
        EToF[k1, f1] = f2
        EToE[k2, f2] = k1
        EToF[k2, f2] = f1
    return EToE, EToF


def build_maps_2d(Np, Nfp, K, Fmask, x, y, EToE, EToF, EToV, VX, VY, node_tol=1e-10):
    """``src/ddg/dg2d/mesh.py:574-627``: per-face nearest-node matching
    within ``node_tol * edge_length``; unmatched nodes fall back to vmapM."""
    node_ids = np.arange(K * Np).reshape(K, Np).T
    vmapM = np.zeros((Nfp, 3, K), dtype=np.int64)
    vmapP = np.zeros((Nfp, 3, K), dtype=np.int64)
    for k in range(K):
        for f in range(3):
            vmapM[:, f, k] = node_ids[Fmask[:, f], k]
    xf = x.flatten(order="F")
    yf = y.flatten(order="F")
    for k1 in range(K):
        for f1 in range(3):
            k2, f2 = EToE[k1, f1], EToF[k1, f1]
            v1, v2 = EToV[k1, f1], EToV[k1, (f1 + 1) % 3]
            ref_d = np.sqrt((VX[v1] - VX[v2]) ** 2 + (VY[v1] - VY[v2]) ** 2)
            idM = vmapM[:, f1, k1]
            idP = vmapM[:, f2, k2]
            D2 = (xf[idM][:, None] - xf[idP][None, :]) ** 2 + \
                 (yf[idM][:, None] - yf[idP][None, :]) ** 2
            ok = np.sqrt(D2) < node_tol * ref_d
            for fp in range(Nfp):
                hit = np.where(ok[fp])[0]
                vmapP[fp, f1, k1] = idP[hit[0]] if hit.size > 0 else idM[fp]
    vmapM = vmapM.flatten(order="F")
    vmapP = vmapP.flatten(order="F")
    mapB = np.where(vmapP == vmapM)[0]
    return vmapM, vmapP, vmapM[mapB], mapB


def geometric_factors_2d(x, y, Dr, Ds):
    """``src/ddg/dg2d/mesh.py:634-644``."""
    xr, xs, yr, ys = Dr @ x, Ds @ x, Dr @ y, Ds @ y
    J = xr * ys - xs * yr
    return ys / J, -yr / J, -xs / J, xr / J, J


def normals_2d(x, y, Dr, Ds, Fmask, Nfp, K):
    """``src/ddg/dg2d/mesh.py:647-684``."""
    xr, xs, yr, ys = Dr @ x, Ds @ x, Dr @ y, Ds @ y
    ff = Fmask.flatten(order="F")
    fxr, fxs, fyr, fys = xr[ff], xs[ff], yr[ff], ys[ff]
    nx = np.zeros((3 * Nfp, K))
    ny = np.zeros((3 * Nfp, K))
    a, b, c = slice(0, Nfp), slice(Nfp, 2 * Nfp), slice(2 * Nfp, 3 * Nfp)
    nx[a], ny[a] = fyr[a], -fxr[a]
    nx[b], ny[b] = fys[b] - fyr[b], -fxs[b] + fxr[b]
    nx[c], ny[c] = -fys[c], fxs[c]
    sJ = np.sqrt(nx ** 2 + ny ** 2)
    return nx / sJ, ny / sJ, sJ


@dataclass
class Mesh2D:
    """Field-for-field restatement of ``src/ddg/dg2d/mesh.py:50-101``."""
    N: int
    Np: int
    K: int
    Nfp: int
    Nfaces: int
    VX: np.ndarray
    VY: np.ndarray
    EToV: np.ndarray
    ref: RefElement
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

    # reference-element shortcuts (same names as the reference's Mesh2D)
    @property
    def r(self): return self.ref.r
    @property
    def s(self): return self.ref.s
    @property
    def V(self): return self.ref.V
    @property
    def invV(self): return self.ref.invV
    @property
    def Dr(self): return self.ref.Dr
    @property
    def Ds(self): return self.ref.Ds
    @property
    def LIFT(self): return self.ref.LIFT
    @property
    def Fmask(self): return self.ref.Fmask


_REF_CACHE: dict[int, RefElement] = {}


def ref_element(N: int) -> RefElement:
    if N not in _REF_CACHE:
        _REF_CACHE[N] = RefElement(N)
    return _REF_CACHE[N]


def build_mesh_2d(VX, VY, EToV, N: int) -> Mesh2D:
    """``src/ddg/dg2d/mesh.py:691-760`` (StartUp2D)."""
    EToV = np.asarray(EToV, dtype=np.int64)
    VX = np.asarray(VX, dtype=np.float64)
    VY = np.asarray(VY, dtype=np.float64)
    K = EToV.shape[0]
    ref = ref_element(N)
    Np, Nfp = ref.Np, ref.Nfp
    va, vb, vc = EToV[:, 0], EToV[:, 1], EToV[:, 2]
    r, s = ref.r, ref.s
    x = 0.5 * (np.outer(-(r + s), VX[va]) + np.outer(1.0 + r, VX[vb]) + np.outer(1.0 + s, VX[vc]))
    y = 0.5 * (np.outer(-(r + s), VY[va]) + np.outer(1.0 + r, VY[vb]) + np.outer(1.0 + s, VY[vc]))
    rx, sx, ry, sy, J = geometric_factors_2d(x, y, ref.Dr, ref.Ds)
    nx, ny, sJ = normals_2d(x, y, ref.Dr, ref.Ds, ref.Fmask, Nfp, K)
    Fscale = sJ / J[ref.Fmask.flatten(order="F"), :]
    EToE, EToF = ti_connect_2d(EToV)
    vmapM, vmapP, vmapB, mapB = build_maps_2d(Np, Nfp, K, ref.Fmask, x, y, EToE, EToF, EToV, VX, VY)
    return Mesh2D(N=N, Np=Np, K=K, Nfp=Nfp, Nfaces=3, VX=VX, VY=VY, EToV=EToV, ref=ref,
                  x=x, y=y, rx=rx, sx=sx, ry=ry, sy=sy, J=J, nx=nx, ny=ny, sJ=sJ,
                  Fscale=Fscale, EToE=EToE, EToF=EToF, vmapM=vmapM, vmapP=vmapP,
                  vmapB=vmapB, mapB=mapB)
