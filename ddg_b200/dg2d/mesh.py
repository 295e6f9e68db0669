"""2D triangle mesh (host setup) with the field names of ddg's ``Mesh2D``.

Mirrors ``src/ddg/dg2d/mesh.py``: ``uniform_rectangle_mesh_2d`` (:125-156),
the hole-bounded builders ``rectangle_with_square_hole_mesh_2d`` (:159-212)
and ``channel_with_circle_mesh_2d`` (:307-513), and ``build_mesh_2d``
(:691-760) produce the same arrays (volume fields
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


def _prune(VX, VY, EToV):
    """Drop unused vertices and renumber (``mesh.py:205-212``)."""
    used = np.unique(EToV.reshape(-1))
    remap = -np.ones(VX.shape[0], dtype=np.int64)
    remap[used] = np.arange(used.shape[0])
    return VX[used], VY[used], remap[EToV]


def _cell_triangles(Kx: int, keep: np.ndarray) -> np.ndarray:
    """The two triangles of every kept cell (j, i) of the structured split,
    in row-major cell order (``mesh.py:125-156``)."""
    j, i = np.nonzero(keep)
    v00 = j * (Kx + 1) + i
    v10, v01 = v00 + 1, v00 + Kx + 1
    v11 = v01 + 1
    lower = np.stack([v00, v10, v11], axis=1)
    upper = np.stack([v00, v11, v01], axis=1)
    return np.stack([lower, upper], axis=1).reshape(-1, 3).astype(np.int64)


def rectangle_with_square_hole_mesh_2d(xmin, xmax, ymin, ymax, Kx: int, Ky: int,
                                       hole_xmin, hole_xmax, hole_ymin, hole_ymax):
    """The uniform split without the cells whose centre lies in the hole box,
    unused vertices pruned (``src/ddg/dg2d/mesh.py:159-212``)."""
    xs = np.linspace(xmin, xmax, Kx + 1)
    ys = np.linspace(ymin, ymax, Ky + 1)
    cx = 0.5 * (xs[:-1] + xs[1:])
    cy = 0.5 * (ys[:-1] + ys[1:])
    inside = ((hole_xmin <= cx[None, :]) & (cx[None, :] <= hole_xmax)
              & (hole_ymin <= cy[:, None]) & (cy[:, None] <= hole_ymax))
    E = _cell_triangles(Kx, ~inside)
    return _prune(np.tile(xs, Ky + 1), np.repeat(ys, Kx + 1), E)


def channel_with_circle_mesh_2d(xmin, xmax, ymin, ymax, Kx: int, Ky: int, *, cx, cy, radius, R_outer,
                                n_radial: int = 4, radial_growth: float = 1.0):
    """Channel with a circular hole, body-fitted by an O-grid
    (``src/ddg/dg2d/mesh.py:307-513``): the Cartesian split minus the
    grid-aligned bounding square of half-side ``R_outer``, plus
    ``n_radial`` layers of wedges between the square's perimeter and the
    polygonal cylinder (inner vertices at the perimeter vertices' angles).
    Call ``curved.apply_circular_hole_2d`` to bend the inner faces."""
    if not radius < R_outer:
        raise ValueError(f"radius={radius} must be < R_outer={R_outer}")
    if not (cx - R_outer > xmin and cx + R_outer < xmax and cy - R_outer > ymin and cy + R_outer < ymax):
        raise ValueError("Bounding square must lie strictly inside the channel")
    hx, hy = (xmax - xmin) / Kx, (ymax - ymin) / Ky
    idx = {}
    for name, v in (("i_lo", (cx - R_outer - xmin) / hx), ("i_hi", (cx + R_outer - xmin) / hx),
                    ("j_lo", (cy - R_outer - ymin) / hy), ("j_hi", (cy + R_outer - ymin) / hy)):
        if abs(v - round(v)) > 1e-9:
            raise ValueError(f"Bounding square not grid-aligned: {name}={v} (must be integral)")
        idx[name] = int(round(v))
    i_lo, i_hi, j_lo, j_hi = idx["i_lo"], idx["i_hi"], idx["j_lo"], idx["j_hi"]
    xs = np.linspace(xmin, xmax, Kx + 1)
    ys = np.linspace(ymin, ymax, Ky + 1)
    VXf, VYf = np.tile(xs, Ky + 1), np.repeat(ys, Kx + 1)
    jj, ii = np.meshgrid(np.arange(Ky), np.arange(Kx), indexing="ij")
    E_outer = _cell_triangles(Kx, ~((i_lo <= ii) & (ii < i_hi) & (j_lo <= jj) & (jj < j_hi)))
    vid = lambda i, j: j * (Kx + 1) + i  # noqa: E731
    # perimeter of the square, counter-clockwise from its bottom-left corner (mesh.py:280-304)
    outer = np.concatenate([vid(np.arange(i_lo, i_hi), j_lo), vid(i_hi, np.arange(j_lo, j_hi)),
                            vid(np.arange(i_hi, i_lo, -1), j_hi), vid(i_lo, np.arange(j_hi, j_lo, -1))]
                           ).astype(np.int64)
    nc = outer.shape[0]
    if nc < 8:
        raise ValueError(f"Bounding square has only {nc} perimeter vertices; need at least 8")
    OX, OY = VXf[outer], VYf[outer]
    th = np.arctan2(OY - cy, OX - cx)
    IX, IY = cx + radius * np.cos(th), cy + radius * np.sin(th)
    if abs(radial_growth - 1.0) < 1e-12:
        frac = np.linspace(0.0, 1.0, n_radial + 1)
    else:
        g = radial_growth
        w0 = 1.0 / ((g ** n_radial - 1.0) / (g - 1.0))
        frac = np.concatenate(([0.0], np.cumsum(w0 * g ** np.arange(n_radial))))
    n0 = VXf.shape[0]
    layers = [n0 + L * nc + np.arange(nc, dtype=np.int64) for L in range(n_radial)] + [outer]
    LX = [IX + frac[L] * (OX - IX) for L in range(n_radial)]
    LY = [IY + frac[L] * (OY - IY) for L in range(n_radial)]
    i = np.arange(nc)
    ip = (i + 1) % nc
    wedge = []
    for L in range(n_radial):
        A, B = layers[L][i], layers[L][ip]
        C, D = layers[L + 1][ip], layers[L + 1][i]
        wedge.append(np.stack([np.stack([A, D, C], 1), np.stack([A, C, B], 1)], 1).reshape(-1, 3))
    E = np.concatenate([E_outer] + wedge)
    return _prune(np.concatenate([VXf] + LX), np.concatenate([VYf] + LY), E)


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
    # device operators built on this mesh (not copied by dataclasses.replace)
    _ops: dict = field(default_factory=dict, init=False, repr=False, compare=False)
    _affine: object = field(default=None, init=False, repr=False, compare=False)

    @property
    def ref(self) -> RefElement:
        return ref_element(self.N)

    @property
    def is_affine(self) -> bool:
        """True when the straight-sided (affine) kernels apply: every element
        is a straight-sided triangle -- the geometric factors are constant
        over each element (to 1e-10 of their magnitude) and so are the
        normals and sJ of each face -- and the two sides of every interior
        face see the same face (equal sJ, opposite normals).  Curved meshes
        (``curved.project_to_curve_2d``) are not: bent elements, and at
        degree 1 (where bending moves only vertices) the faces whose two
        sides no longer meet."""
        if self._affine is None:
            def const(a, rows):
                a = np.asarray(a)
                ref = a[rows]
                scale = max(float(np.max(np.abs(a))), 1e-300)
                return float(np.max(np.abs(a - ref))) <= 1e-10 * scale
            Nfp = self.Nfp
            first = np.repeat(np.arange(3) * Nfp, Nfp)
            ok = all(const(a, np.zeros(self.Np, dtype=np.int64)) for a in (self.rx, self.sx, self.ry, self.sy, self.J))
            ok = ok and all(const(a, first) for a in (self.nx, self.ny, self.sJ, self.Fscale))
            if ok:
                f0 = np.arange(3) * Nfp
                nx1, ny1, sJ1 = (np.asarray(a)[f0] for a in (self.nx, self.ny, self.sJ))   # (3, K)
                kp, fp = np.asarray(self.EToE).T, np.asarray(self.EToF).T
                inner = kp != np.arange(self.K)[None, :]
                scale = max(float(np.max(sJ1)), 1e-300)
                ok = (float(np.max(np.abs(nx1 + nx1[fp, kp])[inner], initial=0.0)) <= 1e-10
                      and float(np.max(np.abs(ny1 + ny1[fp, kp])[inner], initial=0.0)) <= 1e-10
                      and float(np.max(np.abs(sJ1 - sJ1[fp, kp])[inner], initial=0.0)) <= 1e-10 * scale)
            object.__setattr__(self, "_affine", bool(ok))
        return self._affine

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
        cached per (tau_scale, device, BC tags); a few BC sets are kept.
        A curved mesh gets the curved-element operator with the nodal
        quadrature (the reference's ``cub=None`` on such a mesh)."""
        if not self.is_affine:
            return self.curved_operator(bc_types, tau_scale, None, device)
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

    def curved_operator(self, bc_types, tau_scale: float = 200.0, cub=None, device: int | None = None):
        """The curved-element operator (per-node geometric factors; nodal
        quadrature, plus the cubature rule of ``cub`` when given), cached per
        (tau_scale, device, BC tags, cub) like :meth:`device_operator`."""
        from .curved_operator import CurvedOperator
        import torch
        dev = torch.cuda.current_device() if device is None else int(device)
        bc = np.ascontiguousarray(np.asarray(bc_types), dtype=np.int32)
        if bc.shape != (self.K, 3):
            raise ValueError(f"bc_types must have shape (K, 3) = ({self.K}, 3), got {bc.shape}")
        if cub is not None:
            from .cubature import MeshCubature
            if not isinstance(cub, MeshCubature):
                raise ValueError("cub must be the MeshCubature of attach_cubature(mesh)")
            if cub.mesh is not self:
                raise ValueError("cub was attached to a different mesh")
        key = ("curved", float(tau_scale), dev, bc.tobytes(), id(cub) if cub is not None else None)
        op = self._ops.pop(key, None)
        if op is None or op.cub is not cub:
            op = CurvedOperator(self, bc, tau_scale=tau_scale, cub=cub, device=dev)
            while len(self._ops) >= 4:
                self._ops.pop(next(iter(self._ops)))
        self._ops[key] = op
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


def geometry_2d(ref: RefElement, x, y):
    """Geometric factors at the nodes and face normals of elements with node
    coordinates (x, y) (``src/ddg/dg2d/mesh.py:634-684``): returns
    rx, sx, ry, sy, J (Np, K) and nx, ny, sJ, Fscale (3 Nfp, K)."""
    Nfp, K = ref.Nfp, x.shape[1]
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
    return rx, sx, ry, sy, J, nx, ny, sJ, Fscale


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
    rx, sx, ry, sy, J, nx, ny, sJ, Fscale = geometry_2d(ref, x, y)
    EToE, EToF = _connect(EToV)
    vmapM, vmapP = _maps(N, ref.Fmask, x, y, EToE, EToF, EToV, VX, VY)
    mapB = np.flatnonzero(vmapP == vmapM)
    return Mesh2D(N=N, Np=Np, K=K, Nfp=Nfp, Nfaces=3, VX=VX, VY=VY, EToV=EToV,
                  r=r, s=s, V=ref.V, invV=ref.invV, Dr=ref.Dr, Ds=ref.Ds, LIFT=ref.LIFT,
                  Fmask=ref.Fmask, x=x, y=y, rx=rx, sx=sx, ry=ry, sy=sy, J=J,
                  nx=nx, ny=ny, sJ=sJ, Fscale=Fscale, EToE=EToE, EToF=EToF,
                  vmapM=vmapM, vmapP=vmapP, vmapB=vmapM[mapB], mapB=mapB)
