"""Oracle: curved-boundary meshes (boundary-face projection with Gordon-Hall
blending) and the two hole-bounded mesh builders, float64 numpy.

Test infrastructure only (see ``oracle/__init__.py``).

Restates ``src/ddg/dg2d/curved.py`` (``_blending_weight_for_face`` :64-86,
``project_to_curve_2d`` :93-236, ``circle_projection`` :243-252,
``apply_circular_hole_2d`` :255-268) and ``src/ddg/dg2d/mesh.py``
(``rectangle_with_square_hole_mesh_2d`` :159-212,
``_square_perimeter_ccw_indices`` :280-304, ``channel_with_circle_mesh_2d``
:307-513) step for step.
"""

from __future__ import annotations

import dataclasses

import numpy as np

from .mesh import geometric_factors_2d, normals_2d
from .refelem import vandermonde_1d


def rectangle_with_square_hole_mesh_2d(xmin, xmax, ymin, ymax, Kx, Ky, hxmin, hxmax, hymin, hymax):
    """``mesh.py:159-212``: the uniform split without the cells whose centre
    lies in the hole box, unused vertices pruned and renumbered."""
    xs = np.linspace(xmin, xmax, Kx + 1)
    ys = np.linspace(ymin, ymax, Ky + 1)
    VXf, VYf = np.tile(xs, Ky + 1), np.repeat(ys, Kx + 1)
    tris = []
    for j in range(Ky):
        for i in range(Kx):
            cx, cy = 0.5 * (xs[i] + xs[i + 1]), 0.5 * (ys[j] + ys[j + 1])
            if hxmin <= cx <= hxmax and hymin <= cy <= hymax:
                continue
            v00 = j * (Kx + 1) + i
            v10, v01 = v00 + 1, v00 + Kx + 1
            v11 = v01 + 1
            tris += [(v00, v10, v11), (v00, v11, v01)]
    E = np.array(tris, dtype=np.int64)
    used = np.unique(E.reshape(-1))
    remap = -np.ones(VXf.shape[0], dtype=np.int64)
    remap[used] = np.arange(used.shape[0])
    return VXf[used], VYf[used], remap[E]


def _perimeter_ccw(Kx, i_lo, i_hi, j_lo, j_hi):
    """``mesh.py:280-304``."""
    vid = lambda i, j: j * (Kx + 1) + i  # noqa: E731
    ids = [vid(i, j_lo) for i in range(i_lo, i_hi)]
    ids += [vid(i_hi, j) for j in range(j_lo, j_hi)]
    ids += [vid(i, j_hi) for i in range(i_hi, i_lo, -1)]
    ids += [vid(i_lo, j) for j in range(j_hi, j_lo, -1)]
    return np.asarray(ids, dtype=np.int64)


def channel_with_circle_mesh_2d(xmin, xmax, ymin, ymax, Kx, Ky, *, cx, cy, radius, R_outer,
                                n_radial=4, radial_growth=1.0):
    """``mesh.py:307-513``: Cartesian channel minus a grid-aligned square,
    plus an O-grid of ``n_radial`` layers between the square's perimeter
    and the polygonal cylinder."""
    if not radius < R_outer:
        raise ValueError("radius must be < R_outer")
    hx, hy = (xmax - xmin) / Kx, (ymax - ymin) / Ky
    lo_hi = [(cx - R_outer - xmin) / hx, (cx + R_outer - xmin) / hx,
             (cy - R_outer - ymin) / hy, (cy + R_outer - ymin) / hy]
    if any(abs(v - round(v)) > 1e-9 for v in lo_hi):
        raise ValueError("bounding square not grid-aligned")
    i_lo, i_hi, j_lo, j_hi = (int(round(v)) for v in lo_hi)
    xs = np.linspace(xmin, xmax, Kx + 1)
    ys = np.linspace(ymin, ymax, Ky + 1)
    VXf, VYf = np.tile(xs, Ky + 1), np.repeat(ys, Kx + 1)
    tris = []
    for j in range(Ky):
        for i in range(Kx):
            if i_lo <= i < i_hi and j_lo <= j < j_hi:
                continue
            v00 = j * (Kx + 1) + i
            v10, v01 = v00 + 1, v00 + Kx + 1
            v11 = v01 + 1
            tris += [(v00, v10, v11), (v00, v11, v01)]
    outer = _perimeter_ccw(Kx, i_lo, i_hi, j_lo, j_hi)
    nc = outer.shape[0]
    if nc < 8:
        raise ValueError("bounding square has fewer than 8 perimeter vertices")
    OX, OY = VXf[outer], VYf[outer]
    th = np.arctan2(OY - cy, OX - cx)
    IX, IY = cx + radius * np.cos(th), cy + radius * np.sin(th)
    if abs(radial_growth - 1.0) < 1e-12:
        frac = np.linspace(0.0, 1.0, n_radial + 1)
    else:
        g = radial_growth
        w0 = 1.0 / ((g ** n_radial - 1.0) / (g - 1.0))
        frac = np.concatenate(([0.0], np.cumsum(w0 * g ** np.arange(n_radial))))
    ids_l, xl, yl = [], [], []
    nid = VXf.shape[0]
    for L in range(n_radial + 1):
        if L == n_radial:
            ids_l.append(outer)
            continue
        xl.append(IX + frac[L] * (OX - IX))
        yl.append(IY + frac[L] * (OY - IY))
        ids_l.append(np.arange(nid, nid + nc, dtype=np.int64))
        nid += nc
    for L in range(n_radial):
        for i in range(nc):
            ip = (i + 1) % nc
            A, B = int(ids_l[L][i]), int(ids_l[L][ip])
            C, D = int(ids_l[L + 1][ip]), int(ids_l[L + 1][i])
            tris += [(A, D, C), (A, C, B)]
    E = np.array(tris, dtype=np.int64)
    VX = np.concatenate([VXf] + xl)
    VY = np.concatenate([VYf] + yl)
    used = np.unique(E.reshape(-1))
    remap = -np.ones(VX.shape[0], dtype=np.int64)
    remap[used] = np.arange(used.shape[0])
    return VX[used], VY[used], remap[E]


def _blending_weight(r, s, f):
    """``curved.py:64-86``: 1 on face f, 0 at the opposite vertex."""
    return [(1.0 - s) / 2.0, (r + s + 2.0) / 2.0, (1.0 - r) / 2.0][f]


def project_to_curve_2d(mesh, *, face_on_curve, project_fn, blend_interior=True):
    """``curved.py:93-236``: project the selected boundary faces' nodes,
    blend the offsets into the element with the face weight and the 1D
    face-node interpolant, restore the face nodes, recompute the
    geometric factors, normals and Fscale."""
    K, Nfp = mesh.K, mesh.Nfp
    ref = mesh.ref
    Fm_all = ref.Fmask
    xf = np.stack([mesh.x[Fm_all[:, f], :].mean(axis=0) for f in range(3)])
    yf = np.stack([mesh.y[Fm_all[:, f], :].mean(axis=0) for f in range(3)])
    is_bdy = (mesh.EToE == np.arange(K)[:, None]).T
    curved = np.asarray(face_on_curve(xf, yf)) & is_bdy
    x, y = mesh.x.copy(), mesh.y.copy()
    r, s = ref.r, ref.s
    for f in range(3):
        ks = np.where(curved[f])[0]
        if ks.size == 0:
            continue
        Fm = Fm_all[:, f]
        xo, yo = mesh.x[Fm[:, None], ks[None, :]], mesh.y[Fm[:, None], ks[None, :]]
        xp, yp = project_fn(xo, yo)
        x[Fm[:, None], ks[None, :]] = xp
        y[Fm[:, None], ks[None, :]] = yp
        if not blend_interior:
            continue
        wgt = _blending_weight(r, s, f)
        t = s if f == 2 else r
        I = vandermonde_1d(mesh.N, t) @ np.linalg.inv(vandermonde_1d(mesh.N, t[Fm]))
        x[:, ks] = x[:, ks] + wgt[:, None] * (I @ (xp - xo))
        y[:, ks] = y[:, ks] + wgt[:, None] * (I @ (yp - yo))
        x[Fm[:, None], ks[None, :]] = xp
        y[Fm[:, None], ks[None, :]] = yp
    rx, sx, ry, sy, J = geometric_factors_2d(x, y, ref.Dr, ref.Ds)
    nx, ny, sJ = normals_2d(x, y, ref.Dr, ref.Ds, Fm_all, Nfp, K)
    Fscale = sJ / J[Fm_all.flatten(order="F"), :]
    return dataclasses.replace(mesh, x=x, y=y, rx=rx, sx=sx, ry=ry, sy=sy, J=J,
                               nx=nx, ny=ny, sJ=sJ, Fscale=Fscale)


def circle_projection(cx, cy, radius):
    """``curved.py:243-252``."""
    def project(x, y):
        dx, dy = x - cx, y - cy
        rr = np.sqrt(dx ** 2 + dy ** 2)
        sc = radius / np.where(rr > 1e-14, rr, 1.0)
        return cx + dx * sc, cy + dy * sc
    return project


def apply_circular_hole_2d(mesh, *, cx, cy, radius, blend_interior=True, detection_tol=0.1):
    """``curved.py:255-268``: faces whose centre lies within
    radius (1 + detection_tol) of the centre are bent onto the circle."""
    def pred(xf, yf):
        return (xf - cx) ** 2 + (yf - cy) ** 2 < (radius * (1 + detection_tol)) ** 2
    return project_to_curve_2d(mesh, face_on_curve=pred, project_fn=circle_projection(cx, cy, radius),
                               blend_interior=blend_interior)
