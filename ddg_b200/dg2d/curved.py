"""Curved-boundary meshes with the call surface of ddg's ``src/ddg/dg2d/curved.py``.

``project_to_curve_2d`` moves the nodes of selected boundary faces onto a
curve and blends each face's displacement into its element (Gordon-Hall
style: the face weight is 1 on the face and 0 at the opposite vertex, the
displacement is carried into the element by the 1D interpolant of the face
nodes), then recomputes the geometric factors and normals from the moved
nodes (``curved.py:93-236``).  Host set-up, vectorised over the elements of
each face index; the resulting ``Mesh2D`` is not affine, so every SIPG call
on it runs the curved-element kernels (nodal quadrature, or the cubature
branch with ``cub=attach_cubature(mesh)``).
"""

from __future__ import annotations

import dataclasses
from typing import Callable

import numpy as np

from .mesh import Mesh2D, geometry_2d
from .reference import vandermonde_1d


def _blend_weight(r, s, f: int):
    """1 on face f, 0 at the opposite vertex, linear in between (``curved.py:64-86``)."""
    if f == 0:
        return (1.0 - s) / 2.0
    if f == 1:
        return (r + s + 2.0) / 2.0
    if f == 2:
        return (1.0 - r) / 2.0
    raise ValueError(f"face must be 0, 1, or 2, got {f}")


def project_to_curve_2d(mesh: Mesh2D, *, face_on_curve: Callable, project_fn: Callable,
                        blend_interior: bool = True) -> Mesh2D:
    """Bend the boundary faces selected by ``face_on_curve(x_face_avg,
    y_face_avg) -> bool (3, K)`` onto ``project_fn(x, y) -> (x', y')``.
    Connectivity is unchanged; node coordinates, geometric factors,
    normals, sJ and Fscale are recomputed."""
    K = mesh.K
    ref = mesh.ref
    Fm_all = ref.Fmask
    xf = np.stack([mesh.x[Fm_all[:, f], :].mean(axis=0) for f in range(3)])
    yf = np.stack([mesh.y[Fm_all[:, f], :].mean(axis=0) for f in range(3)])
    on_bdy = (np.asarray(mesh.EToE) == np.arange(K)[:, None]).T
    curved = np.asarray(face_on_curve(xf, yf)) & on_bdy
    x, y = np.array(mesh.x, dtype=np.float64), np.array(mesh.y, dtype=np.float64)
    r, s = ref.r, ref.s
    for f in range(3):
        ks = np.flatnonzero(curved[f])
        if ks.size == 0:
            continue
        Fm = Fm_all[:, f]
        x0, y0 = mesh.x[np.ix_(Fm, ks)], mesh.y[np.ix_(Fm, ks)]
        xp, yp = project_fn(x0, y0)
        xp, yp = np.asarray(xp, dtype=np.float64), np.asarray(yp, dtype=np.float64)
        x[np.ix_(Fm, ks)] = xp
        y[np.ix_(Fm, ks)] = yp
        if not blend_interior:
            continue
        t = s if f == 2 else r                                        # face parameter (curved.py:183-201)
        interp = np.linalg.solve(vandermonde_1d(mesh.N, t[Fm]).T, vandermonde_1d(mesh.N, t).T).T
        wgt = _blend_weight(r, s, f)[:, None]
        x[:, ks] += wgt * (interp @ (xp - x0))
        y[:, ks] += wgt * (interp @ (yp - y0))
        x[np.ix_(Fm, ks)] = xp                                        # the face nodes exactly on the curve
        y[np.ix_(Fm, ks)] = yp
    rx, sx, ry, sy, J, nx, ny, sJ, Fscale = geometry_2d(ref, x, y)
    return dataclasses.replace(mesh, x=x, y=y, rx=rx, sx=sx, ry=ry, sy=sy, J=J,
                               nx=nx, ny=ny, sJ=sJ, Fscale=Fscale)


def circle_projection(cx: float, cy: float, radius: float):
    """Orthogonal projection onto the circle of ``radius`` about (cx, cy)
    (``curved.py:243-252``)."""
    def project(x, y):
        dx, dy = x - cx, y - cy
        rr = np.sqrt(dx * dx + dy * dy)
        scale = radius / np.where(rr > 1e-14, rr, 1.0)
        return cx + dx * scale, cy + dy * scale
    return project


def apply_circular_hole_2d(mesh: Mesh2D, *, cx: float, cy: float, radius: float,
                           blend_interior: bool = True, detection_tol: float = 0.1) -> Mesh2D:
    """Bend the boundary faces whose centre lies within
    ``radius (1 + detection_tol)`` of (cx, cy) onto that circle
    (``curved.py:255-268``)."""
    def face_pred(xf, yf):
        return (xf - cx) ** 2 + (yf - cy) ** 2 < (radius * (1 + detection_tol)) ** 2
    return project_to_curve_2d(mesh, face_on_curve=face_pred, project_fn=circle_projection(cx, cy, radius),
                               blend_interior=blend_interior)
