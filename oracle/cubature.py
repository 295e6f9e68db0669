"""Oracle: high-order cubature on the reference triangle and the per-mesh
cubature data of curved elements, float64 numpy.

Test infrastructure only (see ``oracle/__init__.py``).

Restates ``src/ddg/dg2d/cubature.py``: ``triangle_cubature`` (:48-66, the
Stroud conical product of Gauss-Legendre in a and Gauss-Jacobi(1, 0) in b),
``MeshCubature`` (:73-107), ``attach_cubature`` (:110-223: Lagrange basis and
reference derivatives at the volume points, geometric factors there, 1D face
rule with per-face traversal, face-nodal -> face-cubature interpolation and
the surface Jacobian / normals at the face points), ``per_element_mass``
(:230-240) and ``cubature_mass_apply`` (:243-254).  The 1D rules come from
numpy's ``leggauss`` and scipy's ``roots_jacobi``, the library calls the
reference makes.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
from numpy.polynomial.legendre import leggauss
from scipy.special import roots_jacobi

from .refelem import grad_vandermonde_2d, vandermonde_1d, vandermonde_2d


def triangle_cubature(degree: int):
    """``cubature.py:48-66``: n = ceil((degree+1)/2) points per direction,
    r = (1+a)(1-b)/2 - 1, s = b, weights a_w b_w / 2 (sum 2)."""
    n = max(1, (degree + 2) // 2)
    a, aw = leggauss(n)
    b, bw = roots_jacobi(n, 1, 0)
    A, B = np.meshgrid(a, b, indexing="ij")
    r = (1.0 + A) * (1.0 - B) / 2.0 - 1.0
    return r.reshape(-1), B.reshape(-1), (np.outer(aw, bw) / 2.0).reshape(-1)


@dataclass(frozen=True)
class MeshCubature:
    """Field-for-field ``cubature.py:73-107``."""
    r: np.ndarray
    s: np.ndarray
    w: np.ndarray
    Lq: np.ndarray
    Drq: np.ndarray
    Dsq: np.ndarray
    J: np.ndarray
    rx: np.ndarray
    sx: np.ndarray
    ry: np.ndarray
    sy: np.ndarray
    face_w: np.ndarray
    face_Lq: np.ndarray
    face_L1d: np.ndarray
    face_sJ: np.ndarray
    face_nx: np.ndarray
    face_ny: np.ndarray


def attach_cubature(mesh, degree=None, face_degree=None) -> MeshCubature:
    """``cubature.py:110-223``: volume rule of degree max(degree, 2N)
    (default 4N - 2), face rule of (face_degree + 2) // 2 Gauss points
    (default face_degree 2N + 1)."""
    N = int(mesh.N)
    ref = mesh.ref
    if degree is None:
        degree = 4 * N - 2
    if face_degree is None:
        face_degree = 2 * N + 1
    rq, sq, wq = triangle_cubature(max(degree, 2 * N))
    Lq = vandermonde_2d(N, rq, sq) @ ref.invV
    Vr, Vs = grad_vandermonde_2d(N, rq, sq)
    Drq, Dsq = Vr @ ref.invV, Vs @ ref.invV
    xr, xs, yr, ys = Drq @ mesh.x, Dsq @ mesh.x, Drq @ mesh.y, Dsq @ mesh.y
    J = xr * ys - xs * yr
    t, fw = leggauss(max(1, (face_degree + 2) // 2))
    one = np.ones_like(t)
    face_rs = [(t, -one), (-t, t), (-one, -t)]                     # cubature.py:173-177
    drsdt = [(1.0, 0.0), (-1.0, 1.0), (0.0, -1.0)]
    Fm = ref.Fmask
    t_nodes = [ref.r[Fm[:, 0]], -ref.r[Fm[:, 1]], -ref.s[Fm[:, 2]]]  # cubature.py:184-188
    fLq, fL1, fsJ, fnx, fny = [], [], [], [], []
    for f in range(3):
        rf, sf = face_rs[f]
        fLq.append(vandermonde_2d(N, rf, sf) @ ref.invV)
        fL1.append(vandermonde_1d(N, t) @ np.linalg.inv(vandermonde_1d(N, t_nodes[f])))
        Vrf, Vsf = grad_vandermonde_2d(N, rf, sf)
        Drf, Dsf = Vrf @ ref.invV, Vsf @ ref.invV
        dr, ds = drsdt[f]
        xt = dr * (Drf @ mesh.x) + ds * (Dsf @ mesh.x)
        yt = dr * (Drf @ mesh.y) + ds * (Dsf @ mesh.y)
        sJ = np.sqrt(xt ** 2 + yt ** 2)
        fsJ.append(sJ)
        fnx.append(yt / sJ)
        fny.append(-xt / sJ)
    return MeshCubature(r=rq, s=sq, w=wq, Lq=Lq, Drq=Drq, Dsq=Dsq, J=J,
                        rx=ys / J, sx=-yr / J, ry=-xs / J, sy=xr / J,
                        face_w=fw, face_Lq=np.stack(fLq), face_L1d=np.stack(fL1),
                        face_sJ=np.stack(fsJ), face_nx=np.stack(fnx), face_ny=np.stack(fny))


def per_element_mass(cub: MeshCubature) -> np.ndarray:
    """``cubature.py:230-240``: (K, Np, Np)."""
    return np.einsum("q,qk,qi,qj->kij", cub.w, cub.J, cub.Lq, cub.Lq)


def cubature_mass_apply(cub: MeshCubature, f: np.ndarray) -> np.ndarray:
    """``cubature.py:243-254``: Lq^T (w J (Lq f)); f is (Np, K) or (Np, K, B)."""
    if f.ndim == 3:
        fq = np.einsum("qi,ikb->qkb", cub.Lq, f)
        return np.einsum("qi,qkb->ikb", cub.Lq, (cub.w[:, None] * cub.J)[:, :, None] * fq)
    return cub.Lq.T @ (cub.w[:, None] * cub.J * (cub.Lq @ f))
