"""High-order cubature for curved elements, with the call surface of ddg's
``src/ddg/dg2d/cubature.py``.

``triangle_cubature`` is the Stroud conical product rule of the reference
(``cubature.py:48-66``): Gauss-Legendre in ``a``, Gauss-Jacobi with weight
``(1 - b)`` in ``b``, mapped by ``r = (1+a)(1-b)/2 - 1, s = b``.  Both 1D
rules are computed here by Newton iteration on the orthonormal Jacobi
polynomials (roots) and the Christoffel numbers ``1 / sum_k p_k(x_i)^2``
(weights), instead of the library routines the reference calls; the two
agree to rounding.

``attach_cubature`` builds the per-mesh data of ``MeshCubature``
(``cubature.py:73-223``) on the host, once per mesh.  ``cubature_mass_apply``
and ``per_element_mass`` run on the GPU (the curved operator's mass kernel,
``libddg_sipg.so``).
"""

from __future__ import annotations

import weakref
from dataclasses import dataclass, field

import numpy as np

from .reference import djacobi, grad_vandermonde_2d, jacobi, vandermonde_1d, vandermonde_2d


def gauss_jacobi(n: int, a: float, b: float):
    """n-point Gauss-Jacobi rule for the weight (1 - x)^a (1 + x)^b on
    [-1, 1]: nodes ascending, weights summing to the weight's integral."""
    if n < 1:
        raise ValueError("n must be >= 1")
    x = -np.cos(np.pi * (np.arange(n) + 0.75 - 0.25 * (b - a) / max(n, 1)) / (n + 0.5))
    x = np.sort(x)
    for _ in range(100):
        f = jacobi(x, a, b, n)
        df = djacobi(x, a, b, n)
        # Newton with deflation by the other current roots (Ehrlich-Aberth)
        diff = x[:, None] - x[None, :]
        np.fill_diagonal(diff, np.inf)
        corr = f / (df - f * np.sum(1.0 / diff, axis=1))
        x = x - corr
        if np.max(np.abs(corr)) < 1e-15:
            break
    x = np.sort(x)
    P = np.stack([jacobi(x, a, b, k) for k in range(n)])
    w = 1.0 / np.sum(P * P, axis=0)
    return x, w


def triangle_cubature(degree: int):
    """Rule exact for total degree ``<= degree`` on the reference triangle
    (-1,-1), (1,-1), (-1,1): ``n = ceil((degree+1)/2)`` points per direction,
    ``n^2`` in all, weights summing to 2 (``cubature.py:48-66``)."""
    n = max(1, (degree + 2) // 2)
    a, aw = gauss_jacobi(n, 0.0, 0.0)
    b, bw = gauss_jacobi(n, 1.0, 0.0)
    A, B = np.meshgrid(a, b, indexing="ij")
    r = (1.0 + A) * (1.0 - B) / 2.0 - 1.0
    return r.reshape(-1), B.reshape(-1), (np.outer(aw, bw) / 2.0).reshape(-1)


@dataclass(frozen=True, eq=False)
class MeshCubature:
    """Per-mesh cubature data (the fields of ``cubature.py:73-107``): the
    reference points and weights, Lagrange basis / derivatives there, the
    geometric factors of every element at the points, and the 1D face rule
    with the surface Jacobian and normals at the face points.  numpy float64."""
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
    _mesh: object = field(default=None, repr=False, compare=False)

    @property
    def mesh(self):
        m = self._mesh() if self._mesh is not None else None
        if m is None:
            raise ValueError("the mesh this cubature was attached to no longer exists")
        return m


# face traversal of the reference triangle (cubature.py:168-188): face f runs
# from vertex f to vertex f+1; (dr/dt, ds/dt) of the parameter t
_FACE_DRS = ((1.0, 0.0), (-1.0, 1.0), (0.0, -1.0))


def attach_cubature(mesh, degree: int | None = None, face_degree: int | None = None) -> MeshCubature:
    """Cubature data of ``mesh`` (``cubature.py:110-223``): a volume rule of
    degree ``max(degree, 2N)`` (default ``4N - 2``, the mass integrand on a
    curved element) and ``(face_degree + 2) // 2`` Gauss points per face
    (default ``face_degree = 2N + 1``)."""
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
    xr, xs = Drq @ mesh.x, Dsq @ mesh.x
    yr, ys = Drq @ mesh.y, Dsq @ mesh.y
    J = xr * ys - xs * yr
    t, fw = gauss_jacobi(max(1, (face_degree + 2) // 2), 0.0, 0.0)
    one = np.ones_like(t)
    face_rs = ((t, -one), (-t, t), (-one, -t))
    Fm = ref.Fmask
    t_nodes = (ref.r[Fm[:, 0]], -ref.r[Fm[:, 1]], -ref.s[Fm[:, 2]])
    V1q = vandermonde_1d(N, t)
    fLq, fL1, fsJ, fnx, fny = [], [], [], [], []
    for f in range(3):
        rf, sf = face_rs[f]
        fLq.append(vandermonde_2d(N, rf, sf) @ ref.invV)
        fL1.append(np.linalg.solve(vandermonde_1d(N, t_nodes[f]).T, V1q.T).T)
        Vrf, Vsf = grad_vandermonde_2d(N, rf, sf)
        Drf, Dsf = Vrf @ ref.invV, Vsf @ ref.invV
        dr, ds = _FACE_DRS[f]
        xt = dr * (Drf @ mesh.x) + ds * (Dsf @ mesh.x)
        yt = dr * (Drf @ mesh.y) + ds * (Dsf @ mesh.y)
        sJ = np.sqrt(xt * xt + yt * yt)
        fsJ.append(sJ)
        fnx.append(yt / sJ)
        fny.append(-xt / sJ)
    return MeshCubature(r=rq, s=sq, w=wq, Lq=Lq, Drq=Drq, Dsq=Dsq, J=J,
                        rx=ys / J, sx=-yr / J, ry=-xs / J, sy=xr / J,
                        face_w=fw, face_Lq=np.stack(fLq), face_L1d=np.stack(fL1),
                        face_sJ=np.stack(fsJ), face_nx=np.stack(fnx), face_ny=np.stack(fny),
                        _mesh=weakref.ref(mesh))


def _mass_op(cub: MeshCubature):
    mesh = cub.mesh
    return mesh.curved_operator(np.zeros((mesh.K, 3), dtype=np.int32), 200.0, cub)


def cubature_mass_apply(cub: MeshCubature, f):
    """``(M_K f)`` on every element by the cubature rule, ``Lq^T (w J (Lq f))``
    (``cubature.py:243-254``); ``f`` is an ``(Np, K)`` field (numpy or torch
    CUDA); the result is the same kind."""
    from .sipg import _flat, _unflat
    op = _mass_op(cub)
    y = op.mass(_flat(f, op._dev()), quad="cubature")
    return _unflat(y, cub.mesh, f)


def per_element_mass(cub: MeshCubature):
    """``M_K[k, i, j] = sum_q w_q J_q L_i L_j`` (``cubature.py:230-240``) as
    a (K, Np, Np) torch CUDA tensor: the mass kernel applied to each unit
    nodal vector (the element masses are block-diagonal)."""
    import torch
    op = _mass_op(cub)
    mesh = cub.mesh
    Np, K = mesh.Np, mesh.K
    out = torch.empty((K, Np, Np), dtype=torch.float64, device=op._dev())
    e = torch.zeros((K, Np), dtype=torch.float64, device=op._dev())
    for j in range(Np):
        e.zero_()
        e[:, j] = 1.0
        out[:, :, j] = op.mass(e.reshape(-1), quad="cubature").reshape(K, Np)
    return out
