"""Oracle: reference-element operators (1D and 2D triangle), float64 numpy.

Test infrastructure only (see ``oracle/__init__.py``).

Restates, function by function:
  * ``src/ddg/dg1d/reference.py:20-142`` (Jacobi polynomials, Gauss and
    Gauss-Lobatto nodes, 1D Vandermonde);
  * ``src/ddg/dg2d/reference.py:27-255`` (warp-and-blend nodes, the
    Koornwinder basis and its gradient, Vandermonde, Dr/Ds, Fmask, LIFT).
"""

from __future__ import annotations

import math

import numpy as np


# ---------------------------------------------------------------- 1D ------

def jacobi_p(x, alpha: float, beta: float, N: int) -> np.ndarray:
    """Orthonormal Jacobi polynomial P_N^(alpha,beta)(x).

    Follows ``src/ddg/dg1d/reference.py:20-68`` (normalised three-term
    recurrence, gamma0/gamma1 start values)."""
    x = np.asarray(x, dtype=np.float64).reshape(-1)
    g0 = (2.0 ** (alpha + beta + 1) / (alpha + beta + 1)
          * math.gamma(alpha + 1) * math.gamma(beta + 1)
          / math.gamma(alpha + beta + 1))
    p0 = np.full_like(x, 1.0 / math.sqrt(g0))
    if N == 0:
        return p0
    g1 = (alpha + 1) * (beta + 1) / (alpha + beta + 3) * g0
    p1 = ((alpha + beta + 2) * x / 2 + (alpha - beta) / 2) / math.sqrt(g1)
    if N == 1:
        return p1
    aold = 2.0 / (2 + alpha + beta) * math.sqrt(
        (alpha + 1) * (beta + 1) / (alpha + beta + 3))
    for i in range(1, N):
        h1 = 2 * i + alpha + beta
        anew = 2.0 / (h1 + 2) * math.sqrt(
            (i + 1) * (i + 1 + alpha + beta) * (i + 1 + alpha)
            * (i + 1 + beta) / (h1 + 1) / (h1 + 3))
        bnew = -(alpha ** 2 - beta ** 2) / h1 / (h1 + 2)
        p2 = (1.0 / anew) * (-aold * p0 + (x - bnew) * p1)
        p0, p1 = p1, p2
        aold = anew
    return p1


def grad_jacobi_p(r, alpha: float, beta: float, N: int) -> np.ndarray:
    """``src/ddg/dg1d/reference.py:71-76``."""
    r = np.asarray(r, dtype=np.float64).reshape(-1)
    if N == 0:
        return np.zeros_like(r)
    return math.sqrt(N * (N + alpha + beta + 1)) * jacobi_p(r, alpha + 1, beta + 1, N - 1)


def jacobi_gauss_quadrature(alpha: float, beta: float, N: int):
    """Golub-Welsch Gauss-Jacobi rule, ``src/ddg/dg1d/reference.py:79-122``."""
    if N == 0:
        return (np.array([-(alpha - beta) / (alpha + beta + 2.0)]), np.array([2.0]))
    n = np.arange(N + 1, dtype=np.float64)
    h1 = 2.0 * n + alpha + beta
    with np.errstate(divide="ignore", invalid="ignore"):
        diag = -0.5 * (alpha ** 2 - beta ** 2) / (h1 + 2.0) / h1
    if abs(alpha + beta) < 10 * np.finfo(np.float64).eps:
        diag[0] = 0.0
    i = np.arange(1, N + 1, dtype=np.float64)
    h = h1[:N]
    off = 2.0 / (h + 2.0) * np.sqrt(
        i * (i + alpha + beta) * (i + alpha) * (i + beta) / (h + 1.0) / (h + 3.0))
    Jm = np.diag(diag) + np.diag(off, 1)
    Jm = Jm + Jm.T
    lam, vec = np.linalg.eigh(Jm)
    w = (vec[0, :] ** 2 * (2.0 ** (alpha + beta + 1) / (alpha + beta + 1))
         * math.gamma(alpha + 1) * math.gamma(beta + 1) / math.gamma(alpha + beta + 1))
    return lam, w


def jacobi_gauss_lobatto_nodes(alpha: float, beta: float, N: int) -> np.ndarray:
    """``src/ddg/dg1d/reference.py:125-135``."""
    if N == 1:
        return np.array([-1.0, 1.0])
    xi, _ = jacobi_gauss_quadrature(alpha + 1, beta + 1, N - 2)
    return np.concatenate([[-1.0], xi, [1.0]])


def vandermonde_1d(N: int, r) -> np.ndarray:
    """``src/ddg/dg1d/reference.py:138-142``."""
    r = np.asarray(r, dtype=np.float64).reshape(-1)
    return np.stack([jacobi_p(r, 0.0, 0.0, j) for j in range(N + 1)], axis=1)


# ---------------------------------------------------------------- 2D ------

ALPHA_OPT = np.array([0.0000, 0.0000, 1.4152, 0.1001, 0.2751, 0.9800, 1.0999,
                      1.2832, 1.3648, 1.4773, 1.4959, 1.5743, 1.5770, 1.6223,
                      1.6258])
"""Warp-and-blend blending constants, ``src/ddg/dg2d/reference.py:27-30``."""


def _alpha_for(N: int) -> float:
    return float(ALPHA_OPT[N - 1]) if 1 <= N <= 15 else 5.0 / 3.0


def warpfactor(N: int, rout) -> np.ndarray:
    """``src/ddg/dg2d/reference.py:39-59``."""
    rout = np.asarray(rout, dtype=np.float64)
    LGLr = jacobi_gauss_lobatto_nodes(0.0, 0.0, N)
    req = np.linspace(-1.0, 1.0, N + 1)
    Veq = vandermonde_1d(N, req)
    Pmat = np.stack([jacobi_p(rout, 0.0, 0.0, i) for i in range(N + 1)], axis=0)
    Lmat = np.linalg.solve(Veq.T, Pmat)
    warp = Lmat.T @ (LGLr - req)
    zerof = np.abs(rout) < 1.0 - 1e-10
    sf = 1.0 - np.where(zerof, rout, 0.0) ** 2
    return warp / sf + warp * (zerof.astype(np.float64) - 1.0)


def equilateral_nodes_2d(N: int):
    """``src/ddg/dg2d/reference.py:62-101``."""
    Np = (N + 1) * (N + 2) // 2
    a = _alpha_for(N)
    L1 = np.zeros(Np)
    L3 = np.zeros(Np)
    sk = 0
    for n in range(1, N + 2):
        for m in range(1, N + 3 - n):
            L1[sk] = (n - 1) / N if N > 0 else 0.0
            L3[sk] = (m - 1) / N if N > 0 else 0.0
            sk += 1
    L2 = 1.0 - L1 - L3
    x = -L2 + L3
    y = (-L2 - L3 + 2.0 * L1) / math.sqrt(3.0)
    if N == 0:
        return x, y
    b1, b2, b3 = 4.0 * L2 * L3, 4.0 * L1 * L3, 4.0 * L1 * L2
    w1 = b1 * warpfactor(N, L3 - L2) * (1.0 + (a * L1) ** 2)
    w2 = b2 * warpfactor(N, L1 - L3) * (1.0 + (a * L2) ** 2)
    w3 = b3 * warpfactor(N, L2 - L1) * (1.0 + (a * L3) ** 2)
    x = x + w1 + math.cos(2 * math.pi / 3) * w2 + math.cos(4 * math.pi / 3) * w3
    y = y + math.sin(2 * math.pi / 3) * w2 + math.sin(4 * math.pi / 3) * w3
    return x, y


def xy_to_rs(x, y):
    """``src/ddg/dg2d/reference.py:104-111``."""
    L1 = (math.sqrt(3.0) * y + 1.0) / 3.0
    L2 = (-3.0 * x - math.sqrt(3.0) * y + 2.0) / 6.0
    L3 = (3.0 * x - math.sqrt(3.0) * y + 2.0) / 6.0
    return -L2 + L3 - L1, -L2 - L3 + L1


def rs_to_ab(r, s):
    """``src/ddg/dg2d/reference.py:114-121``."""
    r = np.asarray(r, dtype=np.float64)
    s = np.asarray(s, dtype=np.float64)
    with np.errstate(divide="ignore", invalid="ignore"):
        a = np.where(np.abs(s - 1.0) > 1e-12, 2.0 * (1.0 + r) / (1.0 - s) - 1.0, -1.0)
    return a, s


def simplex_2d_p(a, b, i: int, j: int) -> np.ndarray:
    """``src/ddg/dg2d/reference.py:124-131``."""
    h1 = jacobi_p(a, 0.0, 0.0, i)
    h2 = jacobi_p(b, 2 * i + 1.0, 0.0, j)
    fac = (1.0 - b) ** i if i > 0 else 1.0
    return math.sqrt(2.0) * h1 * h2 * fac


def grad_simplex_2d_p(a, b, i: int, j: int):
    """``src/ddg/dg2d/reference.py:134-161``."""
    a = np.asarray(a, dtype=np.float64).reshape(-1)
    b = np.asarray(b, dtype=np.float64).reshape(-1)
    fa = jacobi_p(a, 0.0, 0.0, i)
    dfa = grad_jacobi_p(a, 0.0, 0.0, i)
    gb = jacobi_p(b, 2 * i + 1.0, 0.0, j)
    dgb = grad_jacobi_p(b, 2 * i + 1.0, 0.0, j)
    dr = dfa * gb
    if i > 0:
        dr = dr * ((0.5 * (1.0 - b)) ** (i - 1))
    ds = dfa * (gb * (0.5 * (1.0 + a)))
    if i > 0:
        ds = ds * ((0.5 * (1.0 - b)) ** (i - 1))
    t = dgb * ((0.5 * (1.0 - b)) ** i)
    if i > 0:
        t = t - 0.5 * i * gb * ((0.5 * (1.0 - b)) ** (i - 1))
    ds = ds + fa * t
    nrm = 2.0 ** (i + 0.5)
    return nrm * dr, nrm * ds


def vandermonde_2d(N: int, r, s) -> np.ndarray:
    """``src/ddg/dg2d/reference.py:164-171`` (mode order i outer, j inner)."""
    a, b = rs_to_ab(r, s)
    return np.stack([simplex_2d_p(a, b, i, j)
                     for i in range(N + 1) for j in range(N - i + 1)], axis=1)


def grad_vandermonde_2d(N: int, r, s):
    """``src/ddg/dg2d/reference.py:174-185``."""
    a, b = rs_to_ab(r, s)
    cr, cs = [], []
    for i in range(N + 1):
        for j in range(N - i + 1):
            dr, ds = grad_simplex_2d_p(a, b, i, j)
            cr.append(dr)
            cs.append(ds)
    return np.stack(cr, axis=1), np.stack(cs, axis=1)


def d_matrices_2d(N: int, r, s, V):
    """``src/ddg/dg2d/reference.py:188-195``: Dr = Vr V^-1, Ds = Vs V^-1."""
    Vr, Vs = grad_vandermonde_2d(N, r, s)
    return np.linalg.solve(V.T, Vr.T).T, np.linalg.solve(V.T, Vs.T).T


def face_masks_2d(N: int, r, s) -> np.ndarray:
    """``src/ddg/dg2d/reference.py:198-210`` (tolerance 1e-12), (Nfp, 3)."""
    tol = 1e-12
    f0 = np.where(np.abs(s + 1.0) < tol)[0]
    f1 = np.where(np.abs(r + s) < tol)[0]
    f2 = np.where(np.abs(r + 1.0) < tol)[0]
    return np.stack([f0, f1, f2], axis=1)


def lift_2d(N: int, r, s, V, Fmask) -> np.ndarray:
    """``src/ddg/dg2d/reference.py:213-255``: LIFT = V (V^T E)."""
    Np = (N + 1) * (N + 2) // 2
    Nfp = N + 1
    E = np.zeros((Np, 3 * Nfp))
    for f in range(3):
        param = s[Fmask[:, f]] if f == 2 else r[Fmask[:, f]]
        V1 = vandermonde_1d(N, param)
        E[np.ix_(Fmask[:, f], np.arange(f * Nfp, (f + 1) * Nfp))] = np.linalg.inv(V1 @ V1.T)
    return V @ (V.T @ E)


class RefElement:
    """All reference-element data for degree N, as ``build_mesh_2d`` computes
    it (``src/ddg/dg2d/mesh.py:704-711``), plus the SIPG mass matrices
    (``src/ddg/dg2d/sipg.py:78-110``)."""

    def __init__(self, N: int):
        self.N = N
        self.Np = (N + 1) * (N + 2) // 2
        self.Nfp = N + 1
        xe, ye = equilateral_nodes_2d(N)
        self.r, self.s = xy_to_rs(xe, ye)
        self.V = vandermonde_2d(N, self.r, self.s)
        self.invV = np.linalg.inv(self.V)
        self.Dr, self.Ds = d_matrices_2d(N, self.r, self.s, self.V)
        self.Fmask = face_masks_2d(N, self.r, self.s)
        self.LIFT = lift_2d(N, self.r, self.s, self.V, self.Fmask)
        # sipg.py:78-80 and :98-110
        self.M = np.linalg.inv(self.V @ self.V.T)
        m1d = []
        for f in range(3):
            param = self.r[self.Fmask[:, f]] if f < 2 else self.s[self.Fmask[:, f]]
            V1 = vandermonde_1d(N, param)
            m1d.append(np.linalg.inv(V1 @ V1.T))
        self.m1d = np.stack(m1d, axis=0)
