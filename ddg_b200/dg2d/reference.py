"""Reference-element operators for nodal DG on the triangle (host setup).

Same operators as ddg's ``src/ddg/dg2d/reference.py`` (warp-and-blend
nodes, orthonormal Koornwinder basis with mode order ``i`` outer / ``j``
inner, ``Dr = Vr V^-1``, ``Ds = Vs V^-1``, ``Fmask``, ``LIFT``) and the
SIPG mass matrices of ``src/ddg/dg2d/sipg.py:78-110``.  The Gauss-Lobatto
nodes are found by Newton iteration on ``(1 - x^2) P_N'(x)`` instead of the
reference's eigenvalue solve (``src/ddg/dg1d/reference.py:79-135``); the two
agree to rounding.  Everything here runs once per polynomial degree and is
cached; the GPU kernels receive the matrices through constant memory.
"""

from __future__ import annotations

import functools
import math

import numpy as np

# Warp-and-blend blending constants for N = 1..15
# (``src/ddg/dg2d/reference.py:27-30``).
_WB_ALPHA = (0.0, 0.0, 1.4152, 0.1001, 0.2751, 0.9800, 1.0999, 1.2832,
             1.3648, 1.4773, 1.4959, 1.5743, 1.5770, 1.6223, 1.6258)


def jacobi(x, a: float, b: float, n: int) -> np.ndarray:
    """Orthonormal Jacobi polynomial of degree ``n`` for weight (a, b)."""
    x = np.asarray(x, dtype=np.float64).reshape(-1)
    lg = (math.lgamma(a + 1) + math.lgamma(b + 1) - math.lgamma(a + b + 1))
    g0 = 2.0 ** (a + b + 1) / (a + b + 1) * math.exp(lg)
    prev = np.full(x.shape, 1.0 / math.sqrt(g0))
    if n == 0:
        return prev
    g1 = (a + 1) * (b + 1) / (a + b + 3) * g0
    cur = ((a + b + 2) * x / 2 + (a - b) / 2) / math.sqrt(g1)
    a_old = 2.0 / (2 + a + b) * math.sqrt((a + 1) * (b + 1) / (a + b + 3))
    for i in range(1, n):
        h = 2 * i + a + b
        a_new = 2.0 / (h + 2) * math.sqrt((i + 1) * (i + 1 + a + b) * (i + 1 + a)
                                          * (i + 1 + b) / (h + 1) / (h + 3))
        b_new = -(a * a - b * b) / h / (h + 2)
        prev, cur = cur, ((x - b_new) * cur - a_old * prev) / a_new
        a_old = a_new
    return cur


def djacobi(x, a: float, b: float, n: int) -> np.ndarray:
    x = np.asarray(x, dtype=np.float64).reshape(-1)
    if n == 0:
        return np.zeros_like(x)
    return math.sqrt(n * (n + a + b + 1)) * jacobi(x, a + 1, b + 1, n - 1)


def gauss_lobatto(n: int) -> np.ndarray:
    """Legendre-Gauss-Lobatto nodes, ascending, endpoints exactly +-1."""
    if n == 1:
        return np.array([-1.0, 1.0])
    # interior nodes are the roots of P_n'(x) ~ P^{(1,1)}_{n-1}
    x = -np.cos(np.pi * np.arange(1, n) / n)
    for _ in range(100):
        f = jacobi(x, 1.0, 1.0, n - 1)
        df = djacobi(x, 1.0, 1.0, n - 1)
        dx = f / df
        x = x - dx
        if np.max(np.abs(dx)) < 1e-16:
            break
    return np.concatenate([[-1.0], np.sort(x), [1.0]])


def vandermonde_1d(n: int, x) -> np.ndarray:
    x = np.asarray(x, dtype=np.float64).reshape(-1)
    return np.column_stack([jacobi(x, 0.0, 0.0, j) for j in range(n + 1)])


def _warp(n: int, rout: np.ndarray) -> np.ndarray:
    gll = gauss_lobatto(n)
    req = np.linspace(-1.0, 1.0, n + 1)
    L = np.linalg.solve(vandermonde_1d(n, req).T,
                        np.vstack([jacobi(rout, 0.0, 0.0, i) for i in range(n + 1)]))
    warp = L.T @ (gll - req)
    inside = np.abs(rout) < 1.0 - 1e-10
    return np.where(inside, warp / (1.0 - np.where(inside, rout, 0.0) ** 2), 0.0)


def triangle_nodes(n: int):
    """Warp-and-blend nodes on the reference triangle (-1,-1),(1,-1),(-1,1)."""
    lam1, lam3 = [], []
    for i in range(n + 1):
        for j in range(n + 1 - i):
            lam1.append(i / n)
            lam3.append(j / n)
    L1, L3 = np.array(lam1), np.array(lam3)
    L2 = 1.0 - L1 - L3
    x = L3 - L2
    y = (2.0 * L1 - L2 - L3) / math.sqrt(3.0)
    al = _WB_ALPHA[n - 1] if n <= 15 else 5.0 / 3.0
    w1 = 4.0 * L2 * L3 * _warp(n, L3 - L2) * (1.0 + (al * L1) ** 2)
    w2 = 4.0 * L1 * L3 * _warp(n, L1 - L3) * (1.0 + (al * L2) ** 2)
    w3 = 4.0 * L1 * L2 * _warp(n, L2 - L1) * (1.0 + (al * L3) ** 2)
    c2, s2 = math.cos(2 * math.pi / 3), math.sin(2 * math.pi / 3)
    c4, s4 = math.cos(4 * math.pi / 3), math.sin(4 * math.pi / 3)
    x = x + w1 + c2 * w2 + c4 * w3
    y = y + s2 * w2 + s4 * w3
    # equilateral -> reference (r, s)
    b1 = (math.sqrt(3.0) * y + 1.0) / 3.0
    b2 = (-3.0 * x - math.sqrt(3.0) * y + 2.0) / 6.0
    b3 = (3.0 * x - math.sqrt(3.0) * y + 2.0) / 6.0
    return -b2 + b3 - b1, -b2 - b3 + b1


def _collapsed(r, s):
    with np.errstate(divide="ignore", invalid="ignore"):
        a = np.where(np.abs(s - 1.0) > 1e-12, 2.0 * (1.0 + r) / (1.0 - s) - 1.0, -1.0)
    return a, s


def vandermonde_2d(n: int, r, s) -> np.ndarray:
    a, b = _collapsed(np.asarray(r, dtype=np.float64), np.asarray(s, dtype=np.float64))
    cols = []
    for i in range(n + 1):
        for j in range(n + 1 - i):
            cols.append(math.sqrt(2.0) * jacobi(a, 0, 0, i) * jacobi(b, 2 * i + 1.0, 0, j)
                        * ((1.0 - b) ** i))
    return np.column_stack(cols)


def grad_vandermonde_2d(n: int, r, s):
    a, b = _collapsed(np.asarray(r, dtype=np.float64), np.asarray(s, dtype=np.float64))
    Vr, Vs = [], []
    for i in range(n + 1):
        fa, dfa = jacobi(a, 0, 0, i), djacobi(a, 0, 0, i)
        hb = 0.5 * (1.0 - b)
        for j in range(n + 1 - i):
            gb, dgb = jacobi(b, 2 * i + 1.0, 0, j), djacobi(b, 2 * i + 1.0, 0, j)
            pm1 = hb ** (i - 1) if i > 0 else np.ones_like(b)
            dr = dfa * gb * (pm1 if i > 0 else 1.0)
            ds = dfa * gb * 0.5 * (1.0 + a) * (pm1 if i > 0 else 1.0)
            t = dgb * hb ** i - (0.5 * i * gb * pm1 if i > 0 else 0.0)
            ds = ds + fa * t
            c = 2.0 ** (i + 0.5)
            Vr.append(c * dr)
            Vs.append(c * ds)
    return np.column_stack(Vr), np.column_stack(Vs)


def fmask_closed_form(n: int) -> np.ndarray:
    """Face-node indices (Nfp, 3) implied by the row-by-row node numbering:
    face 0 is the first row, face 1 the last node of each row, face 2 the
    first node of each row (the kernels hard-code this; ``RefElement``
    checks it against the tolerance search of ``reference.py:198-210``)."""
    rs = [i * (n + 1) - i * (i - 1) // 2 for i in range(n + 1)]
    return np.array([[p, rs[p] + (n - p), rs[p]] for p in range(n + 1)], dtype=np.int64)


class RefElement:
    """Reference-element operators for degree ``N`` (``Np`` nodes)."""

    def __init__(self, N: int):
        if N < 1:
            raise ValueError("polynomial degree must be >= 1")
        self.N, self.Np, self.Nfp = N, (N + 1) * (N + 2) // 2, N + 1
        self.r, self.s = triangle_nodes(N)
        self.V = vandermonde_2d(N, self.r, self.s)
        self.invV = np.linalg.inv(self.V)
        Vr, Vs = grad_vandermonde_2d(N, self.r, self.s)
        self.Dr = np.linalg.solve(self.V.T, Vr.T).T
        self.Ds = np.linalg.solve(self.V.T, Vs.T).T
        tol = 1e-12
        fm = np.stack([np.flatnonzero(np.abs(self.s + 1.0) < tol),
                       np.flatnonzero(np.abs(self.r + self.s) < tol),
                       np.flatnonzero(np.abs(self.r + 1.0) < tol)], axis=1)
        if not np.array_equal(fm, fmask_closed_form(N)):
            raise RuntimeError("face-node numbering differs from the closed form")
        self.Fmask = fm
        self.M = np.linalg.inv(self.V @ self.V.T)
        m1d = []
        E = np.zeros((self.Np, 3 * self.Nfp))
        for f in range(3):
            t = (self.s if f == 2 else self.r)[fm[:, f]]
            V1 = vandermonde_1d(N, t)
            m1d.append(np.linalg.inv(V1 @ V1.T))
            E[np.ix_(fm[:, f], np.arange(f * self.Nfp, (f + 1) * self.Nfp))] = m1d[-1]
        self.m1d = np.stack(m1d)
        self.LIFT = self.V @ (self.V.T @ E)
        self.rot_perm = self._rotation_permutations()

    def _rotation_permutations(self) -> np.ndarray:
        """(3, Np) node permutations: row f lists, for each node of the element
        relabelled so that its face f becomes face 0 (vertices v_f, v_f+1,
        v_f+2), the index of the same node in the original numbering."""
        r, s = self.r, self.s
        # relabelled barycentric (lam_A, lam_B, lam_C) of node i: lam_B=(1+r)/2, lam_C=(1+s)/2
        lb, lc = 0.5 * (1 + r), 0.5 * (1 + s)
        la = 1.0 - lb - lc
        out = np.zeros((3, self.Np), dtype=np.int64)
        for f in range(3):
            lam = [None, None, None]
            lam[f % 3], lam[(f + 1) % 3], lam[(f + 2) % 3] = la, lb, lc
            ro, so = 2.0 * lam[1] - 1.0, 2.0 * lam[2] - 1.0       # original (r, s)
            d = (ro[:, None] - r[None, :]) ** 2 + (so[:, None] - s[None, :]) ** 2
            out[f] = np.argmin(d, axis=1)
            if np.max(np.min(d, axis=1)) > 1e-20:
                raise RuntimeError("node set is not rotation symmetric")
        return out


@functools.lru_cache(maxsize=None)
def ref_element(N: int) -> RefElement:
    return RefElement(N)
