"""Oracle: p- and hp-multigrid V-cycle preconditioners.

Test infrastructure only (see ``oracle/__init__.py``).

Restates ``src/ddg/dg2d/multigrid.py``: level operator ``alpha M + A``
(:53-74), level = operator + block-Jacobi smoother from matrix-free probing
(:77-99), nodal p-interpolation I = V_lo(r_hi, s_hi) invV_lo (:106-134),
four red-child interpolants (:137-184), the V-cycle with a dense LU coarse
solve and optional ``eps*max|diag|`` shift (:211-246), and the two builders
(:253-367).
"""

from __future__ import annotations

import numpy as np
import scipy.linalg as sla

from .mesh import build_mesh_2d
from .refelem import vandermonde_2d
from .refinement import build_h_meshes
from .sipg import extract_block_diag_matfree, flat_op


class Level:
    def __init__(self, mesh, bc, tau_scale, alpha):
        self.mesh = mesh
        self.apply = flat_op(mesh, bc_types=bc, tau_scale=tau_scale, alpha=alpha)
        blocks = extract_block_diag_matfree(self.apply, mesh)
        self.blocks = blocks
        self.binv = np.linalg.inv(blocks)
        Np = mesh.Np
        self.smooth_inv = lambda v: np.einsum("kij,kj->ki", self.binv, v.reshape(-1, Np)).reshape(-1)
        self.prolong = None
        self.restrict = None


def p_interp_matrix(mesh_lo, mesh_hi):
    """``multigrid.py:106-114``."""
    return vandermonde_2d(mesh_lo.N, mesh_hi.r, mesh_hi.s) @ mesh_lo.invV


def p_transfer(I):
    Nh, Nl = I.shape
    pro = lambda c: np.einsum("hl,kl->kh", I, c.reshape(-1, Nl)).reshape(-1)  # noqa: E731
    res = lambda f: np.einsum("hl,kh->kl", I, f.reshape(-1, Nh)).reshape(-1)  # noqa: E731
    return pro, res


def h_child_interp_matrices(mesh):
    """``multigrid.py:137-163``."""
    A, B, C = np.array([-1.0, -1.0]), np.array([1.0, -1.0]), np.array([-1.0, 1.0])
    mAB, mBC, mCA = 0.5 * (A + B), 0.5 * (B + C), 0.5 * (C + A)
    kids = [(A, mAB, mCA), (mAB, B, mBC), (mCA, mBC, C), (mAB, mBC, mCA)]
    r, s = mesh.r, mesh.s
    mats = []
    for P0, P1, P2 in kids:
        pr = (-(r + s) / 2) * P0[0] + ((1 + r) / 2) * P1[0] + ((1 + s) / 2) * P2[0]
        ps = (-(r + s) / 2) * P0[1] + ((1 + r) / 2) * P1[1] + ((1 + s) / 2) * P2[1]
        mats.append(vandermonde_2d(mesh.N, pr, ps) @ mesh.invV)
    return np.stack(mats)


def h_transfer(Ic):
    Np = Ic.shape[1]
    pro = lambda c: np.einsum("cij,kj->kci", Ic, c.reshape(-1, Np)).reshape(-1)  # noqa: E731
    res = lambda f: np.einsum("cij,kci->kj", Ic, f.reshape(-1, 4, Np)).reshape(-1)  # noqa: E731
    return pro, res


def assemble_vcycle(levels, *, nu_smooth, omega, regularize, eps):
    """``multigrid.py:211-246``."""
    co = levels[-1]
    n = co.mesh.Np * co.mesh.K
    Ac = co.apply(np.eye(n))
    if regularize:
        Ac = Ac + eps * np.max(np.abs(np.diag(Ac))) * np.eye(n)
    lu = sla.lu_factor(Ac)
    L = len(levels)

    def vc(li, b):
        if li == L - 1:
            return sla.lu_solve(lu, b)
        lv = levels[li]
        x = np.zeros_like(b)
        for _ in range(nu_smooth):
            x = x + omega * lv.smooth_inv(b - lv.apply(x))
        e = vc(li + 1, lv.restrict(b - lv.apply(x)))
        x = x + lv.prolong(e)
        for _ in range(nu_smooth):
            x = x + omega * lv.smooth_inv(b - lv.apply(x))
        return x
    return lambda v: vc(0, v)


def make_pmg(mesh, *, bc_types, tau_scale=200.0, alpha=0.0, p_coarse=1, nu_smooth=2,
             omega=0.7, regularize=False, eps=1e-8):
    """``multigrid.py:253-294``."""
    pf = mesh.N
    if p_coarse < 1 or p_coarse > pf:
        raise ValueError(f"p_coarse must be in [1, {pf}], got {p_coarse}")
    deg = list(range(pf, p_coarse - 1, -1))
    meshes = {d: mesh if d == pf else build_mesh_2d(mesh.VX, mesh.VY, mesh.EToV, d) for d in deg}
    levels = [Level(meshes[d], bc_types, tau_scale, alpha) for d in deg]
    for li in range(len(deg) - 1):
        levels[li].prolong, levels[li].restrict = p_transfer(
            p_interp_matrix(meshes[deg[li + 1]], meshes[deg[li]]))
    return assemble_vcycle(levels, nu_smooth=nu_smooth, omega=omega, regularize=regularize, eps=eps)


def make_hpmg(base_mesh, n_h_levels, *, bc_fn, tau_scale=200.0, alpha=0.0, p_coarse=1,
              nu_smooth=2, omega=0.7, regularize=False, eps=1e-8):
    """``multigrid.py:301-367``.  Returns ``(preconditioner, finest_mesh)``."""
    hm = build_h_meshes(base_mesh.VX, base_mesh.VY, base_mesh.EToV, base_mesh.N, n_h_levels)
    fin = hm[-1]
    pf = fin.N
    if p_coarse < 1 or p_coarse > pf:
        raise ValueError(f"p_coarse must be in [1, {pf}], got {p_coarse}")
    deg = list(range(pf, p_coarse - 1, -1))
    bcf = bc_fn(fin)
    pm = {d: fin if d == pf else build_mesh_2d(fin.VX, fin.VY, fin.EToV, d) for d in deg}
    levels = [Level(pm[d], bcf, tau_scale, alpha) for d in deg]
    hl = [build_mesh_2d(m.VX, m.VY, m.EToV, p_coarse) for m in hm[-2::-1]]
    levels += [Level(m, bc_fn(m), tau_scale, alpha) for m in hl]
    n_p = len(deg)
    for li in range(n_p - 1):
        levels[li].prolong, levels[li].restrict = p_transfer(p_interp_matrix(pm[deg[li + 1]], pm[deg[li]]))
    hp, hr = h_transfer(h_child_interp_matrices(pm[p_coarse]))
    for li in range(n_p - 1, len(levels) - 1):
        levels[li].prolong, levels[li].restrict = hp, hr
    return assemble_vcycle(levels, nu_smooth=nu_smooth, omega=omega, regularize=regularize, eps=eps), fin


def pcg_count(A, b, Minv, *, tol=1e-8, maxiter=2000):
    """The iteration-counting PCG of ``test/test_multigrid_2d.py:49-68``."""
    bn = np.linalg.norm(b)
    x = np.zeros_like(b)
    r = b.copy()
    z = Minv(r)
    p = z.copy()
    rz = float(r @ z)
    for it in range(1, maxiter + 1):
        Ap = A(p)
        a = rz / float(p @ Ap)
        x = x + a * p
        r = r - a * Ap
        if np.linalg.norm(r) / bn < tol:
            return x, it
        z = Minv(r)
        rz2 = float(r @ z)
        p = z + (rz2 / rz) * p
        rz = rz2
    return x, maxiter
