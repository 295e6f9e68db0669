"""Diffusivity extension and hand-written adjoint on the GPU."""

import numpy as np
import pytest

from oracle import mesh as om
from oracle import sipg as osp

pytestmark = pytest.mark.gpu


def _pair(K, N):
    from ddg_b200.dg2d import mesh as pm
    VX, VY, E = om.uniform_rectangle_mesh_2d(0.0, 1.0, 0.0, 1.0, K, K)
    return om.build_mesh_2d(VX, VY, E, N), pm.build_mesh_2d(VX, VY, E, N)


def _t(a):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


@pytest.mark.parametrize("N", [2, 3, 4])
def test_kappa_apply_and_grad_kernel_match_oracle(N):
    o, p = _pair(5, N)
    isb = o.EToE == np.arange(o.K)[:, None]
    rng = np.random.default_rng(N)
    for bc in (np.where(isb, 1, 0).astype(np.int32),
               np.where(isb, np.where(rng.random((o.K, 3)) > 0.5, 1, 2), 0).astype(np.int32)):
        kap = np.exp(0.5 * rng.standard_normal(o.K))
        u = rng.standard_normal((o.Np, o.K))
        lam = rng.standard_normal((o.Np, o.K))
        op = p.device_operator(bc, 0.5)
        op.set_kappa(kap)
        y = op.apply(_t(u.T.reshape(-1)), alpha=2.0).cpu().numpy()
        ref = osp.flat_op(o, bc_types=bc, tau_scale=0.5, alpha=2.0, kappa=kap)(u.T.reshape(-1))
        assert np.max(np.abs(y - ref)) < 1e-12 * np.max(np.abs(ref))
        g = op.grad_kappa(_t(u.T.reshape(-1)), _t(lam.T.reshape(-1))).cpu().numpy()
        g_ref = osp.grad_kappa(o, u, lam, bc_types=bc, tau_scale=0.5, kappa=kap)
        assert np.max(np.abs(g - g_ref)) < 1e-11 * np.max(np.abs(g_ref))
        y32 = op.apply(_t(u.T.reshape(-1)).float(), alpha=2.0).double().cpu().numpy()
        assert np.max(np.abs(y32 - ref)) < 2e-5 * np.max(np.abs(ref))
        op.set_kappa(None)


def _problem(K=8, N=3, seed=0):
    o, p = _pair(K, N)
    bc = osp.boundary_bc(o)
    f = np.sin(np.pi * o.x) * np.sin(np.pi * o.y) + 0.5
    rng = np.random.default_rng(seed)
    g_obs = 0.5 * rng.standard_normal(o.K)
    g = 0.5 * np.random.default_rng(seed + 1).standard_normal(o.K)
    return o, p, bc, f, g_obs, g


def test_adjoint_gradient_matches_dense_oracle():
    from ddg_b200 import adjoint
    o, p, bc, f, g_obs, g = _problem(K=4, N=3)
    # oracle: dense solves + autograd contraction
    def solve(kap, rhs):
        return np.linalg.solve(osp.dense_matrix(o, bc_types=bc, tau_scale=0.5, kappa=kap), rhs)
    b = osp.mass_apply(o, f).T.reshape(-1)
    u_obs = solve(np.exp(g_obs), b)
    kap = np.exp(g)
    u = solve(kap, b)
    Mr = osp.mass_apply(o, (u - u_obs).reshape(o.K, o.Np).T).T.reshape(-1)
    lam = solve(kap, Mr)
    g_ref = -kap * osp.grad_kappa(o, u.reshape(o.K, o.Np).T, lam.reshape(o.K, o.Np).T, bc_types=bc,
                                  tau_scale=0.5, kappa=kap)
    op = p.device_operator(bc, 0.5)
    adjoint._state(op).use(op, np.exp(g_obs))
    uo, _ = adjoint._cg(op, adjoint.mass_apply(op, _t(f.T.reshape(-1))), 1e-14, 20000)
    L, G, _ = adjoint.loss_and_grad(op, _t(g[None, :]), _t(f.T.reshape(-1)), uo, tol=1e-14)
    assert np.max(np.abs(G[0].cpu().numpy() - g_ref)) < 1e-8 * np.max(np.abs(g_ref))
    r = u - u_obs
    assert abs(float(L[0]) - 0.5 * r @ Mr) < 1e-8 * abs(0.5 * r @ Mr)


def test_adjoint_gradient_vs_centred_differences():
    """Directional derivatives along random directions, step 1e-6, float64."""
    from ddg_b200 import adjoint
    o, p, bc, f, g_obs, g = _problem(K=8, N=4, seed=3)
    op = p.device_operator(bc, 0.5)
    ft = _t(f.T.reshape(-1))
    adjoint._state(op).use(op, np.exp(g_obs))
    uo, _ = adjoint._cg(op, adjoint.mass_apply(op, ft), 1e-14, 40000)
    gt = _t(g)
    _, G, _ = adjoint.loss_and_grad(op, gt[None, :], ft, uo, tol=1e-14, maxiter=40000)
    rng = np.random.default_rng(11)
    h = 1e-6
    for _ in range(4):
        d = _t(rng.standard_normal(o.K))
        Lp = adjoint.loss_only(op, gt + h * d, ft, uo, tol=1e-14)
        Lm = adjoint.loss_only(op, gt - h * d, ft, uo, tol=1e-14)
        fd = (Lp - Lm) / (2 * h)
        ad = float((G[0] * d).sum())
        assert abs(fd - ad) <= 1e-5 * abs(ad), (fd, ad)


def test_autograd_function_backward():
    import torch
    from ddg_b200 import adjoint
    o, p, bc, f, g_obs, g = _problem(K=6, N=3, seed=5)
    op = p.device_operator(bc, 0.5)
    ft = _t(f.T.reshape(-1)).requires_grad_(True)
    w = _t(np.random.default_rng(2).random(o.K * o.Np))
    gt = _t(g).requires_grad_(True)
    u = adjoint.kappa_solve(gt, ft, op, tol=1e-14)
    loss = 0.5 * torch.sum(w * u * u)
    loss.backward()
    h = 1e-6
    d = _t(np.random.default_rng(4).standard_normal(o.K))
    with torch.no_grad():
        lp = 0.5 * torch.sum(w * adjoint.kappa_solve(gt + h * d, ft, op, tol=1e-14) ** 2)
        lm = 0.5 * torch.sum(w * adjoint.kappa_solve(gt - h * d, ft, op, tol=1e-14) ** 2)
    fd = float((lp - lm) / (2 * h))
    assert abs(fd - float((gt.grad * d).sum())) <= 1e-5 * abs(fd)
    df = _t(np.random.default_rng(6).standard_normal(o.K * o.Np))
    with torch.no_grad():
        lp = 0.5 * torch.sum(w * adjoint.kappa_solve(gt, ft + h * df, op, tol=1e-14) ** 2)
        lm = 0.5 * torch.sum(w * adjoint.kappa_solve(gt, ft - h * df, op, tol=1e-14) ** 2)
    fd = float((lp - lm) / (2 * h))
    assert abs(fd - float((ft.grad * df).sum())) <= 1e-5 * abs(fd)
