"""Differentiable SIPG solves with a per-element diffusivity kappa = exp(g).

Extension with no reference counterpart: ddg's SIPG operator has no
coefficient, and ddg differentiates its solves with ``jax.grad`` through
``jax.scipy.sparse.linalg.cg`` (an implicit linear-solve rule).  Here the
derivative is written by hand:

    A(kappa) u = J M f                     (forward block-Jacobi PCG)
    A(kappa) lam = dL/du                   (adjoint: A is symmetric, so the
                                            same operator and preconditioner)
    dL/dkappa_k = -d a(u, lam; kappa)/d kappa_k      (device contraction kernel)
    dL/dg = kappa * dL/dkappa,   dL/df = J M lam

``KappaSolve`` wraps this in a ``torch.autograd.Function``; ``loss_and_grad``
is the fused form for L = 1/2 ||u - u_obs||_M^2 over a batch of kappas.
"""

from __future__ import annotations

import numpy as np

from .dg2d.operator import SipgOperator, axpby, dot


def _cg(op, b, tol, maxiter):
    import torch
    x = torch.zeros_like(b)
    st, its, rr, bb = op.cg(b, x, tol=tol, maxiter=maxiter, pc=True)
    if st != "converged":
        raise RuntimeError(f"kappa solve did not converge ({st} after {its} iterations)")
    return x, its


class _KappaState:
    """Keeps the handle's diffusivity and preconditioner in sync with the
    kappa a forward or backward pass needs.  Stored on the operator itself,
    so it lives exactly as long as the handle (no module-level registry
    keeps operators alive)."""

    def __init__(self):
        self.current = None

    def use(self, op: SipgOperator, kappa):
        if self.current is None or not np.array_equal(self.current, kappa):
            self.op_set(op, kappa)
            self.current = kappa.copy()

    @staticmethod
    def op_set(op, kappa):
        op.set_kappa(kappa)
        op.pc_build(0.0)


def _state(op):
    if not isinstance(op, SipgOperator):
        raise ValueError("the per-element diffusivity (kappa) is built for straight-sided (affine) meshes only")
    s = getattr(op, "_kappa_state", None)
    if s is None:
        s = op._kappa_state = _KappaState()
    return s


def mass_apply(op, v):
    """J M v on a flat float64 device vector (the RHS kernel with f = v)."""
    return op.rhs(f=v)


def _torch_fn():
    import torch

    class KappaSolve(torch.autograd.Function):
        """u = A(exp(g))^-1 (J M f) with a hand-written adjoint.

        g: (K,) float64 CUDA tensor; f: flat (K*Np,) nodal source (element
        major); returns the flat solution u.  ``op`` is the mesh's device
        operator (its BC tags; homogeneous boundary data)."""

        @staticmethod
        def forward(ctx, g, f, op, tol=1e-12, maxiter=20000):
            kappa = torch.exp(g)
            k_np = kappa.detach().cpu().numpy()
            st = _state(op)
            st.use(op, k_np)
            u, _ = _cg(op, mass_apply(op, f.detach().contiguous()), tol, maxiter)
            ctx.op, ctx.tol, ctx.maxiter, ctx.k_np = op, tol, maxiter, k_np
            ctx.save_for_backward(u, kappa)
            return u

        @staticmethod
        def backward(ctx, gu):
            u, kappa = ctx.saved_tensors
            op = ctx.op
            _state(op).use(op, ctx.k_np)
            lam, _ = _cg(op, gu.contiguous(), ctx.tol, ctx.maxiter)
            gk = op.grad_kappa(u, lam)
            return -gk * kappa, mass_apply(op, lam), None, None, None

    return KappaSolve


KappaSolve = None


def kappa_solve(g, f, op, tol=1e-12, maxiter=20000):
    """Differentiable solve (see :class:`KappaSolve`)."""
    global KappaSolve
    if KappaSolve is None:
        KappaSolve = _torch_fn()
    return KappaSolve.apply(g, f, op, tol, maxiter)


def loss_and_grad(op, g_batch, f, u_obs, tol=1e-12, maxiter=20000):
    """L_b = 1/2 (u_b - u_obs)^T J M (u_b - u_obs) and dL_b/dg_b for every row
    of ``g_batch`` (B, K); one forward and one adjoint solve per row.
    Returns (losses (B,), grads (B, K), total CG iterations)."""
    import torch
    st = _state(op)
    B = g_batch.shape[0]
    losses = torch.empty(B, dtype=torch.float64, device=g_batch.device)
    grads = torch.empty_like(g_batch)
    b = mass_apply(op, f)
    its = 0
    for i in range(B):
        kappa = torch.exp(g_batch[i])
        st.use(op, kappa.cpu().numpy())
        u, i1 = _cg(op, b, tol, maxiter)
        r = u.clone()
        axpby(-1.0, u_obs, 1.0, r)
        Mr = mass_apply(op, r)
        losses[i] = 0.5 * dot(r, Mr)
        lam, i2 = _cg(op, Mr, tol, maxiter)
        grads[i] = -op.grad_kappa(u, lam) * kappa
        its += i1 + i2
    return losses, grads, its


def loss_only(op, g, f, u_obs, tol=1e-13, maxiter=40000):
    """L for one kappa = exp(g) (the finite-difference check's evaluations)."""
    import torch
    st = _state(op)
    st.use(op, torch.exp(g).cpu().numpy())
    u, _ = _cg(op, mass_apply(op, f), tol, maxiter)
    r = u.clone()
    axpby(-1.0, u_obs, 1.0, r)
    return 0.5 * dot(r, mass_apply(op, r))
