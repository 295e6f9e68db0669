"""SIPG Poisson / Helmholtz operator and solves on the GPU, with the call
surface of ddg's ``src/ddg/dg2d/sipg.py``.

Every function keeps the reference's name, argument names, defaults and
error behaviour; the arithmetic runs in ``libddg_sipg.so`` (sm_100a).
Fields may be numpy arrays or torch tensors; results come back as the same
kind (numpy in -> numpy out, torch CUDA in -> torch CUDA out), float64,
shape ``(Np, K)``.

Differences (extensions, all opt-in):
  * ``IterativeConfig`` accepts ``method="gmres"`` (restarted GMRES,
    ``restart``) and ``precision="mixed"``: float32 PCG iterations that keep
    their search direction across float64 residual replacements (reliable
    updates, every ``inner_tol`` reduction of the float32 residual), so the
    iteration count stays near the float64 one and the result is float64
    accurate.  ``precision="mixed-restart"`` is plain iterative refinement
    (float32 CG restarted from each float64 residual).  The defaults
    reproduce the reference (``method="cg"``, float64).
  * Solves can return their Krylov status (``return_info=True``): the
    reference discards jax's ``info`` (``sipg.py:604,910``).

Curved meshes (``curved.project_to_curve_2d``; ``Mesh2D.is_affine`` False)
and the cubature branch (``cub=cubature.attach_cubature(mesh)``) run the
curved-element kernels (``curved_operator.CurvedOperator``): nodal
quadrature without ``cub``, the cubature rule with it; the loads always use
the nodal face rule, as in the reference.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .. import _lib
from .curved_operator import CurvedOperator
from .mesh import Mesh2D
from .operator import SipgOperator, axpby, cast, dot

BC_INTERIOR = 0
BC_DIRICHLET = 1
BC_NEUMANN = 2


@dataclass(frozen=True)
class IterativeConfig:
    """``src/ddg/dg2d/sipg.py:59-71`` plus opt-in extensions."""
    method: str = "cg"
    tol: float = 1e-9
    atol: float = 0.0
    maxiter: int = 1000
    precision: str = "fp64"      # "fp64" | "mixed" | "mixed-restart"
    inner_tol: float = 0.7       # mixed: float32 residual reduction between float64 updates
    max_refinements: int = 50    # mixed-restart: outer iteration cap
    restart: int = 30            # gmres
    # pure-Neumann (singular) Poisson: "shift" is the reference's epsilon
    # shift (sipg.py:891-906); "project" solves the consistent singular system
    # exactly (RHS projected onto range(A) = 1-perp, no shift) and returns the
    # solution with zero mean over the DOFs -- the limit the shifted solution
    # approaches as epsilon -> 0
    nullspace: str = "shift"


@dataclass
class SolveInfo:
    status: str
    iterations: int
    residual: float      # ||r||_2 at exit
    b_norm: float
    refinements: int = 0
    inner_iterations: int = 0


# ---------------------------------------------------------------- helpers

def _torch():
    import torch
    return torch


def _is_torch(a) -> bool:
    return hasattr(a, "data_ptr") and hasattr(a, "device")


def _flat(field, dev):
    """(Np, K) field -> element-major flat float64 device vector."""
    torch = _torch()
    if field is None:
        return None
    t = torch.as_tensor(field, dtype=torch.float64, device=dev)
    return t.t().contiguous().reshape(-1)


def _unflat(v, mesh, like):
    u = v.reshape(mesh.K, mesh.Np).t().contiguous()
    if like is not None and _is_torch(like):
        return u
    return u.cpu().numpy()


def _op(mesh: Mesh2D, bc_types, tau_scale, cub=None):
    """The device operator: affine kernels for straight-sided meshes without
    ``cub``, the curved-element operator otherwise."""
    if cub is not None:
        return mesh.curved_operator(_bc_np(bc_types), tau_scale, cub)
    return mesh.device_operator(_bc_np(bc_types), tau_scale)


def _curved(op) -> bool:
    return isinstance(op, CurvedOperator)


def _bc_np(bc_types):
    if _is_torch(bc_types):
        bc_types = bc_types.cpu().numpy()
    return np.ascontiguousarray(np.asarray(bc_types), dtype=np.int32)


# ------------------------------------------------------------- operator

def sipg_apply_2d(mesh: Mesh2D, u, *, bc_types, u_dir=None, tau_scale: float = 200.0,
                  M_ref=None, m1d_per_face=None, cub=None):
    """``M (-Delta_h) u`` with the Dirichlet-load offset when ``u_dir`` is
    given (``src/ddg/dg2d/sipg.py:304-337``).  ``M_ref`` / ``m1d_per_face``
    are accepted for signature compatibility; the device uses the reference
    element's own matrices."""
    op = _op(mesh, bc_types, tau_scale, cub)
    if _curved(op):
        dev = op._dev()
        y = op.apply(_flat(u, dev)) if u_dir is None else op.apply_dir(_flat(u, dev), _flat(u_dir, dev))
        return _unflat(y, mesh, u)
    if u_dir is None and not _is_torch(u):
        # host (Np, K) arrays: chunked copy / apply / copy-back pipeline
        return op.apply_host(u)
    dev = op._dev()
    y = op.apply(_flat(u, dev))
    if u_dir is not None:
        axpby(-1.0, op.rhs(u_dir=_flat(u_dir, dev)), 1.0, y)   # + L_D
    return _unflat(y, mesh, u)


def sipg_dirichlet_load_2d(mesh: Mesh2D, u_dir, *, bc_types, tau_scale: float = 200.0):
    """``src/ddg/dg2d/sipg.py:398-417``."""
    op = _op(mesh, bc_types, tau_scale)
    r = op.rhs(u_dir=_flat(u_dir, op._dev()))
    axpby(0.0, r, -1.0, r)
    return _unflat(r, mesh, u_dir)


def sipg_neumann_load_2d(mesh: Mesh2D, q_neu, *, bc_types):
    """``src/ddg/dg2d/sipg.py:420-453``; ``q_neu`` is ``(3 Nfp, K)``."""
    op = _op(mesh, bc_types, 200.0)
    return _unflat(op.rhs(q_neu=_flat(q_neu, op._dev())), mesh, q_neu)


def _dense(mesh, bc_types, tau_scale, alpha, cub=None):
    """Dense (alpha M + A) by applying the device operator to unit vectors
    (``sipg_matrix_2d``, ``sipg.py:344-364``; with ``cub`` the mass is the
    cubature one, ``per_element_mass`` at ``sipg.py:485-490``); for small
    meshes only."""
    torch = _torch()
    op = _op(mesh, bc_types, tau_scale, cub)
    n = op.n
    if n > 20000:
        raise ValueError(f"dense SIPG matrix of {n} unknowns is too large; use iterative=IterativeConfig(...)")
    A = torch.empty((n, n), dtype=torch.float64, device=op._dev())
    e = torch.zeros(n, dtype=torch.float64, device=op._dev())
    for j in range(n):
        e.zero_()
        e[j] = 1.0
        A[:, j] = op.apply(e, alpha=alpha)
    return A


def sipg_matrix_2d(mesh: Mesh2D, *, bc_types, tau_scale: float = 200.0, cub=None):
    """``src/ddg/dg2d/sipg.py:344-364`` (torch CUDA tensor)."""
    return _dense(mesh, bc_types, tau_scale, 0.0, cub)


def sipg_helmholtz_matrix_2d(mesh: Mesh2D, *, alpha, nu, bc_types, tau_scale: float = 200.0, cub=None):
    """``src/ddg/dg2d/sipg.py:460-496`` (``nu`` unused, as in the reference)."""
    return _dense(mesh, bc_types, tau_scale, float(alpha), cub)


def factor_sipg_2d(mesh: Mesh2D, *, bc_types, tau_scale: float = 200.0, regularize: bool = False,
                   eps: float = 1.0e-8, cub=None):
    """``src/ddg/dg2d/sipg.py:367-391``: (A, lu, piv) on the GPU."""
    torch = _torch()
    A = sipg_matrix_2d(mesh, bc_types=bc_types, tau_scale=tau_scale, cub=cub)
    if regularize:
        A = A + eps * torch.max(torch.abs(torch.diag(A))) * torch.eye(A.shape[0], dtype=A.dtype, device=A.device)
    lu, piv = torch.linalg.lu_factor(A)
    return A, lu, piv


def factor_sipg_helmholtz_2d(mesh: Mesh2D, *, alpha, nu, bc_types, tau_scale: float = 200.0, cub=None):
    """``src/ddg/dg2d/sipg.py:518-533``."""
    torch = _torch()
    A = sipg_helmholtz_matrix_2d(mesh, alpha=alpha, nu=nu, bc_types=bc_types, tau_scale=tau_scale, cub=cub)
    lu, piv = torch.linalg.lu_factor(A)
    return A, lu, piv


# ------------------------------------------------------- block Jacobi

class BlockJacobiPreconditioner:
    """``M^-1(v_flat) -> v_flat`` with per-element inverse diagonal blocks
    held on the device (``sipg.py:707-715``).  Passing it to a solve on the
    same mesh / BC tags / penalty / alpha runs the fused device PCG."""

    def __init__(self, op, alpha: float):
        op.pc_build(alpha)
        self.op = op
        self.alpha = float(alpha)
        self.bc = op.bc.copy()
        self.quad = getattr(op, "pc_quad", None)

    def valid_for(self, op, alpha) -> bool:
        if _curved(op):
            # the same blocks can be rebuilt inside another curved handle of
            # this mesh / BC tags / penalty (e.g. the cubature solve with the
            # nodal blocks, as the reference pairs them): any solve alpha
            return _curved(self.op) and op.mesh is self.op.mesh and op.tau_scale == self.op.tau_scale \
                and np.array_equal(op.bc, self.bc)
        return op is self.op and float(alpha) == self.alpha and self.op.pc_alpha == self.alpha \
            and np.array_equal(op.bc, self.bc)

    def prepare(self, op):
        """Blocks of this preconditioner in ``op`` (curved handles)."""
        if op.pc_alpha != self.alpha or op.pc_quad != self.quad:
            op.pc_build(self.alpha, quad=self.quad)

    def blocks(self):
        return self.op.pc_blocks()

    def __call__(self, v_flat):
        torch = _torch()
        t = torch.as_tensor(v_flat, device=self.op._dev())
        if t.dtype not in (torch.float32, torch.float64):
            t = t.to(torch.float64)
        z = self.op.pc_apply(t.contiguous())
        return z if _is_torch(v_flat) else z.cpu().numpy()


def make_sipg_block_jacobi_preconditioner(mesh: Mesh2D, *, bc_types, tau_scale: float = 200.0,
                                          A_dense=None, matfree: bool = False, cub=None):
    """``src/ddg/dg2d/sipg.py:718-761``.  The blocks are always computed on
    the device from the element operator (the dense and colour-probed
    variants of the reference give the same blocks), so ``A_dense`` and
    ``matfree`` do not change the result.  On a curved mesh the blocks are
    those of the nodal operator, as in the reference (it takes no ``cub``);
    ``cub=`` (extension) gives the blocks of the cubature operator."""
    return BlockJacobiPreconditioner(_op(mesh, bc_types, tau_scale, cub), 0.0)


def make_helmholtz_block_jacobi_preconditioner(mesh: Mesh2D, *, alpha, nu, bc_types,
                                               tau_scale: float = 200.0, A_dense=None,
                                               matfree: bool = False, cub=None):
    """``src/ddg/dg2d/sipg.py:764-805`` (``cub=`` as in
    :func:`make_sipg_block_jacobi_preconditioner`)."""
    return BlockJacobiPreconditioner(_op(mesh, bc_types, tau_scale, cub), float(alpha))


def _color_elements(mesh: Mesh2D):
    """Greedy element colouring (``sipg.py:651-668``); host setup."""
    K = mesh.K
    col = -np.ones(K, dtype=np.int64)
    E = np.asarray(mesh.EToE)
    for k in range(K):
        used = {int(col[nb]) for nb in E[k] if nb != k and col[nb] >= 0}
        c = 0
        while c in used:
            c += 1
        col[k] = c
    return col, int(col.max()) + 1


def extract_block_diag_matfree(apply_flat, mesh: Mesh2D):
    """Coloured probing of an arbitrary flat apply (``sipg.py:671-704``);
    returns (K, Np, Np) as torch CUDA float64."""
    torch = _torch()
    Np, K = mesh.Np, mesh.K
    col, nc = _color_elements(mesh)
    dev = torch.device("cuda", torch.cuda.current_device())
    colt = torch.as_tensor(col, device=dev)
    blocks = torch.zeros((K, Np, Np), dtype=torch.float64, device=dev)
    for c in range(nc):
        mask = (colt == c)
        for j in range(Np):
            probe = torch.zeros((K, Np), dtype=torch.float64, device=dev)
            probe[:, j] = mask.to(torch.float64)
            r = torch.as_tensor(apply_flat(probe.reshape(-1)), device=dev).reshape(K, Np)
            blocks[:, :, j] += torch.where(mask[:, None], r, torch.zeros_like(r))
    return blocks


# ---------------------------------------------------------------- solves

def _generic_pcg(op, b, x, *, alpha, shift, tol, atol, maxiter, M):
    """PCG for an arbitrary preconditioner callable, same stopping rule as
    jax's cg; every vector operation is a device kernel of the library."""
    torch = _torch()
    bb = dot(b, b)
    atol2 = max(tol * tol * bb, atol * atol)

    def A(v):
        y = op.apply(v, alpha=alpha)
        if shift != 0.0:
            axpby(shift, v, 1.0, y)
        return y

    r = b.clone()
    axpby(-1.0, A(x), 1.0, r)
    z = torch.as_tensor(M(r), dtype=torch.float64, device=b.device).contiguous()
    p = z.clone()
    gamma = dot(r, z)
    k = 0
    status = "converged"
    while True:
        rs = dot(r, r)
        if not (rs > atol2 and k < maxiter):
            if rs > atol2:
                status = "maxiter"
            break
        Ap = A(p)
        pAp = dot(p, Ap)
        if not pAp > 0.0:
            status = "breakdown"
            break
        a = gamma / pAp
        axpby(a, p, 1.0, x)
        axpby(-a, Ap, 1.0, r)
        z = torch.as_tensor(M(r), dtype=torch.float64, device=b.device).contiguous()
        g2 = dot(r, z)
        axpby(1.0, z, g2 / gamma, p)
        gamma = g2
        k += 1
    return SolveInfo(status, k, float(np.sqrt(max(rs, 0.0))), float(np.sqrt(bb)))


def _mixed_ir(op, b, x, *, alpha, shift, cfg, pc):
    """Float64 iterative refinement around float32 device CG solves:
    r = b - A x (float64, the true residual), A d = r in float32 to
    ``inner_tol``, x += d.  Stops at ||r|| <= max(tol ||b||, atol), or when a
    refinement no longer reduces the true residual (the float64 residual
    floor): status "stagnated" with the residual reached."""
    torch = _torch()
    bb = dot(b, b)
    target = max(cfg.tol * cfg.tol * bb, cfg.atol * cfg.atol)
    total_inner = 0
    status = "maxiter"
    history = []
    it = 0
    for it in range(cfg.max_refinements + 1):
        r = op.apply(x, alpha=alpha)
        if shift != 0.0:
            axpby(shift, x, 1.0, r)
        axpby(1.0, b, -1.0, r)
        rr = dot(r, r)
        history.append(rr)
        if rr <= target:
            status = "converged"
            break
        if len(history) >= 3 and history[-1] > 0.5 * history[-2] and history[-2] > 0.5 * history[-3]:
            status = "stagnated"
            break
        if it == cfg.max_refinements or total_inner >= cfg.maxiter:
            break
        r32 = cast(r, torch.float32)
        d32 = torch.zeros_like(r32)
        st, its, _, _ = op.cg(r32, d32, tol=1e-4, atol=0.0, maxiter=cfg.maxiter - total_inner,
                              pc=pc, alpha=alpha, shift=shift, precision="fp32")
        total_inner += its
        if st == "breakdown" or its == 0:
            status = "breakdown" if st == "breakdown" else "stalled"
            break
        axpby(1.0, cast(d32, torch.float64), 1.0, x)
    info = SolveInfo(status, total_inner, float(np.sqrt(history[-1])), float(np.sqrt(bb)), refinements=it,
                     inner_iterations=total_inner)
    info.history = [float(np.sqrt(h / bb)) for h in history]
    return info


def _iterative_solve(mesh, op, b, x0, *, alpha, shift, iterative, preconditioner):
    torch = _torch()
    x = torch.zeros_like(b) if x0 is None else _flat(x0, b.device)
    if iterative.method not in ("cg", "gmres"):
        raise ValueError(f"iterative method {iterative.method!r} not supported for SPD")
    if _curved(op):
        return x, _curved_solve(op, b, x, alpha=alpha, shift=shift, iterative=iterative,
                                preconditioner=preconditioner)
    if iterative.precision not in ("fp64", "mixed", "mixed-restart"):
        raise ValueError(f"precision {iterative.precision!r} must be 'fp64', 'mixed' or 'mixed-restart'")
    from .multigrid import SipgMultigrid
    native_pc = preconditioner is None or (
        isinstance(preconditioner, BlockJacobiPreconditioner) and preconditioner.valid_for(op, alpha))
    if isinstance(preconditioner, SipgMultigrid) and preconditioner.matches(op, alpha) \
            and iterative.method == "cg" and iterative.precision == "fp64":
        st, its, rr, bb = op.cg_mg(preconditioner, b, x, tol=iterative.tol, atol=iterative.atol,
                                   maxiter=iterative.maxiter, alpha=alpha, shift=shift)
        return x, SolveInfo(st, its, float(np.sqrt(max(rr, 0.0))), float(np.sqrt(bb)))
    use_pc = preconditioner is not None
    if iterative.method == "gmres":
        from .krylov import gmres
        M = None if preconditioner is None else preconditioner
        info = gmres(op, b, x, alpha=alpha, shift=shift, tol=iterative.tol, atol=iterative.atol,
                     maxiter=iterative.maxiter, restart=iterative.restart, M=M)
        return x, info
    if iterative.precision in ("mixed", "mixed-restart"):
        if not native_pc:
            raise ValueError("mixed precision needs no preconditioner or a block-Jacobi one built on "
                             "the same mesh, BC tags, penalty and alpha")
        if iterative.precision == "mixed-restart":
            return x, _mixed_ir(op, b, x, alpha=alpha, shift=shift, cfg=iterative, pc=use_pc)
        st, its, rr, bb, upd = op.cg_mixed(b, x, tol=iterative.tol, atol=iterative.atol,
                                           maxiter=iterative.maxiter, pc=use_pc, alpha=alpha, shift=shift,
                                           delta=iterative.inner_tol)
        return x, SolveInfo(st, its, float(np.sqrt(max(rr, 0.0))), float(np.sqrt(bb)), refinements=upd,
                            inner_iterations=its)
    if native_pc:
        st, its, rr, bb = op.cg(b, x, tol=iterative.tol, atol=iterative.atol, maxiter=iterative.maxiter,
                                pc=use_pc, alpha=alpha, shift=shift, precision="fp64")
        return x, SolveInfo(st, its, float(np.sqrt(max(rr, 0.0))), float(np.sqrt(bb)))
    return x, _generic_pcg(op, b, x, alpha=alpha, shift=shift, tol=iterative.tol, atol=iterative.atol,
                           maxiter=iterative.maxiter, M=preconditioner)


def _curved_solve(op, b, x, *, alpha, shift, iterative, preconditioner):
    """Float64 solves on the curved-element operator: the device CG graph
    (no preconditioner, or block-Jacobi from make_*_block_jacobi_* on the
    same mesh), GMRES, or PCG around an arbitrary preconditioner callable."""
    if iterative.precision != "fp64":
        raise ValueError("the curved-element operator solves in float64 (precision='fp64')")
    if iterative.method == "gmres":
        from .krylov import gmres
        return gmres(op, b, x, alpha=alpha, shift=shift, tol=iterative.tol, atol=iterative.atol,
                     maxiter=iterative.maxiter, restart=iterative.restart, M=preconditioner)
    native = preconditioner is None or (isinstance(preconditioner, BlockJacobiPreconditioner)
                                        and preconditioner.valid_for(op, alpha))
    if not native:
        return _generic_pcg(op, b, x, alpha=alpha, shift=shift, tol=iterative.tol, atol=iterative.atol,
                            maxiter=iterative.maxiter, M=preconditioner)
    if preconditioner is not None:
        preconditioner.prepare(op)
    st, its, rr, bb = op.cg(b, x, tol=iterative.tol, atol=iterative.atol, maxiter=iterative.maxiter,
                            pc=preconditioner is not None, alpha=alpha, shift=shift)
    return SolveInfo(st, its, float(np.sqrt(max(rr, 0.0))), float(np.sqrt(bb)))


def _dense_solve(A_factored, b):
    torch = _torch()
    _, lu, piv = A_factored
    return torch.linalg.lu_solve(lu, piv, b.reshape(-1, 1)).reshape(-1)


def solve_sipg_poisson_2d(mesh: Mesh2D, source, *, bc_types, u_dir=None, q_neu=None,
                          tau_scale: float = 200.0, A_factored=None, iterative: IterativeConfig | None = None,
                          x0=None, preconditioner=None, cub=None, return_info: bool = False):
    """``-Delta u = source`` with mixed BCs (``src/ddg/dg2d/sipg.py:812-918``),
    including the singular pure-Neumann branch (eps-shift of
    ``1e-6 ||A probe|| / ||probe||`` and a mean-free RHS, ``:891-906``)."""
    bc = _bc_np(bc_types)
    op = _op(mesh, bc, tau_scale, cub)
    dev = op._dev()
    b = op.rhs(_flat(source, dev), _flat(u_dir, dev), _flat(q_neu, dev))
    if iterative is None:
        if A_factored is None:
            A_factored = factor_sipg_2d(mesh, bc_types=bc, tau_scale=tau_scale, cub=cub)
        u = _unflat(_dense_solve(A_factored, b), mesh, source)
        return (u, None) if return_info else u
    shift = 0.0
    singular = not bool(np.any(bc == BC_DIRICHLET))
    if iterative.nullspace not in ("shift", "project"):
        raise ValueError(f"nullspace {iterative.nullspace!r} must be 'shift' or 'project'")
    if singular:
        torch = _torch()
        ones = torch.ones(op.n, dtype=torch.float64, device=dev)
        if iterative.nullspace == "shift":
            probe = torch.sin(torch.arange(op.n, dtype=torch.float64, device=dev))
            axpby(-dot(probe, ones) / op.n, ones, 1.0, probe)
            Ap = op.apply(probe)
            shift = 1.0e-6 * float(np.sqrt(dot(Ap, Ap) / dot(probe, probe)))
        axpby(-dot(b, ones) / op.n, ones, 1.0, b)
    if singular and iterative.nullspace == "project":
        # CG on the consistent singular system with every preconditioned
        # residual projected onto 1-perp, so the search directions never pick
        # up the constant null vector (pAp stays positive); mean-free result
        torch = _torch()
        x = torch.zeros_like(b) if x0 is None else _flat(x0, dev)

        def proj(v):
            z = (v.clone() if preconditioner is None else
                 torch.as_tensor(preconditioner(v), dtype=torch.float64, device=dev).contiguous())
            axpby(-dot(z, ones) / op.n, ones, 1.0, z)
            return z
        info = _generic_pcg(op, b, x, alpha=0.0, shift=0.0, tol=iterative.tol, atol=iterative.atol,
                            maxiter=iterative.maxiter, M=proj)
        axpby(-dot(x, ones) / op.n, ones, 1.0, x)
    else:
        x, info = _iterative_solve(mesh, op, b, x0, alpha=0.0, shift=shift, iterative=iterative,
                                   preconditioner=preconditioner)
    u = _unflat(x, mesh, source)
    return (u, info) if return_info else u


def solve_sipg_helmholtz_2d(mesh: Mesh2D, rhs_field, *, alpha, nu, bc_types, u_dir=None, q_neu=None,
                            tau_scale: float = 200.0, A_factored=None,
                            iterative: IterativeConfig | None = None, x0=None, preconditioner=None,
                            cub=None, return_info: bool = False):
    """``(alpha M - Delta) u = rhs_field`` (``src/ddg/dg2d/sipg.py:536-612``;
    ``nu`` unused, as in the reference)."""
    bc = _bc_np(bc_types)
    op = _op(mesh, bc, tau_scale, cub)
    dev = op._dev()
    b = op.rhs(_flat(rhs_field, dev), _flat(u_dir, dev), _flat(q_neu, dev))
    if iterative is None:
        if A_factored is None:
            A_factored = factor_sipg_helmholtz_2d(mesh, alpha=alpha, nu=nu, bc_types=bc, tau_scale=tau_scale,
                                                  cub=cub)
        u = _unflat(_dense_solve(A_factored, b), mesh, rhs_field)
        return (u, None) if return_info else u
    x, info = _iterative_solve(mesh, op, b, x0, alpha=float(alpha), shift=0.0, iterative=iterative,
                               preconditioner=preconditioner)
    u = _unflat(x, mesh, rhs_field)
    return (u, info) if return_info else u
