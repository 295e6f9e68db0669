"""p- and hp-multigrid V-cycle preconditioners on the GPU, with the call
surface of ddg's ``src/ddg/dg2d/multigrid.py``.

The hierarchy is set up on the host (meshes, transfer matrices, the dense
inverse of the coarsest operator); the V-cycle itself (weighted
block-Jacobi smoothing, p/h transfers, coarse solve) runs in
``libddg_sipg.so`` (``ddg_mg_*``).  A solve handed this preconditioner runs
CG with the whole V-cycle inside the device loop graph.

Extension: ``precision="fp32"`` runs smoothing, transfers and the coarse
solve in float32 (the outer CG stays float64); the default ``"fp64"``
reproduces the reference.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from .. import _lib
from .mesh import Mesh2D, build_mesh_2d
from .reference import ref_element, vandermonde_2d
from .refinement import uniform_hierarchy


def _p_interp_matrix(N_lo: int, N_hi: int) -> np.ndarray:
    """Nodal interpolation degree N_lo -> N_hi: V_lo(r_hi, s_hi) invV_lo
    (``multigrid.py:106-114``), shape (Np_hi, Np_lo)."""
    hi, lo = ref_element(N_hi), ref_element(N_lo)
    return vandermonde_2d(N_lo, hi.r, hi.s) @ lo.invV


def _h_child_interp_matrices(N: int) -> np.ndarray:
    """(4, Np, Np) red-child interpolants (``multigrid.py:137-163``)."""
    e = ref_element(N)
    A, B, Cc = np.array([-1.0, -1.0]), np.array([1.0, -1.0]), np.array([-1.0, 1.0])
    mAB, mBC, mCA = 0.5 * (A + B), 0.5 * (B + Cc), 0.5 * (Cc + A)
    out = []
    for P0, P1, P2 in ((A, mAB, mCA), (mAB, B, mBC), (mCA, mBC, Cc), (mAB, mBC, mCA)):
        w0, w1, w2 = -(e.r + e.s) / 2, (1 + e.r) / 2, (1 + e.s) / 2
        pr = w0 * P0[0] + w1 * P1[0] + w2 * P2[0]
        ps = w0 * P0[1] + w1 * P1[1] + w2 * P2[1]
        out.append(vandermonde_2d(N, pr, ps) @ e.invV)
    return np.stack(out)


def _coarse_inverse(op, alpha, regularize, eps):
    """Dense (alpha M + A) of the coarsest level by device applies, optional
    ``eps max|diag|`` shift (``multigrid.py:220-225``), inverted in float64."""
    import torch
    n = op.n
    A = torch.empty((n, n), dtype=torch.float64, device=op._dev())
    e = torch.zeros(n, dtype=torch.float64, device=op._dev())
    for j in range(n):
        e.zero_()
        e[j] = 1.0
        A[:, j] = op.apply(e, alpha=alpha)
    A = A.cpu().numpy()
    if regularize:
        A = A + eps * np.max(np.abs(np.diag(A))) * np.eye(n)
    return np.linalg.inv(A)


class SipgMultigrid:
    """A device V-cycle; callable as ``M^-1(v_flat) -> v_flat`` on the
    finest level's element-major vector."""

    def __init__(self, meshes, bcs, *, tau_scale, alpha, nu_smooth, omega, regularize, eps, precision):
        import torch
        if precision not in ("fp64", "fp32"):
            raise ValueError("precision must be 'fp64' or 'fp32'")
        self.alpha = float(alpha)
        self.tau_scale = float(tau_scale)
        self.meshes = meshes
        if not all(m.is_affine for m in meshes):
            raise ValueError("the device multigrid needs straight-sided (affine) levels; use block-Jacobi "
                             "or no preconditioner on curved meshes")
        self.ops = [m.device_operator(bc, tau_scale) for m, bc in zip(meshes, bcs)]
        for op in self.ops[:-1]:
            if op.pc_alpha != self.alpha:
                op.pc_build(self.alpha)
        P, rows, cols = [], [], []
        for f, c in zip(meshes[:-1], meshes[1:]):
            if f.K == c.K:
                M = _p_interp_matrix(c.N, f.N)
            elif f.K == 4 * c.K and f.N == c.N:
                M = _h_child_interp_matrices(c.N).reshape(4 * c.Np, c.Np)
            else:
                raise ValueError("consecutive levels must share the mesh (p) or be a uniform refinement (h)")
            P.append(np.ascontiguousarray(M))
            rows.append(M.shape[0])
            cols.append(M.shape[1])
        Ainv = np.ascontiguousarray(_coarse_inverse(self.ops[-1], self.alpha, regularize, eps))
        L = len(meshes)
        self._keep = (P, Ainv)
        ops_arr = (C.c_void_p * L)(*[op._h.value for op in self.ops])
        P_arr = (C.POINTER(C.c_double) * max(1, L - 1))(*[p.ctypes.data_as(C.POINTER(C.c_double)) for p in P])
        r_arr = (C.c_int32 * max(1, L - 1))(*rows)
        c_arr = (C.c_int32 * max(1, L - 1))(*cols)
        d = _lib.MgDesc(nlevels=L, precision=_lib.DDG_FP32 if precision == "fp32" else _lib.DDG_FP64,
                        nu=int(nu_smooth), reserved=0, omega=float(omega), alpha=self.alpha,
                        ops=ops_arr, prolong=P_arr, prolong_rows=r_arr, prolong_cols=c_arr,
                        coarse_inv=Ainv.ctypes.data_as(C.POINTER(C.c_double)))
        h = C.c_void_p()
        _lib.check(_lib.lib().ddg_mg_create(C.byref(d), C.byref(h)), "ddg_mg_create")
        self._h = h
        self.finest = meshes[0]
        self.precision = precision
        self._torch = torch

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.lib().ddg_mg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def matches(self, op, alpha) -> bool:
        return (op.mesh is self.finest or (op.K == self.ops[0].K and op.N == self.ops[0].N)) \
            and float(alpha) == self.alpha

    def apply_device(self, r, out=None):
        torch = self._torch
        z = torch.empty_like(r) if out is None else out
        _lib.check(_lib.lib().ddg_mg_apply(self._h, r.data_ptr(), z.data_ptr(), _lib.stream_handle(None)),
                   "ddg_mg_apply")
        return z

    def __call__(self, v_flat):
        torch = self._torch
        t = torch.as_tensor(v_flat, dtype=torch.float64, device=self.ops[0]._dev()).contiguous()
        z = self.apply_device(t)
        return z if hasattr(v_flat, "data_ptr") else z.cpu().numpy()


def make_sipg_mg_preconditioner(mesh: Mesh2D, *, bc_types, tau_scale: float = 200.0, alpha: float = 0.0,
                                p_coarse: int = 1, nu_smooth: int = 2, omega: float = 0.7,
                                regularize: bool = False, eps: float = 1.0e-8, precision: str = "fp64"):
    """p-multigrid V-cycle over degrees N, N-1, ..., p_coarse on one mesh
    (``multigrid.py:253-294``)."""
    pf = int(mesh.N)
    if p_coarse < 1 or p_coarse > pf:
        raise ValueError(f"p_coarse must be in [1, {pf}], got {p_coarse}")
    degrees = list(range(pf, p_coarse - 1, -1))
    meshes = [mesh if d == pf else build_mesh_2d(mesh.VX, mesh.VY, mesh.EToV, d) for d in degrees]
    bc = np.asarray(bc_types)
    return SipgMultigrid(meshes, [bc] * len(meshes), tau_scale=tau_scale, alpha=alpha, nu_smooth=nu_smooth,
                         omega=omega, regularize=regularize, eps=eps, precision=precision)


def make_sipg_hpmg_preconditioner(base_mesh: Mesh2D, n_h_levels: int, *, bc_fn, tau_scale: float = 200.0,
                                  alpha: float = 0.0, p_coarse: int = 1, nu_smooth: int = 2,
                                  omega: float = 0.7, regularize: bool = False, eps: float = 1.0e-8,
                                  precision: str = "fp64"):
    """hp-multigrid: p-levels on the uniformly refined finest mesh, then
    h-levels at ``p_coarse`` down to ``base_mesh`` (``multigrid.py:301-367``).
    Returns ``(preconditioner, finest_mesh)``."""
    hier = uniform_hierarchy(base_mesh.VX, base_mesh.VY, base_mesh.EToV, n_h_levels)
    N = int(base_mesh.N)
    finest = build_mesh_2d(*hier[-1], N)
    if p_coarse < 1 or p_coarse > N:
        raise ValueError(f"p_coarse must be in [1, {N}], got {p_coarse}")
    degrees = list(range(N, p_coarse - 1, -1))
    meshes = [finest if d == N else build_mesh_2d(*hier[-1], d) for d in degrees]
    bc_fine = np.asarray(bc_fn(finest))
    bcs = [bc_fine] * len(meshes)
    for h in hier[-2::-1]:
        m = build_mesh_2d(*h, p_coarse)
        meshes.append(m)
        bcs.append(np.asarray(bc_fn(m)))
    mg = SipgMultigrid(meshes, bcs, tau_scale=tau_scale, alpha=alpha, nu_smooth=nu_smooth, omega=omega,
                       regularize=regularize, eps=eps, precision=precision)
    return mg, finest
