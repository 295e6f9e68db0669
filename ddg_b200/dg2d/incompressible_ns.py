"""Dual-splitting incompressible Navier-Stokes step on the device SIPG solves.

The production caller of the SIPG path (``src/ddg/dg2d/incompressible_ns.py``
in the reference): per time step one pressure Poisson solve and two viscous
Helmholtz solves (one per velocity component), each through this package's
device operators.  The operators stay resident across steps (one handle per
(mesh, BC tags, penalty) through ``Mesh2D.device_operator``; the block-Jacobi
inverses and captured CG graphs are rebuilt only when ``alpha`` changes, at
the BDF1 -> BDF2 switch), and the viscous solves warm-start from the previous
velocity as in the reference.

The explicit parts of the step -- the Lax-Friedrichs advection term, the
divergence and gradient, and the consistent pressure-Neumann data -- are
elementwise float64 numpy on the host, restated from the reference
(``incompressible_ns.py:100-320``, ``maxwell.py:31-42``); they are not part
of the SIPG solve path this package accelerates.  Curved meshes run with or
without ``cub``; velocity reconstruction and the penalty post-projection are
not supported.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .mesh import Mesh2D
from .sipg import (BC_DIRICHLET, BC_INTERIOR, BC_NEUMANN, IterativeConfig, factor_sipg_2d,
                   factor_sipg_helmholtz_2d, solve_sipg_helmholtz_2d, solve_sipg_poisson_2d)

# INS boundary codes (incompressible_ns.py:67-71)
BC_INS_INTERIOR = 0
BC_INS_INFLOW = 1
BC_INS_OUTFLOW = 2
BC_INS_WALL = 3
BC_INS_OBSTACLE = 4


def pressure_bc_types_from_ins(ins_bc_types):
    """Inflow / wall / obstacle -> Neumann; outflow -> Dirichlet
    (``incompressible_ns.py:74-82``)."""
    b = np.asarray(ins_bc_types)
    neu = (b == BC_INS_INFLOW) | (b == BC_INS_WALL) | (b == BC_INS_OBSTACLE)
    return np.where(b == BC_INS_OUTFLOW, BC_DIRICHLET, np.where(neu, BC_NEUMANN, BC_INTERIOR)).astype(np.int32)


def viscous_bc_types_from_ins(ins_bc_types):
    """Inflow / wall / obstacle -> Dirichlet; outflow -> Neumann
    (``incompressible_ns.py:85-97``)."""
    b = np.asarray(ins_bc_types)
    dirf = (b == BC_INS_INFLOW) | (b == BC_INS_WALL) | (b == BC_INS_OBSTACLE)
    return np.where(dirf, BC_DIRICHLET, np.where(b == BC_INS_OUTFLOW, BC_NEUMANN, BC_INTERIOR)).astype(np.int32)


@dataclass(frozen=True)
class BDFCoeffs:
    """Backward-difference / extrapolation coefficients (``:322-332``)."""
    g0: float
    a0: float
    a1: float
    b0: float
    b1: float


BDF1 = BDFCoeffs(g0=1.0, a0=1.0, a1=0.0, b0=1.0, b1=0.0)
BDF2 = BDFCoeffs(g0=1.5, a0=2.0, a1=-0.5, b0=2.0, b1=-1.0)


# --------------------------------------------------------- explicit parts

def grad_2d(mesh: Mesh2D, u):
    """Physical gradient (``maxwell.py:31-35``)."""
    ur, us = mesh.Dr @ u, mesh.Ds @ u
    return mesh.rx * ur + mesh.sx * us, mesh.ry * ur + mesh.sy * us


def curl_z_2d(mesh: Mesh2D, ux, uy):
    """d uy/dx - d ux/dy (``maxwell.py:38-42``)."""
    ux_y = mesh.ry * (mesh.Dr @ ux) + mesh.sy * (mesh.Ds @ ux)
    uy_x = mesh.rx * (mesh.Dr @ uy) + mesh.sx * (mesh.Ds @ uy)
    return uy_x - ux_y


def _div_2d(mesh: Mesh2D, fx, fy):
    """Strong-form divergence per element (``:100-110``)."""
    return (mesh.rx * (mesh.Dr @ fx) + mesh.sx * (mesh.Ds @ fx)
            + mesh.ry * (mesh.Dr @ fy) + mesh.sy * (mesh.Ds @ fy))


def _face_flat(mesh: Mesh2D, a):
    return np.asarray(a).reshape(-1, order="F")


def _bc_facenodes(mesh: Mesh2D, ins_bc_types):
    """(K, 3) codes -> one per face node, face-trace flat order (``:269-281``)."""
    b = np.asarray(ins_bc_types).T.astype(np.int32)
    return np.broadcast_to(b[None], (mesh.Nfp, 3, mesh.K)).reshape(-1, order="F")


def ns_advection_2d(mesh: Mesh2D, ux, uy, *, ins_bc_types, bc_ux=None, bc_uy=None,
                    velocity_reconstruction=None, convective_form: str = "conservative"):
    """N(U) = div(U (x) U) with the local Lax-Friedrichs face flux, lambda
    taken as the maximum over each face's nodes (``:116-266``); the "+" trace
    on inflow / wall / obstacle faces is the prescribed velocity."""
    if velocity_reconstruction is not None:
        raise ValueError("velocity_reconstruction is not supported")
    ux, uy = np.asarray(ux, dtype=np.float64), np.asarray(uy, dtype=np.float64)
    if convective_form == "conservative":
        nx_vol = _div_2d(mesh, ux * ux, ux * uy)
        ny_vol = _div_2d(mesh, ux * uy, uy * uy)
    elif convective_form == "skew_symmetric":
        dxx, dxy = grad_2d(mesh, ux)
        dyx, dyy = grad_2d(mesh, uy)
        nx_vol = 0.5 * (_div_2d(mesh, ux * ux, ux * uy) + ux * dxx + uy * dxy)
        ny_vol = 0.5 * (_div_2d(mesh, ux * uy, uy * uy) + ux * dyx + uy * dyy)
    else:
        raise ValueError(f"convective_form must be 'conservative' or 'skew_symmetric', got {convective_form!r}")
    uxf, uyf = ux.T.reshape(-1), uy.T.reshape(-1)
    uxM, uyM = uxf[mesh.vmapM], uyf[mesh.vmapM]
    bcn = _bc_facenodes(mesh, ins_bc_types)
    use_bc = (bcn == BC_INS_INFLOW) | (bcn == BC_INS_WALL) | (bcn == BC_INS_OBSTACLE)
    gx = np.asarray(bc_ux).T.reshape(-1)[mesh.vmapM] if bc_ux is not None else 0.0
    gy = np.asarray(bc_uy).T.reshape(-1)[mesh.vmapM] if bc_uy is not None else 0.0
    uxP = np.where(use_bc, gx, uxf[mesh.vmapP])
    uyP = np.where(use_bc, gy, uyf[mesh.vmapP])
    nx, ny = _face_flat(mesh, mesh.nx), _face_flat(mesh, mesh.ny)
    lam = np.maximum(np.abs(uxM * nx + uyM * ny), np.abs(uxP * nx + uyP * ny))
    lam = np.repeat(lam.reshape((mesh.Nfp, 3 * mesh.K), order="F").max(axis=0), mesh.Nfp)
    fx = 0.5 * (-nx * (uxM * uxM - uxP * uxP) - ny * (uxM * uyM - uxP * uyP) - lam * (uxP - uxM))
    fy = 0.5 * (-nx * (uxM * uyM - uxP * uyP) - ny * (uyM * uyM - uyP * uyP) - lam * (uyP - uyM))
    shape = (mesh.Nfp * 3, mesh.K)
    nux = nx_vol + mesh.LIFT @ (mesh.Fscale * fx.reshape(shape, order="F"))
    nuy = ny_vol + mesh.LIFT @ (mesh.Fscale * fy.reshape(shape, order="F"))
    return nux, nuy


def ns_pressure_neumann_data(mesh: Mesh2D, ux, uy, Nux, Nuy, *, nu: float):
    """dp/dn = -n.(N(U) + nu curl curl U) at the face nodes, own-side trace
    (``:284-319``)."""
    w = curl_z_2d(mesh, ux, uy)
    dwdx, dwdy = grad_2d(mesh, w)
    rx = (-np.asarray(Nux) - nu * dwdy).T.reshape(-1)
    ry = (-np.asarray(Nuy) + nu * dwdx).T.reshape(-1)
    d = _face_flat(mesh, mesh.nx) * rx[mesh.vmapM] + _face_flat(mesh, mesh.ny) * ry[mesh.vmapM]
    return d.reshape((mesh.Nfp * 3, mesh.K), order="F")


# -------------------------------------------------------------- operators

@dataclass
class INSOperators:
    """The step's linear-system data (``:400-412``): BC tags, alpha, and
    (only when built) dense factors for the direct path."""
    pressure_factored: tuple | None
    viscous_factored: tuple | None
    pressure_bc_types: np.ndarray
    viscous_bc_types: np.ndarray
    alpha: float


def build_ins_operators(mesh: Mesh2D, *, dt: float, nu: float, g0: float, ins_bc_types, tau_scale: float = 200.0,
                        skip_factor: bool = False, cub=None) -> INSOperators:
    """``build_ins_operators`` (``:415-458``).  With ``skip_factor`` (the
    iterative path) nothing dense is built; the device operators are created
    lazily by the solves and kept resident on the mesh.  ``cub`` (curved
    meshes) factors the cubature operators, as the reference does."""
    p_bc = pressure_bc_types_from_ins(ins_bc_types)
    v_bc = viscous_bc_types_from_ins(ins_bc_types)
    alpha = g0 / (nu * dt)
    p_sing = not bool(np.any(p_bc == BC_DIRICHLET))
    if skip_factor:
        pf = vf = None
    else:
        pf = factor_sipg_2d(mesh, bc_types=p_bc, tau_scale=tau_scale, regularize=p_sing, cub=cub)
        vf = factor_sipg_helmholtz_2d(mesh, alpha=alpha, nu=nu, bc_types=v_bc, tau_scale=tau_scale, cub=cub)
    return INSOperators(pf, vf, p_bc, v_bc, alpha)


def make_ins_mg_preconditioners(mesh: Mesh2D, *, dt: float, nu: float, g0: float, ins_bc_types,
                                tau_scale: float = 200.0, p_coarse: int = 1, nu_smooth: int = 2,
                                omega: float = 0.7):
    """Device p-multigrid V-cycles for the pressure Poisson and the viscous
    Helmholtz (``:461-506``)."""
    from .multigrid import make_sipg_mg_preconditioner
    p_bc = pressure_bc_types_from_ins(ins_bc_types)
    v_bc = viscous_bc_types_from_ins(ins_bc_types)
    alpha = g0 / (nu * dt)
    p_sing = not bool(np.any(p_bc == BC_DIRICHLET))
    pp = make_sipg_mg_preconditioner(mesh, bc_types=p_bc, tau_scale=tau_scale, alpha=0.0, p_coarse=p_coarse,
                                     nu_smooth=nu_smooth, omega=omega, regularize=p_sing)
    vp = make_sipg_mg_preconditioner(mesh, bc_types=v_bc, tau_scale=tau_scale, alpha=alpha, p_coarse=p_coarse,
                                     nu_smooth=nu_smooth, omega=omega)
    return pp, vp


# ------------------------------------------------------------------- step

def ns_step_2d(mesh: Mesh2D, ux_n, uy_n, ux_old, uy_old, Nux_old, Nuy_old, dpdn_old, *, dt: float, nu: float,
               bdf: BDFCoeffs, ops: INSOperators, ins_bc_types, bc_ux, bc_uy, p_dir=None, q_ux_neu=None,
               q_uy_neu=None, tau_scale: float = 200.0, penalty_factored=None, penalty_iterative=None,
               iterative: IterativeConfig | None = None, pressure_preconditioner=None,
               viscous_preconditioner=None, velocity_reconstruction=None, convective_form: str = "conservative",
               body_force=None, cub=None):
    """One dual-splitting step (``:509-666``): advection and BDF
    extrapolation, pressure Poisson with the extrapolated consistent Neumann
    data, pressure-gradient correction, then one viscous Helmholtz solve per
    velocity component warm-started from ``ux_n`` / ``uy_n``.  With ``cub``
    (curved meshes) the three solves use the cubature operator and mass, as
    ``_pressure_solve`` / ``_viscous_solve`` do (``:669-805``).  Returns
    ``(ux, uy, p, Nux, Nuy, dpdn)``."""
    if penalty_factored is not None or penalty_iterative is not None:
        raise ValueError("the penalty post-projection is not supported")
    g0 = bdf.g0
    ux_n, uy_n = np.asarray(ux_n, dtype=np.float64), np.asarray(uy_n, dtype=np.float64)
    nux, nuy = ns_advection_2d(mesh, ux_n, uy_n, ins_bc_types=ins_bc_types, bc_ux=bc_ux, bc_uy=bc_uy,
                               velocity_reconstruction=velocity_reconstruction, convective_form=convective_form)
    ux_t = (bdf.a0 * ux_n + bdf.a1 * np.asarray(ux_old) - dt * (bdf.b0 * nux + bdf.b1 * np.asarray(Nux_old))) / g0
    uy_t = (bdf.a0 * uy_n + bdf.a1 * np.asarray(uy_old) - dt * (bdf.b0 * nuy + bdf.b1 * np.asarray(Nuy_old))) / g0
    if body_force is not None:
        ux_t = ux_t + (dt / g0) * np.asarray(body_force[0])
        uy_t = uy_t + (dt / g0) * np.asarray(body_force[1])
    p_source = -(g0 / dt) * _div_2d(mesh, ux_t, uy_t)
    dpdn_n = ns_pressure_neumann_data(mesh, ux_n, uy_n, nux, nuy, nu=nu)
    dpdn_x = bdf.b0 * dpdn_n + bdf.b1 * np.asarray(dpdn_old)
    p = solve_sipg_poisson_2d(mesh, p_source, bc_types=ops.pressure_bc_types, u_dir=p_dir, q_neu=dpdn_x,
                              tau_scale=tau_scale, A_factored=ops.pressure_factored, iterative=iterative,
                              preconditioner=pressure_preconditioner, cub=cub)
    dpdx, dpdy = grad_2d(mesh, p)
    ux_tt = ux_t - (dt / g0) * dpdx
    uy_tt = uy_t - (dt / g0) * dpdy
    a = ops.alpha
    ux = solve_sipg_helmholtz_2d(mesh, a * ux_tt, alpha=a, nu=nu, bc_types=ops.viscous_bc_types, u_dir=bc_ux,
                                 q_neu=q_ux_neu, tau_scale=tau_scale, A_factored=ops.viscous_factored,
                                 iterative=iterative, x0=ux_n, preconditioner=viscous_preconditioner, cub=cub)
    uy = solve_sipg_helmholtz_2d(mesh, a * uy_tt, alpha=a, nu=nu, bc_types=ops.viscous_bc_types, u_dir=bc_uy,
                                 q_neu=q_uy_neu, tau_scale=tau_scale, A_factored=ops.viscous_factored,
                                 iterative=iterative, x0=uy_n, preconditioner=viscous_preconditioner, cub=cub)
    return ux, uy, p, nux, nuy, dpdn_n
