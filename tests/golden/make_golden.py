"""Generate golden fixtures from the UNMODIFIED reference (ddg) for the SIPG path.

TEST INFRASTRUCTURE ONLY.  Run here, where the reference sources are present::

    python tests/golden/make_golden.py [/path/to/ddg/src]

(default source path: ``/root/reference/src``).  The reference's own modules
``ddg.dg1d.reference``, ``ddg.dg2d.reference``, ``ddg.dg2d.mesh``,
``ddg.dg2d.sipg``, ``ddg.dg2d.multigrid`` and ``ddg.dg2d.refinement`` are
imported unchanged over the numpy-backed JAX stand-in in ``refshim.py``
(JAX itself cannot be installed in this container).  Every number written
here is computed by the reference's code path:

* reference elements N = 1..6: ``equilateral_nodes_2d``, ``vandermonde_2d``,
  ``d_matrices_2d``, ``lift_2d``, ``face_masks_2d`` through ``build_mesh_2d``,
  plus ``sipg._local_mass`` and ``sipg._face_1d_mass_matrices``;
* meshes: ``uniform_rectangle_mesh_2d`` + ``build_mesh_2d`` (connectivity,
  node maps, geometric factors, normals), a vertex-perturbed mesh with
  shuffled element order, and a ``RefinementForest`` hierarchy;
* operator applies: ``sipg_apply_2d`` (``jax.grad`` of ``sipg_bilinear_form``)
  for random ``u`` under several boundary-condition sets and penalties, with
  and without ``u_dir``; the dense ``sipg_matrix_2d`` and
  ``sipg_helmholtz_matrix_2d`` of a tiny mesh;
* loads: ``sipg_dirichlet_load_2d`` and ``sipg_neumann_load_2d``;
* block diagonals: ``extract_block_diag_matfree`` and ``_color_elements``;
* solves: ``solve_sipg_poisson_2d`` by matrix-free CG and by dense LU on the
  plain manufactured-solution workload (12 x 12 quads, N = 4,
  ``tau_scale = 0.5``), the singular (all-Neumann) branch with its epsilon
  shift, ``solve_sipg_helmholtz_2d`` with the block-Jacobi preconditioner,
  and CG preconditioned by the p- and hp-multigrid V-cycles, with the
  iteration counts the CG loop took.

* one dual-splitting Navier-Stokes step (``incompressible_ns.ns_step_2d``) on
  the reference test's channel, by direct LU and by multigrid-preconditioned
  CG, and a second (BDF2) step.

* curved elements (``curved.npz``, also alone with ``--only curved``): the
  hole-bounded builders ``rectangle_with_square_hole_mesh_2d`` and
  ``channel_with_circle_mesh_2d``, the boundary bending of
  ``apply_circular_hole_2d``, ``attach_cubature``, ``per_element_mass``,
  ``cubature_mass_apply``, ``sipg_apply_2d`` with and without ``cub`` on the
  curved meshes, the loads there, block diagonals by coloured probing, and
  ``solve_sipg_poisson_2d`` / ``solve_sipg_helmholtz_2d`` with ``cub`` by LU
  and CG.

Outputs: ``refelem.npz``, ``meshes.npz``, ``applies.npz``, ``solves.npz``,
``ins.npz``, ``curved.npz`` next to this file.
"""

from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import refshim  # noqa: E402

MESH_FIELDS = ("VX", "VY", "EToV", "x", "y", "rx", "sx", "ry", "sy", "J", "nx", "ny", "sJ",
               "Fscale", "EToE", "EToF", "vmapM", "vmapP", "vmapB", "mapB")


def _a(x):
    return np.asarray(x)


def boundary_faces(m):
    K = int(m.K)
    return _a(m.EToE) == np.arange(K)[:, None]


def bc_sets(m, rng):
    """Named (K, 3) int32 boundary-condition arrays for a mesh."""
    K = int(m.K)
    isb = boundary_faces(m)
    nx = _a(m.nx).reshape((int(m.Nfp), 3, K), order="F")[0].T
    rnd = rng.integers(1, 3, size=(K, 3))
    return {
        "dirichlet": np.where(isb, 1, 0).astype(np.int32),
        "neumann": np.where(isb, 2, 0).astype(np.int32),
        "dir_x_neu_y": np.where(isb, np.where(np.abs(nx) > 0.5, 1, 2), 0).astype(np.int32),
        "random": np.where(isb, rnd, 0).astype(np.int32),
    }


CUB_FIELDS = ("r", "s", "w", "Lq", "Drq", "Dsq", "J", "rx", "sx", "ry", "sy", "face_w", "face_Lq",
              "face_L1d", "face_sJ", "face_nx", "face_ny")


def curved_fixtures(imp) -> dict:
    """Fixtures of the curved-element (cubature) branch."""
    rmesh = imp("ddg.dg2d.mesh")
    rsipg = imp("ddg.dg2d.sipg")
    rcur = imp("ddg.dg2d.curved")
    rcub = imp("ddg.dg2d.cubature")
    IC = rsipg.IterativeConfig
    out = {}
    t0 = time.time()
    rng = np.random.default_rng(31)
    # the reference test's annulus (square hole bent onto its inscribed
    # circle), coarser, and a cylinder-in-channel O-grid mesh
    VX, VY, E = rmesh.rectangle_with_square_hole_mesh_2d(-2.0, 2.0, -2.0, 2.0, 8, 8, -0.5, 0.5, -0.5, 0.5)
    base = rmesh.build_mesh_2d(VX, VY, E, 3)
    ann = rcur.apply_circular_hole_2d(base, cx=0.0, cy=0.0, radius=0.5, detection_tol=0.5)
    VX2, VY2, E2 = rmesh.channel_with_circle_mesh_2d(0.0, 2.0, 0.0, 2.0, 8, 8, cx=1.0, cy=1.0, radius=0.25,
                                                     R_outer=0.5, n_radial=3, radial_growth=1.3)
    base2 = rmesh.build_mesh_2d(VX2, VY2, E2, 4)
    cyl = rcur.apply_circular_hole_2d(base2, cx=1.0, cy=1.0, radius=0.25, detection_tol=0.1)
    meshes = {"annulus8_N3": (ann, (VX, VY, E)), "cyl8_N4": (cyl, (VX2, VY2, E2))}
    # the other degrees on the same annulus
    for Nx in (1, 2, 5):
        mx = rcur.apply_circular_hole_2d(rmesh.build_mesh_2d(VX, VY, E, Nx), cx=0.0, cy=0.0, radius=0.5,
                                         detection_tol=0.5)
        meshes[f"annulus8_N{Nx}"] = (mx, (VX, VY, E))
    cubs = {}
    for name, (m, (vx, vy, ee)) in meshes.items():
        out[f"{name}/VX"], out[f"{name}/VY"], out[f"{name}/EToV"] = _a(vx), _a(vy), _a(ee)
        for f in MESH_FIELDS:
            out[f"{name}/mesh/{f}"] = _a(getattr(m, f))
        out[f"{name}/N"] = np.int64(m.N)
        cub = rcub.attach_cubature(m)
        cubs[name] = cub
        for f in CUB_FIELDS:
            out[f"{name}/cub/{f}"] = _a(getattr(cub, f))
        K, Np = int(m.K), int(m.Np)
        fld = rng.standard_normal((Np, K))
        out[f"{name}/mass/f"] = fld
        out[f"{name}/mass/Mf"] = _a(rcub.cubature_mass_apply(cub, fld))
        if name == "annulus8_N3":
            out[f"{name}/mass/MK"] = _a(rcub.per_element_mass(cub))
        sets = bc_sets(m, rng)
        for bname in ("dirichlet", "random", "neumann"):
            for tau in (200.0, 0.5):
                bc = sets[bname]
                u = rng.standard_normal((Np, K))
                key = f"{name}/apply/{bname}/tau{tau:g}"
                out[key + "/bc"] = bc
                out[key + "/u"] = u
                out[key + "/Au_nodal"] = _a(rsipg.sipg_apply_2d(m, u, bc_types=bc, tau_scale=tau))
                out[key + "/Au_cub"] = _a(rsipg.sipg_apply_2d(m, u, bc_types=bc, tau_scale=tau, cub=cub))
        bc = sets["random"]
        u = rng.standard_normal((Np, K))
        ud = np.sin(1.3 * _a(m.x)) * np.cos(0.7 * _a(m.y))
        q = rng.standard_normal((3 * int(m.Nfp), K))
        out[f"{name}/udir/bc"] = bc
        out[f"{name}/udir/u"] = u
        out[f"{name}/udir/u_dir"] = ud
        out[f"{name}/udir/q_neu"] = q
        out[f"{name}/udir/Au_cub"] = _a(rsipg.sipg_apply_2d(m, u, bc_types=bc, u_dir=ud, tau_scale=200.0, cub=cub))
        out[f"{name}/udir/LD"] = _a(rsipg.sipg_dirichlet_load_2d(m, ud, bc_types=bc, tau_scale=200.0))
        out[f"{name}/udir/LN"] = _a(rsipg.sipg_neumann_load_2d(m, q, bc_types=bc))
        print(f"curved {name} applies {time.time() - t0:.1f}s", flush=True)

    # block diagonals (coloured probing) of the nodal and the cubature operator
    m = ann
    cub = cubs["annulus8_N3"]
    bc = bc_sets(m, rng)["dirichlet"]
    K, Np = int(m.K), int(m.Np)
    for tag, c in (("nodal", None), ("cub", cub)):
        def apply_flat(v, c=c):
            return rsipg.sipg_apply_2d(m, v.reshape(K, Np).T, bc_types=bc, tau_scale=200.0, cub=c).T.reshape(-1)
        out[f"annulus8_N3/blocks/{tag}"] = _a(rsipg.extract_block_diag_matfree(apply_flat, m))
    out["annulus8_N3/blocks/bc"] = bc

    # the reference test's manufactured Poisson solve, all-Dirichlet, with and
    # without cubature, by LU; with cubature also by CG
    ue = np.sin(np.pi * _a(m.x) / 4) * np.sin(np.pi * _a(m.y) / 4)
    src = 2 * (np.pi / 4) ** 2 * ue
    out["annulus8_N3/solve/bc"] = bc
    out["annulus8_N3/solve/u_exact"] = ue
    out["annulus8_N3/solve/u_lu_nodal"] = _a(rsipg.solve_sipg_poisson_2d(m, src, bc_types=bc, u_dir=ue))
    out["annulus8_N3/solve/u_lu_cub"] = _a(rsipg.solve_sipg_poisson_2d(m, src, bc_types=bc, u_dir=ue, cub=cub))
    x = rsipg.solve_sipg_poisson_2d(m, src, bc_types=bc, u_dir=ue, cub=cub, iterative=IC(tol=1e-10, maxiter=5000))
    out["annulus8_N3/solve/u_cg_cub"] = _a(x)
    out["annulus8_N3/solve/cg_iterations"] = np.int64(refshim.cg_last_iterations())
    print(f"curved poisson CG {refshim.cg_last_iterations()} its {time.time() - t0:.1f}s", flush=True)
    # Helmholtz with cubature (mass by cubature), mixed BCs, CG and LU
    m = cyl
    cub = cubs["cyl8_N4"]
    bc = bc_sets(m, rng)["random"]
    rhs = np.cos(2.0 * _a(m.x)) * np.sin(1.5 * _a(m.y)) + 0.2
    out["cyl8_N4/helm/bc"] = bc
    out["cyl8_N4/helm/rhs"] = rhs
    x = rsipg.solve_sipg_helmholtz_2d(m, rhs, alpha=5.0, nu=1.0, bc_types=bc, tau_scale=0.5, cub=cub,
                                      iterative=IC(tol=1e-10, maxiter=8000))
    out["cyl8_N4/helm/u_cg"] = _a(x)
    out["cyl8_N4/helm/cg_iterations"] = np.int64(refshim.cg_last_iterations())
    print(f"curved helmholtz CG {refshim.cg_last_iterations()} its {time.time() - t0:.1f}s", flush=True)
    out["cyl8_N4/helm/u_lu"] = _a(rsipg.solve_sipg_helmholtz_2d(m, rhs, alpha=5.0, nu=1.0, bc_types=bc,
                                                                 tau_scale=0.5, cub=cub))
    # one dual-splitting step on the cylinder mesh (N = 3) with cubature:
    # inflow x = 0, outflow x = 2, walls y = 0, 2, the cylinder an obstacle;
    # direct LU and matrix-free CG
    rins = imp("ddg.dg2d.incompressible_ns")
    VX2, VY2, E2 = _a(out["cyl8_N4/VX"]), _a(out["cyl8_N4/VY"]), _a(out["cyl8_N4/EToV"])
    m3 = rcur.apply_circular_hole_2d(rmesh.build_mesh_2d(VX2, VY2, E2, 3), cx=1.0, cy=1.0, radius=0.25,
                                     detection_tol=0.1)
    cub3 = rcub.attach_cubature(m3)
    K3 = int(m3.K)
    isb = boundary_faces(m3)
    xf = _a(m3.x)[_a(m3.Fmask)]                                    # (Nfp, 3, K)
    yf = _a(m3.y)[_a(m3.Fmask)]
    on = lambda a, v: np.all(np.abs(a - v) < 1e-7, axis=0).T       # noqa: E731  (K, 3)
    code = np.where(on(xf, 0.0), rins.BC_INS_INFLOW,
                    np.where(on(xf, 2.0), rins.BC_INS_OUTFLOW,
                             np.where(on(yf, 0.0) | on(yf, 2.0), rins.BC_INS_WALL, rins.BC_INS_OBSTACLE)))
    ins_bc = np.where(isb, code, rins.BC_INS_INTERIOR).astype(np.int32)
    x3, y3 = _a(m3.x), _a(m3.y)
    ux0 = 0.2 * y3 * (2.0 - y3)
    uy0 = 0.05 * np.sin(np.pi * x3) * y3 * (2.0 - y3)
    bcux = np.where(np.abs(x3) < 1e-9, y3 * (2.0 - y3), 0.0)
    zero = np.zeros_like(x3)
    dt, nu = 0.01, 0.05
    nxo, nyo = rins.ns_advection_2d(m3, ux0, uy0, ins_bc_types=ins_bc, bc_ux=bcux, bc_uy=zero)
    dpdn0 = np.zeros((3 * int(m3.Nfp), K3))
    args = (m3, ux0, uy0, ux0, uy0, nxo, nyo, dpdn0)
    kw = dict(dt=dt, nu=nu, bdf=rins.BDF1, ins_bc_types=ins_bc, bc_ux=bcux, bc_uy=zero, cub=cub3)
    ops = rins.build_ins_operators(m3, dt=dt, nu=nu, g0=1.0, ins_bc_types=ins_bc, cub=cub3)
    res_lu = rins.ns_step_2d(*args, ops=ops, **kw)
    ops_mf = rins.build_ins_operators(m3, dt=dt, nu=nu, g0=1.0, ins_bc_types=ins_bc, skip_factor=True, cub=cub3)
    res_cg = rins.ns_step_2d(*args, ops=ops_mf, iterative=IC(tol=1e-12, maxiter=20000), **kw)
    out["ins_cyl_N3/ins_bc"] = ins_bc
    out["ins_cyl_N3/ux0"], out["ins_cyl_N3/uy0"], out["ins_cyl_N3/bc_ux"] = ux0, uy0, bcux
    out["ins_cyl_N3/Nux_old"], out["ins_cyl_N3/Nuy_old"] = _a(nxo), _a(nyo)
    for tag, res in (("lu", res_lu), ("cg", res_cg)):
        for name, v in zip(("ux", "uy", "p", "Nux", "Nuy", "dpdn"), res):
            out[f"ins_cyl_N3/{tag}/{name}"] = _a(v)
    print(f"curved done {time.time() - t0:.1f}s", flush=True)
    return out


def main(src: str, only: str | None = None) -> None:
    imp = refshim.install(src)
    if only == "curved":
        d = curved_fixtures(imp)
        np.savez_compressed(os.path.join(HERE, "curved.npz"), **{k: np.asarray(v) for k, v in d.items()})
        return
    rmesh = imp("ddg.dg2d.mesh")
    rsipg = imp("ddg.dg2d.sipg")
    rmg = imp("ddg.dg2d.multigrid")
    rref = imp("ddg.dg2d.refinement")
    t0 = time.time()
    out_ref, out_mesh, out_app, out_sol = {}, {}, {}, {}

    # ---- reference elements
    for N in range(1, 7):
        VX, VY, E = rmesh.uniform_rectangle_mesh_2d(0.0, 1.0, 0.0, 1.0, 1, 1)
        m = rmesh.build_mesh_2d(VX, VY, E, N)
        for f in ("r", "s", "V", "invV", "Dr", "Ds", "LIFT", "Fmask"):
            out_ref[f"N{N}_{f}"] = _a(getattr(m, f))
        out_ref[f"N{N}_M"] = _a(rsipg._local_mass(m))
        out_ref[f"N{N}_m1d"] = _a(rsipg._face_1d_mass_matrices(m))

    # ---- meshes
    meshes = {}
    VX, VY, E = rmesh.uniform_rectangle_mesh_2d(0.0, 1.0, 0.0, 1.0, 12, 12)
    meshes["plain12_N4"] = rmesh.build_mesh_2d(VX, VY, E, 4)
    VX, VY, E = rmesh.uniform_rectangle_mesh_2d(0.0, 1.0, 0.0, 2.0, 4, 8)
    meshes["rect4x8_N3"] = rmesh.build_mesh_2d(VX, VY, E, 3)
    # perturbed interior vertices + shuffled element order (seeded)
    rng = np.random.default_rng(2024)
    VX, VY, E = rmesh.uniform_rectangle_mesh_2d(0.0, 1.0, 0.0, 1.0, 5, 5)
    VX, VY, E = _a(VX).copy(), _a(VY).copy(), _a(E).copy()
    inner = (VX > 1e-12) & (VX < 1 - 1e-12) & (VY > 1e-12) & (VY < 1 - 1e-12)
    h = 1.0 / 5
    VX[inner] += 0.2 * h * rng.uniform(-1, 1, inner.sum())
    VY[inner] += 0.2 * h * rng.uniform(-1, 1, inner.sum())
    E = E[rng.permutation(E.shape[0])]
    meshes["perturbed5_N2"] = rmesh.build_mesh_2d(VX, VY, E, 2)
    # forest refinement (leaf-ordered active mesh), 2 uniform levels on [0,1]x[0,2]
    VX, VY, E = rmesh.uniform_rectangle_mesh_2d(0.0, 1.0, 0.0, 2.0, 2, 3)
    base = rmesh.build_mesh_2d(VX, VY, E, 4)
    hm = rmg._build_h_meshes(base, 2)
    meshes["refined2x3x2_N4"] = hm[-1]
    VX, VY, E = rmesh.uniform_rectangle_mesh_2d(0.0, 1.0, 0.0, 1.0, 2, 2)
    meshes["tiny2_N2"] = rmesh.build_mesh_2d(VX, VY, E, 2)
    for name, m in meshes.items():
        for f in MESH_FIELDS:
            out_mesh[f"{name}/{f}"] = _a(getattr(m, f))
        out_mesh[f"{name}/N"] = np.int64(m.N)
    print(f"meshes done {time.time() - t0:.1f}s", flush=True)

    # ---- applies
    rng = np.random.default_rng(7)
    for name, m in meshes.items():
        sets = bc_sets(m, rng)
        if name == "plain12_N4":
            combos = [("dirichlet", 0.5), ("dir_x_neu_y", 0.5), ("neumann", 200.0)]
        else:
            combos = [(b, t) for b in sets for t in (200.0, 0.5)]
        for bname, tau in combos:
            bc = sets[bname]
            u = rng.standard_normal((int(m.Np), int(m.K)))
            y = _a(rsipg.sipg_apply_2d(m, u, bc_types=bc, tau_scale=tau))
            key = f"{name}/{bname}/tau{tau:g}"
            out_app[key + "/bc"] = bc
            out_app[key + "/u"] = u
            out_app[key + "/Au"] = y
        # affine apply with u_dir on the Dirichlet set
        bc = sets["dir_x_neu_y"]
        u = rng.standard_normal((int(m.Np), int(m.K)))
        ud = np.sin(np.pi * _a(m.x)) * np.cos(np.pi * _a(m.y))
        y = _a(rsipg.sipg_apply_2d(m, u, bc_types=bc, u_dir=ud, tau_scale=200.0))
        out_app[f"{name}/udir/bc"] = bc
        out_app[f"{name}/udir/u"] = u
        out_app[f"{name}/udir/u_dir"] = ud
        out_app[f"{name}/udir/Au"] = y
        # loads
        q = rng.standard_normal((3 * int(m.Nfp), int(m.K)))
        out_app[f"{name}/loads/bc"] = bc
        out_app[f"{name}/loads/u_dir"] = ud
        out_app[f"{name}/loads/q_neu"] = q
        out_app[f"{name}/loads/LD"] = _a(rsipg.sipg_dirichlet_load_2d(m, ud, bc_types=bc, tau_scale=200.0))
        out_app[f"{name}/loads/LN"] = _a(rsipg.sipg_neumann_load_2d(m, q, bc_types=bc))
    print(f"applies done {time.time() - t0:.1f}s", flush=True)

    # ---- dense matrices of a tiny mesh
    m = meshes["tiny2_N2"]
    bc = bc_sets(m, rng)["dir_x_neu_y"]
    out_app["tiny2_N2/dense/bc"] = bc
    out_app["tiny2_N2/dense/A"] = _a(rsipg.sipg_matrix_2d(m, bc_types=bc, tau_scale=200.0))
    out_app["tiny2_N2/dense/H"] = _a(rsipg.sipg_helmholtz_matrix_2d(m, alpha=5.0, nu=1.0, bc_types=bc,
                                                                    tau_scale=200.0))

    # ---- block diagonals by coloured probing
    for name in ("rect4x8_N3", "perturbed5_N2"):
        m = meshes[name]
        bc = bc_sets(m, rng)["dir_x_neu_y"]
        col, ncol = rsipg._color_elements(m)
        out_app[f"{name}/blocks/colors"] = _a(col)
        out_app[f"{name}/blocks/ncolors"] = np.int64(ncol)
        Np, K = int(m.Np), int(m.K)

        def apply_flat(v, m=m, bc=bc):
            return rsipg.sipg_apply_2d(m, v.reshape(K, Np).T, bc_types=bc, tau_scale=200.0).T.reshape(-1)
        out_app[f"{name}/blocks/bc"] = bc
        out_app[f"{name}/blocks/B"] = _a(rsipg.extract_block_diag_matfree(apply_flat, m))
    print(f"dense + blocks done {time.time() - t0:.1f}s", flush=True)

    # ---- solves
    IC = rsipg.IterativeConfig
    m = meshes["plain12_N4"]
    bc = bc_sets(m, rng)["dirichlet"]
    ue = np.sin(np.pi * _a(m.x)) * np.sin(np.pi * _a(m.y))
    f = 2 * np.pi ** 2 * ue
    x = rsipg.solve_sipg_poisson_2d(m, f, bc_types=bc, u_dir=ue, tau_scale=0.5, iterative=IC(tol=1e-9))
    out_sol["plain/bc"] = bc
    out_sol["plain/u_cg"] = _a(x)
    out_sol["plain/cg_iterations"] = np.int64(refshim.cg_last_iterations())
    print(f"plain CG {refshim.cg_last_iterations()} its {time.time() - t0:.1f}s", flush=True)
    x = rsipg.solve_sipg_poisson_2d(m, f, bc_types=bc, u_dir=ue, tau_scale=0.5)
    out_sol["plain/u_lu"] = _a(x)
    print(f"plain LU done {time.time() - t0:.1f}s", flush=True)

    # singular all-Neumann Poisson (eps shift + mean deflation branch)
    m = meshes["rect4x8_N3"]
    bc = bc_sets(m, rng)["neumann"]
    src = np.cos(np.pi * _a(m.x)) * np.cos(0.5 * np.pi * _a(m.y)) + 0.3
    x = rsipg.solve_sipg_poisson_2d(m, src, bc_types=bc, tau_scale=200.0, iterative=IC(tol=1e-10))
    out_sol["singular/bc"] = bc
    out_sol["singular/source"] = src
    out_sol["singular/u"] = _a(x)
    out_sol["singular/cg_iterations"] = np.int64(refshim.cg_last_iterations())

    # Helmholtz, Dirichlet x / Neumann y, block-Jacobi PCG (precision workload shape, small)
    VX, VY, E = rmesh.uniform_rectangle_mesh_2d(0.0, 1.0, 0.0, 1.0, 16, 16)
    m = rmesh.build_mesh_2d(VX, VY, E, 4)
    bc = bc_sets(m, rng)["dir_x_neu_y"]
    frng = np.random.default_rng(0)
    kx = frng.integers(1, 7, 8)
    ky = frng.integers(1, 7, 8)
    amp = frng.standard_normal(8)
    rhs = sum(a * np.sin(np.pi * i * _a(m.x)) * np.cos(np.pi * j * _a(m.y)) for a, i, j in zip(amp, kx, ky))
    pc = rsipg.make_helmholtz_block_jacobi_preconditioner(m, alpha=5.0, nu=1.0, bc_types=bc, tau_scale=0.5)
    x = rsipg.solve_sipg_helmholtz_2d(m, rhs, alpha=5.0, nu=1.0, bc_types=bc, tau_scale=0.5,
                                      iterative=IC(tol=1e-10, maxiter=5000), preconditioner=pc)
    out_sol["helmholtz16/bc"] = bc
    out_sol["helmholtz16/rhs"] = rhs
    out_sol["helmholtz16/u"] = _a(x)
    out_sol["helmholtz16/cg_iterations"] = np.int64(refshim.cg_last_iterations())
    print(f"helmholtz {refshim.cg_last_iterations()} its {time.time() - t0:.1f}s", flush=True)

    # p-multigrid PCG (N = 3 -> 2 -> 1) on the 4x8 rectangle, Dirichlet x / Neumann y
    m = meshes["rect4x8_N3"]
    bc = bc_sets(m, rng)["dir_x_neu_y"]
    src = np.sin(np.pi * _a(m.x)) * np.cos(np.pi * _a(m.y)) + 0.5
    pc = rmg.make_sipg_mg_preconditioner(m, bc_types=bc, tau_scale=200.0)
    x = rsipg.solve_sipg_poisson_2d(m, src, bc_types=bc, tau_scale=200.0, iterative=IC(tol=1e-8),
                                    preconditioner=pc)
    out_sol["pmg/bc"] = bc
    out_sol["pmg/source"] = src
    out_sol["pmg/u"] = _a(x)
    out_sol["pmg/cg_iterations"] = np.int64(refshim.cg_last_iterations())
    r = np.random.default_rng(11).standard_normal(int(m.Np) * int(m.K))
    out_sol["pmg/vcycle_in"] = r
    out_sol["pmg/vcycle_out"] = _a(pc(r))
    print(f"pmg {refshim.cg_last_iterations()} its {time.time() - t0:.1f}s", flush=True)

    # hp-multigrid PCG: base 2x4 on [0,1]x[0,2], 2 h-levels, N = 3, Dirichlet everywhere
    VX, VY, E = rmesh.uniform_rectangle_mesh_2d(0.0, 1.0, 0.0, 2.0, 2, 4)
    base = rmesh.build_mesh_2d(VX, VY, E, 3)

    def bc_fn(mm):
        return np.where(boundary_faces(mm), 1, 0).astype(np.int32)
    pc, fine = rmg.make_sipg_hpmg_preconditioner(base, 2, bc_fn=bc_fn, tau_scale=200.0)
    bc = bc_fn(fine)
    src = np.sin(np.pi * _a(fine.x)) * np.sin(0.5 * np.pi * _a(fine.y)) * 5.0
    x = rsipg.solve_sipg_poisson_2d(fine, src, bc_types=bc, tau_scale=200.0, iterative=IC(tol=1e-8),
                                    preconditioner=pc)
    for f_ in ("VX", "VY", "EToV"):
        out_sol[f"hpmg/fine_{f_}"] = _a(getattr(fine, f_))
    out_sol["hpmg/bc"] = bc
    out_sol["hpmg/source"] = src
    out_sol["hpmg/u"] = _a(x)
    out_sol["hpmg/cg_iterations"] = np.int64(refshim.cg_last_iterations())
    r = np.random.default_rng(12).standard_normal(int(fine.Np) * int(fine.K))
    out_sol["hpmg/vcycle_in"] = r
    out_sol["hpmg/vcycle_out"] = _a(pc(r))
    print(f"hpmg {refshim.cg_last_iterations()} its {time.time() - t0:.1f}s", flush=True)

    # ---- one dual-splitting INS step (incompressible_ns.py:509-666) on the
    # reference test's channel (walls on three sides, outflow on x = 1; 6x6
    # quads, N = 3, dt = 0.01, nu = 0.02): direct-LU and matrix-free CG with
    # the p-multigrid preconditioners, then a BDF2 step from the LU result
    out_ins = {}
    rins = imp("ddg.dg2d.incompressible_ns")
    VX, VY, E = rmesh.uniform_rectangle_mesh_2d(0.0, 1.0, 0.0, 1.0, 6, 6)
    m = rmesh.build_mesh_2d(VX, VY, E, 3)
    isb = boundary_faces(m)
    xf = _a(m.x)[_a(m.Fmask)]                       # (Nfp, 3, K) face-node x
    outflow = np.all(np.abs(xf - 1.0) < 1e-7, axis=0).T
    ins_bc = np.where(isb, np.where(outflow, rins.BC_INS_OUTFLOW, rins.BC_INS_WALL),
                      rins.BC_INS_INTERIOR).astype(np.int32)
    dt, nu = 0.01, 0.02
    zero = np.zeros((int(m.Np), int(m.K)))
    ux = 0.2 * np.sin(np.pi * _a(m.x)) * np.cos(np.pi * _a(m.y))
    uy = -0.2 * np.cos(np.pi * _a(m.x)) * np.sin(np.pi * _a(m.y))
    nxo, nyo = rins.ns_advection_2d(m, ux, uy, ins_bc_types=ins_bc, bc_ux=zero, bc_uy=zero)
    dpdn0 = np.zeros((3 * int(m.Nfp), int(m.K)))
    args = (m, ux, uy, ux, uy, nxo, nyo, dpdn0)
    kw = dict(dt=dt, nu=nu, bdf=rins.BDF1, ins_bc_types=ins_bc, bc_ux=zero, bc_uy=zero)
    ops = rins.build_ins_operators(m, dt=dt, nu=nu, g0=1.0, ins_bc_types=ins_bc)
    res_lu = rins.ns_step_2d(*args, ops=ops, **kw)
    ops_mf = rins.build_ins_operators(m, dt=dt, nu=nu, g0=1.0, ins_bc_types=ins_bc, skip_factor=True)
    pp, vp = rins.make_ins_mg_preconditioners(m, dt=dt, nu=nu, g0=1.0, ins_bc_types=ins_bc)
    res_mg = rins.ns_step_2d(*args, ops=ops_mf, iterative=IC(tol=1e-11, maxiter=3000),
                             pressure_preconditioner=pp, viscous_preconditioner=vp, **kw)
    ops2 = rins.build_ins_operators(m, dt=dt, nu=nu, g0=rins.BDF2.g0, ins_bc_types=ins_bc)
    res2 = rins.ns_step_2d(m, res_lu[0], res_lu[1], ux, uy, res_lu[3], res_lu[4], res_lu[5], dt=dt, nu=nu,
                           bdf=rins.BDF2, ops=ops2, ins_bc_types=ins_bc, bc_ux=zero, bc_uy=zero)
    out_ins.update(VX=_a(VX), VY=_a(VY), EToV=_a(E), ins_bc=ins_bc, ux0=ux, uy0=uy, Nux_old=_a(nxo), Nuy_old=_a(nyo))
    for tag, res in (("lu", res_lu), ("mg", res_mg), ("bdf2", res2)):
        for name, v in zip(("ux", "uy", "p", "Nux", "Nuy", "dpdn"), res):
            out_ins[f"{tag}/{name}"] = _a(v)
    print(f"ins done {time.time() - t0:.1f}s", flush=True)

    out_cur = curved_fixtures(imp)
    for fname, d in (("refelem.npz", out_ref), ("meshes.npz", out_mesh), ("applies.npz", out_app),
                     ("solves.npz", out_sol), ("ins.npz", out_ins), ("curved.npz", out_cur)):
        np.savez_compressed(os.path.join(HERE, fname), **{k: np.asarray(v) for k, v in d.items()})
    print(f"wrote fixtures in {time.time() - t0:.1f}s")


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--only")]
    only = next((a.split("=", 1)[1] for a in sys.argv[1:] if a.startswith("--only=")), None)
    main(args[0] if args else "/root/reference/src", only)
