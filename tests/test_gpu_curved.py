"""GPU parity of the curved-element operator (per-node geometry, nodal and
cubature quadrature) against fixtures from the reference's own code
(``tests/golden/curved.npz``) and against the oracle, through the product's
reference-named functions: ``sipg_apply_2d`` with and without ``cub``, the
loads, ``cubature_mass_apply`` / ``per_element_mass``, the block-Jacobi
blocks, and the Poisson / Helmholtz solves with ``cub`` (device CG graph and
LU).  Float64 throughout; tolerances are max-abs relative."""

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
NAMES = ("annulus8_N1", "annulus8_N2", "annulus8_N3", "annulus8_N5", "cyl8_N4")
RTOL = 2e-12          # curved operator vs the reference (the product's curved geometry differs by <= 7e-13)


def _g():
    return np.load(os.path.join(GOLD, "curved.npz"))


def _rel(a, b):
    a = a.detach().cpu().numpy() if hasattr(a, "detach") else np.asarray(a)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _bend(name, m, mod):
    if name.startswith("annulus"):
        return mod.apply_circular_hole_2d(m, cx=0.0, cy=0.0, radius=0.5, detection_tol=0.5)
    return mod.apply_circular_hole_2d(m, cx=1.0, cy=1.0, radius=0.25, detection_tol=0.1)


def _pmesh(g, name):
    from ddg_b200.dg2d import cubature as pcub
    from ddg_b200.dg2d import curved as pcur
    from ddg_b200.dg2d import mesh as pm
    m = pm.build_mesh_2d(g[f"{name}/VX"], g[f"{name}/VY"], g[f"{name}/EToV"], int(g[f"{name}/N"]))
    m = _bend(name, m, pcur)
    return m, pcub.attach_cubature(m)


def _annulus(N, Kx, which="both"):
    """Product and oracle curved annulus meshes built independently."""
    from ddg_b200.dg2d import cubature as pcub
    from ddg_b200.dg2d import curved as pcur
    from ddg_b200.dg2d import mesh as pm
    from oracle import cubature as ocub
    from oracle import curved as ocur
    from oracle import mesh as om
    VX, VY, E = pm.rectangle_with_square_hole_mesh_2d(-2.0, 2.0, -2.0, 2.0, Kx, Kx, -0.5, 0.5, -0.5, 0.5)
    p = _bend("annulus", pm.build_mesh_2d(VX, VY, E, N), pcur)
    o = _bend("annulus", om.build_mesh_2d(VX, VY, E, N), ocur)
    return p, pcub.attach_cubature(p), o, ocub.attach_cubature(o)


@pytest.mark.parametrize("name", NAMES)
def test_curved_apply_matches_reference(name):
    from ddg_b200.dg2d import sipg
    g = _g()
    m, cub = _pmesh(g, name)
    for b in ("dirichlet", "random", "neumann"):
        for tau in (200.0, 0.5):
            k = f"{name}/apply/{b}/tau{tau:g}"
            bc, u = g[k + "/bc"], g[k + "/u"]
            y = sipg.sipg_apply_2d(m, u, bc_types=bc, tau_scale=tau)
            assert _rel(y, g[k + "/Au_nodal"]) < RTOL, ("nodal", k)
            y = sipg.sipg_apply_2d(m, u, bc_types=bc, tau_scale=tau, cub=cub)
            assert _rel(y, g[k + "/Au_cub"]) < RTOL, ("cubature", k)


@pytest.mark.parametrize("name", NAMES)
def test_curved_dirichlet_ghost_loads_and_mass_match_reference(name):
    from ddg_b200.dg2d import cubature as pcub
    from ddg_b200.dg2d import sipg
    g = _g()
    m, cub = _pmesh(g, name)
    k = f"{name}/udir"
    bc = g[k + "/bc"]
    y = sipg.sipg_apply_2d(m, g[k + "/u"], bc_types=bc, u_dir=g[k + "/u_dir"], tau_scale=200.0, cub=cub)
    assert _rel(y, g[k + "/Au_cub"]) < RTOL
    assert _rel(sipg.sipg_dirichlet_load_2d(m, g[k + "/u_dir"], bc_types=bc, tau_scale=200.0), g[k + "/LD"]) < RTOL
    assert _rel(sipg.sipg_neumann_load_2d(m, g[k + "/q_neu"], bc_types=bc), g[k + "/LN"]) < RTOL
    assert _rel(pcub.cubature_mass_apply(cub, g[f"{name}/mass/f"]), g[f"{name}/mass/Mf"]) < RTOL
    if name == "annulus8_N3":
        assert _rel(pcub.per_element_mass(cub), g[f"{name}/mass/MK"]) < RTOL


def test_curved_block_diagonals_match_reference():
    import torch
    from ddg_b200.dg2d import sipg
    g = _g()
    m, cub = _pmesh(g, "annulus8_N3")
    bc = g["annulus8_N3/blocks/bc"]
    # reference-named builder on the curved mesh: blocks of the nodal operator
    pc = sipg.make_sipg_block_jacobi_preconditioner(m, bc_types=bc, tau_scale=200.0)
    assert _rel(pc.blocks(), g["annulus8_N3/blocks/nodal"]) < RTOL
    # device coloured probing of the cubature operator, and the generic
    # extract_block_diag_matfree over the cubature apply
    op = m.curved_operator(bc, 200.0, cub)
    op.pc_build(0.0, quad="cubature")
    assert _rel(op.pc_blocks(), g["annulus8_N3/blocks/cub"]) < RTOL
    Np, K = m.Np, m.K

    def apply_flat(v):
        return op.apply(torch.as_tensor(v, device="cuda"))
    assert _rel(sipg.extract_block_diag_matfree(apply_flat, m), g["annulus8_N3/blocks/cub"]) < RTOL
    # the inverse blocks: B^-1 (B e) = e
    r = torch.randn(Np * K, dtype=torch.float64, device="cuda")
    Bt = op.pc_blocks()
    Br = torch.einsum("kij,kj->ki", Bt, r.reshape(K, Np)).reshape(-1)
    assert _rel(op.pc_apply(Br), r.cpu().numpy()) < 1e-10


def test_curved_poisson_solves_match_reference():
    from ddg_b200.dg2d import sipg
    g = _g()
    m, cub = _pmesh(g, "annulus8_N3")
    bc, ue = g["annulus8_N3/solve/bc"], g["annulus8_N3/solve/u_exact"]
    src = 2 * (np.pi / 4) ** 2 * ue
    u = sipg.solve_sipg_poisson_2d(m, src, bc_types=bc, u_dir=ue)
    assert _rel(u, g["annulus8_N3/solve/u_lu_nodal"]) < 1e-10
    u = sipg.solve_sipg_poisson_2d(m, src, bc_types=bc, u_dir=ue, cub=cub)
    assert _rel(u, g["annulus8_N3/solve/u_lu_cub"]) < 1e-10
    u, info = sipg.solve_sipg_poisson_2d(m, src, bc_types=bc, u_dir=ue, cub=cub, return_info=True,
                                         iterative=sipg.IterativeConfig(tol=1e-10, maxiter=5000))
    ref_its = int(g["annulus8_N3/solve/cg_iterations"])
    assert info.status == "converged"
    # tau_scale 200 makes this a 1.8k-iteration CG: rounding moves the count
    # by ~1% and the solution (tol 1e-10 on the residual) by a few 1e-8
    assert abs(info.iterations - ref_its) <= max(3, int(0.02 * ref_its))
    assert _rel(u, g["annulus8_N3/solve/u_cg_cub"]) < 1e-7
    assert _rel(u, g["annulus8_N3/solve/u_lu_cub"]) < 1e-6


def test_curved_helmholtz_solves_match_reference():
    from ddg_b200.dg2d import sipg
    g = _g()
    m, cub = _pmesh(g, "cyl8_N4")
    bc, rhs = g["cyl8_N4/helm/bc"], g["cyl8_N4/helm/rhs"]
    u, info = sipg.solve_sipg_helmholtz_2d(m, rhs, alpha=5.0, nu=1.0, bc_types=bc, tau_scale=0.5, cub=cub,
                                           iterative=sipg.IterativeConfig(tol=1e-10, maxiter=8000),
                                           return_info=True)
    ref_its = int(g["cyl8_N4/helm/cg_iterations"])
    assert info.status == "converged"
    assert abs(info.iterations - ref_its) <= max(3, int(0.02 * ref_its))
    assert _rel(u, g["cyl8_N4/helm/u_cg"]) < 1e-8
    u = sipg.solve_sipg_helmholtz_2d(m, rhs, alpha=5.0, nu=1.0, bc_types=bc, tau_scale=0.5, cub=cub)
    assert _rel(u, g["cyl8_N4/helm/u_lu"]) < 1e-10


@pytest.mark.parametrize("blocks", ["nodal", "cubature"])
def test_curved_block_jacobi_pcg_matches_oracle(blocks):
    """Block-Jacobi PCG on the cubature operator.  "nodal": the reference's
    pairing -- make_helmholtz_block_jacobi_preconditioner takes no cub, so
    its blocks are the nodal operator's; the device graph rebuilds those
    blocks inside the cubature handle.  "cubature": the extension ``cub=``
    gives the cubature operator's own blocks.  Same iterates as the oracle's
    PCG with the same blocks, and fewer iterations than plain CG."""
    from ddg_b200.dg2d import sipg
    from oracle import sipg as osp
    p, pcub_, o, ocub_ = _annulus(3, 16)
    assert p.J.min() > 0 and pcub_.J.min() > 0
    bc = np.where(p.EToE == np.arange(p.K)[:, None], 1, 0).astype(np.int32)
    src = np.cos(p.x) * np.sin(0.7 * p.y) + 0.1
    cfg = sipg.IterativeConfig(tol=1e-10, maxiter=4000)
    pc = sipg.make_helmholtz_block_jacobi_preconditioner(p, alpha=2.0, nu=1.0, bc_types=bc, tau_scale=0.5,
                                                         cub=pcub_ if blocks == "cubature" else None)
    u, info = sipg.solve_sipg_helmholtz_2d(p, src, alpha=2.0, nu=1.0, bc_types=bc, tau_scale=0.5, cub=pcub_,
                                           iterative=cfg, preconditioner=pc, return_info=True)
    B = osp.extract_block_diag_matfree(
        osp.flat_op(o, bc_types=bc, tau_scale=0.5, alpha=2.0, cub=ocub_ if blocks == "cubature" else None), o)
    uo, its = osp.solve_helmholtz(o, src, alpha=2.0, bc_types=bc, tau_scale=0.5, cub=ocub_,
                                  preconditioner=osp.block_jacobi_from_blocks(B),
                                  iterative=osp.IterativeConfig(tol=1e-10, maxiter=4000), return_info=True)
    assert info.status == "converged"
    assert abs(info.iterations - its) <= max(2, int(0.02 * its))
    assert _rel(u, uo) < 1e-8
    _, plain = sipg.solve_sipg_helmholtz_2d(p, src, alpha=2.0, nu=1.0, bc_types=bc, tau_scale=0.5, cub=pcub_,
                                            iterative=cfg, return_info=True)
    assert info.iterations < plain.iterations


@pytest.mark.parametrize("N", [1, 2, 3, 4, 5])
def test_curved_every_degree_matches_oracle(N):
    """Every built degree, both quadratures, with the Helmholtz mass term, on
    an annulus whose element count leaves a partial last tile."""
    import torch
    from oracle import sipg as osp
    p, pc_, o, oc_ = _annulus(N, 16)
    assert p.K % 128 != 0 and p.J.min() > 0
    rng = np.random.default_rng(N)
    isb = p.EToE == np.arange(p.K)[:, None]
    bc = np.where(isb, rng.integers(1, 3, size=(p.K, 3)), 0).astype(np.int32)
    u = rng.standard_normal(p.K * p.Np)
    for quad, c_p, c_o in (("nodal", None, None), ("cubature", pc_, oc_)):
        op = p.curved_operator(bc, 0.5, c_p)
        y = op.apply(torch.as_tensor(u, device="cuda"), alpha=3.0, quad=quad)
        ref = osp.flat_op(o, bc_types=bc, tau_scale=0.5, alpha=3.0, cub=c_o)(u)
        assert _rel(y, ref) < RTOL, (N, quad)


def test_curved_cylinder_many_elements_matches_oracle():
    import torch
    from ddg_b200.dg2d import cubature as pcub
    from ddg_b200.dg2d import curved as pcur
    from ddg_b200.dg2d import mesh as pm
    from oracle import cubature as ocub
    from oracle import curved as ocur
    from oracle import mesh as om
    from oracle import sipg as osp
    args = (0.0, 8.0, 0.0, 4.0, 64, 32)
    kw = dict(cx=2.0, cy=2.0, radius=0.35, R_outer=1.0, n_radial=6, radial_growth=1.2)
    VX, VY, E = pm.channel_with_circle_mesh_2d(*args, **kw)
    p = pcur.apply_circular_hole_2d(pm.build_mesh_2d(VX, VY, E, 4), cx=2.0, cy=2.0, radius=0.35)
    o = ocur.apply_circular_hole_2d(om.build_mesh_2d(VX, VY, E, 4), cx=2.0, cy=2.0, radius=0.35)
    assert p.K > 4000 and not p.is_affine
    bc = np.where(p.EToE == np.arange(p.K)[:, None], 1, 0).astype(np.int32)
    u = np.random.default_rng(5).standard_normal(p.K * p.Np)
    op = p.curved_operator(bc, 200.0, pcub.attach_cubature(p))
    y = op.apply(torch.as_tensor(u, device="cuda"))
    ref = osp.flat_op(o, bc_types=bc, cub=ocub.attach_cubature(o))(u)
    assert _rel(y, ref) < RTOL


def test_affine_mesh_cubature_equals_affine_kernels():
    """On straight-sided elements the cubature branch and the nodal rule are
    the same operator (both exact): the curved kernels with cub agree with
    the affine tensor-core kernel."""
    from ddg_b200.dg2d import cubature as pcub
    from ddg_b200.dg2d import mesh as pm
    from ddg_b200.dg2d import sipg
    VX, VY, E = pm.uniform_rectangle_mesh_2d(0.0, 1.0, 0.0, 1.0, 9, 7)
    m = pm.build_mesh_2d(VX, VY, E, 4)
    assert m.is_affine
    bc = np.where(m.EToE == np.arange(m.K)[:, None], 1, 0).astype(np.int32)
    u = np.random.default_rng(2).standard_normal((m.Np, m.K))
    y_aff = sipg.sipg_apply_2d(m, u, bc_types=bc, tau_scale=0.5)
    y_cub = sipg.sipg_apply_2d(m, u, bc_types=bc, tau_scale=0.5, cub=pcub.attach_cubature(m))
    assert _rel(y_cub, y_aff) < 1e-12


def test_curved_cg_zero_rhs_and_errors():
    import torch
    from ddg_b200 import _lib
    from ddg_b200.dg2d import multigrid, sipg
    p, pc_, _, _ = _annulus(3, 8)
    assert p.J.min() > 0
    bc = np.where(p.EToE == np.arange(p.K)[:, None], 1, 0).astype(np.int32)
    op = p.curved_operator(bc, 200.0, pc_)
    b = torch.zeros(p.K * p.Np, dtype=torch.float64, device="cuda")
    x = torch.zeros_like(b)
    st, its, rr, bb = op.cg(b, x, tol=1e-10)
    assert st == "converged" and its == 0 and float(x.abs().max()) == 0.0
    nodal_only = p.curved_operator(bc, 200.0, None)
    with pytest.raises(_lib.DdgError):
        nodal_only.apply(b, quad="cubature")
    with pytest.raises(ValueError):
        multigrid.make_sipg_mg_preconditioner(p, bc_types=bc, tau_scale=200.0)
    with pytest.raises(ValueError):
        sipg.solve_sipg_poisson_2d(p, np.ones((p.Np, p.K)), bc_types=bc, cub=pc_,
                                   iterative=sipg.IterativeConfig(precision="mixed"))


@pytest.mark.parametrize("path", ["lu", "cg"])
def test_curved_ins_step_with_cubature_matches_reference(path):
    """One dual-splitting step (BDF1) of flow past the bent cylinder with
    cub=attach_cubature(mesh): pressure Poisson (outflow Dirichlet) and the
    two viscous Helmholtz solves on the cubature operator, by LU and by the
    device CG, against the reference's own ns_step_2d with cub."""
    from ddg_b200.dg2d import cubature as pcub
    from ddg_b200.dg2d import curved as pcur
    from ddg_b200.dg2d import incompressible_ns as pins
    from ddg_b200.dg2d import mesh as pm
    from ddg_b200.dg2d import sipg
    g = _g()
    m = pcur.apply_circular_hole_2d(pm.build_mesh_2d(g["cyl8_N4/VX"], g["cyl8_N4/VY"], g["cyl8_N4/EToV"], 3),
                                    cx=1.0, cy=1.0, radius=0.25, detection_tol=0.1)
    cub = pcub.attach_cubature(m)
    k = "ins_cyl_N3/"
    ins_bc, zero = g[k + "ins_bc"], np.zeros_like(m.x)
    dpdn0 = np.zeros((3 * m.Nfp, m.K))
    ops = pins.build_ins_operators(m, dt=0.01, nu=0.05, g0=1.0, ins_bc_types=ins_bc, skip_factor=(path == "cg"),
                                   cub=cub)
    it = sipg.IterativeConfig(tol=1e-12, maxiter=20000) if path == "cg" else None
    res = pins.ns_step_2d(m, g[k + "ux0"], g[k + "uy0"], g[k + "ux0"], g[k + "uy0"], g[k + "Nux_old"],
                          g[k + "Nuy_old"], dpdn0, dt=0.01, nu=0.05, bdf=pins.BDF1, ops=ops, ins_bc_types=ins_bc,
                          bc_ux=g[k + "bc_ux"], bc_uy=zero, iterative=it, cub=cub)
    tol = 1e-9 if path == "lu" else 1e-8
    for name, v in zip(("ux", "uy", "p"), res[:3]):
        assert _rel(v, g[f"{k}{path}/{name}"]) < tol, (path, name)


def test_reference_curved_poisson_known_answer():
    """The reference's test_curved_poisson_solve_well_behaved at its own size
    (24 x 24 annulus, N = 3, all-Dirichlet, u = sin(pi x / 4) sin(pi y / 4),
    direct LU of the nodal-rule operator): relative L2 error < 2e-2 --
    and with the cubature rule too."""
    from ddg_b200.dg2d import cubature as pcub
    from ddg_b200.dg2d import curved as pcur
    from ddg_b200.dg2d import mesh as pm
    from ddg_b200.dg2d import sipg
    VX, VY, E = pm.rectangle_with_square_hole_mesh_2d(-2.0, 2.0, -2.0, 2.0, 24, 24, -0.5, 0.5, -0.5, 0.5)
    m = pcur.apply_circular_hole_2d(pm.build_mesh_2d(VX, VY, E, 3), cx=0.0, cy=0.0, radius=0.5, detection_tol=0.5)
    ue = np.sin(np.pi * m.x / 4) * np.sin(np.pi * m.y / 4)
    src = 2 * (np.pi / 4) ** 2 * ue
    bc = np.where(m.EToE == np.arange(m.K)[:, None], 1, 0).astype(np.int32)
    for cub in (None, pcub.attach_cubature(m)):
        u = sipg.solve_sipg_poisson_2d(m, src, bc_types=bc, u_dir=ue, cub=cub)
        err = np.sqrt(np.sum(m.J * (u - ue) ** 2) / np.sum(m.J * ue ** 2))
        assert err < 2e-2, (cub is not None, err)
