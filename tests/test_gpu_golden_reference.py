"""GPU parity against fixtures computed by the reference's own, unmodified code
(``tests/golden/make_golden.py``): the CUDA applies on both engines and both
precisions, the loads, the dense probing path, the block-Jacobi blocks (the
device closed-form blocks and the reference-named
``extract_block_diag_matfree``), and the solves (plain CG and LU on the
manufactured-solution workload, the singular branch, block-Jacobi PCG and
p/hp-multigrid PCG) through the product's reference-named functions."""

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
RTOL64 = 1e-12          # float64 operator vs the reference (max-abs relative)
RTOL32 = 2e-5           # float32 operator vs the reference


def _load(name):
    return np.load(os.path.join(GOLD, name))


def _rel(a, b):
    a = a.detach().cpu().numpy() if hasattr(a, "detach") else np.asarray(a)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _pmesh(g, name):
    from ddg_b200.dg2d import mesh as pm
    return pm.build_mesh_2d(g[f"{name}/VX"], g[f"{name}/VY"], g[f"{name}/EToV"], int(g[f"{name}/N"]))


def _cases(a):
    return sorted({k.rsplit("/", 1)[0] for k in a.files if k.endswith("/Au") and "/udir" not in k})


@pytest.mark.parametrize("engine", ["tensor", "cuda"])
def test_apply_fp64_matches_reference(engine):
    import torch
    g, a = _load("meshes.npz"), _load("applies.npz")
    meshes, n = {}, 0
    for case in _cases(a):
        name = case.split("/")[0]
        p = meshes.setdefault(name, _pmesh(g, name))
        tau = float(case.rsplit("tau", 1)[1])
        from ddg_b200.dg2d.operator import SipgOperator
        op = SipgOperator(p, a[case + "/bc"], tau_scale=tau)
        op.set_engine(engine)
        u = torch.as_tensor(a[case + "/u"].T.reshape(-1), device="cuda")
        y = op.apply(u).cpu().numpy().reshape(p.K, p.Np).T
        assert _rel(y, a[case + "/Au"]) < RTOL64, (engine, case)
        op.close()
        n += 1
    assert n >= 30


@pytest.mark.parametrize("engine", ["tensor", "cuda"])
def test_apply_fp32_matches_reference(engine):
    import torch
    from ddg_b200.dg2d.operator import SipgOperator
    g, a = _load("meshes.npz"), _load("applies.npz")
    for case in _cases(a):
        name = case.split("/")[0]
        p = _pmesh(g, name)
        if engine == "tensor" and p.N > 4:
            continue
        tau = float(case.rsplit("tau", 1)[1])
        op = SipgOperator(p, a[case + "/bc"], tau_scale=tau)
        op.set_engine(engine)
        u = torch.as_tensor(a[case + "/u"].T.reshape(-1), device="cuda", dtype=torch.float32)
        y = op.apply(u).double().cpu().numpy().reshape(p.K, p.Np).T
        assert _rel(y, a[case + "/Au"]) < RTOL32, (engine, case)
        op.close()


def test_affine_apply_and_loads_match_reference():
    from ddg_b200.dg2d.sipg import sipg_apply_2d, sipg_dirichlet_load_2d, sipg_neumann_load_2d
    g, a = _load("meshes.npz"), _load("applies.npz")
    names = sorted({k.split("/")[0] for k in g.files})
    for name in names:
        p = _pmesh(g, name)
        c = f"{name}/udir"
        y = sipg_apply_2d(p, a[c + "/u"], bc_types=a[c + "/bc"], u_dir=a[c + "/u_dir"], tau_scale=200.0)
        assert _rel(y, a[c + "/Au"]) < RTOL64, name
        c = f"{name}/loads"
        LD = sipg_dirichlet_load_2d(p, a[c + "/u_dir"], bc_types=a[c + "/bc"], tau_scale=200.0)
        LN = sipg_neumann_load_2d(p, a[c + "/q_neu"], bc_types=a[c + "/bc"])
        assert _rel(LD, a[c + "/LD"]) < RTOL64, name
        assert _rel(LN, a[c + "/LN"]) < RTOL64, name


def test_dense_matrices_match_reference():
    from ddg_b200.dg2d.sipg import sipg_helmholtz_matrix_2d, sipg_matrix_2d
    g, a = _load("meshes.npz"), _load("applies.npz")
    p = _pmesh(g, "tiny2_N2")
    bc = a["tiny2_N2/dense/bc"]
    assert _rel(sipg_matrix_2d(p, bc_types=bc, tau_scale=200.0), a["tiny2_N2/dense/A"]) < RTOL64
    assert _rel(sipg_helmholtz_matrix_2d(p, alpha=5.0, nu=1.0, bc_types=bc, tau_scale=200.0),
                a["tiny2_N2/dense/H"]) < RTOL64


@pytest.mark.parametrize("name", ["rect4x8_N3", "perturbed5_N2"])
def test_block_diagonals_match_reference(name):
    """Both the device closed-form self-blocks (``k_self_blocks``) and the
    reference-named coloured probing ``extract_block_diag_matfree`` over the
    device apply reproduce the reference's probed blocks."""
    import torch
    from ddg_b200.dg2d.operator import SipgOperator
    from ddg_b200.dg2d.sipg import extract_block_diag_matfree
    g, a = _load("meshes.npz"), _load("applies.npz")
    p = _pmesh(g, name)
    bc = a[f"{name}/blocks/bc"]
    ref = a[f"{name}/blocks/B"]
    op = SipgOperator(p, bc, tau_scale=200.0)
    B = extract_block_diag_matfree(lambda v: op.apply(v), p)
    assert isinstance(B, torch.Tensor) and B.is_cuda
    assert _rel(B, ref) < 1e-11
    op.pc_build(0.0)
    Bd = op.pc_blocks()
    assert _rel(Bd, ref) < 1e-11
    op.close()


def test_plain_workload_solves_match_reference():
    """Plain manufactured-solution workload exactly as specified: 12x12 quads
    -> 288 triangles, N=4, tau_scale=0.5, Dirichlet from sin(pi x) sin(pi y),
    f = 2 pi^2 u, unpreconditioned CG to tol 1e-9; also the dense LU path."""
    from ddg_b200.dg2d import sipg as ps
    g, s = _load("meshes.npz"), _load("solves.npz")
    p = _pmesh(g, "plain12_N4")
    bc = s["plain/bc"]
    ue = np.sin(np.pi * p.x) * np.sin(np.pi * p.y)
    u, info = ps.solve_sipg_poisson_2d(p, 2 * np.pi ** 2 * ue, bc_types=bc, u_dir=ue, tau_scale=0.5,
                                       iterative=ps.IterativeConfig(tol=1e-9), return_info=True)
    assert info.status == "converged"
    assert abs(info.iterations - int(s["plain/cg_iterations"])) <= 2
    assert _rel(u, s["plain/u_cg"]) < 1e-8
    # L2 error against the exact solution equals the reference's to 1e-6 relative
    M = p.ref.M
    e_ref = s["plain/u_cg"] - ue
    e = u - ue
    l2 = lambda d: float(np.sqrt(np.sum(p.J * d * (M @ d))))  # noqa: E731
    assert abs(l2(e) - l2(e_ref)) <= 1e-6 * l2(e_ref)
    assert l2(e) < 1e-3
    ulu = ps.solve_sipg_poisson_2d(p, 2 * np.pi ** 2 * ue, bc_types=bc, u_dir=ue, tau_scale=0.5)
    assert _rel(ulu, s["plain/u_lu"]) < 1e-10


def test_singular_and_helmholtz_solves_match_reference():
    from ddg_b200.dg2d import mesh as pm
    from ddg_b200.dg2d import sipg as ps
    g, s = _load("meshes.npz"), _load("solves.npz")
    p = _pmesh(g, "rect4x8_N3")
    u, info = ps.solve_sipg_poisson_2d(p, s["singular/source"], bc_types=s["singular/bc"], tau_scale=200.0,
                                       iterative=ps.IterativeConfig(tol=1e-10), return_info=True)
    assert abs(info.iterations - int(s["singular/cg_iterations"])) <= 2
    assert _rel(u, s["singular/u"]) < 1e-8
    VX, VY, E = pm.uniform_rectangle_mesh_2d(0.0, 1.0, 0.0, 1.0, 16, 16)
    p = pm.build_mesh_2d(VX, VY, E, 4)
    bc = s["helmholtz16/bc"]
    pc = ps.make_helmholtz_block_jacobi_preconditioner(p, alpha=5.0, nu=1.0, bc_types=bc, tau_scale=0.5)
    u, info = ps.solve_sipg_helmholtz_2d(p, s["helmholtz16/rhs"], alpha=5.0, nu=1.0, bc_types=bc,
                                         tau_scale=0.5, iterative=ps.IterativeConfig(tol=1e-10, maxiter=5000),
                                         preconditioner=pc, return_info=True)
    assert abs(info.iterations - int(s["helmholtz16/cg_iterations"])) <= 3
    assert _rel(u, s["helmholtz16/u"]) < 1e-8


def test_multigrid_matches_reference():
    from ddg_b200.dg2d import mesh as pm
    from ddg_b200.dg2d import multigrid as pmg
    from ddg_b200.dg2d import sipg as ps
    g, s = _load("meshes.npz"), _load("solves.npz")
    p = _pmesh(g, "rect4x8_N3")
    bc = s["pmg/bc"]
    pc = pmg.make_sipg_mg_preconditioner(p, bc_types=bc, tau_scale=200.0)
    assert _rel(pc(s["pmg/vcycle_in"]), s["pmg/vcycle_out"]) < 1e-10
    u, info = ps.solve_sipg_poisson_2d(p, s["pmg/source"], bc_types=bc, tau_scale=200.0,
                                       iterative=ps.IterativeConfig(tol=1e-8), preconditioner=pc,
                                       return_info=True)
    # The 2-norm residual of MG-preconditioned CG swings by up to 10x from one
    # iteration to the next (CG minimises the energy norm); the reference's
    # run crosses tol at iteration 54 with 9.7e-9, so a 1e-10 perturbation of
    # the V-cycle can move the first crossing by a few iterations.
    assert abs(info.iterations - int(s["pmg/cg_iterations"])) <= 4
    assert _rel(u, s["pmg/u"]) < 1e-8
    VX, VY, E = pm.uniform_rectangle_mesh_2d(0.0, 1.0, 0.0, 2.0, 2, 4)
    base = pm.build_mesh_2d(VX, VY, E, 3)

    def bc_fn(m):
        return np.where(np.asarray(m.EToE) == np.arange(m.K)[:, None], 1, 0).astype(np.int32)
    pc, fine = pmg.make_sipg_hpmg_preconditioner(base, 2, bc_fn=bc_fn, tau_scale=200.0)
    assert np.array_equal(fine.EToV, s["hpmg/fine_EToV"])
    assert _rel(pc(s["hpmg/vcycle_in"]), s["hpmg/vcycle_out"]) < 1e-10
    u, info = ps.solve_sipg_poisson_2d(fine, s["hpmg/source"], bc_types=s["hpmg/bc"], tau_scale=200.0,
                                       iterative=ps.IterativeConfig(tol=1e-8), preconditioner=pc,
                                       return_info=True)
    assert abs(info.iterations - int(s["hpmg/cg_iterations"])) <= 4
    assert _rel(u, s["hpmg/u"]) < 1e-8


@pytest.mark.parametrize("precision", ["mixed", "mixed-restart"])
def test_mixed_precision_solve_matches_reference_fp64_solution(precision):
    """The mixed-precision block-Jacobi PCG (float32 iterations, float64
    refinement) reaches relative L2 error <= 1e-8 against the reference's own
    float64 solution of the same Helmholtz system (16x16 quads, N=4, alpha=5,
    Dirichlet x / Neumann y, tau_scale=0.5, 8-mode RHS)."""
    from ddg_b200.dg2d import mesh as pm
    from ddg_b200.dg2d import sipg as ps
    s = _load("solves.npz")
    VX, VY, E = pm.uniform_rectangle_mesh_2d(0.0, 1.0, 0.0, 1.0, 16, 16)
    p = pm.build_mesh_2d(VX, VY, E, 4)
    bc = s["helmholtz16/bc"]
    pc = ps.make_helmholtz_block_jacobi_preconditioner(p, alpha=5.0, nu=1.0, bc_types=bc, tau_scale=0.5)
    u, info = ps.solve_sipg_helmholtz_2d(p, s["helmholtz16/rhs"], alpha=5.0, nu=1.0, bc_types=bc, tau_scale=0.5,
                                         iterative=ps.IterativeConfig(tol=1e-10, maxiter=20000, precision=precision),
                                         preconditioner=pc, return_info=True)
    ref = s["helmholtz16/u"]
    assert info.status == "converged"
    assert np.linalg.norm(u - ref) / np.linalg.norm(ref) <= 1e-8
