"""GPU p- and hp-multigrid: V-cycle parity with the oracle's restatement of
``src/ddg/dg2d/multigrid.py`` and the reference's own multigrid properties
(``test/test_multigrid_2d.py``) through the device MG-preconditioned CG."""

import numpy as np
import pytest

from oracle import mesh as om
from oracle import multigrid as omg
from oracle import sipg as osp

pytestmark = pytest.mark.gpu


def _pair(K, N, Ky=None):
    from ddg_b200.dg2d import mesh as pm
    VX, VY, E = om.uniform_rectangle_mesh_2d(0.0, 1.0, 0.0, 1.0, K, Ky or K)
    return om.build_mesh_2d(VX, VY, E, N), pm.build_mesh_2d(VX, VY, E, N)


def _dir(m):
    return osp.boundary_bc(m)


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("alpha", [0.0, 50.0])
def test_pmg_vcycle_matches_oracle(alpha):
    from ddg_b200.dg2d import multigrid as pmg
    o, p = _pair(6, 4)
    bc = _dir(o)
    v = np.random.default_rng(0).standard_normal(o.Np * o.K)
    z_ref = omg.make_pmg(o, bc_types=bc, alpha=alpha)(v)
    z = pmg.make_sipg_mg_preconditioner(p, bc_types=bc, alpha=alpha)(v)
    assert _rel(z, z_ref) < 1e-10


def test_hpmg_vcycle_matches_oracle():
    from ddg_b200.dg2d import multigrid as pmg
    o, p = _pair(2, 3)
    mg_ref, fin_o = omg.make_hpmg(o, 2, bc_fn=osp.boundary_bc)
    mg, fin = pmg.make_sipg_hpmg_preconditioner(p, 2, bc_fn=osp.boundary_bc)
    assert np.array_equal(fin.EToV, fin_o.EToV) and np.array_equal(fin.vmapP, fin_o.vmapP)
    v = np.random.default_rng(1).standard_normal(fin.Np * fin.K)
    assert _rel(mg(v), mg_ref(v)) < 1e-10


def test_pmg_fp32_vcycle_close_to_fp64():
    from ddg_b200.dg2d import multigrid as pmg
    o, p = _pair(6, 4)
    bc = _dir(o)
    v = np.random.default_rng(2).standard_normal(o.Np * o.K)
    z64 = pmg.make_sipg_mg_preconditioner(p, bc_types=bc)(v)
    z32 = pmg.make_sipg_mg_preconditioner(p, bc_types=bc, precision="fp32")(v)
    assert _rel(z32, z64) < 1e-4


def _solve_iters(p, bc, b_field, pc, tol=1e-8, alpha=0.0):
    from ddg_b200.dg2d import sipg as ps
    cfg = ps.IterativeConfig(tol=tol, maxiter=5000)
    if alpha == 0.0:
        return ps.solve_sipg_poisson_2d(p, b_field, bc_types=bc, iterative=cfg, preconditioner=pc,
                                        return_info=True)
    return ps.solve_sipg_helmholtz_2d(p, b_field, alpha=alpha, nu=1.0, bc_types=bc, iterative=cfg,
                                      preconditioner=pc, return_info=True)


def test_pmg_pcg_matches_direct():
    """test_multigrid_2d.py:77-93 through the product's device MG-PCG."""
    from ddg_b200.dg2d import multigrid as pmg
    from ddg_b200.dg2d import sipg as ps
    o, p = _pair(8, 4)
    bc = _dir(o)
    src = np.random.default_rng(0).standard_normal((o.Np, o.K))
    u_lu = ps.solve_sipg_poisson_2d(p, src, bc_types=bc)
    mg = pmg.make_sipg_mg_preconditioner(p, bc_types=bc)
    u, info = _solve_iters(p, bc, src, mg, tol=1e-10)
    assert info.status == "converged" and _rel(u, u_lu) < 1e-7


def test_pmg_beats_block_jacobi_and_is_degree_robust():
    """test_multigrid_2d.py:98-125."""
    from ddg_b200.dg2d import multigrid as pmg
    from ddg_b200.dg2d import sipg as ps
    pm_it, bj_it = {}, {}
    for N in (2, 3, 4, 5):
        o, p = _pair(8, N)
        bc = _dir(o)
        src = np.random.default_rng(1).standard_normal((o.Np, o.K))
        _, i_bj = _solve_iters(p, bc, src, ps.make_sipg_block_jacobi_preconditioner(p, bc_types=bc))
        _, i_mg = _solve_iters(p, bc, src, pmg.make_sipg_mg_preconditioner(p, bc_types=bc))
        bj_it[N], pm_it[N] = i_bj.iterations, i_mg.iterations
    assert pm_it[5] < 0.5 * bj_it[5] and pm_it[4] < 0.5 * bj_it[4], (pm_it, bj_it)
    assert pm_it[5] < 2.0 * pm_it[2] and bj_it[5] > 1.5 * bj_it[2], (pm_it, bj_it)


def test_pmg_helmholtz():
    """test_multigrid_2d.py:130-152."""
    from ddg_b200.dg2d import multigrid as pmg
    from ddg_b200.dg2d import sipg as ps
    o, p = _pair(8, 4)
    bc = _dir(o)
    src = np.random.default_rng(2).standard_normal((o.Np, o.K))
    u_lu = ps.solve_sipg_helmholtz_2d(p, src, alpha=50.0, nu=1.0, bc_types=bc)
    u, i_mg = _solve_iters(p, bc, src, pmg.make_sipg_mg_preconditioner(p, bc_types=bc, alpha=50.0),
                           tol=1e-10, alpha=50.0)
    _, i_bj = _solve_iters(p, bc, src, ps.make_helmholtz_block_jacobi_preconditioner(
        p, alpha=50.0, nu=1.0, bc_types=bc), tol=1e-10, alpha=50.0)
    assert _rel(u, u_lu) < 1e-7 and i_mg.iterations <= i_bj.iterations


def test_hpmg_correct_and_mesh_independent():
    """test_multigrid_2d.py:157-202."""
    from ddg_b200.dg2d import multigrid as pmg
    from ddg_b200.dg2d import sipg as ps
    hp, bj = {}, {}
    for nh in (1, 2, 3):
        o, p = _pair(2, 3)
        mg, fin = pmg.make_sipg_hpmg_preconditioner(p, nh, bc_fn=osp.boundary_bc)
        bc = osp.boundary_bc(fin)
        src = np.random.default_rng(5).standard_normal((fin.Np, fin.K))
        u, info = _solve_iters(fin, bc, src, mg)
        hp[nh] = info.iterations
        _, ib = _solve_iters(fin, bc, src, ps.make_sipg_block_jacobi_preconditioner(fin, bc_types=bc))
        bj[nh] = ib.iterations
        if nh == 2:
            u_lu = ps.solve_sipg_poisson_2d(fin, src, bc_types=bc)
            u10, _ = _solve_iters(fin, bc, src, mg, tol=1e-10)
            assert _rel(u10, u_lu) < 1e-7
    assert hp[3] < 1.6 * hp[1] and bj[3] > 1.8 * bj[1] and hp[3] < 0.3 * bj[3], (hp, bj)


def test_hpmg_fp32_smoothing_same_solution():
    """float32 V-cycle inside float64 CG: same answer to 1e-8, similar count."""
    from ddg_b200.dg2d import multigrid as pmg
    o, p = _pair(2, 3)
    mg64, fin = pmg.make_sipg_hpmg_preconditioner(p, 3, bc_fn=osp.boundary_bc)
    mg32, _ = pmg.make_sipg_hpmg_preconditioner(p, 3, bc_fn=osp.boundary_bc, precision="fp32")
    bc = osp.boundary_bc(fin)
    src = np.random.default_rng(6).standard_normal((fin.Np, fin.K))
    u64, i64 = _solve_iters(fin, bc, src, mg64, tol=1e-12)
    u32, i32 = _solve_iters(fin, bc, src, mg32, tol=1e-12)
    assert i32.status == "converged" and _rel(u32, u64) < 1e-8
    assert i32.iterations <= 1.5 * i64.iterations + 2


def test_hpmg_pure_neumann_regularised():
    """Singular pressure Poisson: eps-shifted CG with a regularised coarse
    solve (sipg.py:891-906, multigrid.py:223-224) matches the oracle."""
    from ddg_b200.dg2d import multigrid as pmg
    from ddg_b200.dg2d import sipg as ps
    o, p = _pair(2, 2)
    nbc = lambda m: osp.boundary_bc(m, osp.BC_NEUMANN)  # noqa: E731
    mg, fin = pmg.make_sipg_hpmg_preconditioner(p, 2, bc_fn=nbc, regularize=True, tau_scale=0.5)
    om_fin = om.build_mesh_2d(fin.VX, fin.VY, fin.EToV, fin.N)
    bc = nbc(fin)
    src = np.cos(np.pi * fin.x) * np.cos(np.pi * fin.y)
    u, info = ps.solve_sipg_poisson_2d(fin, src, bc_types=bc, tau_scale=0.5, preconditioner=mg,
                                       iterative=ps.IterativeConfig(tol=1e-12, maxiter=2000), return_info=True)
    u_ref = osp.solve_poisson(om_fin, src, bc_types=bc, tau_scale=0.5,
                              iterative=osp.IterativeConfig(tol=1e-12, maxiter=5000))
    assert info.status == "converged" and _rel(u, u_ref) < 1e-7
    assert abs(u.sum()) < 1e-8 * np.abs(u).sum()


def test_mesh_cache_eviction_keeps_multigrid_levels_alive():
    """Filling the mesh's operator cache with other (BC, penalty) pairs drops
    the cache's reference to a multigrid level operator but must not free the
    handle the V-cycle still uses; the MG-PCG solve afterwards still matches
    the direct solve."""
    import gc
    from ddg_b200.dg2d import multigrid as pmg
    from ddg_b200.dg2d import sipg as ps
    o, p = _pair(6, 3)
    bc = _dir(o)
    src = np.random.default_rng(1).standard_normal((o.Np, o.K))
    mg = pmg.make_sipg_mg_preconditioner(p, bc_types=bc)
    for tau in (1.0, 2.0, 3.0, 4.0, 5.0):           # five other keys evict the level operator
        p.device_operator(bc, tau)
    gc.collect()
    u, info = _solve_iters(p, bc, src, mg, tol=1e-10)
    u_lu = ps.solve_sipg_poisson_2d(p, src, bc_types=bc)
    assert info.status == "converged" and _rel(u, u_lu) < 1e-7


def test_operator_destroyed_before_multigrid():
    """A user operator that captured an MG-CG graph is destroyed before the
    multigrid object (and the other way round); neither destroy may touch
    freed memory, and a fresh solve still works."""
    import torch
    from ddg_b200.dg2d import multigrid as pmg
    from ddg_b200.dg2d.operator import SipgOperator
    o, p = _pair(5, 3)
    bc = _dir(o)
    b = torch.as_tensor(np.random.default_rng(2).standard_normal(o.Np * o.K), device="cuda")
    for order in ("op_first", "mg_first"):
        mg = pmg.make_sipg_mg_preconditioner(p, bc_types=bc)
        user = SipgOperator(p, bc, tau_scale=200.0)
        x = torch.zeros_like(b)
        st, its, _, _ = user.cg_mg(mg, b, x, tol=1e-10)
        assert st == "converged"
        if order == "op_first":
            user.close()
            mg.close()
        else:
            mg.close()
            user.close()
    mg = pmg.make_sipg_mg_preconditioner(p, bc_types=bc)
    user = SipgOperator(p, bc, tau_scale=200.0)
    x = torch.zeros_like(b)
    st, its2, _, _ = user.cg_mg(mg, b, x, tol=1e-10)
    assert st == "converged" and its2 == its
