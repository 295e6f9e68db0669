"""Pin the CPU oracle against every known-answer test the reference's own
suite holds for the SIPG solve path (ddg ships no golden data files).

Each test names the reference test it restates; the tolerances are the
reference's.  These run on CPU only (no GPU, no library).
"""

import numpy as np
import pytest

from oracle import mesh as om
from oracle import multigrid as omg
from oracle import refelem as ore
from oracle import sipg as osp
from oracle import refinement as orf

_MESH = {}


def mesh(Kx, Ky, N, x0=0.0, x1=1.0, y0=0.0, y1=1.0):
    key = (Kx, Ky, N, x0, x1, y0, y1)
    if key not in _MESH:
        _MESH[key] = om.build_mesh_2d(*om.uniform_rectangle_mesh_2d(x0, x1, y0, y1, Kx, Ky), N)
    return _MESH[key]


def rel_l2(m, u, ue):
    return float(np.sqrt(np.sum(m.J * (u - ue) ** 2) / np.sum(m.J * ue ** 2)))


def bc_by_normal(m, dir_pred, neu_pred):
    """test/test_sipg_poisson_2d.py:41-64."""
    nx = m.nx.reshape((m.Nfp, 3, m.K), order="F")[0]
    ny = m.ny.reshape((m.Nfp, 3, m.K), order="F")[0]
    isb = (m.EToE == np.arange(m.K)[:, None]).T
    bc = np.full((3, m.K), osp.BC_INTERIOR, dtype=np.int32)
    bc = np.where(dir_pred(nx, ny) & isb, osp.BC_DIRICHLET, bc)
    bc = np.where(neu_pred(nx, ny) & isb, osp.BC_NEUMANN, bc)
    return bc.T.copy()


def full_dir(m):
    return bc_by_normal(m, lambda a, b: np.ones_like(a, dtype=bool), lambda a, b: np.zeros_like(a, dtype=bool))


def mixed_dir_x(m):
    return bc_by_normal(m, lambda a, b: np.abs(a) > 0.5, lambda a, b: np.abs(b) > 0.5)


def neu_top(m):
    """test/test_sipg_poisson_2d.py:83-102."""
    ny = m.ny.reshape((m.Nfp, 3, m.K), order="F")[0]
    yf = np.stack([m.y[m.Fmask[:, f], :].mean(axis=0) for f in range(3)])
    isb = (m.EToE == np.arange(m.K)[:, None]).T
    neu = isb & (np.abs(ny) > 0.5) & (yf > 0.5)
    bc = np.where(isb & ~neu, osp.BC_DIRICHLET, np.where(neu, osp.BC_NEUMANN, osp.BC_INTERIOR))
    return bc.T.astype(np.int32).copy()


# ------------------------------------------- test/test_reference_2d.py

def test_reference_triangle_area():
    r, s = ore.xy_to_rs(*ore.equilateral_nodes_2d(5))
    V = ore.vandermonde_2d(5, r, s)
    Mm = np.linalg.inv(V @ V.T)
    assert abs(np.ones(21) @ Mm @ np.ones(21) - 2.0) < 1e-10


@pytest.mark.parametrize("N", [2, 3, 4, 6])
def test_d_matrices_exact_on_polynomials(N):
    r, s = ore.xy_to_rs(*ore.equilateral_nodes_2d(N))
    V = ore.vandermonde_2d(N, r, s)
    Dr, Ds = ore.d_matrices_2d(N, r, s, V)
    for p in range(N + 1):
        for q in range(N - p + 1):
            f = r ** p * s ** q
            dfr = p * r ** max(p - 1, 0) * s ** q if p > 0 else 0 * r
            dfs = q * r ** p * s ** max(q - 1, 0) if q > 0 else 0 * r
            assert np.max(np.abs(Dr @ f - dfr)) < 1e-10
            assert np.max(np.abs(Ds @ f - dfs)) < 1e-10


def test_face_masks_positions():
    r, s = ore.xy_to_rs(*ore.equilateral_nodes_2d(5))
    Fm = ore.face_masks_2d(5, r, s)
    assert Fm.shape == (6, 3)
    assert np.max(np.abs(s[Fm[:, 0]] + 1)) < 1e-12
    assert np.max(np.abs(r[Fm[:, 1]] + s[Fm[:, 1]])) < 1e-12
    assert np.max(np.abs(r[Fm[:, 2]] + 1)) < 1e-12


def test_lift_shape():
    e = ore.RefElement(4)
    assert e.LIFT.shape == (15, 15)


def test_grad_simplex_central_differences():
    r = np.array([0.0, 0.1, -0.3, -0.2])
    s = np.array([0.0, -0.5, 0.0, 0.3])
    h = 1e-5
    for (i, j) in [(1, 0), (0, 1), (1, 1), (2, 0), (2, 1)]:
        a, b = ore.rs_to_ab(r, s)
        dr, ds = ore.grad_simplex_2d_p(a, b, i, j)
        f = lambda rr, ss: ore.simplex_2d_p(*ore.rs_to_ab(rr, ss), i, j)  # noqa: E731
        assert np.max(np.abs(dr - (f(r + h, s) - f(r - h, s)) / (2 * h))) < 1e-6
        assert np.max(np.abs(ds - (f(r, s + h) - f(r, s - h)) / (2 * h))) < 1e-6


# ------------------------------------------------- test/test_mesh_2d.py

def test_mesh_shapes_and_jacobian():
    m = mesh(4, 4, 3)
    assert m.Np == 10 and m.K == 32 and m.x.shape == (10, 32) and m.nx.shape == (12, 32)
    np.testing.assert_allclose(m.J, 0.25 * 0.25 / 4.0, atol=1e-12)


def test_internal_face_matching():
    m = mesh(3, 3, 4, -1.0, 1.0, -1.0, 1.0)
    xf, yf = m.x.flatten(order="F"), m.y.flatten(order="F")
    d = np.hypot(xf[m.vmapM] - xf[m.vmapP], yf[m.vmapM] - yf[m.vmapP])
    internal = ~np.isin(np.arange(len(m.vmapM)), m.mapB)
    assert d[internal].max() < 1e-13


def test_unit_normals_and_symmetric_connectivity():
    m = mesh(4, 4, 4)
    assert np.max(np.abs(np.hypot(m.nx, m.ny) - 1.0)) < 1e-13
    for k in range(m.K):
        for f in range(3):
            kp, fp = m.EToE[k, f], m.EToF[k, f]
            if kp == k and fp == f:
                continue
            assert m.EToE[kp, fp] == k and m.EToF[kp, fp] == f


def test_boundary_node_count():
    m = mesh(4, 4, 3)
    assert len(m.mapB) == 4 * (2 * 4 + 2 * 4)


# ------------------------------------------ test/test_sipg_poisson_2d.py

@pytest.mark.parametrize("bcf", [full_dir, mixed_dir_x])
def test_sipg_matrix_symmetric(bcf):
    m = mesh(6, 6, 3)
    A = osp.dense_matrix(m, bc_types=bcf(m))
    assert np.max(np.abs(A - A.T)) < 1e-10


def test_explicit_operator_equals_autograd_form():
    """The explicit restatement equals d a(u,v)/dv of the literal form."""
    m = mesh(3, 4, 3)
    rng = np.random.default_rng(0)
    for bc in (full_dir(m), mixed_dir_x(m), neu_top(m), osp.boundary_bc(m, osp.BC_NEUMANN)):
        u = rng.standard_normal((m.Np, m.K))
        ud = rng.standard_normal((m.Np, m.K))
        for kw in ({}, {"u_dir": ud}):
            a = osp.apply(m, u, bc_types=bc, tau_scale=7.0, **kw)
            b = osp.apply_autograd(m, u, bc_types=bc, tau_scale=7.0, **kw)
            assert np.max(np.abs(a - b)) <= 1e-13 * np.max(np.abs(b))


@pytest.mark.parametrize("N,Kx,Ky", [(3, 6, 6), (3, 10, 10), (4, 8, 8)])
def test_full_dirichlet_manufactured(N, Kx, Ky):
    m = mesh(Kx, Ky, N)
    ue = np.sin(np.pi * m.x) * np.sin(np.pi * m.y)
    u = osp.solve_poisson(m, 2 * np.pi ** 2 * ue, bc_types=full_dir(m))
    assert rel_l2(m, u, ue) < 1e-3


@pytest.mark.parametrize("N,Kx,Ky", [(3, 6, 6), (4, 8, 8)])
def test_mixed_homog_neumann_manufactured(N, Kx, Ky):
    m = mesh(Kx, Ky, N)
    ue = np.sin(np.pi * m.x) * np.cos(np.pi * m.y)
    u = osp.solve_poisson(m, 2 * np.pi ** 2 * ue, bc_types=mixed_dir_x(m))
    assert rel_l2(m, u, ue) < 1e-3


@pytest.mark.parametrize("N", [3, 4])
def test_mixed_nonhomog_neumann_manufactured(N):
    m = mesh(8, 8, N)
    ue = m.x * (1 - m.x) * m.y
    xf = m.x.reshape(-1, order="F")[m.vmapM]
    q = (xf * (1 - xf)).reshape((3 * m.Nfp, m.K), order="F")
    u = osp.solve_poisson(m, 2.0 * m.y, bc_types=neu_top(m), q_neu=q)
    assert rel_l2(m, u, ue) < 1e-3


@pytest.mark.parametrize("alpha", [1.0, 100.0])
def test_helmholtz_manufactured(alpha):
    m = mesh(8, 8, 3)
    ue = np.sin(np.pi * m.x) * np.sin(np.pi * m.y)
    u = osp.solve_helmholtz(m, (2 * np.pi ** 2 + alpha) * ue, alpha=alpha, bc_types=full_dir(m))
    assert rel_l2(m, u, ue) < 1e-3


def test_nonhomog_dirichlet_harmonic():
    m = mesh(8, 8, 3)
    ue = m.x ** 2 - m.y ** 2
    u = osp.solve_poisson(m, 0 * ue, bc_types=full_dir(m), u_dir=ue)
    assert rel_l2(m, u, ue) < 1e-6


def test_cg_matches_lu_poisson_and_helmholtz():
    m = mesh(8, 8, 3)
    ue = np.sin(np.pi * m.x) * np.sin(np.pi * m.y)
    bc = full_dir(m)
    cfg = osp.IterativeConfig(tol=1e-12, maxiter=2000)
    d1 = np.max(np.abs(osp.solve_poisson(m, 2 * np.pi ** 2 * ue, bc_types=bc, iterative=cfg)
                       - osp.solve_poisson(m, 2 * np.pi ** 2 * ue, bc_types=bc)))
    f = (2 * np.pi ** 2 + 100) * ue
    d2 = np.max(np.abs(osp.solve_helmholtz(m, f, alpha=100.0, bc_types=bc, iterative=cfg)
                       - osp.solve_helmholtz(m, f, alpha=100.0, bc_types=bc)))
    assert d1 < 1e-8 and d2 < 1e-8


def test_unsupported_method_raises():
    m = mesh(2, 2, 2)
    with pytest.raises(ValueError):
        osp.solve_poisson(m, 0 * m.x, bc_types=full_dir(m), iterative=osp.IterativeConfig(method="bicg"))


# -------------------------- test/test_block_jacobi_preconditioner.py

def _bj_setup(N=2, K=4, seed=0):
    m = mesh(K, K, N)
    bc = osp.boundary_bc(m)
    src = np.random.default_rng(seed).standard_normal((m.Np, m.K))
    return m, bc, src


def test_pc_matches_unpreconditioned_and_lu():
    m, bc, src = _bj_setup(seed=0)
    cfg = osp.IterativeConfig(tol=1e-11, maxiter=5000)
    pc = osp.make_block_jacobi(m, bc_types=bc)
    u0 = osp.solve_poisson(m, src, bc_types=bc, iterative=cfg)
    u1 = osp.solve_poisson(m, src, bc_types=bc, iterative=cfg, preconditioner=pc)
    ul = osp.solve_poisson(m, src, bc_types=bc)
    assert np.max(np.abs(u0 - u1)) / np.max(np.abs(u0)) < 1e-7
    assert np.max(np.abs(ul - u1)) / np.max(np.abs(ul)) < 1e-7


def test_helmholtz_pc_matches_lu():
    m, bc, src = _bj_setup(seed=2)
    pc = osp.make_block_jacobi(m, bc_types=bc, alpha=50.0)
    cfg = osp.IterativeConfig(tol=1e-11, maxiter=5000)
    u = osp.solve_helmholtz(m, src, alpha=50.0, bc_types=bc, iterative=cfg, preconditioner=pc)
    ul = osp.solve_helmholtz(m, src, alpha=50.0, bc_types=bc)
    assert np.max(np.abs(u - ul)) / np.max(np.abs(ul)) < 1e-7


def test_adjoint_gradient_through_pcg_matches_lu():
    """test_block_jacobi_preconditioner.py:110-138: grad of sum(u^2) wrt the
    source; u = A^-1 (J M f), so grad = (J M)^T A^-T (2u)."""
    m, bc, src = _bj_setup(N=2, K=3, seed=3)
    A = osp.dense_matrix(m, bc_types=bc)
    cfg = osp.IterativeConfig(tol=1e-11, maxiter=5000)
    pc = osp.make_block_jacobi(m, bc_types=bc)
    op = osp.flat_op(m, bc_types=bc)

    def grad(solver):
        u = solver(osp._rhs(m, src, bc, None, None, 200.0))
        lam = solver(2.0 * u)                             # A symmetric: A^-T = A^-1
        return osp._flat(osp.mass_apply(m, osp._unflat(lam[:, None], m.Np, m.K)[:, :, 0]))[:, 0]

    g_lu = grad(lambda b: np.linalg.solve(A, b))
    g_pc = grad(lambda b: osp.cg(op, b, tol=cfg.tol, maxiter=cfg.maxiter, M=pc)[0])
    assert np.max(np.abs(g_lu - g_pc)) / np.max(np.abs(g_lu)) < 1e-6


# ----------------------------- test/test_matfree_preconditioner.py

def test_colouring_valid():
    m = mesh(8, 8, 3)
    col, nc = osp.color_elements(m)
    assert nc <= 4
    for k in range(m.K):
        for nb in m.EToE[k]:
            assert nb == k or col[nb] != col[k]


@pytest.mark.parametrize("alpha", [0.0, 37.0])
def test_matfree_blocks_equal_dense(alpha):
    m = mesh(8, 8, 3)
    bc = osp.boundary_bc(m)
    A = osp.dense_matrix(m, bc_types=bc, alpha=alpha)
    b1 = osp.extract_block_diag_dense(A, m.Np, m.K)
    b2 = osp.extract_block_diag_matfree(osp.flat_op(m, bc_types=bc, alpha=alpha), m)
    v = np.random.default_rng(0).standard_normal(m.Np * m.K)
    z1 = osp.block_jacobi_from_blocks(b1)(v)
    z2 = osp.block_jacobi_from_blocks(b2)(v)
    assert np.max(np.abs(z1 - z2)) < 1e-11
    assert float(v @ z2) > 0.0


# ------------------------------------------ test/test_multigrid_2d.py

def test_pmg_solve_correct():
    m = mesh(8, 8, 4)
    bc = osp.boundary_bc(m)
    A = osp.flat_op(m, bc_types=bc)
    b = np.random.default_rng(0).standard_normal(m.Np * m.K)
    xd = np.linalg.solve(osp.dense_matrix(m, bc_types=bc), b)
    x, it = omg.pcg_count(A, b, omg.make_pmg(m, bc_types=bc), tol=1e-10)
    assert np.linalg.norm(x - xd) / np.linalg.norm(xd) < 1e-7


def test_pmg_beats_block_jacobi_degree_robust():
    pm, bj = {}, {}
    for p in (2, 3, 4, 5):
        m = mesh(8, 8, p)
        bc = osp.boundary_bc(m)
        A = osp.flat_op(m, bc_types=bc)
        b = np.random.default_rng(1).standard_normal(m.Np * m.K)
        _, bj[p] = omg.pcg_count(A, b, osp.make_block_jacobi(m, bc_types=bc))
        _, pm[p] = omg.pcg_count(A, b, omg.make_pmg(m, bc_types=bc))
    assert pm[5] < 0.5 * bj[5] and pm[4] < 0.5 * bj[4]
    assert pm[5] < 2.0 * pm[2] and bj[5] > 1.5 * bj[2]


def test_pmg_helmholtz():
    m = mesh(8, 8, 4)
    bc = osp.boundary_bc(m)
    A = osp.flat_op(m, bc_types=bc, alpha=50.0)
    b = np.random.default_rng(2).standard_normal(m.Np * m.K)
    xd = np.linalg.solve(osp.dense_matrix(m, bc_types=bc, alpha=50.0), b)
    x, itm = omg.pcg_count(A, b, omg.make_pmg(m, bc_types=bc, alpha=50.0), tol=1e-10)
    _, itb = omg.pcg_count(A, b, osp.make_block_jacobi(m, bc_types=bc), tol=1e-10)
    assert np.linalg.norm(x - xd) / np.linalg.norm(xd) < 1e-7 and itm <= itb


def test_hpmg_correct_and_mesh_independent():
    hp, bj = {}, {}
    for nh in (1, 2, 3):
        base = mesh(2, 2, 3)
        mg, fin = omg.make_hpmg(base, nh, bc_fn=osp.boundary_bc)
        bc = osp.boundary_bc(fin)
        A = osp.flat_op(fin, bc_types=bc)
        b = np.random.default_rng(5).standard_normal(fin.Np * fin.K)
        if nh == 2:
            xd = np.linalg.solve(osp.dense_matrix(fin, bc_types=bc), b)
            x, _ = omg.pcg_count(A, b, mg, tol=1e-10)
            assert np.linalg.norm(x - xd) / np.linalg.norm(xd) < 1e-7
        _, hp[nh] = omg.pcg_count(A, b, mg)
        _, bj[nh] = omg.pcg_count(A, b, osp.make_block_jacobi(fin, bc_types=bc))
    assert hp[3] < 1.6 * hp[1] and bj[3] > 1.8 * bj[1] and hp[3] < 0.3 * bj[3]


def test_refined_children_ordering():
    """Element 4k+c of a refined level is child c of element k
    (multigrid.py:187-204): its centroid lies inside the parent."""
    VX, VY, E = om.uniform_rectangle_mesh_2d(0, 1, 0, 1, 2, 2)
    f = orf.UniformForest(VX, VY, E, 1)
    c0 = np.stack([VX[E].mean(1), VY[E].mean(1)], 1)
    f.refine_all()
    VX2, VY2, E2 = f.active()
    for k in range(E.shape[0]):
        for c in range(4):
            t = E2[4 * k + c]
            cx, cy = VX2[t].mean(), VY2[t].mean()
            P = np.stack([VX[E[k]], VY[E[k]]], 1)
            lam = np.linalg.solve(np.vstack([P.T, np.ones(3)]), np.array([cx, cy, 1.0]))
            assert np.all(lam > 0)
    assert np.allclose(c0[0], [VX2[E2[3]].mean(), VY2[E2[3]].mean()])


# ----------------- singular pure-Neumann branch (sipg.py:891-906)

def test_singular_neumann_shifted_solution_is_mean_free():
    """The reference's singular branch solves (A + eps I) x = b - mean(b) with
    eps = 1e-6 ||A probe|| / ||probe||: the solution is exactly mean-free and
    solves the shifted system; it is NOT the exact mean-free solution of
    A x = b (the gap is O(eps / lambda_min), ~10% at this size)."""
    m = mesh(6, 6, 3)
    bc = osp.boundary_bc(m, osp.BC_NEUMANN)
    src = np.cos(np.pi * m.x) * np.cos(np.pi * m.y)
    u, it = osp.solve_poisson(m, src, bc_types=bc, iterative=osp.IterativeConfig(tol=1e-12, maxiter=5000),
                              return_info=True)
    x = u.T.reshape(-1)
    assert abs(x.sum()) < 1e-8 * np.abs(x).sum()
    raw = osp.flat_op(m, bc_types=bc)
    probe = np.sin(np.arange(x.size, dtype=np.float64))
    probe -= probe.mean()
    eps = 1e-6 * np.linalg.norm(raw(probe)) / np.linalg.norm(probe)
    b = osp._rhs(m, src, bc, None, None, 200.0)
    b = b - b.mean()
    assert np.linalg.norm(raw(x) + eps * x - b) < 1e-10 * np.linalg.norm(b)
