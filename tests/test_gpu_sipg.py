"""GPU parity of the SIPG operator, loads, block-Jacobi and CG against the
CPU oracle (tolerances in each test), plus the reference's manufactured-
solution tests run through the product API."""

import numpy as np
import pytest

from oracle import mesh as om
from oracle import refinement as orf
from oracle import sipg as osp

pytestmark = pytest.mark.gpu

APPLY_RTOL64 = 1e-12       # float64 operator vs oracle (max-abs relative)
APPLY_RTOL32 = 2e-5        # float32 operator vs oracle


def _pair(Kx, Ky, N, x1=1.0, y1=1.0):
    from ddg_b200.dg2d import mesh as pm
    VX, VY, E = om.uniform_rectangle_mesh_2d(0.0, x1, 0.0, y1, Kx, Ky)
    return om.build_mesh_2d(VX, VY, E, N), pm.build_mesh_2d(VX, VY, E, N)


def _refined_pair(N):
    from ddg_b200.dg2d import mesh as pm
    f = orf.UniformForest(*om.uniform_rectangle_mesh_2d(0.0, 1.0, 0.0, 2.0, 2, 3), N)
    f.refine_all()
    f.refine_all()
    a = f.active()
    return om.build_mesh_2d(*a, N), pm.build_mesh_2d(*a, N)


def _bcs(m):
    K = m.K
    isb = m.EToE == np.arange(K)[:, None]
    nx = m.nx.reshape((m.Nfp, 3, K), order="F")[0].T
    out = {
        "dirichlet": np.where(isb, 1, 0).astype(np.int32),
        "neumann": np.where(isb, 2, 0).astype(np.int32),
        "mixed": np.where(isb, np.where(np.abs(nx) > 0.5, 1, 2), 0).astype(np.int32),
        "interior_tagged_boundary": np.zeros((K, 3), dtype=np.int32),
    }
    return out


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("N", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("bcname", ["dirichlet", "neumann", "mixed", "interior_tagged_boundary"])
def test_apply_fp64_matches_oracle(N, bcname):
    from ddg_b200.dg2d.sipg import sipg_apply_2d
    o, p = _pair(5, 4, N)
    bc = _bcs(o)[bcname]
    rng = np.random.default_rng(N)
    u = rng.standard_normal((o.Np, o.K))
    for tau in (200.0, 0.5):
        ref = osp.apply(o, u, bc_types=bc, tau_scale=tau)
        got = sipg_apply_2d(p, u, bc_types=bc, tau_scale=tau)
        assert _rel(got, ref) < APPLY_RTOL64, (N, bcname, tau)


@pytest.mark.parametrize("N", [2, 3, 4])
def test_apply_refined_mesh_and_helmholtz(N):
    import torch
    o, p = _refined_pair(N)
    bc = osp.boundary_bc(o)
    op = p.device_operator(bc, 200.0)
    u = np.random.default_rng(7).standard_normal((o.Np, o.K))
    for alpha in (0.0, 5.0):
        ref = osp.flat_op(o, bc_types=bc, alpha=alpha)(u.T.reshape(-1))
        got = op.apply(torch.as_tensor(u.T.reshape(-1), device="cuda"), alpha=alpha).cpu().numpy()
        assert _rel(got, ref) < APPLY_RTOL64


@pytest.mark.parametrize("N", [1, 3, 4])
def test_apply_fp32_matches_oracle(N):
    import torch
    o, p = _pair(6, 5, N)
    bc = _bcs(o)["mixed"]
    op = p.device_operator(bc, 200.0)
    u = np.random.default_rng(3).standard_normal((o.Np, o.K))
    ref = osp.flat_op(o, bc_types=bc, alpha=3.0)(u.T.reshape(-1))
    got = op.apply(torch.as_tensor(u.T.reshape(-1), dtype=torch.float32, device="cuda"), alpha=3.0)
    assert _rel(got.double().cpu().numpy(), ref) < APPLY_RTOL32


def test_apply_ragged_tail_and_unaligned_pointer():
    """K not a multiple of the tile and a vector that is not 16-byte aligned
    take the plain-load path; results must not change."""
    import torch
    o, p = _pair(7, 3, 3)        # K = 42
    bc = _bcs(o)["dirichlet"]
    op = p.device_operator(bc, 200.0)
    u = np.random.default_rng(1).standard_normal(o.Np * o.K)
    ref = osp.flat_op(o, bc_types=bc)(u)
    buf = torch.zeros(u.size + 1, dtype=torch.float64, device="cuda")
    buf[1:] = torch.as_tensor(u, device="cuda")
    out = torch.zeros(u.size + 1, dtype=torch.float64, device="cuda")
    op.apply(buf[1:], out=out[1:])
    assert _rel(out[1:].cpu().numpy(), ref) < APPLY_RTOL64


def test_loads_match_oracle():
    from ddg_b200.dg2d import sipg as ps
    o, p = _pair(6, 6, 4)
    bc = _bcs(o)["mixed"]
    rng = np.random.default_rng(11)
    ud = rng.standard_normal((o.Np, o.K))
    q = rng.standard_normal((3 * o.Nfp, o.K))
    assert _rel(ps.sipg_dirichlet_load_2d(p, ud, bc_types=bc), osp.dirichlet_load(o, ud, bc_types=bc)) < 1e-12
    assert _rel(ps.sipg_neumann_load_2d(p, q, bc_types=bc), osp.neumann_load(o, q, bc_types=bc)) < 1e-12
    u = rng.standard_normal((o.Np, o.K))
    ref = osp.apply(o, u, bc_types=bc, u_dir=ud)
    assert _rel(ps.sipg_apply_2d(p, u, bc_types=bc, u_dir=ud), ref) < 1e-12


@pytest.mark.parametrize("alpha", [0.0, 37.0])
def test_block_jacobi_blocks_and_apply(alpha):
    from ddg_b200.dg2d import sipg as ps
    o, p = _pair(8, 8, 3)
    bc = osp.boundary_bc(o)
    A = osp.dense_matrix(o, bc_types=bc, alpha=alpha)
    ref_blocks = osp.extract_block_diag_dense(A, o.Np, o.K)
    pc = (ps.make_sipg_block_jacobi_preconditioner(p, bc_types=bc) if alpha == 0.0 else
          ps.make_helmholtz_block_jacobi_preconditioner(p, alpha=alpha, nu=0.01, bc_types=bc))
    got = pc.blocks().cpu().numpy()
    assert np.max(np.abs(got - ref_blocks)) < 1e-11 * max(1.0, np.max(np.abs(ref_blocks)))
    v = np.random.default_rng(0).standard_normal(o.Np * o.K)
    z_ref = osp.block_jacobi_from_blocks(ref_blocks)(v)
    assert np.max(np.abs(pc(v) - z_ref)) < 1e-11 * max(1.0, np.max(np.abs(z_ref)))
    assert float(v @ pc(v)) > 0.0


@pytest.mark.parametrize("use_pc", [False, True])
def test_cg_matches_oracle_cg(use_pc):
    from ddg_b200.dg2d import sipg as ps
    o, p = _pair(8, 8, 3)
    bc = osp.boundary_bc(o)
    src = np.random.default_rng(4).standard_normal((o.Np, o.K))
    cfg_o = osp.IterativeConfig(tol=1e-10, maxiter=3000)
    pco = osp.make_block_jacobi(o, bc_types=bc) if use_pc else None
    u_ref, it_ref = osp.solve_poisson(o, src, bc_types=bc, iterative=cfg_o, preconditioner=pco, return_info=True)
    pcp = ps.make_sipg_block_jacobi_preconditioner(p, bc_types=bc) if use_pc else None
    u, info = ps.solve_sipg_poisson_2d(p, src, bc_types=bc, iterative=ps.IterativeConfig(tol=1e-10, maxiter=3000),
                                       preconditioner=pcp, return_info=True)
    assert info.status == "converged"
    # long CG runs are rounding-sensitive: counts agree to a few percent
    assert abs(info.iterations - it_ref) <= max(2, 0.03 * it_ref)
    assert _rel(u, u_ref) < 1e-8


def test_cg_x0_and_maxiter_and_atol():
    from ddg_b200.dg2d import sipg as ps
    o, p = _pair(6, 6, 2)
    bc = osp.boundary_bc(o)
    src = np.random.default_rng(5).standard_normal((o.Np, o.K))
    u1, i1 = ps.solve_sipg_poisson_2d(p, src, bc_types=bc, iterative=ps.IterativeConfig(tol=1e-12, maxiter=5000),
                                      return_info=True)
    u2, i2 = ps.solve_sipg_poisson_2d(p, src, bc_types=bc, iterative=ps.IterativeConfig(tol=1e-12, maxiter=5000),
                                      x0=u1, return_info=True)
    assert i2.iterations <= 5 and _rel(u2, u1) < 1e-10
    _, i3 = ps.solve_sipg_poisson_2d(p, src, bc_types=bc, iterative=ps.IterativeConfig(tol=1e-14, maxiter=7),
                                     return_info=True)
    assert i3.iterations == 7 and i3.status == "maxiter"
    _, i4 = ps.solve_sipg_poisson_2d(p, src, bc_types=bc, iterative=ps.IterativeConfig(tol=0.0, atol=1e30),
                                     return_info=True)
    assert i4.iterations == 0


# ----------------- the reference's own solve tests, through the product API

def _rel_l2(m, u, ue):
    return float(np.sqrt(np.sum(m.J * (u - ue) ** 2) / np.sum(m.J * ue ** 2)))


@pytest.mark.parametrize("N,Kx,Ky", [(3, 6, 6), (3, 10, 10), (4, 8, 8)])
def test_full_dirichlet_manufactured(N, Kx, Ky):
    from ddg_b200.dg2d import sipg as ps
    o, p = _pair(Kx, Ky, N)
    bc = _bcs(o)["dirichlet"]
    ue = np.sin(np.pi * p.x) * np.sin(np.pi * p.y)
    u_lu = ps.solve_sipg_poisson_2d(p, 2 * np.pi ** 2 * ue, bc_types=bc)
    u_cg = ps.solve_sipg_poisson_2d(p, 2 * np.pi ** 2 * ue, bc_types=bc,
                                    iterative=ps.IterativeConfig(tol=1e-12, maxiter=4000))
    assert _rel_l2(p, u_lu, ue) < 1e-3 and _rel_l2(p, u_cg, ue) < 1e-3
    assert np.max(np.abs(u_cg - u_lu)) < 1e-8


def test_mixed_nonhomog_neumann_and_harmonic_dirichlet():
    from ddg_b200.dg2d import sipg as ps
    o, p = _pair(8, 8, 3)
    ue = p.x * (1 - p.x) * p.y
    xf = p.x.reshape(-1, order="F")[p.vmapM]
    q = (xf * (1 - xf)).reshape((3 * p.Nfp, p.K), order="F")
    ny = p.ny.reshape((p.Nfp, 3, p.K), order="F")[0]
    yf = np.stack([p.y[p.Fmask[:, f], :].mean(axis=0) for f in range(3)])
    isb = (p.EToE == np.arange(p.K)[:, None]).T
    neu = isb & (np.abs(ny) > 0.5) & (yf > 0.5)
    bc = np.where(isb & ~neu, 1, np.where(neu, 2, 0)).T.astype(np.int32)
    cfg = ps.IterativeConfig(tol=1e-12, maxiter=4000)
    u = ps.solve_sipg_poisson_2d(p, 2.0 * p.y, bc_types=bc, q_neu=q, iterative=cfg)
    assert _rel_l2(p, u, ue) < 1e-3
    uh = p.x ** 2 - p.y ** 2
    u2 = ps.solve_sipg_poisson_2d(p, 0 * uh, bc_types=osp.boundary_bc(o), u_dir=uh, iterative=cfg)
    assert _rel_l2(p, u2, uh) < 1e-6


@pytest.mark.parametrize("alpha", [1.0, 100.0])
def test_helmholtz_cg_vs_lu(alpha):
    from ddg_b200.dg2d import sipg as ps
    o, p = _pair(8, 8, 3)
    bc = osp.boundary_bc(o)
    ue = np.sin(np.pi * p.x) * np.sin(np.pi * p.y)
    f = (2 * np.pi ** 2 + alpha) * ue
    u_lu = ps.solve_sipg_helmholtz_2d(p, f, alpha=alpha, nu=1.0, bc_types=bc)
    u_cg = ps.solve_sipg_helmholtz_2d(p, f, alpha=alpha, nu=1.0, bc_types=bc,
                                      iterative=ps.IterativeConfig(tol=1e-12, maxiter=2000))
    assert _rel_l2(p, u_lu, ue) < 1e-3 and np.max(np.abs(u_cg - u_lu)) < 1e-8


def test_singular_neumann_matches_oracle():
    from ddg_b200.dg2d import sipg as ps
    o, p = _pair(6, 6, 3)
    bc = osp.boundary_bc(o, osp.BC_NEUMANN)
    src = np.cos(np.pi * o.x) * np.cos(np.pi * o.y)
    cfg = ps.IterativeConfig(tol=1e-12, maxiter=5000)
    u_ref = osp.solve_poisson(o, src, bc_types=bc, iterative=osp.IterativeConfig(tol=1e-12, maxiter=5000))
    u = ps.solve_sipg_poisson_2d(p, src, bc_types=bc, iterative=cfg)
    assert _rel(u, u_ref) < 1e-7
    assert abs(u.sum()) < 1e-8 * np.abs(u).sum()


@pytest.mark.parametrize("precision", ["mixed", "mixed-restart"])
def test_mixed_precision_reaches_fp64_accuracy(precision):
    """float32 iterations, float64 accuracy: relative error <= 1e-8 against
    the float64 device solve (tau = (N+1)^2/h penalty, mixed BCs)."""
    from ddg_b200.dg2d import sipg as ps
    o, p = _pair(32, 32, 4)
    bc = _bcs(o)["mixed"]
    rng = np.random.default_rng(9)
    src = rng.standard_normal((o.Np, o.K))
    pc = ps.make_helmholtz_block_jacobi_preconditioner(p, alpha=5.0, nu=1.0, bc_types=bc, tau_scale=0.5)
    u64, i64 = ps.solve_sipg_helmholtz_2d(p, src, alpha=5.0, nu=1.0, bc_types=bc, preconditioner=pc,
                                          tau_scale=0.5, iterative=ps.IterativeConfig(tol=1e-13, maxiter=20000),
                                          return_info=True)
    um, info = ps.solve_sipg_helmholtz_2d(p, src, alpha=5.0, nu=1.0, bc_types=bc, preconditioner=pc,
                                          tau_scale=0.5, return_info=True,
                                          iterative=ps.IterativeConfig(tol=1e-12, maxiter=20000,
                                                                       precision=precision))
    assert info.status == "converged", info
    assert np.linalg.norm(um - u64) / np.linalg.norm(u64) < 1e-8
    if precision == "mixed":   # reliable updates keep the iteration count near float64 CG
        assert info.iterations < 1.5 * i64.iterations, (info, i64)


def test_gmres_extension_matches_cg():
    from ddg_b200.dg2d import sipg as ps
    o, p = _pair(6, 6, 3)
    bc = osp.boundary_bc(o)
    src = np.random.default_rng(2).standard_normal((o.Np, o.K))
    u_cg = ps.solve_sipg_poisson_2d(p, src, bc_types=bc, tau_scale=0.5,
                                    iterative=ps.IterativeConfig(tol=1e-11, maxiter=4000))
    u_gm, info = ps.solve_sipg_poisson_2d(p, src, bc_types=bc, return_info=True, tau_scale=0.5,
                                          iterative=ps.IterativeConfig(method="gmres", tol=1e-11, maxiter=4000,
                                                                       restart=60))
    assert info.status == "converged" and _rel(u_gm, u_cg) < 1e-7


def test_errors_are_raised():
    from ddg_b200.dg2d import sipg as ps
    o, p = _pair(2, 2, 2)
    bc = osp.boundary_bc(o)
    with pytest.raises(ValueError):
        ps.solve_sipg_poisson_2d(p, 0 * p.x, bc_types=bc, iterative=ps.IterativeConfig(method="bicg"))
    with pytest.raises(ValueError):
        ps.sipg_apply_2d(p, 0 * p.x, bc_types=bc[:3])
    with pytest.raises(ValueError):
        ps.sipg_apply_2d(p, 0 * p.x, bc_types=bc, cub=object())


# ------------------------- size-independent properties at full size

def test_full_size_operator_symmetry_and_linearity():
    """K = 131072, N = 4 (the precision workload's mesh): u.Av = v.Au and
    A(au + bv) = aAu + bAv, float64, through the C ABI."""
    import torch
    from ddg_b200.dg2d import mesh as pm
    m = pm.build_mesh_2d(*pm.uniform_rectangle_mesh_2d(0, 1, 0, 1, 256, 256), 4)
    isb = m.EToE == np.arange(m.K)[:, None]
    nx = m.nx.reshape((m.Nfp, 3, m.K), order="F")[0].T
    bc = np.where(isb, np.where(np.abs(nx) > 0.5, 1, 2), 0).astype(np.int32)
    op = m.device_operator(bc, 0.5)
    g = torch.Generator(device="cuda").manual_seed(0)
    u = torch.randn(op.n, dtype=torch.float64, device="cuda", generator=g)
    v = torch.randn(op.n, dtype=torch.float64, device="cuda", generator=g)
    Au, Av = op.apply(u, alpha=5.0), op.apply(v, alpha=5.0)
    s1, s2 = float(u @ Av), float(v @ Au)
    assert abs(s1 - s2) <= 1e-12 * (abs(s1) + abs(s2))
    w = op.apply(2.0 * u - 3.0 * v, alpha=5.0)
    assert float(torch.max(torch.abs(w - (2.0 * Au - 3.0 * Av)))) <= 1e-12 * float(torch.max(torch.abs(w)))
    assert float(u @ Au) > 0.0


@pytest.mark.parametrize("shuffle", [False, True])
@pytest.mark.parametrize("Kx,Ky,N", [(64, 64, 4), (96, 48, 3), (67, 65, 4), (37, 23, 2)])
def test_apply_host_chunked_pipeline(Kx, Ky, N, shuffle):
    """Host-buffer apply (chunked copy / apply / copy-back on three streams)
    gives identical results on every call and matches the device apply and
    the oracle to 1e-12, for pinned
    and pageable arrays; shuffled element numbering makes every chunk depend
    on far-away chunks."""
    import torch
    import ddg_b200
    from ddg_b200.dg2d import mesh as pm
    VX, VY, E = om.uniform_rectangle_mesh_2d(0.0, 1.0, 0.0, 1.0, Kx, Ky)
    if shuffle:
        E = E[np.random.default_rng(3).permutation(E.shape[0])]
    o, p = om.build_mesh_2d(VX, VY, E, N), pm.build_mesh_2d(VX, VY, E, N)
    bc = _bcs(o)["mixed"]
    op = p.device_operator(bc, 0.5)
    u = np.random.default_rng(11).standard_normal((o.Np, o.K))
    dev = op.apply(torch.as_tensor(u.T.reshape(-1), device="cuda"), alpha=5.0).cpu().numpy()
    dev = dev.reshape(o.K, o.Np).T
    ref = osp.flat_op(o, bc_types=bc, alpha=5.0, tau_scale=0.5)(u.T.reshape(-1)).reshape(o.K, o.Np).T
    up = ddg_b200.pinned_empty(u.shape)
    up[...] = u
    yp = ddg_b200.pinned_empty(u.shape)
    first = None
    for src, out in ((u, None), (up, yp), (u, yp), (up, None)):
        for _ in range(2):
            got = op.apply_host(src, alpha=5.0, out=out)
            if first is None:
                first = got.copy()
            assert np.array_equal(got, first)       # every call identical
            assert _rel(got, dev) < APPLY_RTOL64    # same operator as the device path
    assert _rel(dev, ref) < APPLY_RTOL64


@pytest.mark.parametrize("N", [1, 2, 3, 4])
@pytest.mark.parametrize("bcname", ["dirichlet", "neumann", "mixed"])
def test_apply_fp32_tensor_cores_match_oracle(N, bcname):
    """float32 apply on the tcgen05 tensor cores (3xTF32) vs the float64
    oracle, and vs the CUDA-core float32 engine; a mesh whose element count
    is not a multiple of the 128-element tile exercises the partial tile."""
    import torch
    o, p = _pair(13, 11, N)
    bc = _bcs(o)[bcname]
    op = p.device_operator(bc, 0.5)
    u = np.random.default_rng(N + 20).standard_normal((o.Np, o.K))
    flat = torch.as_tensor(u.T.reshape(-1).copy(), device="cuda").float()
    for alpha in (0.0, 5.0):
        ref = osp.flat_op(o, bc_types=bc, alpha=alpha, tau_scale=0.5)(u.T.reshape(-1))
        op.set_engine("tensor")
        got_tc = op.apply(flat, alpha=alpha).double().cpu().numpy()
        op.set_engine("cuda")
        got_cc = op.apply(flat, alpha=alpha).double().cpu().numpy()
        op.set_engine("tensor")
        assert _rel(got_cc, ref) < APPLY_RTOL32, (N, bcname, alpha)
        assert _rel(got_tc, ref) < APPLY_RTOL32, (N, bcname, alpha, _rel(got_tc, ref))


def test_apply_fp32_tensor_cores_large_and_repeated():
    """Persistent tensor-core kernel over many tiles (more tiles than CTAs),
    run twice in a row: identical results, float32 accuracy."""
    import torch
    o, p = _pair(96, 80, 4)
    bc = _bcs(o)["mixed"]
    op = p.device_operator(bc, 0.5)
    u = np.random.default_rng(5).standard_normal((o.Np, o.K))
    flat = torch.as_tensor(u.T.reshape(-1).copy(), device="cuda").float()
    y1 = op.apply(flat, alpha=5.0)
    y2 = op.apply(flat, alpha=5.0)
    torch.cuda.synchronize()
    assert torch.equal(y1, y2)
    ref = osp.flat_op(o, bc_types=bc, alpha=5.0, tau_scale=0.5)(u.T.reshape(-1))
    assert _rel(y1.double().cpu().numpy(), ref) < APPLY_RTOL32


def test_fp32_cg_tensor_and_cuda_engines_agree():
    """float32 block-Jacobi PCG whose fused direction-update + apply runs on
    the tensor cores converges like the CUDA-core one (same tolerance,
    iteration counts within 10 %, solutions within float32 accuracy of the
    float64 solve)."""
    import torch
    o, p = _pair(24, 20, 4)
    bc = _bcs(o)["mixed"]
    op = p.device_operator(bc, 0.5)
    op.pc_build(alpha=5.0)
    b = torch.as_tensor(np.random.default_rng(9).standard_normal(op.n), device="cuda")
    x64 = torch.zeros_like(b)
    st, it64, _, _ = op.cg(b, x64, tol=1e-10, maxiter=5000, pc=True, alpha=5.0)
    assert st == "converged"
    res = {}
    for eng in ("tensor", "cuda"):
        op.set_engine(eng)
        x = torch.zeros_like(b, dtype=torch.float32)
        st, its, _, _ = op.cg(b.float(), x, tol=1e-5, maxiter=5000, pc=True, alpha=5.0, precision="fp32")
        assert st == "converged", eng
        res[eng] = (its, x.double())
    op.set_engine("tensor")
    assert abs(res["tensor"][0] - res["cuda"][0]) <= max(3, 0.1 * res["cuda"][0])
    for eng, (its, x) in res.items():
        err = float((x - x64).norm() / x64.norm())
        assert err < 1e-4, (eng, err)
    # mixed precision (float32 iterations on the tensor cores, float64
    # reliable updates) reaches the float64 tolerance
    xm = torch.zeros_like(b)
    st, its, rr, bb, upd = op.cg_mixed(b, xm, tol=1e-10, maxiter=20000, pc=True, alpha=5.0)
    assert st == "converged"
    assert float((xm - x64).norm() / x64.norm()) < 1e-8


@pytest.mark.parametrize("N", [1, 2, 3, 4, 5])
def test_apply_engines_match_oracle(N):
    """Every apply engine against the oracle: float64 (1e-12), float32 CUDA
    cores and tensor cores (float32 tolerance), with Helmholtz mass, mixed
    BCs and a per-element diffusivity; odd element count (partial tiles)."""
    import torch
    o, p = _pair(9, 7, N)
    bc = _bcs(o)["mixed"]
    op = p.device_operator(bc, 0.5)
    rng = np.random.default_rng(N + 40)
    u = rng.standard_normal((o.Np, o.K))
    flat = torch.as_tensor(u.T.reshape(-1).copy(), device="cuda")
    for kappa in (None, np.exp(0.5 * rng.standard_normal(o.K))):
        op.set_kappa(kappa)
        ref = osp.flat_op(o, bc_types=bc, alpha=3.0, tau_scale=0.5, kappa=kappa)(u.T.reshape(-1))
        got = op.apply(flat, alpha=3.0).cpu().numpy()
        assert _rel(got, ref) < APPLY_RTOL64, (N, kappa is None)
        for eng in ["cuda"] + (["tensor"] if N <= 4 else []):
            op.set_engine(eng)
            got = op.apply(flat.float(), alpha=3.0).double().cpu().numpy()
            assert _rel(got, ref) < APPLY_RTOL32, (N, eng, kappa is None)
    op.set_kappa(None)
    if N <= 4:
        op.set_engine("tensor")


@pytest.mark.parametrize("N", [1, 2, 3, 4, 5])
def test_fp64_engines_match_oracle_and_each_other(N):
    """float64 apply on the FP64 tensor cores (the default engine) and on the
    CUDA cores against the oracle (1e-12) for Poisson and Helmholtz under
    every BC set, switched with set_bc (which rebuilds the tensor-core
    kernel's face table), on an odd element count (partial row blocks)."""
    import torch
    o, p = _pair(9, 7, N)
    bcs = _bcs(o)
    op = p.device_operator(bcs["mixed"], 0.5)
    rng = np.random.default_rng(N + 70)
    u = rng.standard_normal((o.Np, o.K))
    flat = torch.as_tensor(u.T.reshape(-1).copy(), device="cuda")
    for name in ("mixed", "dirichlet", "neumann", "interior_tagged_boundary", "mixed"):
        op.set_bc(bcs[name])
        for alpha in (0.0, 3.0):
            ref = osp.flat_op(o, bc_types=bcs[name], alpha=alpha, tau_scale=0.5)(u.T.reshape(-1))
            got = {}
            for eng in ("tensor", "cuda"):
                op.set_engine(eng)
                got[eng] = op.apply(flat, alpha=alpha).cpu().numpy()
                assert _rel(got[eng], ref) < APPLY_RTOL64, (N, name, alpha, eng)
            assert _rel(got["tensor"], got["cuda"]) < 1e-13, (N, name, alpha)
    op.set_engine("tensor")


@pytest.mark.parametrize("N", [2, 4])
def test_fp64_cg_engines_agree(N):
    """float64 block-Jacobi PCG through the FP64 tensor-core kernel's CG
    modes (direction update fused with the apply, residual with norms)
    against the CUDA-core engine: iteration counts within 2, solutions
    within 1e-9 relative."""
    import torch
    o, p = _pair(12, 10, N)
    bc = _bcs(o)["mixed"]
    op = p.device_operator(bc, 0.5)
    op.pc_build(alpha=2.0)
    b = torch.as_tensor(np.random.default_rng(5).standard_normal(op.n), device="cuda")
    res = {}
    for eng in ("tensor", "cuda"):
        op.set_engine(eng)
        x = torch.zeros_like(b)
        st = op.cg(b, x, tol=1e-12, maxiter=5000, pc=True, alpha=2.0)
        assert st[0] == "converged", (eng, st)
        res[eng] = (st[1], x.cpu().numpy())
    op.set_engine("tensor")
    assert abs(res["tensor"][0] - res["cuda"][0]) <= 2
    assert np.linalg.norm(res["tensor"][1] - res["cuda"][1]) / np.linalg.norm(res["cuda"][1]) < 1e-9


def test_apply_host_follows_engine_switch():
    """The host-buffer apply recaptures its pipeline after set_engine: results
    stay equal to the device apply of the engine in force after each switch."""
    import torch
    from ddg_b200.dg2d import mesh as pm
    VX, VY, E = om.uniform_rectangle_mesh_2d(0.0, 1.0, 0.0, 1.0, 24, 20)
    o, p = om.build_mesh_2d(VX, VY, E, 4), pm.build_mesh_2d(VX, VY, E, 4)
    bc = _bcs(o)["mixed"]
    from ddg_b200.dg2d.operator import SipgOperator
    op = SipgOperator(p, bc, tau_scale=0.5)
    u = np.random.default_rng(5).standard_normal((o.Np, o.K))
    ref = osp.flat_op(o, bc_types=bc, alpha=5.0, tau_scale=0.5)(u.T.reshape(-1)).reshape(o.K, o.Np).T
    for engine in ("tensor", "cuda", "tensor", "cuda"):
        op.set_engine(engine)
        dev = op.apply(torch.as_tensor(u.T.reshape(-1), device="cuda"), alpha=5.0).cpu().numpy()
        dev = dev.reshape(o.K, o.Np).T
        got = op.apply_host(u, alpha=5.0)
        assert np.array_equal(got, dev), engine
        assert _rel(got, ref) < APPLY_RTOL64
    op.close()


@pytest.mark.parametrize("use_pc", [False, True])
def test_projected_singular_mode_is_exact_mean_free_solution(use_pc):
    """Pure-Neumann Poisson: nullspace="project" returns the exact solution of
    the consistent system A u = P b (P = projection onto 1-perp) with zero mean,
    checked against the oracle's dense bordered solve; the reference's
    epsilon-shift solution differs from it by a small, stated gap."""
    from ddg_b200.dg2d import sipg as ps
    o, p = _pair(6, 5, 3)
    bc = osp.boundary_bc(o, osp.BC_NEUMANN)
    src = np.cos(np.pi * o.x) * np.cos(np.pi * o.y) + 0.2 * o.x
    A = osp.dense_matrix(o, bc_types=bc, tau_scale=200.0)
    b = osp._rhs(o, src, bc, None, None, 200.0)
    n = b.size
    b = b - b.mean()
    K = np.zeros((n + 1, n + 1))
    K[:n, :n] = A
    K[:n, n] = K[n, :n] = 1.0
    ue = np.linalg.solve(K, np.concatenate([b, [0.0]]))[:n].reshape(o.K, o.Np).T
    pc = ps.make_sipg_block_jacobi_preconditioner(p, bc_types=bc) if use_pc else None
    u, info = ps.solve_sipg_poisson_2d(p, src, bc_types=bc, preconditioner=pc, return_info=True,
                                       iterative=ps.IterativeConfig(tol=1e-12, maxiter=5000, nullspace="project"))
    assert info.status == "converged"
    assert abs(u.mean()) < 1e-12 * np.abs(u).max()
    assert np.linalg.norm(u - ue) / np.linalg.norm(ue) < 1e-9
    # the reference's epsilon-shift mode solves (A + eps I) u = P b, eps =
    # 1e-6 ||A probe|| / ||probe||: it matches the dense shifted solve, and its
    # distance to the exact mean-free solution is the shift's bias
    # (eps / lambda_1 relative on the slowest mode; about 9 % here, where
    # tau_scale = 200 makes ||A|| large against lambda_1)
    probe = np.sin(np.arange(n, dtype=np.float64))
    probe -= probe.mean()
    eps = 1e-6 * np.linalg.norm(A @ probe) / np.linalg.norm(probe)
    ush = np.linalg.solve(A + eps * np.eye(n), b).reshape(o.K, o.Np).T
    us = ps.solve_sipg_poisson_2d(p, src, bc_types=bc, preconditioner=pc,
                                  iterative=ps.IterativeConfig(tol=1e-12, maxiter=5000))
    assert np.linalg.norm(us - ush) / np.linalg.norm(ush) < 1e-8
    gap = np.linalg.norm(us - ue) / np.linalg.norm(ue)
    gap_dense = np.linalg.norm(ush - ue) / np.linalg.norm(ue)
    assert abs(gap - gap_dense) < 1e-6 and gap > 1e-3
