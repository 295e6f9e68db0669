"""Sharded solve (one process per GPU), host side: the strip partition, the
ghost layer and halo slices, and the distributed CG itself, run as gloo
ranks on the CPU with the oracle as each rank's local operator (the device
local operator is exercised by the single-rank GPU test).  The distributed
solve must reproduce the single-process oracle solve: same CG iterations
(up to one, from the reduction order) and the same solution."""

import os
import socket

import numpy as np
import pytest

from oracle import sipg as osp


def _mesh(kx=12, ky=6, N=2, lx=2.0):
    from ddg_b200.dg2d import mesh as pm
    VX, VY, E = pm.uniform_rectangle_mesh_2d(0.0, lx, 0.0, 1.0, kx, ky)
    return pm.build_mesh_2d(VX, VY, E, N)


def _bc(m, code):
    return np.where(m.EToE == np.arange(m.K)[:, None], code, 0).astype(np.int32)


@pytest.mark.parametrize("world", [1, 2, 3, 4])
def test_shard_plan_partition_and_halo_slices(world):
    from ddg_b200.dg2d.sharded import ShardPlan
    m = _mesh()
    P = ShardPlan(m, world)
    owned = np.concatenate([p.elements[:p.n_own] for p in P.parts])
    assert np.array_equal(np.sort(owned), np.arange(m.K))              # a partition
    for r, p in enumerate(P.parts):
        lm = P.local_mesh(r)
        L = p.elements
        assert np.array_equal(P.owner[L[:p.n_own]], np.full(p.n_own, r))
        assert np.all(P.owner[L[p.n_own:]] != r)
        assert np.array_equal(lm.x, m.x[:, L]) and np.array_equal(lm.J, m.J[:, L])
        # every owned element keeps its global neighbours (now local ids)
        for kl in range(p.n_own):
            assert np.array_equal(np.sort(L[lm.EToE[kl]]), np.sort(m.EToE[L[kl]]))
            assert np.array_equal(lm.EToF[kl], m.EToF[L[kl]])
        # halo slices: what r sends to q is what q receives from r, in order
        for q, (a, b) in p.send.items():
            qa, qb = P.parts[q].recv[r]
            assert np.array_equal(L[a:b], P.parts[q].elements[qa:qb])
        ghosts = np.concatenate([L[a:b] for a, b in p.recv.values()]) if p.recv else np.zeros(0, int)
        assert np.array_equal(np.sort(ghosts), np.sort(L[p.n_own:]))


class OracleLocalOps:
    """A rank's local operator and vector kernels computed by the oracle on
    the CPU (test stand-in for the device local operator)."""

    def __init__(self, lm, lbc, tau, cub=None):
        import torch
        self.torch = torch
        self.lm, self.bc, self.tau, self.cub = lm, lbc, tau, cub
        self.n = lm.K * lm.Np
        self.device = None

    def vector(self, f):
        if f is None:
            return None
        return self.torch.tensor(np.asarray(f, dtype=np.float64).T.reshape(-1).copy())

    def zeros(self):
        return self.torch.zeros(self.n, dtype=self.torch.float64)

    def _field(self, v):
        return v.numpy().reshape(self.lm.K, self.lm.Np).T

    def apply(self, v, alpha):
        U = self._field(v)
        Y = osp.apply(self.lm, U, bc_types=self.bc, tau_scale=self.tau, cub=self.cub)
        if alpha != 0.0:
            Y = Y + alpha * osp.mass_apply(self.lm, U, self.cub)
        return self.torch.tensor(Y.T.reshape(-1).copy())

    def rhs(self, f, u_dir, q_neu):
        fld = lambda v: None if v is None else self._field(v)  # noqa: E731
        q = None if q_neu is None else q_neu.numpy().reshape(self.lm.K, -1).T
        return self.torch.tensor(osp._rhs(self.lm, fld(f), self.bc, fld(u_dir), q, self.tau, self.cub).copy())

    def pc_build(self, alpha):
        B = osp.extract_block_diag_matfree(osp.flat_op(self.lm, bc_types=self.bc, tau_scale=self.tau,
                                                       alpha=alpha, cub=self.cub), self.lm)
        self.Binv = np.linalg.inv(B)

    def pc_apply(self, r):
        Z = np.einsum("kij,kj->ki", self.Binv, r.numpy().reshape(self.lm.K, self.lm.Np))
        return self.torch.tensor(Z.reshape(-1).copy())

    def dot(self, a, b, n):
        return float(a[:n] @ b[:n])

    def axpby(self, a, x, b, y):
        y.mul_(b).add_(x, alpha=a)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, name, q):
    import torch.distributed as dist
    from ddg_b200.dg2d.sharded import ShardedSipg
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        case = CASES[name]
        m, cub = case.get("mesh", lambda: (_mesh(), None))()
        kw = case["kw"]
        bc = case["bc"](m)
        tau = kw["tau"]
        sh = ShardedSipg(m, bc, tau_scale=tau, local_ops=OracleLocalOps, cub=cub)
        u, info = sh.solve(case["src"](m), alpha=kw["alpha"], u_dir=case.get("udir", lambda m: None)(m),
                           tol=kw["tol"], maxiter=2000, preconditioner=kw["pc"])
        if rank == 0:
            q.put((u, info.iterations, info.status))
    finally:
        dist.destroy_process_group()


def _curved_mesh():
    """A bent annulus (degree 2) with its cubature: the curved branch."""
    from ddg_b200.dg2d import cubature as pcub
    from ddg_b200.dg2d import curved as pcur
    from ddg_b200.dg2d import mesh as pm
    VX, VY, E = pm.rectangle_with_square_hole_mesh_2d(-2.0, 2.0, -2.0, 2.0, 16, 16, -0.5, 0.5, -0.5, 0.5)
    m = pcur.apply_circular_hole_2d(pm.build_mesh_2d(VX, VY, E, 2), cx=0.0, cy=0.0, radius=0.5, detection_tol=0.5)
    return m, pcub.attach_cubature(m)


CASES = {
    "curved_helmholtz_cub": dict(kw=dict(tau=0.5, alpha=2.0, tol=1e-11, pc="block_jacobi"),
                                 mesh=_curved_mesh, bc=lambda m: _bc(m, 1),
                                 src=lambda m: np.cos(m.x) * np.sin(0.7 * m.y) + 0.1),
    "helmholtz_bj": dict(kw=dict(tau=0.5, alpha=3.0, tol=1e-11, pc="block_jacobi"),
                         bc=lambda m: _bc(m, 1),
                         src=lambda m: np.sin(2 * m.x) * np.cos(3 * m.y) + 0.2),
    "poisson_dirichlet_plain": dict(kw=dict(tau=200.0, alpha=0.0, tol=1e-10, pc=None),
                                    bc=lambda m: _bc(m, 1),
                                    src=lambda m: np.ones_like(m.x),
                                    udir=lambda m: np.sin(m.x) * m.y),
    "poisson_neumann_singular": dict(kw=dict(tau=200.0, alpha=0.0, tol=1e-9, pc="block_jacobi"),
                                     bc=lambda m: _bc(m, 2),
                                     src=lambda m: np.cos(np.pi * m.x / 2) * np.cos(np.pi * m.y) + 0.3),
}


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("name", sorted(CASES))
def test_sharded_cg_matches_single_process(world, name):
    import torch.multiprocessing as mp
    case = CASES[name]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, name, q)) for r in range(world)]
    for p in procs:
        p.start()
    u, its, status = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    # the single-process oracle solve of the same system
    m, cub = case.get("mesh", lambda: (_mesh(), None))()
    kw = case["kw"]
    bc = case["bc"](m)
    udir = case.get("udir", lambda m: None)(m)
    M = None
    if kw["pc"]:
        B = osp.extract_block_diag_matfree(osp.flat_op(m, bc_types=bc, tau_scale=kw["tau"], alpha=kw["alpha"],
                                                       cub=cub), m)
        M = osp.block_jacobi_from_blocks(B)
    cfg = osp.IterativeConfig(tol=kw["tol"], maxiter=2000)
    if kw["alpha"] > 0:
        ref, rits = osp.solve_helmholtz(m, case["src"](m), alpha=kw["alpha"], bc_types=bc, tau_scale=kw["tau"],
                                        iterative=cfg, preconditioner=M, return_info=True, cub=cub)
    else:
        ref, rits = osp.solve_poisson(m, case["src"](m), bc_types=bc, u_dir=udir, tau_scale=kw["tau"],
                                      iterative=cfg, preconditioner=M, return_info=True)
    assert status == "converged"
    assert abs(its - rits) <= 1
    assert np.linalg.norm(u - ref) <= 1e-8 * np.linalg.norm(ref)
