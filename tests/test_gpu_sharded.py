"""The sharded solve's device path on one GPU (a single NCCL rank): the
rank-local operator, RHS, block-Jacobi and vector kernels of
``libddg_sipg.so`` under the distributed CG give the same solution as the
single-GPU solve.  The multi-rank halo exchange and reductions are tested
as gloo ranks on the CPU (``tests/test_sharded.py``); this run has one GPU."""

import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.parametrize("case", ["helmholtz_bj", "poisson_neumann", "curved_cub"])
def test_sharded_single_rank_matches_single_gpu_solve(case):
    import torch.distributed as dist
    from ddg_b200.dg2d import mesh as pm
    from ddg_b200.dg2d import sipg as ps
    from ddg_b200.dg2d.sharded import ShardedSipg
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_port()}", rank=0, world_size=1)
    try:
        VX, VY, E = pm.uniform_rectangle_mesh_2d(0.0, 2.0, 0.0, 1.0, 24, 12)
        m = pm.build_mesh_2d(VX, VY, E, 3)
        isb = m.EToE == np.arange(m.K)[:, None]
        if case == "helmholtz_bj":
            bc = np.where(isb, 1, 0).astype(np.int32)
            f = np.sin(2 * m.x) * np.cos(3 * m.y) + 0.2
            sh = ShardedSipg(m, bc, tau_scale=0.5)
            u, info = sh.solve(f, alpha=3.0, tol=1e-10, maxiter=3000)
            pc = ps.make_helmholtz_block_jacobi_preconditioner(m, alpha=3.0, nu=1.0, bc_types=bc, tau_scale=0.5)
            ref, rinfo = ps.solve_sipg_helmholtz_2d(m, f, alpha=3.0, nu=1.0, bc_types=bc, tau_scale=0.5,
                                                    preconditioner=pc, return_info=True,
                                                    iterative=ps.IterativeConfig(tol=1e-10, maxiter=3000))
        elif case == "curved_cub":
            from ddg_b200.dg2d import cubature as pcub
            from ddg_b200.dg2d import curved as pcur
            VX, VY, E = pm.rectangle_with_square_hole_mesh_2d(-2.0, 2.0, -2.0, 2.0, 16, 16, -0.5, 0.5, -0.5, 0.5)
            m = pcur.apply_circular_hole_2d(pm.build_mesh_2d(VX, VY, E, 3), cx=0.0, cy=0.0, radius=0.5,
                                            detection_tol=0.5)
            cub = pcub.attach_cubature(m)
            bc = np.where(m.EToE == np.arange(m.K)[:, None], 1, 0).astype(np.int32)
            f = np.cos(m.x) * np.sin(0.7 * m.y) + 0.1
            sh = ShardedSipg(m, bc, tau_scale=0.5, cub=cub)
            u, info = sh.solve(f, alpha=2.0, tol=1e-10, maxiter=3000)
            pc = ps.make_helmholtz_block_jacobi_preconditioner(m, alpha=2.0, nu=1.0, bc_types=bc, tau_scale=0.5,
                                                               cub=cub)
            ref, rinfo = ps.solve_sipg_helmholtz_2d(m, f, alpha=2.0, nu=1.0, bc_types=bc, tau_scale=0.5, cub=cub,
                                                    preconditioner=pc, return_info=True,
                                                    iterative=ps.IterativeConfig(tol=1e-10, maxiter=3000))
        else:
            bc = np.where(isb, 2, 0).astype(np.int32)
            f = np.cos(np.pi * m.x / 2) * np.cos(np.pi * m.y) + 0.3
            sh = ShardedSipg(m, bc, tau_scale=200.0)
            u, info = sh.solve(f, tol=1e-9, maxiter=3000)
            pc = ps.make_sipg_block_jacobi_preconditioner(m, bc_types=bc, tau_scale=200.0)
            ref, rinfo = ps.solve_sipg_poisson_2d(m, f, bc_types=bc, tau_scale=200.0, preconditioner=pc,
                                                  return_info=True,
                                                  iterative=ps.IterativeConfig(tol=1e-9, maxiter=3000))
        assert info.status == "converged" and rinfo.status == "converged"
        # different reduction orders: the 2k-iteration singular solve moves by a few iterations
        assert abs(info.iterations - rinfo.iterations) <= max(2, int(0.01 * rinfo.iterations))
        assert np.linalg.norm(u - ref) <= 1e-6 * np.linalg.norm(ref)
    finally:
        dist.destroy_process_group()
