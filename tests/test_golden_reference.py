"""Pin the oracle and the product's host-side builders to fixtures computed by
the reference's own, unmodified code (``tests/golden/make_golden.py`` runs
ddg's ``dg1d/reference.py``, ``dg2d/reference.py``, ``dg2d/mesh.py``,
``dg2d/sipg.py``, ``dg2d/multigrid.py`` and ``dg2d/refinement.py`` over a
numpy-backed JAX stand-in and writes the ``.npz`` files beside it).

CPU only: reference elements, meshes and node maps (bit-exact), operator
applies, loads, dense matrices, coloured block diagonals, and the solves
(CG, LU, singular branch, block-Jacobi PCG, p/hp-multigrid PCG) of the
oracle against the reference's numbers.
"""

import os

import numpy as np
import pytest

from oracle import mesh as om
from oracle import multigrid as omg
from oracle import refelem as ore
from oracle import sipg as osp

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
RTOL_APPLY = 1e-12


def _load(name):
    return np.load(os.path.join(GOLD, name))


def _rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - b)) / max(np.max(np.abs(b)), 1e-300))


def _mesh_names(g):
    return sorted({k.split("/")[0] for k in g.files})


def _oracle_mesh(g, name):
    return om.build_mesh_2d(g[f"{name}/VX"], g[f"{name}/VY"], g[f"{name}/EToV"], int(g[f"{name}/N"]))


@pytest.mark.parametrize("N", range(1, 7))
def test_reference_element_matches_reference(N):
    g = _load("refelem.npz")
    o = ore.RefElement(N)
    for f in ("r", "s", "V", "invV", "Dr", "Ds", "LIFT", "M", "m1d"):
        assert _rel(getattr(o, f), g[f"N{N}_{f}"]) < 1e-12, f
    assert np.array_equal(o.Fmask, g[f"N{N}_Fmask"])


@pytest.mark.parametrize("N", range(1, 7))
def test_product_reference_element_matches_reference(N):
    from ddg_b200.dg2d.reference import ref_element
    g = _load("refelem.npz")
    p = ref_element(N)
    for f in ("r", "s", "V", "invV", "Dr", "Ds", "LIFT", "M", "m1d"):
        assert _rel(getattr(p, f), g[f"N{N}_{f}"]) < 1e-12, f
    assert np.array_equal(p.Fmask, g[f"N{N}_Fmask"])


MAPS = ("EToE", "EToF", "vmapM", "vmapP", "vmapB", "mapB")
GEOM = ("x", "y", "rx", "sx", "ry", "sy", "J", "nx", "ny", "sJ", "Fscale")


@pytest.mark.parametrize("name", ["plain12_N4", "rect4x8_N3", "perturbed5_N2", "refined2x3x2_N4", "tiny2_N2"])
def test_meshes_match_reference(name):
    from ddg_b200.dg2d import mesh as pm
    g = _load("meshes.npz")
    o = _oracle_mesh(g, name)
    p = pm.build_mesh_2d(g[f"{name}/VX"], g[f"{name}/VY"], g[f"{name}/EToV"], int(g[f"{name}/N"]))
    for m in (o, p):
        for f in MAPS:
            assert np.array_equal(np.asarray(getattr(m, f)), g[f"{name}/{f}"]), (name, f)
        for f in GEOM:
            assert _rel(getattr(m, f), g[f"{name}/{f}"]) < 1e-12, (name, f)


def test_uniform_refinement_order_matches_reference():
    """The reference's RefinementForest hierarchy (``multigrid.py:187-204``) and
    the product's / oracle's uniform refinement produce the same vertices and
    the same element order (element 4k+c is child c of k)."""
    from ddg_b200.dg2d import refinement as prf
    from oracle import refinement as orf
    g = _load("meshes.npz")
    name = "refined2x3x2_N4"
    VX, VY, E = om.uniform_rectangle_mesh_2d(0.0, 1.0, 0.0, 2.0, 2, 3)
    hp = prf.uniform_hierarchy(VX, VY, E, 2)[-1]
    ho = orf.build_h_meshes(VX, VY, E, 4, 2)[-1]
    for vx, vy, ev in ((hp[0], hp[1], hp[2]), (ho.VX, ho.VY, ho.EToV)):
        assert np.array_equal(np.asarray(ev), g[f"{name}/EToV"])
        assert np.array_equal(np.asarray(vx), g[f"{name}/VX"])
        assert np.array_equal(np.asarray(vy), g[f"{name}/VY"])


def _apply_cases(a):
    return sorted({k.rsplit("/", 1)[0] for k in a.files if k.endswith("/Au")})


def test_oracle_apply_matches_reference():
    g, a = _load("meshes.npz"), _load("applies.npz")
    meshes = {}
    n = 0
    for case in _apply_cases(a):
        name = case.split("/")[0]
        m = meshes.setdefault(name, _oracle_mesh(g, name))
        tau = 200.0 if case.endswith("udir") else float(case.rsplit("tau", 1)[1])
        ud = a[case + "/u_dir"] if case.endswith("udir") else None
        y = osp.apply(m, a[case + "/u"], bc_types=a[case + "/bc"], u_dir=ud, tau_scale=tau)
        assert _rel(y, a[case + "/Au"]) < RTOL_APPLY, case
        n += 1
    assert n >= 30


def test_oracle_autograd_form_matches_reference():
    """The oracle's literal bilinear form under torch autograd agrees with the
    reference's ``jax.grad`` of its own form."""
    g, a = _load("meshes.npz"), _load("applies.npz")
    for case in ("rect4x8_N3/random/tau0.5", "perturbed5_N2/dir_x_neu_y/tau200"):
        m = _oracle_mesh(g, case.split("/")[0])
        tau = float(case.rsplit("tau", 1)[1])
        y = osp.apply_autograd(m, a[case + "/u"], bc_types=a[case + "/bc"], tau_scale=tau)
        assert _rel(y, a[case + "/Au"]) < RTOL_APPLY, case


def test_oracle_loads_match_reference():
    g, a = _load("meshes.npz"), _load("applies.npz")
    for name in _mesh_names(g):
        m = _oracle_mesh(g, name)
        bc = a[f"{name}/loads/bc"]
        LD = osp.dirichlet_load(m, a[f"{name}/loads/u_dir"], bc_types=bc, tau_scale=200.0)
        LN = osp.neumann_load(m, a[f"{name}/loads/q_neu"], bc_types=bc)
        assert _rel(LD, a[f"{name}/loads/LD"]) < RTOL_APPLY, name
        assert _rel(LN, a[f"{name}/loads/LN"]) < RTOL_APPLY, name


def test_oracle_dense_matrices_match_reference():
    g, a = _load("meshes.npz"), _load("applies.npz")
    m = _oracle_mesh(g, "tiny2_N2")
    bc = a["tiny2_N2/dense/bc"]
    A = osp.dense_matrix(m, bc_types=bc, tau_scale=200.0)
    H = osp.dense_matrix(m, bc_types=bc, tau_scale=200.0, alpha=5.0)
    assert _rel(A, a["tiny2_N2/dense/A"]) < RTOL_APPLY
    assert _rel(H, a["tiny2_N2/dense/H"]) < RTOL_APPLY


@pytest.mark.parametrize("name", ["rect4x8_N3", "perturbed5_N2"])
def test_oracle_block_diagonal_matches_reference(name):
    g, a = _load("meshes.npz"), _load("applies.npz")
    m = _oracle_mesh(g, name)
    col, nc = osp.color_elements(m)
    assert np.array_equal(col, a[f"{name}/blocks/colors"]) and nc == int(a[f"{name}/blocks/ncolors"])
    B = osp.extract_block_diag_matfree(osp.flat_op(m, bc_types=a[f"{name}/blocks/bc"]), m)
    assert _rel(B, a[f"{name}/blocks/B"]) < 1e-11


def test_product_color_elements_matches_reference():
    from ddg_b200.dg2d import mesh as pm
    from ddg_b200.dg2d.sipg import _color_elements
    g, a = _load("meshes.npz"), _load("applies.npz")
    for name in ("rect4x8_N3", "perturbed5_N2"):
        p = pm.build_mesh_2d(g[f"{name}/VX"], g[f"{name}/VY"], g[f"{name}/EToV"], int(g[f"{name}/N"]))
        col, nc = _color_elements(p)
        assert np.array_equal(col, a[f"{name}/blocks/colors"]) and nc == int(a[f"{name}/blocks/ncolors"])


def test_oracle_plain_solves_match_reference():
    """Plain manufactured-solution workload (12x12 quads, N=4, tau_scale=0.5,
    Dirichlet from sin(pi x) sin(pi y), CG tol 1e-9, no preconditioner):
    the oracle's CG and LU solutions against the reference's."""
    g, s = _load("meshes.npz"), _load("solves.npz")
    m = _oracle_mesh(g, "plain12_N4")
    bc = s["plain/bc"]
    ue = np.sin(np.pi * m.x) * np.sin(np.pi * m.y)
    u, it = osp.solve_poisson(m, 2 * np.pi ** 2 * ue, bc_types=bc, u_dir=ue, tau_scale=0.5,
                              iterative=osp.IterativeConfig(tol=1e-9), return_info=True)
    assert abs(it - int(s["plain/cg_iterations"])) <= 2
    assert _rel(u, s["plain/u_cg"]) < 1e-8
    ulu = osp.solve_poisson(m, 2 * np.pi ** 2 * ue, bc_types=bc, u_dir=ue, tau_scale=0.5)
    assert _rel(ulu, s["plain/u_lu"]) < 1e-10


def test_oracle_singular_and_helmholtz_solves_match_reference():
    g, s = _load("meshes.npz"), _load("solves.npz")
    m = _oracle_mesh(g, "rect4x8_N3")
    u, it = osp.solve_poisson(m, s["singular/source"], bc_types=s["singular/bc"], tau_scale=200.0,
                              iterative=osp.IterativeConfig(tol=1e-10), return_info=True)
    assert abs(it - int(s["singular/cg_iterations"])) <= 2
    assert _rel(u, s["singular/u"]) < 1e-8
    VX, VY, E = om.uniform_rectangle_mesh_2d(0.0, 1.0, 0.0, 1.0, 16, 16)
    m = om.build_mesh_2d(VX, VY, E, 4)
    bc = s["helmholtz16/bc"]
    pc = osp.make_block_jacobi(m, bc_types=bc, tau_scale=0.5, alpha=5.0)
    u, it = osp.solve_helmholtz(m, s["helmholtz16/rhs"], alpha=5.0, bc_types=bc, tau_scale=0.5,
                                iterative=osp.IterativeConfig(tol=1e-10, maxiter=5000), preconditioner=pc,
                                return_info=True)
    assert abs(it - int(s["helmholtz16/cg_iterations"])) <= 3
    assert _rel(u, s["helmholtz16/u"]) < 1e-8


def test_oracle_multigrid_matches_reference():
    g, s = _load("meshes.npz"), _load("solves.npz")
    m = _oracle_mesh(g, "rect4x8_N3")
    bc = s["pmg/bc"]
    pc = omg.make_pmg(m, bc_types=bc, tau_scale=200.0)
    assert _rel(pc(s["pmg/vcycle_in"]), s["pmg/vcycle_out"]) < 1e-10
    u, it = osp.solve_poisson(m, s["pmg/source"], bc_types=bc, tau_scale=200.0,
                              iterative=osp.IterativeConfig(tol=1e-8), preconditioner=pc, return_info=True)
    assert it == int(s["pmg/cg_iterations"])
    assert _rel(u, s["pmg/u"]) < 1e-8
    VX, VY, E = om.uniform_rectangle_mesh_2d(0.0, 1.0, 0.0, 2.0, 2, 4)
    base = om.build_mesh_2d(VX, VY, E, 3)
    pc, fine = omg.make_hpmg(base, 2, bc_fn=osp.boundary_bc, tau_scale=200.0)
    assert np.array_equal(fine.EToV, s["hpmg/fine_EToV"])
    assert np.array_equal(osp.boundary_bc(fine), s["hpmg/bc"])
    assert _rel(pc(s["hpmg/vcycle_in"]), s["hpmg/vcycle_out"]) < 1e-10
    u, it = osp.solve_poisson(fine, s["hpmg/source"], bc_types=s["hpmg/bc"], tau_scale=200.0,
                              iterative=osp.IterativeConfig(tol=1e-8), preconditioner=pc, return_info=True)
    assert it == int(s["hpmg/cg_iterations"])
    assert _rel(u, s["hpmg/u"]) < 1e-8
