"""The dual-splitting Navier-Stokes step (row f2) against the reference's own
``ns_step_2d`` (fixture ``tests/golden/ins.npz``, generated from the
unmodified reference): the explicit advection and pressure-Neumann terms on
the host (CPU tests), and whole steps through the device solves (GPU tests),
at the reference test's tolerance (``test/test_ins_multigrid_2d.py``: 1e-6)."""

import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ins.npz")


def _setup():
    from ddg_b200.dg2d import mesh as pm
    g = np.load(GOLD)
    m = pm.build_mesh_2d(g["VX"], g["VY"], g["EToV"], 3)
    return g, m


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - b) / np.linalg.norm(b))


def test_bc_conversions():
    from ddg_b200.dg2d import incompressible_ns as ins
    b = np.array([[0, 1, 2], [3, 4, 0]])
    assert np.array_equal(ins.pressure_bc_types_from_ins(b), [[0, 2, 1], [2, 2, 0]])
    assert np.array_equal(ins.viscous_bc_types_from_ins(b), [[0, 1, 2], [1, 1, 0]])


def test_explicit_terms_match_reference():
    from ddg_b200.dg2d import incompressible_ns as ins
    g, m = _setup()
    zero = np.zeros((m.Np, m.K))
    nux, nuy = ins.ns_advection_2d(m, g["ux0"], g["uy0"], ins_bc_types=g["ins_bc"], bc_ux=zero, bc_uy=zero)
    assert _rel(nux, g["Nux_old"]) < 1e-12 and _rel(nuy, g["Nuy_old"]) < 1e-12
    d = ins.ns_pressure_neumann_data(m, g["ux0"], g["uy0"], nux, nuy, nu=0.02)
    assert _rel(d, g["lu/dpdn"]) < 1e-12


def _step(m, g, **kw):
    from ddg_b200.dg2d import incompressible_ns as ins
    zero = np.zeros((m.Np, m.K))
    dpdn0 = np.zeros((3 * m.Nfp, m.K))
    return ins.ns_step_2d(m, g["ux0"], g["uy0"], g["ux0"], g["uy0"], g["Nux_old"], g["Nuy_old"], dpdn0,
                          dt=0.01, nu=0.02, bdf=ins.BDF1, ins_bc_types=g["ins_bc"], bc_ux=zero, bc_uy=zero, **kw)


@pytest.mark.gpu
def test_ins_step_direct_matches_reference():
    from ddg_b200.dg2d import incompressible_ns as ins
    g, m = _setup()
    ops = ins.build_ins_operators(m, dt=0.01, nu=0.02, g0=1.0, ins_bc_types=g["ins_bc"])
    ux, uy, p, *_ = _step(m, g, ops=ops)
    assert _rel(ux, g["lu/ux"]) < 1e-9 and _rel(uy, g["lu/uy"]) < 1e-9 and _rel(p, g["lu/p"]) < 1e-9


@pytest.mark.gpu
def test_ins_step_multigrid_cg_matches_reference():
    """Matrix-free device CG with the device p-multigrid preconditioners and
    warm-started viscous solves, against both of the reference's paths."""
    from ddg_b200.dg2d import incompressible_ns as ins
    from ddg_b200.dg2d.sipg import IterativeConfig
    g, m = _setup()
    ops = ins.build_ins_operators(m, dt=0.01, nu=0.02, g0=1.0, ins_bc_types=g["ins_bc"], skip_factor=True)
    pp, vp = ins.make_ins_mg_preconditioners(m, dt=0.01, nu=0.02, g0=1.0, ins_bc_types=g["ins_bc"])
    ux, uy, p, nux, nuy, dpdn = _step(m, g, ops=ops, iterative=IterativeConfig(tol=1e-11, maxiter=3000),
                                      pressure_preconditioner=pp, viscous_preconditioner=vp)
    for tag in ("mg", "lu"):
        assert _rel(ux, g[f"{tag}/ux"]) < 1e-6 and _rel(uy, g[f"{tag}/uy"]) < 1e-6
        assert _rel(p, g[f"{tag}/p"]) < 1e-6
    assert _rel(dpdn, g["mg/dpdn"]) < 1e-12


@pytest.mark.gpu
def test_ins_second_step_bdf2_matches_reference():
    from ddg_b200.dg2d import incompressible_ns as ins
    from ddg_b200.dg2d.sipg import IterativeConfig
    g, m = _setup()
    zero = np.zeros((m.Np, m.K))
    ops = ins.build_ins_operators(m, dt=0.01, nu=0.02, g0=ins.BDF2.g0, ins_bc_types=g["ins_bc"],
                                  skip_factor=True)
    ux, uy, p, *_ = ins.ns_step_2d(m, g["lu/ux"], g["lu/uy"], g["ux0"], g["uy0"], g["lu/Nux"], g["lu/Nuy"],
                                   g["lu/dpdn"], dt=0.01, nu=0.02, bdf=ins.BDF2, ops=ops,
                                   ins_bc_types=g["ins_bc"], bc_ux=zero, bc_uy=zero,
                                   iterative=IterativeConfig(tol=1e-12, maxiter=5000))
    assert _rel(ux, g["bdf2/ux"]) < 1e-6 and _rel(uy, g["bdf2/uy"]) < 1e-6 and _rel(p, g["bdf2/p"]) < 1e-6
