"""Host-side (CPU) checks of the product: reference element, mesh and maps
against the oracle, and the C ABI library's exported symbols."""

import os
import re

import numpy as np
import pytest

from ddg_b200 import _lib
from ddg_b200.dg2d import mesh as pm
from ddg_b200.dg2d import reference as pref
from oracle import mesh as om
from oracle import refelem as ore
from oracle import refinement as orf

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("N", [1, 2, 3, 4, 5, 6])
def test_reference_element_matches_oracle(N):
    p, o = pref.RefElement(N), ore.RefElement(N)
    for name in ("r", "s", "V", "invV", "Dr", "Ds", "M", "m1d", "LIFT"):
        a, b = getattr(p, name), getattr(o, name)
        assert np.max(np.abs(a - b)) <= 1e-13 * max(1.0, np.max(np.abs(b))), name
    assert np.array_equal(p.Fmask, o.Fmask)


@pytest.mark.parametrize("N", [1, 2, 3, 4, 5])
def test_rotation_permutations_relabel_faces(N):
    """rot_perm[f] maps the element re-labelled (v_f, v_f+1, v_f+2) back to
    the original numbering: its face-0 nodes are the original face f nodes."""
    e = pref.RefElement(N)
    for f in range(3):
        face0 = e.rot_perm[f][: N + 1]
        assert sorted(face0.tolist()) == sorted(e.Fmask[:, f].tolist())
        assert sorted(e.rot_perm[f].tolist()) == list(range(e.Np))


def _cmp_mesh(VX, VY, E, N):
    o, p = om.build_mesh_2d(VX, VY, E, N), pm.build_mesh_2d(VX, VY, E, N)
    for name in ("EToE", "EToF", "vmapM", "vmapP", "vmapB", "mapB"):
        assert np.array_equal(getattr(o, name), getattr(p, name)), name
    for name in ("x", "y", "rx", "sx", "ry", "sy", "J", "nx", "ny", "sJ", "Fscale"):
        a, b = getattr(p, name), getattr(o, name)
        assert np.max(np.abs(a - b)) <= 1e-12 * max(1.0, np.max(np.abs(b))), name


@pytest.mark.parametrize("Kx,Ky,N", [(1, 1, 1), (3, 3, 2), (4, 5, 3), (12, 12, 4), (7, 3, 5)])
def test_mesh_maps_bit_exact(Kx, Ky, N):
    VX, VY, E = om.uniform_rectangle_mesh_2d(0.0, 1.0, 0.0, 2.0, Kx, Ky)
    VX2, VY2, E2 = pm.uniform_rectangle_mesh_2d(0.0, 1.0, 0.0, 2.0, Kx, Ky)
    assert np.array_equal(VX, VX2) and np.array_equal(VY, VY2) and np.array_equal(E, E2)
    _cmp_mesh(VX, VY, E, N)


def test_refined_mesh_maps_bit_exact():
    f = orf.UniformForest(*om.uniform_rectangle_mesh_2d(0.0, 1.0, 0.0, 2.0, 2, 3), 3)
    f.refine_all()
    f.refine_all()
    _cmp_mesh(*f.active(), 3)


def test_perturbed_vertices_maps_bit_exact():
    VX, VY, E = om.uniform_rectangle_mesh_2d(0.0, 1.0, 0.0, 1.0, 5, 4)
    rng = np.random.default_rng(0)
    inner = (VX > 0) & (VX < 1) & (VY > 0) & (VY < 1)
    VX = VX + 0.03 * rng.standard_normal(VX.shape) * inner
    VY = VY + 0.03 * rng.standard_normal(VY.shape) * inner
    _cmp_mesh(VX, VY, E, 3)


def test_element_geometry_layout():
    m = pm.build_mesh_2d(*pm.uniform_rectangle_mesh_2d(0, 1, 0, 1, 2, 2), 2)
    g = m.element_geometry()
    assert g.shape == (m.K, 14)
    np.testing.assert_array_equal(g[:, 4], m.J[0])
    np.testing.assert_array_equal(g[:, 10], m.sJ[m.Nfp])       # sJ of face 1
    np.testing.assert_array_equal(g[:, 11], m.nx[2 * m.Nfp])    # nx of face 2


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    header = open(os.path.join(ROOT, "include", "ddg_sipg.h")).read()
    declared = sorted(set(re.findall(r"\b(ddg_[a-z0-9_]+)\s*\(", header)))
    assert declared, "no declarations parsed"
    for name in declared:
        assert hasattr(L, name), name
    assert set(_lib.exported_symbols()) <= set(declared)
    assert L.ddg_version().decode().startswith("ddg_sipg")


def test_mesh_connect_rejects_bad_input():
    L = _lib.lib()
    E = np.array([[0, 1, -2]], dtype=np.int64)
    out = np.zeros((1, 3), dtype=np.int64)
    rc = L.ddg_mesh_connect(1, E.ctypes.data, out.ctypes.data, out.ctypes.data)
    assert rc == 1 and b"negative" in L.ddg_last_error()


def test_no_cpu_fallback_in_product():
    """The product never imports the oracle."""
    for dirpath, _, files in os.walk(os.path.join(ROOT, "ddg_b200")):
        for fn in files:
            if fn.endswith(".py"):
                src = open(os.path.join(dirpath, fn)).read()
                assert "oracle" not in re.findall(r"^\s*(?:from|import)\s+(\w+)", src, re.M), fn
