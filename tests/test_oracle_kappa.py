"""CPU pins of the diffusivity extension (no reference counterpart): the
explicit kappa operator equals torch autograd of the literal kappa-weighted
form, reduces to the reference operator at kappa = 1, stays symmetric, and
the form is linear in kappa (so a(u, v) = sum_k kappa_k da/dkappa_k)."""

import numpy as np
import pytest

from oracle import mesh as om
from oracle import sipg as osp


def _mesh():
    return om.build_mesh_2d(*om.uniform_rectangle_mesh_2d(0, 1, 0, 1, 3, 4), 3)


@pytest.mark.parametrize("which", ["dirichlet", "neumann", "mixed"])
def test_kappa_operator_pins(which):
    m = _mesh()
    rng = np.random.default_rng(0)
    isb = m.EToE == np.arange(m.K)[:, None]
    bc = {"dirichlet": np.where(isb, 1, 0), "neumann": np.where(isb, 2, 0),
          "mixed": np.where(isb, np.where(rng.random((m.K, 3)) > 0.5, 1, 2), 0)}[which].astype(np.int32)
    u = rng.standard_normal((m.Np, m.K))
    lam = rng.standard_normal((m.Np, m.K))
    kap = np.exp(0.5 * rng.standard_normal(m.K))
    a = osp.apply(m, u, bc_types=bc, tau_scale=3.0, kappa=kap)
    b = osp.apply_autograd(m, u, bc_types=bc, tau_scale=3.0, kappa=kap)
    assert np.max(np.abs(a - b)) <= 1e-13 * np.max(np.abs(b))
    assert np.array_equal(osp.apply(m, u, bc_types=bc, kappa=np.ones(m.K)), osp.apply(m, u, bc_types=bc))
    A = osp.dense_matrix(m, bc_types=bc, kappa=kap)
    assert np.max(np.abs(A - A.T)) <= 1e-13 * np.max(np.abs(A))
    g = osp.grad_kappa(m, u, lam, bc_types=bc, kappa=kap)
    v, uu = lam.T.reshape(-1), u.T.reshape(-1)
    assert abs(v @ A @ uu - kap @ g) <= 1e-12 * abs(v @ A @ uu)
