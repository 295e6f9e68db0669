"""Uniform red refinement of a triangle mesh (host setup for hp-multigrid).

Produces the hierarchy ddg's ``multigrid._build_h_meshes`` gets from its
``RefinementForest`` (``src/ddg/dg2d/multigrid.py:187-204``,
``src/ddg/dg2d/refinement.py:210-453``) when every leaf is refined:

* leaves are refined in element order; edge midpoints get new vertex ids in
  order of first use, edges visited (v0,v1), (v1,v2), (v2,v0) per element;
* element k yields children (v0,m01,m20), (m01,v1,m12), (m20,m12,v2),
  (m01,m12,m20) as elements 4k .. 4k+3 (so fine element 4k+c is child c of
  coarse element k);
* every vertex stays in use, so the active-mesh renumbering is the identity.

Vectorised numpy instead of the forest's per-leaf Python loop.
"""

from __future__ import annotations

import numpy as np


def refine_uniform(VX, VY, EToV):
    """One level of red refinement; returns (VX, VY, EToV) of the children."""
    VX = np.asarray(VX, dtype=np.float64)
    VY = np.asarray(VY, dtype=np.float64)
    E = np.asarray(EToV, dtype=np.int64)
    nv, K = VX.shape[0], E.shape[0]
    a = E[:, [0, 1, 2]].reshape(-1)
    b = E[:, [1, 2, 0]].reshape(-1)
    lo, hi = np.minimum(a, b), np.maximum(a, b)
    key = lo * nv + hi
    uniq, first, inv = np.unique(key, return_index=True, return_inverse=True)
    rank = np.empty(uniq.shape[0], dtype=np.int64)
    rank[np.argsort(first, kind="stable")] = np.arange(uniq.shape[0])
    mid = (nv + rank[inv]).reshape(K, 3)                       # m01, m12, m20
    ea, eb = a[first[np.argsort(first, kind="stable")]], b[first[np.argsort(first, kind="stable")]]
    VX2 = np.concatenate([VX, 0.5 * (VX[ea] + VX[eb])])
    VY2 = np.concatenate([VY, 0.5 * (VY[ea] + VY[eb])])
    v0, v1, v2 = E[:, 0], E[:, 1], E[:, 2]
    m01, m12, m20 = mid[:, 0], mid[:, 1], mid[:, 2]
    kids = np.stack([np.stack([v0, m01, m20], 1), np.stack([m01, v1, m12], 1),
                     np.stack([m20, m12, v2], 1), np.stack([m01, m12, m20], 1)], axis=1)
    return VX2, VY2, kids.reshape(4 * K, 3)


def uniform_hierarchy(VX, VY, EToV, n_levels: int):
    """[(VX, VY, EToV)] from the base mesh (coarsest) to n_levels refinements."""
    out = [(np.asarray(VX, dtype=np.float64), np.asarray(VY, dtype=np.float64),
            np.asarray(EToV, dtype=np.int64))]
    for _ in range(n_levels):
        out.append(refine_uniform(*out[-1]))
    return out
