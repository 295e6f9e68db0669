"""Oracle: uniform red refinement (the h-hierarchy source of hp-multigrid).

Test infrastructure only (see ``oracle/__init__.py``).

Restates the part of ``RefinementForest`` (``src/ddg/dg2d/refinement.py``)
that ``multigrid._build_h_meshes`` (``src/ddg/dg2d/multigrid.py:187-204``)
exercises: refine every leaf (:210-244; with every leaf marked, the 2:1 and
green-closability closure :246-346 adds nothing), shared edge midpoints
created once in refinement order (:348-357), children
(v0,m01,m20),(m01,v1,m12),(m20,m12,v2),(m01,m12,m20) (:359-380), and the
active mesh of leaves in node-id order with unused vertices pruned
(:389-453).  Element 4k+c of a refined level is child c of element k.
"""

from __future__ import annotations

import numpy as np

from .mesh import build_mesh_2d


def _edge(a, b):
    return (a, b) if a < b else (b, a)


class UniformForest:
    def __init__(self, VX, VY, EToV, N):
        self.N = N
        self.vx = [float(v) for v in VX]
        self.vy = [float(v) for v in VY]
        self.leaves = [tuple(int(t) for t in tri) for tri in np.asarray(EToV)]
        self.mid = {}

    def _midpoint(self, a, b):
        e = _edge(a, b)
        m = self.mid.get(e)
        if m is None:
            m = len(self.vx)
            self.vx.append(0.5 * (self.vx[a] + self.vx[b]))
            self.vy.append(0.5 * (self.vy[a] + self.vy[b]))
            self.mid[e] = m
        return m

    def refine_all(self):
        new = []
        for v0, v1, v2 in self.leaves:
            m01 = self._midpoint(v0, v1)
            m12 = self._midpoint(v1, v2)
            m20 = self._midpoint(v2, v0)
            new += [(v0, m01, m20), (m01, v1, m12), (m20, m12, v2), (m01, m12, m20)]
        self.leaves = new

    def active(self):
        E = np.asarray(self.leaves, dtype=np.int64)
        used = np.unique(E.reshape(-1))
        remap = -np.ones(len(self.vx), dtype=np.int64)
        remap[used] = np.arange(used.shape[0])
        return (np.asarray(self.vx)[used], np.asarray(self.vy)[used], remap[E])


def build_h_meshes(base_VX, base_VY, base_EToV, N, n_levels):
    """``multigrid.py:187-204``: [coarsest, ..., finest] meshes of degree N."""
    f = UniformForest(base_VX, base_VY, base_EToV, N)
    out = [build_mesh_2d(*f.active(), N)]
    for _ in range(n_levels):
        f.refine_all()
        out.append(build_mesh_2d(*f.active(), N))
    return out
