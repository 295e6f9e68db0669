"""CPU oracle for the matrix-free SIPG Poisson/Helmholtz path of ddg.

TEST INFRASTRUCTURE ONLY.  Nothing in the ``ddg_b200`` product imports,
links or executes this package.  Only ``tests/``, ``__graft_entry__.smoke()``
and the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` use it,
and only as the checker or the timed CPU baseline, never as the thing
measured on the GPU.

It is a float64 restatement of the reference's algorithm (ddg is pure
Python on JAX; JAX is not installable here, so the reference itself
cannot be run).  Every function cites the reference file:line it follows.

Parity pinning: the reference ships no golden data files.  The oracle is
pinned against every known-answer test the reference's own suite holds for
this path (reference-element identities, mesh known answers, operator
symmetry, manufactured-solution error bounds, CG-vs-LU agreement,
preconditioner equivalences, multigrid iteration properties); see
``tests/test_oracle_kats.py``.  The operator itself is pinned twice: the
literal bilinear form differentiated by torch autograd (the stand-in for
``jax.grad`` in ``src/ddg/dg2d/sipg.py:331-337``) and an explicit
gather/scatter restatement must agree to 1e-13.
"""

from . import refelem, mesh, sipg, multigrid, refinement, cubature, curved  # noqa: F401
