"""A numpy-backed stand-in for the small part of JAX that ddg's SIPG path uses.

TEST INFRASTRUCTURE ONLY: it lets ``make_golden.py`` import the UNMODIFIED
reference sources (``src/ddg/dg1d/reference.py``, ``src/ddg/dg2d/reference.py``,
``src/ddg/dg2d/mesh.py``, ``src/ddg/dg2d/sipg.py``, ``src/ddg/dg2d/multigrid.py``,
``src/ddg/dg2d/refinement.py``) in a container where JAX cannot be installed,
so that golden fixtures come from the reference's own code rather than from a
restatement of it.  Nothing in the product or in the GPU tests imports it.

What it provides, and how each piece relates to JAX's documented behaviour:

* ``jax.numpy``: numpy, with arrays returned as an ndarray subclass that
  carries JAX's functional update syntax ``x.at[idx].set/add/multiply/get``
  (each returns a new array, as JAX's does).
* ``jax.grad``: reverse-mode differentiation of a scalar function of one
  array argument, over a recorded tape of the operations the reference's
  bilinear form (``sipg.py:142-301``) applies to its argument: products with
  constant arrays (``*``, ``@``, ``einsum``), sums, differences, transposes,
  C/F-order reshapes, integer-array gathers, ``where`` and ``sum``.  A product
  of two recorded values (not needed by a bilinear form) is supported by the
  product rule.  Any other operation on a recorded value raises, so a silent
  wrong gradient is not possible.
* ``jax.jacobian``: column probing ``J[:, i] = f(x0 + e_i) - f(x0)``, which
  is exact for the affine maps the reference passes to it
  (``sipg.py:356-364``, ``multigrid.py:222``); affinity is checked on a
  random combination of columns.
* ``jax.vmap``: a Python loop over the leading axis, stacked.
* ``jax.scipy.linalg.lu_factor / lu_solve``: scipy's (same LAPACK getrf/getrs).
* ``jax.scipy.sparse.linalg.cg``: JAX's documented preconditioned CG
  (x0 defaults to zero, r0 = b - A x0, z = M r, p = z, stop when
  ``r.r <= max(tol^2 b.b, atol^2)`` or after ``maxiter`` iterations, default
  ``10 n``; returns ``(x, None)``), restated from its published algorithm.
* ``jax.config.update``, ``jax.tree_util.register_pytree_node``,
  ``jax.jit``: no-ops / identity.

``install(ref_src)`` registers these modules and empty ``ddg``, ``ddg.dg1d``,
``ddg.dg2d`` packages (so the reference's package ``__init__`` files, which
pull in unrelated solvers, are not executed) and returns an import helper.
"""

from __future__ import annotations

import importlib
import os
import sys
import types

import numpy as np
import scipy.linalg as sla


# ---------------------------------------------------------------------------
# arrays with JAX's .at[] functional updates
# ---------------------------------------------------------------------------

class _AtRef:
    def __init__(self, arr, idx):
        self.arr, self.idx = arr, idx

    def set(self, val):
        out = np.array(self.arr, copy=True).view(JArray)
        out[self.idx] = _val(val)
        return out

    def add(self, val):
        out = np.array(self.arr, copy=True).view(JArray)
        np.add.at(out, self.idx, _val(val)) if _is_fancy(self.idx) else out.__setitem__(
            self.idx, out[self.idx] + _val(val))
        return out

    def multiply(self, val):
        out = np.array(self.arr, copy=True).view(JArray)
        out[self.idx] = out[self.idx] * _val(val)
        return out

    def get(self):
        return self.arr[self.idx]


def _is_fancy(idx):
    items = idx if isinstance(idx, tuple) else (idx,)
    return any(isinstance(i, (np.ndarray, list)) for i in items)


class _AtIndexer:
    def __init__(self, arr):
        self.arr = arr

    def __getitem__(self, idx):
        return _AtRef(self.arr, idx)


class JArray(np.ndarray):
    """ndarray with JAX's ``.at[idx].set(...)`` style functional updates."""

    @property
    def at(self):
        return _AtIndexer(self)


def _wrap(x):
    if isinstance(x, np.ndarray) and not isinstance(x, JArray):
        return x.view(JArray)
    if isinstance(x, tuple):
        return tuple(_wrap(e) for e in x)
    if isinstance(x, list):
        return [_wrap(e) for e in x]
    return x


# ---------------------------------------------------------------------------
# reverse-mode tape
# ---------------------------------------------------------------------------

class Var:
    """A recorded value: ``val`` plus the vector-Jacobian products of its inputs."""

    __array_ufunc__ = None          # make numpy defer to our reflected operators
    __array_priority__ = 1000

    def __init__(self, val, parents=()):
        self.val = np.asarray(val)
        self.parents = parents      # tuple of (Var, vjp: cotangent -> cotangent of parent)

    # -- shape helpers
    @property
    def shape(self):
        return self.val.shape

    @property
    def ndim(self):
        return self.val.ndim

    @property
    def dtype(self):
        return self.val.dtype

    @property
    def T(self):
        return Var(self.val.T, ((self, lambda g: g.T),))

    def __len__(self):
        return len(self.val)

    def reshape(self, *shape, order="C"):
        if len(shape) == 1 and isinstance(shape[0], (tuple, list)):
            shape = tuple(shape[0])
        old = self.val.shape
        return Var(self.val.reshape(shape, order=order),
                   ((self, lambda g: np.reshape(g, old, order=order)),))

    def __getitem__(self, idx):
        old = self.val.shape

        def vjp(g):
            out = np.zeros(old, dtype=np.result_type(g, np.float64))
            np.add.at(out, idx, g)
            return out
        return Var(self.val[idx], ((self, vjp),))

    # -- arithmetic
    def __neg__(self):
        return Var(-self.val, ((self, lambda g: -g),))

    def __add__(self, o):
        if isinstance(o, Var):
            return Var(self.val + o.val, ((self, _unbroadcast(lambda g: g, self.shape)),
                                          (o, _unbroadcast(lambda g: g, o.shape))))
        o = _val(o)
        return Var(self.val + o, ((self, _unbroadcast(lambda g: g, self.shape)),))

    __radd__ = __add__

    def __sub__(self, o):
        return self + (-o if isinstance(o, Var) else -_val(o))

    def __rsub__(self, o):
        return (-self) + o

    def __mul__(self, o):
        if isinstance(o, Var):
            a, b = self, o
            return Var(a.val * b.val, ((a, _unbroadcast(lambda g: g * b.val, a.shape)),
                                       (b, _unbroadcast(lambda g: g * a.val, b.shape))))
        c = _val(o)
        return Var(self.val * c, ((self, _unbroadcast(lambda g: g * c, self.shape)),))

    __rmul__ = __mul__

    def __truediv__(self, o):
        if isinstance(o, Var):
            raise TypeError("refshim: division by a recorded value is not supported")
        c = _val(o)
        return Var(self.val / c, ((self, _unbroadcast(lambda g: g / c, self.shape)),))

    def __matmul__(self, o):
        if isinstance(o, Var):
            raise TypeError("refshim: product of two recorded values under @ is not supported")
        c = _val(o)
        return Var(self.val @ c, ((self, lambda g: _matmul_vjp_left(g, c, self.shape)),))

    def __rmatmul__(self, o):
        c = _val(o)
        return Var(c @ self.val, ((self, lambda g: _matmul_vjp_right(c, g, self.shape)),))

    def astype(self, dt):
        return Var(self.val.astype(dt), ((self, lambda g: g),))

    def __repr__(self):
        return f"Var(shape={self.shape})"

    # anything else touching a recorded value is an error
    def __array__(self, *a, **k):
        raise TypeError("refshim: a recorded value was converted to a plain array; "
                        "the reference used an operation this shim does not differentiate")


def _matmul_vjp_left(g, c, shape):
    # y = x @ c ; dx = g @ c^T
    if c.ndim == 1:
        return np.multiply.outer(g, c).reshape(shape)
    return g @ np.swapaxes(c, -1, -2)


def _matmul_vjp_right(c, g, shape):
    # y = c @ x ; dx = c^T @ g  (c 1-D: y = sum_i c_i x_i, dx = outer(c, g))
    if c.ndim == 1:
        return np.multiply.outer(c, g).reshape(shape)
    return np.swapaxes(c, -1, -2) @ g


def _unbroadcast(f, shape):
    def vjp(g):
        g = np.asarray(f(g))
        while g.ndim > len(shape):
            g = g.sum(axis=0)
        for ax, n in enumerate(shape):
            if n == 1 and g.shape[ax] != 1:
                g = g.sum(axis=ax, keepdims=True)
        return np.broadcast_to(g, shape)
    return vjp


def _val(x):
    return x.val if isinstance(x, Var) else np.asarray(x) if isinstance(x, (list, tuple)) else x


def _grad(fun, argnums=0):
    if argnums != 0:
        raise NotImplementedError("refshim.grad: argnums other than 0")

    def g(x, *args, **kw):
        x0 = np.asarray(x, dtype=np.float64)
        leaf = Var(x0)
        out = fun(leaf, *args, **kw)
        if not isinstance(out, Var):
            return np.zeros_like(x0).view(JArray)
        if out.val.size != 1:
            raise TypeError("refshim.grad: function output is not a scalar")
        # topological order, then reverse accumulation
        order, seen = [], set()
        stack = [(out, False)]
        while stack:
            node, done = stack.pop()
            if done:
                order.append(node)
                continue
            if id(node) in seen:
                continue
            seen.add(id(node))
            stack.append((node, True))
            for p, _ in node.parents:
                if id(p) not in seen:
                    stack.append((p, False))
        cot = {id(out): np.ones_like(out.val, dtype=np.float64)}
        for node in reversed(order):
            gnode = cot.pop(id(node), None)
            if gnode is None:
                continue
            if node is leaf:
                cot[id(leaf)] = gnode
                continue
            for p, vjp in node.parents:
                gp = vjp(gnode)
                cot[id(p)] = cot[id(p)] + gp if id(p) in cot else np.array(gp, dtype=np.float64)
        res = cot.get(id(leaf))
        if res is None:
            res = np.zeros_like(x0)
        return np.asarray(res, dtype=np.float64).reshape(x0.shape).view(JArray)
    return g


def _jacobian(fun):
    def jac(x0):
        x0 = np.asarray(x0, dtype=np.float64)
        f0 = np.asarray(fun(x0.view(JArray)), dtype=np.float64)
        n = x0.size
        cols = np.empty((f0.size, n))
        for i in range(n):
            e = np.zeros(n)
            e[i] = 1.0
            cols[:, i] = (np.asarray(fun((x0 + e.reshape(x0.shape)).view(JArray)),
                                     dtype=np.float64) - f0).reshape(-1)
        # affinity check on a random combination
        rng = np.random.default_rng(12345)
        c = rng.standard_normal(n)
        lhs = np.asarray(fun((x0 + c.reshape(x0.shape)).view(JArray)), dtype=np.float64).reshape(-1) - f0.reshape(-1)
        rhs = cols @ c
        if np.linalg.norm(lhs - rhs) > 1e-9 * max(1.0, np.linalg.norm(rhs)):
            raise ValueError("refshim.jacobian: the function is not affine; probing is not exact")
        return cols.reshape(f0.shape + x0.shape).view(JArray)
    return jac


def _vmap(fun, in_axes=0, out_axes=0):
    if in_axes != 0 or out_axes != 0:
        raise NotImplementedError("refshim.vmap: only in_axes=out_axes=0")

    def vf(*xs):
        n = len(xs[0])
        outs = [fun(*(x[i] for x in xs)) for i in range(n)]
        if isinstance(outs[0], tuple):
            return tuple(np.stack(o).view(JArray) for o in zip(*outs))
        return np.stack(outs).view(JArray)
    return vf


def _cg(A, b, x0=None, *, tol=1e-5, atol=0.0, maxiter=None, M=None):
    """JAX's documented PCG (see the module docstring for the stopping rule)."""
    b = np.asarray(b, dtype=np.float64)
    Aop = A if callable(A) else (lambda v: np.asarray(A) @ v)
    Mop = (lambda v: v) if M is None else (M if callable(M) else (lambda v: np.asarray(M) @ v))
    x = np.zeros_like(b) if x0 is None else np.asarray(x0, dtype=np.float64).copy()
    if maxiter is None:
        maxiter = 10 * b.size
    bs = float(b @ b)
    atol2 = max(tol * tol * bs, atol * atol)
    r = b - np.asarray(Aop(x))
    z = np.asarray(Mop(r))
    p = z
    gamma = float(r @ z)
    k = 0
    while float(r @ r) > atol2 and k < maxiter:
        Ap = np.asarray(Aop(p))
        alpha = gamma / float(p @ Ap)
        x = x + alpha * p
        r = r - alpha * Ap
        z = np.asarray(Mop(r))
        gamma_new = float(r @ z)
        beta = gamma_new / gamma
        gamma = gamma_new
        p = z + beta * p
        k += 1
    _cg.last_iterations = k
    return x.view(JArray), None


_cg.last_iterations = 0


# ---------------------------------------------------------------------------
# jax.numpy
# ---------------------------------------------------------------------------

def _where(cond, a=None, b=None):
    if a is None and b is None:
        return _wrap(np.where(_val(cond)))
    cond = np.asarray(_val(cond))
    if isinstance(a, Var) or isinstance(b, Var):
        av, bv = _val(a), _val(b)
        out = np.where(cond, av, bv)
        parents = []
        if isinstance(a, Var):
            parents.append((a, _unbroadcast(lambda g: np.where(cond, g, 0.0), a.shape)))
        if isinstance(b, Var):
            parents.append((b, _unbroadcast(lambda g: np.where(cond, 0.0, g), b.shape)))
        return Var(out, tuple(parents))
    return _wrap(np.where(cond, a, b))


def _sum(x, axis=None, **kw):
    if isinstance(x, Var):
        shape = x.shape

        def vjp(g):
            g = np.asarray(g)
            if axis is not None:
                g = np.expand_dims(g, axis)
            return np.broadcast_to(g, shape)
        if kw:
            raise NotImplementedError("refshim.sum: keyword arguments on a recorded value")
        return Var(np.sum(x.val, axis=axis), ((x, vjp),))
    return _wrap(np.sum(x, axis=axis, **kw))


def _einsum(spec, *ops, **kw):
    var_pos = [i for i, o in enumerate(ops) if isinstance(o, Var)]
    vals = [_val(o) for o in ops]
    if not var_pos:
        return _wrap(np.einsum(spec, *vals, **kw))
    if len(var_pos) > 1:
        raise NotImplementedError("refshim.einsum: more than one recorded operand")
    i = var_pos[0]
    ins, out = spec.replace(" ", "").split("->")
    in_specs = ins.split(",")
    res = np.einsum(spec, *vals)
    others = [s for j, s in enumerate(in_specs) if j != i]
    other_vals = [v for j, v in enumerate(vals) if j != i]
    target = in_specs[i]
    avail = set("".join(others) + out)
    if not set(target) <= avail:
        raise NotImplementedError("refshim.einsum: an index appears only in the recorded operand")
    vspec = ",".join(others + [out]) + "->" + target
    shape = ops[i].shape
    return Var(res, ((ops[i], lambda g: np.einsum(vspec, *other_vals, np.asarray(g)).reshape(shape)),))


def _zeros_like(x, *a, **k):
    return _wrap(np.zeros_like(_val(x), *a, **k))


def _asarray(x, dtype=None, **k):
    if isinstance(x, Var):
        if dtype is None:
            return x
        return x.astype(dtype)
    return _wrap(np.asarray(x, dtype=dtype, **k))


def _make_jnp():
    m = types.ModuleType("jax.numpy")
    overrides = {
        "where": _where, "sum": _sum, "einsum": _einsum, "zeros_like": _zeros_like,
        "asarray": _asarray, "array": lambda x, dtype=None, **k: _wrap(np.array(_val(x), dtype=dtype, **k)),
        "ndarray": np.ndarray,
    }

    def __getattr__(name):
        if name in overrides:
            return overrides[name]
        obj = getattr(np, name)
        if callable(obj) and not isinstance(obj, type):
            def f(*a, **k):
                return _wrap(obj(*a, **k))
            f.__name__ = name
            return f
        return obj
    m.__getattr__ = __getattr__
    lin = types.ModuleType("jax.numpy.linalg")

    def lin_getattr(name):
        obj = getattr(np.linalg, name)

        def f(*a, **k):
            return _wrap(obj(*[_val(x) for x in a], **k))
        return f
    lin.__getattr__ = lin_getattr
    m.linalg = lin
    return m, lin


def install(ref_src: str):
    """Register the shim as ``jax`` and bare ``ddg`` packages rooted at ``ref_src``.

    Returns ``importlib.import_module`` for convenience.
    """
    jax = types.ModuleType("jax")
    jnp, jlin = _make_jnp()
    jax.numpy = jnp
    jax.Array = np.ndarray
    jax.grad = _grad
    jax.jacobian = _jacobian
    jax.jacfwd = _jacobian
    jax.jacrev = _jacobian
    jax.vmap = _vmap
    jax.jit = lambda f=None, **k: (f if f is not None else (lambda g: g))
    cfg = types.SimpleNamespace(update=lambda *a, **k: None)
    jax.config = cfg
    tu = types.ModuleType("jax.tree_util")
    tu.register_pytree_node = lambda *a, **k: None
    jax.tree_util = tu
    jsc = types.ModuleType("jax.scipy")
    jsl = types.ModuleType("jax.scipy.linalg")
    jsl.lu_factor = lambda A, **k: _wrap(sla.lu_factor(np.asarray(A)))
    jsl.lu_solve = lambda lp, b, **k: _wrap(sla.lu_solve((np.asarray(lp[0]), np.asarray(lp[1])),
                                                         np.asarray(b)))
    jss = types.ModuleType("jax.scipy.sparse")
    jssl = types.ModuleType("jax.scipy.sparse.linalg")
    jssl.cg = _cg
    jss.linalg = jssl
    jsc.linalg = jsl
    jsc.sparse = jss
    jax.scipy = jsc
    sys.modules.update({
        "jax": jax, "jax.numpy": jnp, "jax.numpy.linalg": jlin, "jax.tree_util": tu,
        "jax.scipy": jsc, "jax.scipy.linalg": jsl, "jax.scipy.sparse": jss,
        "jax.scipy.sparse.linalg": jssl,
    })
    root = os.path.join(ref_src, "ddg")
    for name, path in (("ddg", root), ("ddg.dg1d", os.path.join(root, "dg1d")),
                       ("ddg.dg2d", os.path.join(root, "dg2d"))):
        pkg = types.ModuleType(name)
        pkg.__path__ = [path]
        pkg.__package__ = name
        sys.modules[name] = pkg
    return importlib.import_module


def cg_last_iterations() -> int:
    """Iterations taken by the most recent shim ``cg`` call."""
    return _cg.last_iterations
