"""A NumPy stand-in for the small subset of JAX the reference hot path calls.

TEST INFRASTRUCTURE ONLY (used by ``make_golden.py`` in the build container,
never on the product path). JAX is not installed here, so the reference's own
modules (`jax_step.py`, `solver.py`, `chem.py`, `photo.py`) are imported
unmodified with this module standing in for ``jax``. Each primitive restates
the published semantics of the JAX call it replaces (JAX has no pinned version
in the reference; the semantics below are the documented ones):

* ``jax.ops.segment_sum``          -> zeros + ``numpy.add.at`` (sequential scatter-add)
* ``jax.scipy.linalg.lu_factor/lu_solve`` -> LAPACK getrf/getrs via SciPy
* ``jax.lax.scan``                 -> Python loop, outputs stacked on axis 0
* ``jax.vmap``                     -> loop over the mapped axes, stacked on axis 0
* ``jax.jit`` / ``jax.config``     -> identity / no-op
* ``x.at[idx].set/add``            -> copy-on-write indexed update
* ``jax.custom_vjp``               -> forward call; ``defvjp`` records fwd/bwd
* ``jax.vjp``                      -> exact VJP of a function LINEAR in its
  argument (probes the argument's basis); used only for ``chem_rhs`` in k.
"""
from __future__ import annotations

import sys
import types

import numpy as np
import scipy.linalg as sla


class JArr(np.ndarray):
    """ndarray with JAX's functional ``.at[...]`` update syntax."""

    @property
    def at(self):
        return _At(self)


class _At:
    def __init__(self, a):
        self.a = a

    def __getitem__(self, idx):
        return _AtIdx(self.a, idx)


class _AtIdx:
    def __init__(self, a, idx):
        self.a, self.idx = a, idx

    def _copy(self):
        return np.array(self.a, copy=True).view(JArr)

    def set(self, v):
        out = self._copy()
        out[self.idx] = np.asarray(v)
        return out

    def add(self, v):
        out = self._copy()
        out[self.idx] = out[self.idx] + np.asarray(v)
        return out


def _wrap(x):
    if isinstance(x, np.ndarray) and not isinstance(x, JArr):
        return x.view(JArr)
    if isinstance(x, tuple):
        return type(x)(*[_wrap(v) for v in x]) if hasattr(x, "_fields") else tuple(_wrap(v) for v in x)
    if isinstance(x, list):
        return [_wrap(v) for v in x]
    return x


def _tree_leaves_map(f, *trees):
    t0 = trees[0]
    if isinstance(t0, tuple) and hasattr(t0, "_fields"):
        return type(t0)(*[_tree_leaves_map(f, *[t[i] for t in trees]) for i in range(len(t0))])
    if isinstance(t0, (tuple, list)):
        return type(t0)(_tree_leaves_map(f, *[t[i] for t in trees]) for i in range(len(t0)))
    if t0 is None:
        return None
    return f(*trees)


# ---------------------------------------------------------------- jax.numpy
jnp = types.ModuleType("jax.numpy")


def _jnp_getattr(name):
    obj = getattr(np, name)
    if callable(obj) and not isinstance(obj, type):
        def fn(*a, **k):
            return _wrap(obj(*a, **k))
        fn.__name__ = name
        return fn
    return obj


jnp.__getattr__ = _jnp_getattr
jnp.ndarray = np.ndarray
jnp.float64 = np.float64
jnp.float32 = np.float32
jnp.int32 = np.int32
jnp.int64 = np.int64
jnp.bool_ = np.bool_


def _asarray(x, dtype=None):
    return np.array(x, dtype=dtype).view(JArr)


jnp.asarray = _asarray
jnp.array = _asarray

# ---------------------------------------------------------------- jax
jax = types.ModuleType("jax")
jax.numpy = jnp


class _Config:
    def update(self, *a, **k):
        pass


jax.config = _Config()


def jit(fun=None, **kw):
    if fun is None:
        return lambda f: f
    return fun


jax.jit = jit


def vmap(fun, in_axes=0, out_axes=0):
    def mapped(*args):
        axes = in_axes if isinstance(in_axes, (tuple, list)) else (in_axes,) * len(args)
        n = None
        for a, ax in zip(args, axes):
            if ax is not None:
                n = np.asarray(a).shape[ax]
                break
        outs = []
        for b in range(n):
            sub = [np.take(np.asarray(a), b, axis=ax).view(JArr) if ax is not None else a
                   for a, ax in zip(args, axes)]
            outs.append(fun(*sub))
        return _tree_leaves_map(lambda *xs: np.stack(xs, axis=0).view(JArr), *outs)
    return mapped


jax.vmap = vmap

# lax
lax = types.ModuleType("jax.lax")


def scan(f, init, xs, length=None):
    leaves = []
    _tree_leaves_map(lambda a: leaves.append(a), xs)
    n = length if length is not None else np.asarray(leaves[0]).shape[0]
    carry = init
    ys = []
    for i in range(n):
        x_i = _tree_leaves_map(lambda a: _wrap(np.asarray(a)[i]), xs)
        carry, y = f(carry, x_i)
        ys.append(y)
    stacked = _tree_leaves_map(lambda *vs: np.stack([np.asarray(v) for v in vs], axis=0).view(JArr), *ys)
    return carry, stacked


lax.scan = scan
jax.lax = lax

# ops
ops = types.ModuleType("jax.ops")


def segment_sum(data, segment_ids, num_segments=None, indices_are_sorted=False, **kw):
    data = np.asarray(data)
    out = np.zeros((num_segments,) + data.shape[1:], dtype=data.dtype)
    np.add.at(out, np.asarray(segment_ids), data)
    return out.view(JArr)


ops.segment_sum = segment_sum
jax.ops = ops

# scipy.linalg
jscipy = types.ModuleType("jax.scipy")
jlinalg = types.ModuleType("jax.scipy.linalg")


def lu_factor(a):
    lu, piv = sla.lu_factor(np.asarray(a), check_finite=False)
    return lu.view(JArr), piv.astype(np.int32).view(JArr)


def lu_solve(lu_and_piv, b):
    lu, piv = lu_and_piv
    return sla.lu_solve((np.asarray(lu), np.asarray(piv)), np.asarray(b), check_finite=False).view(JArr)


jlinalg.lu_factor = lu_factor
jlinalg.lu_solve = lu_solve
jscipy.linalg = jlinalg
jax.scipy = jscipy

# tree utilities
tree_util = types.ModuleType("jax.tree_util")
tree_util.register_pytree_node = lambda *a, **k: None
jax.tree_util = tree_util
tree = types.ModuleType("jax.tree")
tree.map = _tree_leaves_map
jax.tree = tree

dtypes = types.ModuleType("jax.dtypes")
dtypes.float0 = np.dtype([("float0", np.void, 0)])
jax.dtypes = dtypes


class custom_vjp:
    def __init__(self, fun, nondiff_argnums=()):
        self.fun = fun
        self.nondiff_argnums = nondiff_argnums
        self.fwd = self.bwd = None

    def __call__(self, *args):
        return self.fun(*args)

    def defvjp(self, fwd, bwd):
        self.fwd, self.bwd = fwd, bwd


jax.custom_vjp = custom_vjp


def vjp(fun, primal):
    """Exact VJP of a function that is LINEAR in ``primal`` (basis probing)."""
    primal = np.asarray(primal)
    out0 = np.asarray(fun(np.zeros_like(primal).view(JArr)))
    cols = []
    flat = np.zeros(primal.size)
    for i in range(primal.size):
        flat[:] = 0.0
        flat[i] = 1.0
        cols.append((np.asarray(fun(flat.reshape(primal.shape).view(JArr))) - out0).reshape(-1))
    A = np.stack(cols, axis=1)                       # d out / d primal

    def vjp_fn(ct):
        return (_wrap((A.T @ np.asarray(ct).reshape(-1)).reshape(primal.shape)),)
    return np.asarray(fun(primal.view(JArr))).view(JArr), vjp_fn


jax.vjp = vjp


def _no_autodiff(*a, **k):
    def fail(*aa, **kk):
        raise NotImplementedError("reverse-mode AD is not available in the NumPy stand-in")
    return fail


jax.jacrev = _no_autodiff
jax.jacfwd = _no_autodiff
jax.grad = _no_autodiff


def install():
    """Register the stand-in under the ``jax`` module names."""
    sys.modules["jax"] = jax
    sys.modules["jax.numpy"] = jnp
    sys.modules["jax.lax"] = lax
    sys.modules["jax.ops"] = ops
    sys.modules["jax.scipy"] = jscipy
    sys.modules["jax.scipy.linalg"] = jlinalg
    sys.modules["jax.tree_util"] = tree_util
    sys.modules["jax.tree"] = tree
    sys.modules["jax.dtypes"] = dtypes
