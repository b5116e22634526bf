"""A numpy-backed stand-in for the subset of the JAX API that jax_fem_cfd calls.

Test infrastructure only: it exists so that the reference's OWN Python modules
(jax_fem_cfd/core, solvers, setup, utils/jax_iterative_solvers.py) can be executed
in a container where jax/jaxlib (pinned upstream as ``jax[cuda12_pip]==0.4.13``,
requirements.txt:3) are not installed, to produce golden input/output vectors.

What is restated here is JAX's published semantics for exactly the calls the
reference makes (with ``jax_enable_x64`` on, as every reference driver sets):

* ``jnp.*``      -> numpy functions returning a ndarray subclass that supports
                    the functional ``x.at[idx].set/add/get`` update syntax.
* ``jax.vmap``   -> a per-example Python loop over the mapped axis, outputs
                    stacked along axis 0 (vmap's definition: f applied to each slice).
* ``jax.jit``    -> identity (tracing/compilation does not change values in x64).
* ``jax.ops.segment_sum`` -> ``np.add.at`` into ``num_segments`` zeros, which
                    accumulates in data order like XLA's CPU scatter-add.
* ``lax.while_loop`` -> Python while loop; ``lax.custom_linear_solve`` -> the
                    forward ``solve(matvec, b)`` (its transpose rule only matters
                    under differentiation).
* tree_util on single arrays / tuples, ``device_put``/``device_get`` identity.

Rounding differs from XLA's (numpy's BLAS/pairwise sums vs XLA's loop order),
so goldens made through this shim pin the reference's algorithm and control
flow, and values to floating-point round-off, not XLA's bits.
"""
from __future__ import annotations

import functools
import importlib.util
import sys
import types

import numpy as np


class JArray(np.ndarray):
    """ndarray with JAX's ``.at[...]`` functional-update property."""

    @property
    def at(self):
        return _AtIndexer(self)

    def block_until_ready(self):
        return self


class _AtRef:
    def __init__(self, arr, idx):
        self.arr, self.idx = arr, _unwrap_idx(idx)

    def set(self, v):
        out = np.array(self.arr, copy=True)
        out[self.idx] = np.asarray(v)
        return _wrap(out)

    def add(self, v):
        out = np.array(self.arr, copy=True)
        np.add.at(out, self.idx, np.asarray(v))
        return _wrap(out)

    def get(self):
        return _wrap(np.asarray(self.arr)[self.idx])


class _AtIndexer:
    def __init__(self, arr):
        self.arr = arr

    def __getitem__(self, idx):
        return _AtRef(self.arr, idx)


def _unwrap_idx(idx):
    if isinstance(idx, tuple):
        return tuple(np.asarray(i) if isinstance(i, np.ndarray) else i for i in idx)
    if isinstance(idx, np.ndarray):
        return np.asarray(idx)
    return idx


def _wrap(x):
    if isinstance(x, JArray):
        return x
    if isinstance(x, np.ndarray):
        return x.view(JArray)
    if isinstance(x, (np.generic, float, int, bool)) and not isinstance(x, (str,)):
        return np.asarray(x).view(JArray)
    if isinstance(x, tuple):
        return tuple(_wrap(v) for v in x)
    if isinstance(x, list):
        return [_wrap(v) for v in x]
    return x


def _wrapped(fn):
    @functools.wraps(fn)
    def inner(*args, **kwargs):
        kwargs.pop("precision", None)
        args = tuple(list(a) if isinstance(a, types.GeneratorType) else a for a in args)
        return _wrap(fn(*args, **kwargs))

    return inner


class _NumpyFacade(types.ModuleType):
    """``jax.numpy``: numpy functions whose array results support ``.at``."""

    def __init__(self, name, target):
        super().__init__(name)
        self._target = target

    def __getattr__(self, item):
        obj = getattr(self._target, item)
        if callable(obj) and not isinstance(obj, type):
            return _wrapped(obj)
        return obj


def _array(obj, dtype=None, **kw):
    return _wrap(np.array(obj, dtype=dtype))


def vmap(fun, in_axes=0, out_axes=0):
    """Per-example loop: stack fun(slice_i) along out_axes (only 0 is used)."""

    def mapped(*args):
        axes = in_axes if isinstance(in_axes, (tuple, list)) else (in_axes,) * len(args)
        n = None
        for a, ax in zip(args, axes):
            if ax is not None:
                n = np.shape(a)[ax]
                break
        outs = []
        for i in range(n):
            sl = [a if ax is None else _wrap(np.take(np.asarray(a), i, axis=ax))
                  for a, ax in zip(args, axes)]
            outs.append(fun(*sl))
        if isinstance(outs[0], tuple):
            return tuple(_wrap(np.stack([np.asarray(o[k]) for o in outs], axis=out_axes))
                         for k in range(len(outs[0])))
        return _wrap(np.stack([np.asarray(o) for o in outs], axis=out_axes))

    return mapped


def jit(fun=None, **_kw):
    if fun is None:
        return lambda f: f
    return fun


def segment_sum(data, segment_ids, num_segments=None, **_kw):
    data = np.asarray(data)
    ids = np.asarray(segment_ids)
    out = np.zeros((num_segments,) + data.shape[1:], dtype=data.dtype)
    np.add.at(out, ids, data)
    return _wrap(out)


def while_loop(cond_fun, body_fun, init_val):
    val = init_val
    while bool(cond_fun(val)):
        val = body_fun(val)
    return val


def scan(f, init, xs, length=None):
    carry = init
    ys = []
    n = length if xs is None else len(xs)
    for i in range(n):
        carry, y = f(carry, None if xs is None else xs[i])
        ys.append(y)
    return carry, ys


def custom_linear_solve(matvec, b, solve, transpose_solve=None, symmetric=False, has_aux=False):
    return solve(matvec, b)


class _Precision:
    HIGHEST = "highest"
    DEFAULT = "default"


def _is_leaf(x):
    return not isinstance(x, (tuple, list, dict)) and x is not None


def tree_leaves(tree):
    if tree is None:
        return []
    if isinstance(tree, (tuple, list)):
        out = []
        for t in tree:
            out.extend(tree_leaves(t))
        return out
    if isinstance(tree, dict):
        out = []
        for k in sorted(tree):
            out.extend(tree_leaves(tree[k]))
        return out
    return [tree]


def tree_map(f, tree, *rest):
    if isinstance(tree, (tuple, list)):
        return type(tree)(tree_map(f, t, *(r[i] for r in rest)) for i, t in enumerate(tree))
    return f(tree, *rest)


def tree_structure(tree):
    if isinstance(tree, (tuple, list)):
        return (type(tree).__name__, tuple(tree_structure(t) for t in tree))
    return "*"


def tree_reduce(f, tree, initializer=None):
    leaves = tree_leaves(tree)
    return functools.reduce(f, leaves) if initializer is None else functools.reduce(f, leaves, initializer)


class Partial(functools.partial):
    pass


def _lattice_result_type(*args):
    return np.result_type(*[np.asarray(a) for a in args]), False


def _convert_element_type(operand, new_dtype=None, weak_type=False, *a, **k):
    return _wrap(np.asarray(operand, dtype=new_dtype))


def _safe_map(f, *args):
    return list(map(f, *args))


def install():
    """Register fake ``jax``, ``jax.numpy`` ... and ``h5py`` modules in sys.modules."""
    if "jax" in sys.modules and getattr(sys.modules["jax"], "__graft_shim__", False):
        return sys.modules["jax"]
    jax = types.ModuleType("jax")
    jax.__graft_shim__ = True
    jnp = _NumpyFacade("jax.numpy", np)
    jnp.array = _array
    jnp.asarray = _array
    jnp.ndarray = JArray
    jnp.newaxis = None
    jnp.pi = np.pi
    jnp.linalg = _NumpyFacade("jax.numpy.linalg", np.linalg)
    jax.numpy = jnp
    jax.vmap = vmap
    jax.jit = jit
    jax.device_put = lambda x, *a, **k: x
    jax.device_get = lambda x: x
    jax.Array = JArray
    jax.ops = types.ModuleType("jax.ops")
    jax.ops.segment_sum = segment_sum
    lax = types.ModuleType("jax.lax")
    lax.while_loop = while_loop
    lax.scan = scan
    lax.custom_linear_solve = custom_linear_solve
    lax.Precision = _Precision
    jax.lax = lax
    jax.config = types.SimpleNamespace(update=lambda *a, **k: None)
    jsp = types.ModuleType("jax.scipy")
    jsp.linalg = types.ModuleType("jax.scipy.linalg")
    jax.scipy = jsp
    tu = types.ModuleType("jax.tree_util")
    tu.tree_leaves, tu.tree_map, tu.tree_structure = tree_leaves, tree_map, tree_structure
    tu.tree_reduce, tu.Partial = tree_reduce, Partial
    jax.tree_util = tu
    src = types.ModuleType("jax._src")
    dtypes = types.ModuleType("jax._src.dtypes")
    dtypes._lattice_result_type = _lattice_result_type
    src_lax_pkg = types.ModuleType("jax._src.lax")
    src_lax = types.ModuleType("jax._src.lax.lax")
    src_lax._convert_element_type = _convert_element_type
    src_lax_pkg.lax = src_lax
    util = types.ModuleType("jax._src.util")
    util.safe_map = _safe_map
    src.dtypes, src.lax, src.util = dtypes, src_lax_pkg, util
    jax._src = src
    mods = {"jax": jax, "jax.numpy": jnp, "jax.numpy.linalg": jnp.linalg, "jax.ops": jax.ops,
            "jax.lax": lax, "jax.scipy": jsp, "jax.scipy.linalg": jsp.linalg,
            "jax.tree_util": tu, "jax._src": src, "jax._src.dtypes": dtypes,
            "jax._src.lax": src_lax_pkg, "jax._src.lax.lax": src_lax, "jax._src.util": util,
            "h5py": types.ModuleType("h5py")}
    sys.modules.update(mods)
    return jax


def load_reference(root):
    """Import the reference's modules from ``root`` without running the package
    ``__init__`` chain (utils/__init__ imports matplotlib/PyQt5 for plotting)."""
    import os

    install()
    pkg_dir = os.path.join(root, "jax_fem_cfd")
    for name, sub in [("jax_fem_cfd", ""), ("jax_fem_cfd.core", "core"),
                      ("jax_fem_cfd.setup", "setup"), ("jax_fem_cfd.solvers", "solvers"),
                      ("jax_fem_cfd.utils", "utils")]:
        if name not in sys.modules:
            m = types.ModuleType(name)
            m.__path__ = [os.path.join(pkg_dir, sub) if sub else pkg_dir]
            sys.modules[name] = m
    out = {}
    for name in ["core.shape_functions", "core.element_calc", "core.element_mult",
                 "utils.jax_iterative_solvers", "core.multigrid", "setup.regular_mesh",
                 "setup.simulation", "solvers.standard", "solvers.passive_transport"]:
        full = "jax_fem_cfd." + name
        if full not in sys.modules:
            path = os.path.join(pkg_dir, *name.split(".")) + ".py"
            spec = importlib.util.spec_from_file_location(full, path)
            mod = importlib.util.module_from_spec(spec)
            sys.modules[full] = mod
            spec.loader.exec_module(mod)
        out[name.split(".")[-1]] = sys.modules[full]
    return out
