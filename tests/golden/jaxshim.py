"""NumPy-backed stand-in for the small part of ``jax`` the DEM hot path uses.

Test infrastructure only.  JAX cannot be installed in this image, so the
golden-vector generator (``make_golden.py``) runs the reference's own
``medea_ice_ship/jax_*.py`` files unmodified on top of this module.  It covers
exactly the API surface those files touch:

* ``jax.jit`` (identity, with or without ``static_argnames``),
  ``jax.block_until_ready``, ``jax.config.update("jax_enable_x64", ...)``;
* ``jax.lax.scan`` and ``jax.lax.fori_loop`` (eager Python loops);
* about 40 ``jax.numpy`` creation / elementwise / reduction functions
  (``jnp.maximum.accumulate`` included);
* the functional scatters ``x.at[idx].add/max/min/set`` mapped onto
  ``np.add.at`` / ``np.maximum.at`` / ``np.minimum.at`` / item assignment,
  which apply updates sequentially in index order.

Precision follows JAX: with ``jax_enable_x64`` on, floats are float64; with it
off, every float64 / int64 request is canonicalised to float32 / int32, as JAX
does.  Python scalars stay weakly typed (NumPy 2 promotion rules match JAX's
weak-type rule for them).
"""
from __future__ import annotations

import sys
import types

import numpy as np

_STATE = {"x64": False}


def _canon(dtype):
    if dtype is None:
        return None
    dt = np.dtype(dtype)
    if not _STATE["x64"]:
        if dt == np.float64:
            return np.dtype(np.float32)
        if dt == np.int64:
            return np.dtype(np.int32)
        if dt == np.uint64:
            return np.dtype(np.uint32)
    return dt


def _default_float():
    return np.dtype(np.float64 if _STATE["x64"] else np.float32)


def _default_int():
    return np.dtype(np.int64 if _STATE["x64"] else np.int32)


class _AtOps:
    def __init__(self, arr, idx):
        self._arr = arr
        self._idx = idx

    def _vals(self, v):
        return np.asarray(v).astype(self._arr.dtype, copy=False)

    def add(self, v):
        out = np.array(self._arr, copy=True)
        np.add.at(out, self._idx, self._vals(v))
        return _w(out)

    def max(self, v):
        out = np.array(self._arr, copy=True)
        np.maximum.at(out, self._idx, self._vals(v))
        return _w(out)

    def min(self, v):
        out = np.array(self._arr, copy=True)
        np.minimum.at(out, self._idx, self._vals(v))
        return _w(out)

    def set(self, v):
        out = np.array(self._arr, copy=True)
        out[self._idx] = self._vals(v)
        return _w(out)


class _AtIndexer:
    def __init__(self, arr):
        self._arr = arr

    def __getitem__(self, idx):
        if isinstance(idx, tuple):
            idx = tuple(np.asarray(i) if isinstance(i, np.ndarray) else i for i in idx)
        elif isinstance(idx, np.ndarray):
            idx = np.asarray(idx)
        return _AtOps(self._arr, idx)


class ShimArray(np.ndarray):
    """ndarray with JAX's ``.at[]`` functional-update indexer."""

    @property
    def at(self):
        return _AtIndexer(self)

    def astype(self, dtype, *args, **kwargs):
        return _w(np.ndarray.astype(np.asarray(self), _canon(dtype), *args, **kwargs))

    def copy(self, *args, **kwargs):
        return _w(np.array(np.asarray(self), copy=True))

    def __array_wrap__(self, arr, context=None, return_scalar=False):
        # ufunc results: JAX in x32 mode never holds a 64-bit array
        out = _w(np.asarray(arr))
        if return_scalar:
            return out[()]
        return out


def _w(x):
    """Wrap a NumPy result as a ShimArray, canonicalising 64-bit dtypes in x32 mode.

    NumPy turns Python scalars into float64 arrays in calls such as
    ``np.where(c, 0.0, -1.0)``; JAX treats them as weakly typed and yields
    the default float (float32 with x64 off).  Casting every result keeps the
    shim's x32 arithmetic in float32 like JAX.
    """
    if isinstance(x, (np.ndarray, np.generic)):
        a = np.asarray(x)
        cd = _canon(a.dtype)
        if cd != a.dtype:
            a = a.astype(cd)
        if isinstance(a, ShimArray):
            return a
        return a.view(ShimArray)
    return x


def _array(obj, dtype=None, copy=True):
    if dtype is not None:
        arr = np.array(obj, dtype=_canon(dtype))
    else:
        arr = np.array(obj)
        if arr.dtype == np.float64 or arr.dtype == np.int64:
            arr = arr.astype(_canon(arr.dtype))
    return _w(arr)


def _make_jnp():
    m = types.ModuleType("jax.numpy")
    m.ndarray = ShimArray
    m.float64 = np.float64
    m.float32 = np.float32
    m.int32 = np.int32
    m.int64 = np.int64
    m.bool_ = np.bool_
    m.pi = float(np.pi)
    m.inf = float(np.inf)

    m.array = _array
    m.asarray = lambda obj, dtype=None: _array(obj, dtype)

    def zeros(shape, dtype=None):
        return _w(np.zeros(shape, dtype=_canon(dtype) or _default_float()))

    def ones(shape, dtype=None):
        return _w(np.ones(shape, dtype=_canon(dtype) or _default_float()))

    def arange(*args, dtype=None):
        r = np.arange(*args)
        return _w(r.astype(_canon(dtype) if dtype is not None else _canon(r.dtype)))

    def linspace(start, stop, num=50, dtype=None):
        return _w(np.linspace(start, stop, num, dtype=_canon(dtype) or _default_float()))

    def eye(n, dtype=None):
        return _w(np.eye(n, dtype=_canon(dtype) or _default_float()))

    m.zeros, m.ones, m.arange, m.linspace, m.eye = zeros, ones, arange, linspace, eye

    def full(shape, fill_value, dtype=None):
        return _w(np.full(shape, fill_value, dtype=_canon(dtype) or _default_float()))

    def meshgrid(*xs, indexing="xy"):
        return tuple(_w(g) for g in np.meshgrid(*[np.asarray(x) for x in xs], indexing=indexing))

    def pad(x, pad_width, mode="constant", **kw):
        return _w(np.pad(np.asarray(x), pad_width, mode=mode, **kw))

    m.full, m.meshgrid, m.pad = full, meshgrid, pad

    def _wrapfn(fn):
        def g(*a, **k):
            return _w(fn(*a, **k))
        g.__name__ = getattr(fn, "__name__", "f")
        return g

    for name in ("abs", "argmax", "argmin", "broadcast_to", "clip", "concatenate",
                 "cos", "sin", "isfinite", "maximum", "minimum", "min", "max",
                 "power", "repeat", "roll", "sign", "sqrt", "stack", "sum", "tile",
                 "where", "exp", "log", "mean", "any", "all", "floor", "ceil",
                 "arctan2", "square", "dot", "matmul", "logical_and", "logical_or",
                 "logical_not", "cumsum", "prod", "diff"):
        setattr(m, name, _wrapfn(getattr(np, name)))
    m.maximum.accumulate = _wrapfn(np.maximum.accumulate)

    linalg = types.ModuleType("jax.numpy.linalg")

    def norm(x, axis=None, keepdims=False):
        x = np.asarray(x)
        return _w(np.linalg.norm(x, axis=axis, keepdims=keepdims))

    linalg.norm = norm
    linalg.inv = _wrapfn(np.linalg.inv)
    m.linalg = linalg
    return m, linalg


def _is_leaf(x):
    return not isinstance(x, (tuple, list, dict)) and x is not None


def _tree_map(fn, *trees):
    t0 = trees[0]
    if t0 is None:
        return None
    if isinstance(t0, tuple) and hasattr(t0, "_fields"):
        return type(t0)(*[_tree_map(fn, *[getattr(t, f) for t in trees]) for f in t0._fields])
    if isinstance(t0, (tuple, list)):
        return type(t0)(_tree_map(fn, *[t[i] for t in trees]) for i in range(len(t0)))
    if isinstance(t0, dict):
        return {k: _tree_map(fn, *[t[k] for t in trees]) for k in t0}
    return fn(*trees)


def _tree_leaves(t):
    if t is None:
        return []
    if isinstance(t, tuple) and hasattr(t, "_fields"):
        return [l for f in t._fields for l in _tree_leaves(getattr(t, f))]
    if isinstance(t, (tuple, list)):
        return [l for x in t for l in _tree_leaves(x)]
    if isinstance(t, dict):
        return [l for k in t for l in _tree_leaves(t[k])]
    return [t]


def _make_lax():
    lax = types.ModuleType("jax.lax")

    def scan(f, init, xs=None, length=None):
        if xs is None:
            n = int(length)
        else:
            n = int(np.shape(_tree_leaves(xs)[0])[0])
        carry = init
        ys = []
        for i in range(n):
            x = None if xs is None else _tree_map(lambda a: _w(np.asarray(a)[i]), xs)
            carry, y = f(carry, x)
            ys.append(y)
        if not ys or ys[0] is None:
            return carry, None
        stacked = _tree_map(lambda *leaves: _w(np.stack([np.asarray(l) for l in leaves])), *ys)
        return carry, stacked

    def fori_loop(lower, upper, body, init):
        val = init
        for i in range(int(lower), int(upper)):
            val = body(i, val)
        return val

    def reduce_window(x, init_value, computation, window_dimensions, window_strides, padding):
        # the max-pool form only: stride 1, VALID padding, computation = lax.max
        x = np.asarray(x)
        if tuple(window_strides) != (1,) * x.ndim or padding != "VALID" or computation is not lax.max:
            raise NotImplementedError("reduce_window: only max, stride 1, VALID")
        win = np.lib.stride_tricks.sliding_window_view(x, tuple(window_dimensions))
        out = win.max(axis=tuple(range(x.ndim, 2 * x.ndim)))
        return _w(np.maximum(out, np.asarray(init_value, dtype=x.dtype)))

    lax.scan = scan
    lax.fori_loop = fori_loop
    lax.max = lambda a, b: _w(np.maximum(a, b))
    lax.reduce_window = reduce_window
    return lax


def install(x64: bool) -> None:
    """Register ``jax``, ``jax.numpy``, ``jax.lax`` shim modules in sys.modules."""
    _STATE["x64"] = bool(x64)
    jax = types.ModuleType("jax")
    jnp, linalg = _make_jnp()
    lax = _make_lax()

    def jit(fun=None, **kwargs):
        if fun is None:
            return lambda f: f
        return fun

    class _Config:
        def update(self, key, value):
            if key == "jax_enable_x64":
                _STATE["x64"] = bool(value)

    jax.jit = jit
    jax.numpy = jnp
    jax.lax = lax
    jax.config = _Config()
    jax.block_until_ready = lambda x: x

    def vmap(f, in_axes=0, out_axes=0):
        def g(*args):
            n = int(np.shape(args[0])[0])
            outs = [f(*[_w(np.asarray(a)[i]) for a in args]) for i in range(n)]
            return _w(np.stack([np.asarray(o) for o in outs]))
        return g

    jax.vmap = vmap
    jax.Array = ShimArray
    sys.modules["jax"] = jax
    sys.modules["jax.numpy"] = jnp
    sys.modules["jax.numpy.linalg"] = linalg
    sys.modules["jax.lax"] = lax


def load_reference(ref_root: str, x64: bool):
    """Import the reference hot-path modules under the shim.

    The package ``__init__`` of ``medea_ice_ship`` imports plotting libraries
    that are absent here, so a bare package object pointing at the reference
    directory is registered instead and only the hot-path modules are loaded.
    """
    import os

    install(x64)
    pkg = types.ModuleType("medea_ice_ship")
    pkg.__path__ = [os.path.join(ref_root, "medea_ice_ship")]
    sys.modules["medea_ice_ship"] = pkg
    import importlib

    mods = {}
    for name in ("properties", "config", "geometry", "auto_icenav_ship", "jax_ice_state",
                 "jax_geometry", "jax_bond_fracture", "jax_vessel_dynamics", "jax_simulation"):
        mods[name] = importlib.import_module(f"medea_ice_ship.{name}")
    return types.SimpleNamespace(**mods)
