"""NumPy-backed stand-in for the small part of the JAX API that the
reference package's hot-path modules use, so that those modules can be
imported and run in a container without JAX (fixture generation only).

What it provides: ``jax.jit`` (identity, any static_argnums),
``jax.numpy`` (NumPy functions whose array results carry JAX's functional
``.at[idx].set(v)`` update), ``jax.random`` (PRNGKey/normal/uniform/split on
``numpy.random.default_rng`` -- NOT JAX's threefry stream, so fixtures never
rely on it), ``jax.tree_util.register_pytree_node`` (no-op), ``jax.lax.scan``
(Python loop), ``jax.config.update`` (no-op) and ``jax.Array``.

Floating point is float64 throughout, as the reference forces
``jax_enable_x64`` on import.  FFTs are NumPy's pocketfft.
"""

from __future__ import annotations

import sys
import types

import numpy as np


class _AtIndexer:
    def __init__(self, arr):
        self._arr = arr

    def __getitem__(self, idx):
        arr = self._arr

        class _Upd:
            def set(self_inner, value):
                out = np.array(arr, copy=True)
                out[idx] = np.asarray(value)
                return out.view(ShimArray)

            def add(self_inner, value):
                out = np.array(arr, copy=True)
                out[idx] = out[idx] + np.asarray(value)
                return out.view(ShimArray)

            def multiply(self_inner, value):
                out = np.array(arr, copy=True)
                out[idx] = out[idx] * np.asarray(value)
                return out.view(ShimArray)

        return _Upd()


class ShimArray(np.ndarray):
    """ndarray with JAX's ``.at[...]`` functional update."""

    @property
    def at(self):
        return _AtIndexer(self)

    def block_until_ready(self):
        return self


def _wrap(x):
    if isinstance(x, np.ndarray) and not isinstance(x, ShimArray):
        return x.view(ShimArray)
    if isinstance(x, tuple):
        return tuple(_wrap(v) for v in x)
    if isinstance(x, list):
        return [_wrap(v) for v in x]
    return x


def _wrapped(fn):
    def f(*a, **k):
        return _wrap(fn(*a, **k))

    f.__name__ = getattr(fn, "__name__", "f")
    return f


class _NumpyModule(types.ModuleType):
    """``jax.numpy``: attribute access falls through to NumPy."""

    def __init__(self, name, base):
        super().__init__(name)
        self._base = base

    def __getattr__(self, name):
        obj = getattr(self._base, name)
        if callable(obj) and not isinstance(obj, type):
            return _wrapped(obj)
        return obj


def _array(x, dtype=None):
    a = np.array(x, dtype=dtype)
    return a.view(ShimArray)


def install() -> types.ModuleType:
    """Register the stand-in as ``jax`` in ``sys.modules`` and return it."""
    jax = types.ModuleType("jax")
    jax.__version__ = "0.4.30"
    jax.Array = np.ndarray

    def jit(fn=None, **kw):
        if fn is None:
            return lambda f: f
        return fn

    jax.jit = jit
    jax.block_until_ready = lambda x: x
    jax.devices = lambda *a, **k: []

    jnp = _NumpyModule("jax.numpy", np)
    jnp.array = _array
    jnp.asarray = _array
    jnp.ndarray = np.ndarray
    fftmod = _NumpyModule("jax.numpy.fft", np.fft)
    jnp.fft = fftmod
    jax.numpy = jnp

    rnd = types.ModuleType("jax.random")
    rnd.PRNGKey = lambda seed: np.array([0, int(seed)], dtype=np.uint32)

    def _rng(key):
        return np.random.default_rng(int(np.asarray(key).ravel()[-1]))

    rnd.normal = lambda key, shape=(), dtype=None: _wrap(_rng(key).standard_normal(shape))
    rnd.uniform = lambda key, shape=(), minval=0.0, maxval=1.0, dtype=None: _wrap(
        _rng(key).uniform(minval, maxval, size=shape)
    )

    def split(key, num=2):
        base = int(np.asarray(key).ravel()[-1])
        return np.array([[0, base * 7919 + i + 1] for i in range(num)], dtype=np.uint32)

    rnd.split = split
    jax.random = rnd

    tu = types.ModuleType("jax.tree_util")
    tu.register_pytree_node = lambda *a, **k: None
    jax.tree_util = tu

    lax = types.ModuleType("jax.lax")

    def scan(f, init, xs, length=None):
        carry = init
        ys = []
        n = length if xs is None else len(xs)
        for i in range(n):
            carry, y = f(carry, None if xs is None else xs[i])
            ys.append(y)
        return carry, ys

    lax.scan = scan
    jax.lax = lax

    cfg = types.SimpleNamespace(update=lambda *a, **k: None)
    jax.config = cfg

    for name, mod in {
        "jax": jax,
        "jax.numpy": jnp,
        "jax.numpy.fft": fftmod,
        "jax.random": rnd,
        "jax.tree_util": tu,
        "jax.lax": lax,
    }.items():
        sys.modules[name] = mod
    return jax
