"""A numpy-backed stand-in for the slice of ``jax`` that beamz's step math uses.

Fixture generation only.  beamz imports ``jax`` at module load, and JAX is not
installable in this image, so ``make_golden.py`` installs this module as
``jax`` / ``jax.numpy`` / ``jax.lax`` before loading individual beamz source
files by path.  The reference's own functions then run unmodified on numpy
arrays.

The stand-in mirrors JAX's default (x64 disabled) dtype policy: every array
that enters through ``jnp.asarray``/``jnp.array``/constructors is canonicalised
to 32-bit (float64 -> float32, int64 -> int32), and ``jnp.result_type`` never
returns a 64-bit type.  numpy 2's NEP 50 weak-scalar promotion matches JAX's
weak typing for Python scalars, so float32 arithmetic stays float32.
"""

from __future__ import annotations

import sys
import types

import numpy as np

_CANON = {
    np.dtype(np.float64): np.dtype(np.float32),
    np.dtype(np.int64): np.dtype(np.int32),
    np.dtype(np.uint64): np.dtype(np.uint32),
    np.dtype(np.complex128): np.dtype(np.complex64),
}


def _canon_dtype(dtype):
    if dtype is None:
        return None
    d = np.dtype(dtype)
    return _CANON.get(d, d)


class _AtIndexer:
    def __init__(self, arr):
        self._arr = arr

    def __getitem__(self, index):
        return _AtOp(self._arr, index)


class _AtOp:
    def __init__(self, arr, index):
        self._arr = arr
        self._index = index

    def set(self, value):
        out = JArray._wrap(np.array(self._arr, copy=True))
        out[self._index] = value
        return out

    def add(self, value):
        out = JArray._wrap(np.array(self._arr, copy=True))
        np.add.at(out, self._index, np.asarray(value, dtype=out.dtype))
        return out

    def get(self):
        return self._arr[self._index]


class JArray(np.ndarray):
    """ndarray with JAX's functional ``.at[...]`` update syntax."""

    @staticmethod
    def _wrap(arr):
        return np.asarray(arr).view(JArray)

    @property
    def at(self):
        return _AtIndexer(self)


def asarray(value, dtype=None):
    if dtype is None:
        arr = np.asarray(value)
        if arr.dtype in _CANON:
            arr = arr.astype(_CANON[arr.dtype])
        elif arr.dtype == object:
            arr = arr.astype(np.float32)
    else:
        arr = np.asarray(value, dtype=_canon_dtype(dtype))
    return JArray._wrap(arr)


def array(value, dtype=None, copy=True):
    return asarray(np.array(value, copy=copy), dtype=dtype)


def result_type(*args):
    return _canon_dtype(np.result_type(*[a if not isinstance(a, (int, float)) else np.asarray(a) for a in args]))


def _ctor(fn):
    def wrapped(*args, dtype=None, **kwargs):
        if dtype is None:
            return asarray(fn(*args, **kwargs))
        return asarray(fn(*args, dtype=_canon_dtype(dtype), **kwargs))

    return wrapped


zeros = _ctor(np.zeros)
ones = _ctor(np.ones)
full = _ctor(np.full)
arange = _ctor(np.arange)
empty = _ctor(np.empty)
linspace = _ctor(np.linspace)


def zeros_like(a, dtype=None):
    return asarray(np.zeros_like(np.asarray(a), dtype=_canon_dtype(dtype)))


def ones_like(a, dtype=None):
    return asarray(np.ones_like(np.asarray(a), dtype=_canon_dtype(dtype)))


def _passthrough(name):
    fn = getattr(np, name)

    def wrapped(*args, **kwargs):
        out = fn(*args, **kwargs)
        if isinstance(out, np.ndarray) and not isinstance(out, JArray):
            return asarray(out)
        return out

    wrapped.__name__ = name
    return wrapped


_jnp = types.ModuleType("jax.numpy")
for _name in dir(np):
    if _name.startswith("_"):
        continue
    _attr = getattr(np, _name)
    if callable(_attr) and not isinstance(_attr, type):
        try:
            setattr(_jnp, _name, _passthrough(_name))
        except Exception:  # pragma: no cover - defensive
            setattr(_jnp, _name, _attr)
    else:
        setattr(_jnp, _name, _attr)
for _name, _fn in {
    "asarray": asarray,
    "array": array,
    "result_type": result_type,
    "zeros": zeros,
    "ones": ones,
    "full": full,
    "arange": arange,
    "empty": empty,
    "linspace": linspace,
    "zeros_like": zeros_like,
    "ones_like": ones_like,
}.items():
    setattr(_jnp, _name, _fn)
_jnp.ndarray = np.ndarray
_jnp.float32 = np.float32
_jnp.float64 = np.float64
_jnp.int32 = np.int32
_jnp.bool_ = np.bool_
_jnp.complex64 = np.complex64


def _cond(pred, true_fn, false_fn, *operands, operand=None):
    if operand is not None and not operands:
        operands = (operand,)
    return true_fn(*operands) if bool(pred) else false_fn(*operands)


def _fori_loop(lower, upper, body, init):
    val = init
    for i in range(int(lower), int(upper)):
        val = body(i, val)
    return val


def _dynamic_slice(arr, starts, sizes):
    index = tuple(slice(int(s), int(s) + int(n)) for s, n in zip(starts, sizes))
    return asarray(np.asarray(arr)[index])


def _dynamic_update_slice(arr, update, starts):
    out = np.array(arr, copy=True)
    update = np.asarray(update)
    index = tuple(slice(int(s), int(s) + int(n)) for s, n in zip(starts, update.shape))
    out[index] = update
    return asarray(out)


_lax = types.ModuleType("jax.lax")
_lax.cond = _cond
_lax.fori_loop = _fori_loop
_lax.dynamic_slice = _dynamic_slice
_lax.dynamic_update_slice = _dynamic_update_slice

_jax = types.ModuleType("jax")
_jax.numpy = _jnp
_jax.lax = _lax
_jax.Array = np.ndarray


class _Config:
    def read(self, name):
        return False


_jax.config = _Config()


def install() -> None:
    """Register the stand-in as ``jax``, ``jax.numpy`` and ``jax.lax``."""
    sys.modules["jax"] = _jax
    sys.modules["jax.numpy"] = _jnp
    sys.modules["jax.lax"] = _lax
