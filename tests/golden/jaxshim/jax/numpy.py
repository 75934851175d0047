"""``jax.numpy`` stand-in: numpy with jax's ``.at[...]`` functional updates,
float shifts accepted by ``roll`` (jax casts them to int32), and float64 as
the default float type.  Used only to run the reference's Python modules for
golden fixtures."""
from __future__ import annotations

import numpy as _np
from numpy import *  # noqa: F401,F403  (the jnp namespace)
from numpy import fft  # noqa: F401


class _AtIndex:
    def __init__(self, arr, idx):
        self._arr, self._idx = arr, idx

    def set(self, values):
        out = _np.array(self._arr, copy=True)
        out[self._idx] = values
        return out.view(JArray)

    def add(self, values):
        out = _np.array(self._arr, copy=True)
        out[self._idx] += values
        return out.view(JArray)


class _At:
    def __init__(self, arr):
        self._arr = arr

    def __getitem__(self, idx):
        return _AtIndex(self._arr, idx)


class JArray(_np.ndarray):
    """ndarray with jax's ``.at`` update helper."""

    @property
    def at(self):
        return _At(self)

    def __rpow__(self, base):
        # ``(-1) ** (alpha // n)`` in schemas/polynomial_jax.py:165 with an
        # integer array exponent that can be negative (parameters_crypto.py:89
        # rotates by arange(-N, N)).  numpy refuses integer ** negative
        # integer; the monomial table only means X^r when this is the
        # mathematical +-1, so the power is taken in float64.
        exp = _np.asarray(self)
        if _np.issubdtype(exp.dtype, _np.integer) and _np.any(exp < 0):
            return _np.power(float(base), exp.astype(_np.float64)).view(JArray)
        return _np.power(base, exp).view(JArray)


def _wrap(fn):
    def inner(*args, **kwargs):
        out = fn(*args, **kwargs)
        return out.view(JArray) if isinstance(out, _np.ndarray) else out
    inner.__name__ = getattr(fn, "__name__", "jnp_fn")
    return inner


array = _wrap(_np.array)
asarray = _wrap(_np.asarray)
zeros = _wrap(_np.zeros)
zeros_like = _wrap(_np.zeros_like)
ones = _wrap(_np.ones)
arange = _wrap(_np.arange)
stack = _wrap(_np.stack)
concatenate = _wrap(_np.concatenate)
concat = _wrap(_np.concatenate)
linspace = _wrap(_np.linspace)
where = _wrap(_np.where)
permute_dims = _wrap(_np.transpose)


def roll(a, shift, axis=None):
    """jnp.roll: a traced (array) shift is cast to int32 as jax does."""
    if not isinstance(shift, (int, _np.integer, tuple, list)):
        s = _np.asarray(shift)
        shift = int(s.reshape(-1)[0]) if s.size == 1 else tuple(int(v) for v in s.reshape(-1))
    return _np.roll(_np.asarray(a), shift, axis=axis).view(JArray)
