"""A numpy-backed stand-in for the subset of ``jax`` that the reference's
PBS-path modules use (``schemas/polynomial_jax.py``, ``schemas/text_jax.py``,
``schemas/LWE_jax.py``, ``schemas/RLWE_jax.py``, ``parameters_crypto.py``).

It exists only so that ``tests/golden/make_golden.py`` can execute the
reference's own Python source in this container, where jax is not installed,
and record its outputs as golden fixtures.  Semantics kept from jax with
``jax_enable_x64``: float64 by default, ``round`` = round-half-to-even,
``vmap`` = map over an axis and stack, ``lax.scan`` = loop and stack,
``jit`` = identity.  FFTs are numpy's (pocketfft) instead of XLA's.
Random-number functions are not provided: keys come from the oracle's
seeded key generation.
"""
from __future__ import annotations

import numpy as _np

from . import numpy  # noqa: F401  (jax.numpy)
from . import lax    # noqa: F401  (jax.lax)
from .numpy import JArray as Array


class _Config:
    def update(self, *args, **kwargs):
        return None


config = _Config()


def jit(fun=None, **kwargs):
    """jax.jit: identity (static_argnames and friends are ignored)."""
    if fun is None:
        return lambda f: f
    return fun


def _is_leaf(x):
    return not isinstance(x, (tuple, list, dict))


def tree_map(f, tree):
    if isinstance(tree, tuple):
        return tuple(tree_map(f, t) for t in tree)
    if isinstance(tree, list):
        return [tree_map(f, t) for t in tree]
    if isinstance(tree, dict):
        return {k: tree_map(f, v) for k, v in tree.items()}
    return f(tree)


def tree_leaves(tree):
    if isinstance(tree, (tuple, list)):
        out = []
        for t in tree:
            out.extend(tree_leaves(t))
        return out
    if isinstance(tree, dict):
        out = []
        for v in tree.values():
            out.extend(tree_leaves(v))
        return out
    return [tree]


def tree_stack(trees, axis=0):
    first = trees[0]
    if first is None:
        return None
    if isinstance(first, tuple):
        return tuple(tree_stack([t[i] for t in trees], axis) for i in range(len(first)))
    if isinstance(first, list):
        return [tree_stack([t[i] for t in trees], axis) for i in range(len(first))]
    if isinstance(first, dict):
        return {k: tree_stack([t[k] for t in trees], axis) for k in first}
    return _np.stack([_np.asarray(t) for t in trees], axis=axis).view(Array)


def vmap(fun, in_axes=0, out_axes=0):
    """jax.vmap: call ``fun`` once per index of the mapped axis and stack
    the results (leaf-wise) on ``out_axes``."""
    def wrapped(*args):
        if isinstance(in_axes, (tuple, list)):
            axes = list(in_axes)
        else:
            axes = [in_axes] * len(args)
        size = None
        for arg, ax in zip(args, axes):
            if ax is None:
                continue
            leaf = _np.asarray(tree_leaves(arg)[0])
            size = leaf.shape[ax]
            break
        if size is None:
            raise ValueError("vmap: no mapped argument")
        outs = []
        for i in range(size):
            call = []
            for arg, ax in zip(args, axes):
                if ax is None:
                    call.append(arg)
                else:
                    call.append(tree_map(lambda x, ax=ax: _np.asarray(_np.take(_np.asarray(x), i, axis=ax)).view(Array)
                                         if _np.ndim(x) else x, arg))
            outs.append(fun(*call))
        return tree_stack(outs, out_axes)
    return wrapped
