"""``jax.lax`` stand-in: ``scan`` as a Python loop, ``stop_gradient`` as
identity.  Used only to run the reference's Python modules for golden
fixtures."""
from __future__ import annotations

import numpy as _np


def stop_gradient(x):
    return x


def scan(f, init, xs=None, length=None, reverse=False, unroll=1, **kwargs):
    from . import tree_map, tree_leaves, tree_stack
    if xs is None:
        n = length
    else:
        n = _np.asarray(tree_leaves(xs)[0]).shape[0]
    carry = init
    ys = []
    order = range(n - 1, -1, -1) if reverse else range(n)
    for i in order:
        x_i = None if xs is None else tree_map(lambda x: _np.asarray(x)[i], xs)
        carry, y = f(carry, x_i)
        ys.append(y)
    if reverse:
        ys = ys[::-1]
    if not ys or ys[0] is None:
        return carry, None
    return carry, tree_stack(ys)
