"""Import environment for executing the REFERENCE's own Python code
(AMIAD-Research/Blind-Spiking-LSTM) in this container, for the golden
fixture generators.

jax and flax are not installed, so the reference modules run under the
numpy-backed stand-ins in ``tests/golden/jaxshim``.  The compiled FFI module
``cuTFHE._core`` cannot be built either; ``cuTFHE.multiply`` is replaced by
a stub that forwards to the reference's own JAX statement of the kernel,
``schemas/text_jax.py:multiply_seq_monomial`` (same signature up to log2
arguments, cuTFHE/multiply.py:54-92 vs schemas/text_jax.py:390-435).
"""
from __future__ import annotations

import os
import sys
import types

HERE = os.path.dirname(os.path.abspath(__file__))
TESTS = os.path.dirname(HERE)
REPO = os.path.dirname(TESTS)
PKG = os.path.join(REPO, "blind-spiking-lstm_b200")


def reference_root():
    root = os.environ.get("REFERENCE_ROOT")
    if not root or not os.path.isdir(root):
        raise SystemExit("set REFERENCE_ROOT to a checkout of AMIAD-Research/Blind-Spiking-LSTM")
    return root


def setup():
    """Put the stand-ins, the reference, the repository and the tests on
    sys.path and install the cuTFHE stub.  Returns the reference root."""
    root = reference_root()
    for p in (PKG, REPO, TESTS, root, os.path.join(HERE, "jaxshim")):
        if p not in sys.path:
            sys.path.insert(0, p)
    from schemas import text_jax as TJ

    cu = types.ModuleType("cuTFHE")
    cum = types.ModuleType("cuTFHE.multiply")

    def multiply_seq_monomial(ciphertext, public_key, BSK, log_q, log_beta, l, degree,
                              collapse, all_rot_fft, n_lut):
        return TJ.multiply_seq_monomial(ciphertext, public_key, BSK, 2.0 ** log_q,
                                        2 ** log_beta, l, degree, collapse, all_rot_fft, n_lut)

    cum.multiply_seq_monomial = multiply_seq_monomial
    cu.multiply = cum
    sys.modules["cuTFHE"] = cu
    sys.modules["cuTFHE.multiply"] = cum
    return root
