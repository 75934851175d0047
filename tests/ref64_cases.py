"""Inputs of the blind rotation at the reference's own parameter set
(q = 2^64 in float64, N = 2048, n = 702, gadget 2^13 x 2, collapse 3,
sigma 2^17; parameters_crypto.py:6-32), rebuilt from fixed seeds for the
fixtures in tests/golden/ref64_golden.npz."""
from __future__ import annotations

import numpy as np

from oracle import tfhe_oracle as O

BATCH = 3          # full-chain ciphertexts
T_MSG = 16         # messages in Z_8 with a padding bit: delta = q / 16
GROUP1_BATCH = 4

_CACHE = {}


def case():
    if "c" in _CACHE:
        return _CACHE["c"]
    p = O.REF64
    q, N = p["q"], p["N"]
    sk_glwe, sk_lwe, bsk = O.keygen_q64(p, 64)
    rng = np.random.default_rng(65)
    msgs = rng.integers(0, T_MSG // 2, size=BATCH)
    delta = np.uint64(1 << 60)                                  # q / 16
    a, b = O.encrypt_lwe_q64(msgs.astype(np.uint64) * delta, sk_lwe, 2.0 ** 40, rng)
    body = O.step_lut(N, T_MSG // 2, T_MSG // 4, q / T_MSG)      # m >= 4 -> q/16
    luts = [np.zeros((BATCH, N)), np.broadcast_to(body, (BATCH, N)).copy()]
    c = dict(sk_glwe=sk_glwe, sk_lwe=sk_lwe, bsk_coeff=bsk, bsk_ordered=O.bsk_coeff_fourier_ordered(bsk),
             all_rot=O.all_rot_possible_fourier(N), lwe_a=a, lwe_b=b, msgs=msgs, luts=luts, body=body)
    _CACHE["c"] = c
    return c


def one_group_inputs(c):
    """Random accumulators and LWE mask triples for the first CMux group,
    with the key restricted to that group (G = 1)."""
    p = O.REF64
    N, L, cc = p["N"], p["l_bs"], p["collapse"]
    G, M = p["n"] // cc, 2 ** cc
    rng = np.random.default_rng(66)
    acc = O.u64_to_centred(rng.integers(0, 2 ** 64, size=(GROUP1_BATCH, 2, N), dtype=np.uint64))
    pk = O.u64_to_centred(rng.integers(0, 2 ** 64, size=(GROUP1_BATCH, cc), dtype=np.uint64))
    bsk1 = c["bsk_ordered"].reshape(2, 2, L, G, M, N // 2)[:, :, :, :1].reshape(2, 2, L, M, N // 2)
    return {"acc": acc, "pk": pk, "bsk1": bsk1}
