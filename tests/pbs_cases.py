"""Shared test cases: keys from the oracle's key generation, canonicalised
to the uint32 torus so the oracle and the engine see identical integers."""
from __future__ import annotations

import numpy as np

from oracle import tfhe_oracle as O

Q = 2.0 ** 32

PARAMS = {
    "tiny_c3": dict(q=Q, N=256, n=24, beta_bs=2 ** 7, l_bs=3, collapse=3, beta_ks=2 ** 3, l_ks=5,
                    sigma_glwe=2.0 ** 7, sigma_lwe=2.0 ** 17),
    "tiny_c2": dict(q=Q, N=512, n=16, beta_bs=2 ** 15, l_bs=2, collapse=2, beta_ks=2 ** 4, l_ks=5,
                    sigma_glwe=1.0, sigma_lwe=2.0 ** 15),
    "cfg1": dict(q=Q, N=1024, n=630, beta_bs=2 ** 7, l_bs=3, collapse=3, beta_ks=2 ** 3, l_ks=5,
                 sigma_glwe=2.0 ** 7, sigma_lwe=2.0 ** 17),
    "cfg2": dict(q=Q, N=2048, n=742, beta_bs=2 ** 15, l_bs=2, collapse=2, beta_ks=2 ** 4, l_ks=5,
                 sigma_glwe=1.0, sigma_lwe=2.0 ** 15),
    "c1_N128": dict(q=Q, N=128, n=12, beta_bs=2 ** 8, l_bs=2, collapse=1, beta_ks=2 ** 4, l_ks=4,
                    sigma_glwe=2.0 ** 6, sigma_lwe=2.0 ** 16),
    "c4_N4096": dict(q=Q, N=4096, n=8, beta_bs=2 ** 10, l_bs=1, collapse=4, beta_ks=2 ** 4, l_ks=4,
                     sigma_glwe=1.0, sigma_lwe=2.0 ** 15),
    # the cluster-of-four kernel's other level counts: one level (the CTAs of
    # odd rank transform nothing) and three (two levels on the even ranks)
    "c1_N1024_l1": dict(q=Q, N=1024, n=12, beta_bs=2 ** 10, l_bs=1, collapse=1, beta_ks=2 ** 4, l_ks=4,
                        sigma_glwe=1.0, sigma_lwe=2.0 ** 15),
    "c3_N2048_l3": dict(q=Q, N=2048, n=18, beta_bs=2 ** 7, l_bs=3, collapse=3, beta_ks=2 ** 3, l_ks=5,
                        sigma_glwe=2.0 ** 7, sigma_lwe=2.0 ** 17),
}
KEY_SEED = {"tiny_c3": 11, "tiny_c2": 12, "cfg1": 13, "cfg2": 14, "c1_N128": 15, "c4_N4096": 16, "c1_N1024_l1": 17,
            "c3_N2048_l3": 18}
INPUT_SEED = {"tiny_c3": 21, "tiny_c2": 22, "cfg1": 23, "cfg2": 24, "c1_N128": 25, "c4_N4096": 26, "c1_N1024_l1": 27,
              "c3_N2048_l3": 28}


def canon(x):
    """torus values -> centred float64 in [-2^31, 2^31) (the uint32 view)."""
    a = np.rint(np.asarray(x, dtype=np.float64)).astype(np.int64)
    return (((a + 2 ** 31) & 0xFFFFFFFF) - 2 ** 31).astype(np.float64)


_KEYS = {}


def keys(name):
    if name not in _KEYS:
        k = O.keygen(PARAMS[name], KEY_SEED[name])
        k.bsk_coeff = canon(k.bsk_coeff)
        k.bsk_ordered = O.bsk_coeff_fourier_ordered(k.bsk_coeff)
        k.ksk = (canon(k.ksk[0]), canon(k.ksk[1]))
        _KEYS[name] = k
    return _KEYS[name]


def inputs(name, batch, t=32, seed_offset=0):
    """Messages in Z_{t/2} (padding bit) encrypted under the GLWE key."""
    p = PARAMS[name]
    rng = np.random.default_rng(INPUT_SEED[name] + seed_offset)
    msgs = rng.integers(0, t // 2, size=batch)
    a, b = O.encrypt_inputs(keys(name), msgs, p["q"] / t, rng)
    return msgs, canon(a), canon(b)


def ks_params(name):
    p = PARAMS[name]
    return {"beta_ks": p["beta_ks"], "l_ks": p["l_ks"], "q": p["q"]}


def step_body(name, t=32):
    """step LUT body for Z_{t/2} + padding: m >= t/4 -> 1, scaled by q/t"""
    p = PARAMS[name]
    return O.step_lut(p["N"], t // 2, t // 4, p["q"] / t)


def many_lut_body(name, n_lut):
    """n_lut step sub-LUTs (get_plain_LUT, nn_tfhe/utils_spike.py:72-87)
    with thresholds spread over [-1.5, 1.5], scaled by q/16"""
    p = PARAMS[name]
    return canon(sum(O.get_plain_LUT(p["N"], n_lut, i, 4.0, g)
                     for i, g in enumerate(np.linspace(-1.5, 1.5, n_lut))) * (p["q"] / 16))
