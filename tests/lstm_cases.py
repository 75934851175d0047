"""Shared cases for the Spike-LSTM operators: a small layer on the tiny_c3
bootstrapping parameters (N=256) with Galois and packing keys from the
client key generation, and the same layer as the oracle's dict."""
from __future__ import annotations

import numpy as np

from oracle import lstm_oracle as LO
from pbs_cases import PARAMS, canon, keys as case_keys

NAME = "tiny_c3"
INPUT_DIM, HIDDEN, N_LUT = 4, 8, 2
GAL_LOG2_BETA, GAL_L = 4, 6
PK_LOG2_BETA, PK_L = 8, 3
BETA_X = 2.0 ** 22          # scale of x, h and c on the torus
S_LUT = 1.0

_CACHE = {}


def cen(u):
    return np.asarray(u, dtype=np.uint32).view(np.int32).astype(np.int64)


def layer_material(seed=5):
    """Keys, weights and LUTs of the small layer (numpy)."""
    if seed in _CACHE:
        return _CACHE[seed]
    from tfhe_b200 import client
    p = PARAMS[NAME]
    N = p["N"]
    k = case_keys(NAME)
    sk = k.sk_glwe.astype(np.int64)
    rng = np.random.default_rng(seed)
    galois = client.galois_keys(sk, GAL_LOG2_BETA, GAL_L, 1.0, rng)
    ksp = client.packing_key(sk, sk, PK_LOG2_BETA, PK_L, 1.0, rng)
    per = HIDDEN // N_LUT
    dim = INPUT_DIM + HIDDEN
    mats = {g: rng.integers(-7, 8, size=(dim, per)) for g in "fio"}
    biases = {g: rng.integers(-3, 4, size=per) * int(BETA_X) for g in "fio"}
    gam = {g: rng.uniform(-0.6, 0.6, size=(N_LUT, per)) for g in "fio"}
    eta = rng.uniform(0.5, 1.5, size=(N_LUT, per))
    plain = {g: np.stack([np.stack([LO.get_plain_LUT(N, N_LUT, i, S_LUT, gam[g][i, kk]) for kk in range(per)])
                          for i in range(N_LUT)]) for g in "fio"}
    lut_f = np.rint(plain["f"]).astype(np.int64)
    lut_o = np.rint(plain["o"]).astype(np.int64)
    lut_i = np.rint(np.sum(plain["i"] * eta[..., None], axis=0) * BETA_X).astype(np.int64)
    layer = {"input_dim": INPUT_DIM, "hidden": HIDDEN, "n_lut": N_LUT, "galois": cen(galois),
             "gal_log2_beta": GAL_LOG2_BETA, "gal_l": GAL_L, "ksp_a": cen(ksp[:, :, 0]), "ksp_b": cen(ksp[:, :, 1]),
             "pk_log2_beta": PK_LOG2_BETA, "pk_l": PK_L, "lut_f": lut_f, "lut_o": lut_o, "lut_i": lut_i}
    for g in "fio":
        kern, bias = LO.linear_kernel_polynomial(mats[g], biases[g], np.ones(per), N)
        layer[f"kern_{g}"], layer[f"bias_{g}"] = kern, bias
    out = dict(p=p, keys=k, sk=sk, galois=galois, ksp=ksp, mats=mats, biases=biases, layer=layer)
    _CACHE[seed] = out
    return out


def encrypt_inputs(sk, T, S, N, seed=7, sigma=1.0):
    """T x S RLWEs of small integer embeddings at coefficients [0, INPUT_DIM)
    scaled by BETA_X: (T, S, 2, N) uint32 and the messages (T, S, INPUT_DIM)."""
    from tfhe_b200 import client
    rng = np.random.default_rng(seed)
    msg = rng.integers(-2, 3, size=(T, S, INPUT_DIM))
    poly = np.zeros((T, S, N), dtype=np.int64)
    poly[..., :INPUT_DIM] = msg * int(BETA_X)
    a, b = client.encrypt_rlwe(poly, sk, sigma, rng)
    return np.stack([a, b], axis=2), msg
