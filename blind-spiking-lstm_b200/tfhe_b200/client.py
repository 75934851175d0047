"""Client side of the engine: secret keys, the public key material the
device needs (bootstrapping and key-switching keys), encryption, decryption
and LUT polynomials, all on the uint32 torus (q = 2^32), host numpy.

The key structure is the reference's:
* key switching key: LWE encryptions under the small key of
  -s_big[i] * q / beta_ks^j (schemas/LWE_jax.py:86-93), as (l_ks, n_big, n)
  masks and (l_ks, n_big) bodies;
* collapsed bootstrapping key: for group g and pattern p (meshgrid 'ij'
  order), e = [s_g == p]; "left" rows GLWE(-e * s_glwe * q / beta^j), "right"
  rows GLWE(e * q / beta^j at coefficient 0), j = 1..l
  (schemas/RLWE_jax.py:162-197), as (2 left/right, 2 mask/body, G*M, l, N).
Outputs of a bootstrap are LWEs under the GLWE key (sk_lut = sk,
setup_crypto.py:19-21), so the big LWE key is the GLWE key.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .params import ParamSet

MASK32 = np.uint64(0xFFFFFFFF)


def _u32(x) -> np.ndarray:
    return (np.asarray(x).astype(np.int64) & 0xFFFFFFFF).astype(np.uint32)


def _centred(u) -> np.ndarray:
    return np.asarray(u, dtype=np.uint32).view(np.int32).astype(np.int64)


def negacyclic_mul_binary(a_u32: np.ndarray, s: np.ndarray) -> np.ndarray:
    """(a * s) mod (X^N + 1, 2^32) for uint32 polynomials a (..., N) and a
    binary s (N,): a is split into two 16-bit halves so every FFT product is
    below 2^28 and rounds to the exact integer."""
    a = np.asarray(a_u32, dtype=np.uint32)
    N = a.shape[-1]
    k = np.arange(N)
    tw = np.exp(-1j * np.pi * k / N)
    fs = np.fft.fft(tw * np.asarray(s, dtype=np.float64))
    out = np.zeros(a.shape, dtype=np.uint64)
    for shift in (0, 16):
        half = ((a >> np.uint32(shift)) & np.uint32(0xFFFF)).astype(np.float64)
        prod = np.fft.ifft(np.fft.fft(tw * half, axis=-1) * fs, axis=-1) * np.conj(tw)
        v = np.rint(prod.real)
        if np.max(np.abs(prod.real - v), initial=0.0) > 0.1:
            raise ArithmeticError("negacyclic product lost exactness")
        out += (v.astype(np.int64).astype(np.uint64) & MASK32) << np.uint64(shift)
    return (out & MASK32).astype(np.uint32)


@dataclass
class ClientKeys:
    params: ParamSet
    sk_glwe: np.ndarray      # (N,) 0/1
    sk_lwe: np.ndarray       # (n,) 0/1
    bsk: np.ndarray          # uint32 (2, 2, G*M, l_bs, N)
    ksk_a: np.ndarray        # uint32 (l_ks, n_big, n)
    ksk_b: np.ndarray        # uint32 (l_ks, n_big)


def _glwe_encrypt(msg_u32, sk, sigma, rng):
    mask = rng.integers(0, 2 ** 32, size=msg_u32.shape, dtype=np.uint64).astype(np.uint32)
    e = np.rint(rng.standard_normal(msg_u32.shape) * sigma).astype(np.int64)
    body = negacyclic_mul_binary(mask, sk).astype(np.int64) + msg_u32.astype(np.int64) + e
    return mask, _u32(body)


def _lwe_encrypt(msg, sk, sigma, rng):
    """LWE encryptions of integer messages (..., ) under sk (n,)."""
    msg = np.asarray(msg, dtype=np.int64)
    n = sk.shape[-1]
    mask = rng.integers(0, 2 ** 32, size=msg.shape + (n,), dtype=np.uint64).astype(np.uint32)
    dot = (_centred(mask).astype(np.float64) @ sk.astype(np.float64)).astype(np.int64)   # exact (< 2^53)
    e = np.rint(rng.standard_normal(msg.shape) * sigma).astype(np.int64)
    return mask, _u32(dot + msg + e)


def keygen(params: ParamSet, seed: int) -> ClientKeys:
    p = params
    rng = np.random.default_rng(seed)
    sk_glwe = rng.integers(0, 2, size=p.N).astype(np.int64)
    sk_lwe = rng.integers(0, 2, size=p.n).astype(np.int64)
    # key switching key
    j = np.arange(1, p.l_ks + 1)
    g = (1 << (32 - j * p.log2_beta_ks)).astype(np.int64)                    # q / beta^j
    msg = -(g[:, None] * sk_glwe[None, : p.big])                             # (l_ks, n_big)
    ksk_a, ksk_b = _lwe_encrypt(msg, sk_lwe, p.sigma_lwe, rng)
    # collapsed bootstrapping key
    c, M, G, L, N = p.collapse, p.M, p.G, p.l_bs, p.N
    patterns = np.stack(np.meshgrid(*([np.array([0, 1])] * c), indexing="ij"), axis=-1).reshape(-1, c)
    groups = sk_lwe.reshape(G, c)
    eq = np.all(groups[:, None, :] == patterns[None, :, :], axis=-1).astype(np.int64).reshape(-1)   # (G*M)
    gj = (1 << (32 - np.arange(1, L + 1) * p.log2_beta_bs)).astype(np.int64)                     # (L,)
    left = -(eq[:, None, None] * gj[None, :, None] * sk_glwe[None, None, :])                      # (GM, L, N)
    right = np.zeros((G * M, L, N), dtype=np.int64)
    right[:, :, 0] = eq[:, None] * gj[None, :]
    bsk = np.empty((2, 2, G * M, L, N), dtype=np.uint32)
    for side, m in enumerate((left, right)):
        mask, body = _glwe_encrypt(_u32(m), sk_glwe, p.sigma_glwe, rng)
        bsk[side, 0], bsk[side, 1] = mask, body
    return ClientKeys(p, sk_glwe, sk_lwe, bsk, ksk_a, ksk_b)


def encrypt(keys: ClientKeys, messages, t: int, rng, sigma=None):
    """LWEs under the GLWE key of messages in Z_t at scale q / t (callers
    keep messages in [0, t/2) for a padding bit).  Returns (a (B, N), b (B))."""
    sigma = keys.params.sigma_glwe if sigma is None else sigma
    delta = 1 << (32 - int(np.log2(t)))
    return _lwe_encrypt(np.asarray(messages, dtype=np.int64) * delta, keys.sk_glwe, sigma, rng)


def phase(a, b, sk) -> np.ndarray:
    """b - <a, s> on the torus, centred int64."""
    dot = (_centred(a).astype(np.float64) @ np.asarray(sk, dtype=np.float64)).astype(np.int64)
    return _centred(_u32(_centred(b) - dot))


def decrypt(a, b, sk, t: int) -> np.ndarray:
    """round(phase / (q/t)) mod t (schemas/LWE_jax.py:30-48, non-negative)."""
    ph = phase(a, b, sk).astype(np.float64)
    return np.mod(np.rint(ph / (2.0 ** 32 / t)), t).astype(np.int64)


def step_lut(N: int, t_in: int, threshold: int, t_out: int) -> np.ndarray:
    """uint32 LUT body: messages m in Z_t_in with a padding bit (phase
    m q / (2 t_in)) map to [m >= threshold] at scale q / t_out; the last half
    box wraps to m = 0 negacyclically."""
    box = N // t_in
    j = np.arange(N)
    m = (j + box // 2) // box
    out_scale = 1 << (32 - int(np.log2(t_out)))
    val = (m >= threshold).astype(np.int64) * out_scale
    val[m >= t_in] = -out_scale * int(0 >= threshold)
    return _u32(val)


def table_lut(N: int, table, t_out: int) -> np.ndarray:
    """uint32 LUT body of an arbitrary table f: Z_t -> Z_t_out, t = len(table),
    for inputs with a padding bit: box m covers [m N/t - N/(2t), m N/t + N/(2t));
    the wrapped half box of m = 0 holds -f(0)."""
    table = np.asarray(table, dtype=np.int64)
    t = len(table)
    box = N // t
    j = np.arange(N)
    m = (j + box // 2) // box
    out_scale = 1 << (32 - int(np.log2(t_out)))
    val = np.where(m < t, table[np.minimum(m, t - 1)] * out_scale, -table[0] * out_scale)
    return _u32(val)


def many_lut(N: int, n_lut: int, thresholds, s: float, t_out: int) -> np.ndarray:
    """uint32 LUT body packing n_lut step tables (nn_tfhe/utils_spike.py:72-87):
    sub-LUT i on positions base*n_lut + i, value [linspace(-s, s) >= thr_i],
    rotated by -N/2 (negacyclic)."""
    sub = N // n_lut
    part = -s + 2 * s * np.arange(sub) / sub
    full = np.zeros(N, dtype=np.int64)
    for i, thr in enumerate(thresholds):
        full[np.arange(sub) * n_lut + i] = (part >= thr).astype(np.int64)
    full *= 1 << (32 - int(np.log2(t_out)))
    # X^(-N/2) * full: coefficient k <- full[k + N/2], negated where it wraps
    rot = np.concatenate([full[N // 2:], -full[: N // 2]])
    return _u32(rot)


def packed_table_lut(N: int, tables, t_out: int) -> np.ndarray:
    """uint32 LUT body packing n_lut arbitrary tables f_i: Z_t -> Z_t_out
    (inputs with a padding bit) for one blind rotation: sub-LUT i sits on
    coefficients base * n_lut + i (the packing of nn_tfhe/utils_spike.py:72-87)
    and holds f_i of the message decoded at position base * n_lut; after the
    rotation by -b~ (a multiple of n_lut) coefficient i is f_i(m)."""
    tables = np.asarray(tables, dtype=np.int64)
    n_lut, t = tables.shape
    box = N // t
    pos = np.arange(0, N, n_lut)
    m = (pos + box // 2) // box
    scale = 1 << (32 - int(np.log2(t_out)))
    body = np.zeros(N, dtype=np.int64)
    for i in range(n_lut):
        body[pos + i] = np.where(m < t, tables[i][np.minimum(m, t - 1)] * scale, -tables[i][0] * scale)
    return _u32(body)


# ---------------------------------------------------------------- RLWE level
def encrypt_rlwe(msg, sk, sigma: float, rng):
    """RLWE encryptions (schemas/RLWE_jax.py:36-54) of integer polynomials
    msg (..., N) under the binary key sk (N,): (mask, body) uint32."""
    return _glwe_encrypt(_u32(msg), np.asarray(sk), sigma, rng)


def rlwe_phase(a, b, sk) -> np.ndarray:
    """b - a * s on the torus, centred int64 (..., N)."""
    prod = negacyclic_mul_binary(np.asarray(a, dtype=np.uint32), np.asarray(sk))
    return _centred(_u32(_centred(b) - _centred(prod)))


def automorphism(poly, k: int) -> np.ndarray:
    """X -> X^k on integer polynomials (schemas/polynomial_jax.py:171-200)."""
    poly = np.asarray(poly, dtype=np.int64)
    N = poly.shape[-1]
    idx = (np.arange(N) * k) % (2 * N)
    out = np.zeros_like(poly)
    out[..., idx % N] = np.where(idx >= N, -poly, poly)
    return out


def galois_keys(sk, log2_beta: int, l: int, sigma: float, rng) -> np.ndarray:
    """Keys of pack_lwe_to_rlwe (get_galois_key, schemas/RLWE_jax.py:218-226):
    for step i, k = 2^(log2 N - i) + 1, the RLWE key switching key
    (get_keyswitch_sk, :91-98) from s(X^k) back to s: rows
    RLWE_s(-s(X^k) q / beta^j), j = 1..l.  Returns uint32 (log2 N, l, 2, N)."""
    sk = np.asarray(sk, dtype=np.int64)
    N = sk.shape[-1]
    steps = int(np.log2(N))
    gj = (1 << (32 - np.arange(1, l + 1) * log2_beta)).astype(np.int64)
    out = np.empty((steps, l, 2, N), dtype=np.uint32)
    for i in range(steps):
        s_auto = automorphism(sk, 2 ** (steps - i) + 1)
        mask, body = encrypt_rlwe(-(gj[:, None] * s_auto[None, :]), sk, sigma, rng)
        out[i, :, 0], out[i, :, 1] = mask, body
    return out


def packing_key(sk_lwe, sk_rlwe, log2_beta: int, l: int, sigma: float, rng) -> np.ndarray:
    """Packing key (get_packing_KSK, schemas/RLWE_jax.py:205-215): for every
    LWE key bit s_i and level j, RLWE_{sk_rlwe}(s_i q / beta^j) as a constant
    polynomial.  Returns uint32 (n_dim, l, 2, N)."""
    sk_lwe = np.asarray(sk_lwe, dtype=np.int64)
    N = np.asarray(sk_rlwe).shape[-1]
    gj = (1 << (32 - np.arange(1, l + 1) * log2_beta)).astype(np.int64)
    msg = np.zeros((sk_lwe.shape[0], l, N), dtype=np.int64)
    msg[:, :, 0] = sk_lwe[:, None] * gj[None, :]
    mask, body = encrypt_rlwe(msg, sk_rlwe, sigma, rng)
    return np.stack([mask, body], axis=2)
