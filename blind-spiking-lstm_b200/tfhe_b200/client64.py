"""Client side on the reference's own torus, q = 2^64 (parameters_crypto.py:6):
secret keys, the device key material (bootstrapping, key-switching, Galois
and packing keys), encryption and decryption, host numpy, exact modulo 2^64
(uint64 wrap-around).

The reference holds these values as float64; here they are uint64 words and
every key is an exact encryption.  Key structures are those of the 2^32
client (client.py) with q / beta^j = 2^(64 - j log2 beta).  The blind
rotation's key is handed to the device in the reference's Fourier layout
(jax_fourier, nn_tfhe/activation.py:49-53, reshaped as cuTFHE/multiply.py:
81-86), because the 2^64 blind rotation is the FP64 kernel of
tfhe_mul_bootstrap at log2_q = 64.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .client import automorphism

M16 = np.uint64(0xFFFF)


@dataclass(frozen=True)
class Params64:
    """A parameter set on Z/2^64."""
    name: str
    N: int
    n: int
    log2_beta_bs: int
    l_bs: int
    collapse: int
    log2_beta_ks: int
    l_ks: int
    sigma_glwe: float
    sigma_lwe: float

    @property
    def big(self) -> int:
        return self.N

    @property
    def M(self) -> int:
        return 1 << self.collapse

    @property
    def G(self) -> int:
        return self.n // self.collapse


# the reference's bootstrapping set (parameters_crypto.py:6-32): N = 2048,
# n = 702, gadget 2^13 x 2, collapse 3, sigma 2^17; the key switch before the
# bootstrap keeps the reference's 20 bits of precision (2 x 20 there) as
# 2^4 x 5
REF64 = Params64("q64_n702_N2048_b13x2_c3", N=2048, n=702, log2_beta_bs=13, l_bs=2, collapse=3, log2_beta_ks=4,
                 l_ks=5, sigma_glwe=2.0 ** 17, sigma_lwe=2.0 ** 40)


def u64(x) -> np.ndarray:
    """Integers (any integer dtype, possibly negative) -> uint64 words mod 2^64."""
    a = np.asarray(x)
    if a.dtype == np.uint64:
        return a
    return a.astype(np.int64).astype(np.uint64)


def centred(u) -> np.ndarray:
    """uint64 words -> centred int64."""
    return np.asarray(u, dtype=np.uint64).view(np.int64)


def negacyclic_mul_binary(a_u64: np.ndarray, s: np.ndarray) -> np.ndarray:
    """(a * s) mod (X^N + 1, 2^64) for uint64 polynomials a (..., N) and a
    binary s (N,): a is split into four 16-bit limbs so every FFT product is
    below 2^27 and rounds to the exact integer."""
    a = np.asarray(a_u64, dtype=np.uint64)
    N = a.shape[-1]
    k = np.arange(N)
    tw = np.exp(-1j * np.pi * k / N)
    fs = np.fft.fft(tw * np.asarray(s, dtype=np.float64))
    out = np.zeros(a.shape, dtype=np.uint64)
    for t in range(4):
        limb = ((a >> np.uint64(16 * t)) & M16).astype(np.float64)
        prod = np.fft.ifft(np.fft.fft(tw * limb, axis=-1) * fs, axis=-1) * np.conj(tw)
        v = np.rint(prod.real)
        if np.max(np.abs(prod.real - v), initial=0.0) > 0.1:
            raise ArithmeticError("negacyclic product lost exactness")
        out += v.astype(np.int64).astype(np.uint64) << np.uint64(16 * t)
    return out


def _noise(rng, shape, sigma):
    return u64(np.rint(rng.standard_normal(shape) * sigma).astype(np.int64))


def encrypt_rlwe(msg, sk, sigma: float, rng):
    """RLWE encryptions (schemas/RLWE_jax.py:36-54) of integer polynomials
    msg (..., N) under the binary key sk (N,): (mask, body) uint64."""
    m = u64(msg)
    mask = rng.integers(0, 2 ** 64, size=m.shape, dtype=np.uint64)
    body = negacyclic_mul_binary(mask, sk) + m + _noise(rng, m.shape, sigma)
    return mask, body


def encrypt_lwe(msg, sk, sigma: float, rng):
    """LWE encryptions (schemas/LWE_jax.py:9-28) of integer messages (...)
    under the binary key sk (n,): (mask (..., n), body (...)) uint64."""
    m = u64(msg)
    sk = np.asarray(sk)
    mask = rng.integers(0, 2 ** 64, size=m.shape + (sk.shape[-1],), dtype=np.uint64)
    dot = (mask * u64(sk)).sum(axis=-1, dtype=np.uint64)
    return mask, dot + m + _noise(rng, m.shape, sigma)


def phase(a, b, sk) -> np.ndarray:
    """b - <a, s> of LWEs (a (..., n), b (...)): centred int64."""
    dot = (np.asarray(a, dtype=np.uint64) * u64(sk)).sum(axis=-1, dtype=np.uint64)
    return centred(np.asarray(b, dtype=np.uint64) - dot)


def rlwe_phase(a, b, sk) -> np.ndarray:
    """b - a * s of RLWEs: centred int64 (..., N)."""
    return centred(np.asarray(b, dtype=np.uint64) - negacyclic_mul_binary(a, sk))


@dataclass
class ClientKeys64:
    params: Params64
    sk_glwe: np.ndarray      # (N,) 0/1
    sk_lwe: np.ndarray       # (n,) 0/1
    bsk: np.ndarray          # uint64 (2 left/right, 2 mask/body, G*M, l_bs, N)
    ksk: np.ndarray          # uint64 (n_big * l_ks, n + 1): row i l + j, columns mask 0..n-1, body n


def keygen(params: Params64, seed: int) -> ClientKeys64:
    """Keys with the reference's structure (schemas/RLWE_jax.py:162-197,
    schemas/LWE_jax.py:86-93) on Z/2^64."""
    p = params
    rng = np.random.default_rng(seed)
    sk_glwe = rng.integers(0, 2, size=p.N).astype(np.int64)
    sk_lwe = rng.integers(0, 2, size=p.n).astype(np.int64)
    # key switching key: LWE_{sk_lwe}(-s_big[i] q / beta^j)
    gj = np.array([1 << (64 - j * p.log2_beta_ks) for j in range(1, p.l_ks + 1)], dtype=np.uint64)
    msg = (np.uint64(0) - u64(sk_glwe[: p.big])[:, None] * gj[None, :])            # (n_big, l_ks)
    ka, kb = encrypt_lwe(msg, sk_lwe, p.sigma_lwe, rng)
    ksk = np.concatenate([ka, kb[..., None]], axis=-1).reshape(p.big * p.l_ks, p.n + 1)
    # collapsed bootstrapping key
    c, L, N = p.collapse, p.l_bs, p.N
    patterns = np.stack(np.meshgrid(*([np.array([0, 1])] * c), indexing="ij"), axis=-1).reshape(-1, c)
    eq = np.all(sk_lwe.reshape(p.G, c)[:, None, :] == patterns[None, :, :], axis=-1).reshape(-1).astype(np.uint64)
    gb = np.array([1 << (64 - j * p.log2_beta_bs) for j in range(1, L + 1)], dtype=np.uint64)
    left = (np.uint64(0) - eq[:, None, None] * gb[None, :, None]) * u64(sk_glwe)[None, None, :]
    right = np.zeros((p.G * p.M, L, N), dtype=np.uint64)
    right[:, :, 0] = eq[:, None] * gb[None, :]
    bsk = np.empty((2, 2, p.G * p.M, L, N), dtype=np.uint64)
    for side, m in enumerate((left, right)):
        bsk[side, 0], bsk[side, 1] = encrypt_rlwe(m, sk_glwe, p.sigma_glwe, rng)
    return ClientKeys64(p, sk_glwe, sk_lwe, bsk, ksk)


def bsk_fourier_grouped(bsk: np.ndarray, params: Params64) -> np.ndarray:
    """The bootstrapping key in the layout tfhe_mul_bootstrap reads:
    jax_fourier (schemas/polynomial_jax.py:11-15) of the centred float64
    values, ordered (G, 2 out, L, 2 in, M, N/2) complex128 (the reference's
    bsk_ordered, nn_tfhe/activation.py:49-53, reshaped and permuted as
    cuTFHE/multiply.py:81-86)."""
    p = params
    N = p.N
    tw = np.exp(-1j * np.pi * np.arange(N) / N)
    vals = centred(bsk).astype(np.float64)                          # (2 side, 2 pk/b, GM, L, N)
    four = np.fft.fft(tw * vals, axis=-1)[..., : N // 2]
    # [side][pk/b][g*M+m][l] -> (G, pk/b (out), l, side (in), M, d)
    four = four.reshape(2, 2, p.G, p.M, p.l_bs, N // 2)
    return np.ascontiguousarray(np.transpose(four, (2, 1, 4, 0, 3, 5)))


def monomial_fourier(N: int) -> np.ndarray:
    """Row r = jax_fourier(X^r), r in [0, 2N) (parameters_crypto.py:86-91):
    exp(-i pi r (2 j + 1) / N), j < N/2, with the angle reduced exactly."""
    r = np.arange(2 * N)[:, None]
    j = np.arange(N // 2)[None, :]
    e = (r * (2 * j + 1)) % (2 * N)
    return np.exp(-1j * np.pi * e / N)


def galois_keys(sk, log2_beta: int, l: int, sigma: float, rng) -> np.ndarray:
    """Keys of pack_lwe_to_rlwe (get_galois_key, schemas/RLWE_jax.py:218-226)
    on Z/2^64: for step i, k = 2^(log2 N - i) + 1, rows RLWE_s(-s(X^k) q /
    beta^j), j = 1..l.  Returns uint64 (log2 N, l, 2, N)."""
    sk = np.asarray(sk, dtype=np.int64)
    N = sk.shape[-1]
    steps = int(np.log2(N))
    gj = np.array([1 << (64 - j * log2_beta) for j in range(1, l + 1)], dtype=np.uint64)
    out = np.empty((steps, l, 2, N), dtype=np.uint64)
    for i in range(steps):
        s_auto = u64(automorphism(sk, 2 ** (steps - i) + 1))
        mask, body = encrypt_rlwe(np.uint64(0) - gj[:, None] * s_auto[None, :], sk, sigma, rng)
        out[i, :, 0], out[i, :, 1] = mask, body
    return out


def packing_key(sk_lwe, sk_rlwe, log2_beta: int, l: int, sigma: float, rng) -> np.ndarray:
    """Packing key (get_packing_KSK, schemas/RLWE_jax.py:205-215) on Z/2^64:
    RLWE_{sk_rlwe}(s_i q / beta^j) as constant polynomials.  Returns uint64
    (n_dim, l, 2, N)."""
    sk_lwe = np.asarray(sk_lwe, dtype=np.int64)
    N = np.asarray(sk_rlwe).shape[-1]
    gj = np.array([1 << (64 - j * log2_beta) for j in range(1, l + 1)], dtype=np.uint64)
    msg = np.zeros((sk_lwe.shape[0], l, N), dtype=np.uint64)
    msg[:, :, 0] = u64(sk_lwe)[:, None] * gj[None, :]
    mask, body = encrypt_rlwe(msg, sk_rlwe, sigma, rng)
    return np.stack([mask, body], axis=2)
