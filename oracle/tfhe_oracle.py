"""CPU oracle for the TFHE programmable-bootstrapping (PBS) path.

TEST INFRASTRUCTURE ONLY.  Nothing in the product imports this module: only
``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl
reference`` legs of ``bench.py`` may use it, and only as the checker or as the
timed CPU restatement of the reference.

What it is
----------
A numpy restatement of the reference's JAX implementation of the PBS path
(AMIAD-Research/Blind-Spiking-LSTM).  Every function names the reference
``file:line`` it follows.  Integers are carried the way the reference carries
them: float64 values centred in [-q/2, q/2] (``centered_mod``), with
``round``/``rint`` meaning round-half-to-even.  With q = 2^32 every integer
stage (decomposition, key switching, modulus switching, rotations, sample
extraction) is exact in float64, so those stages are bit-exact statements of
the reference.  The FFT-based external product is restated with numpy's
pocketfft in place of XLA's FFT; its rounding is pinned separately against an
exact integer negacyclic product (``multiply_seq_monomial_exact``).

How it is pinned
----------------
``tests/golden/make_golden.py`` imports the reference's own Python modules
(``schemas/polynomial_jax.py``, ``schemas/text_jax.py``, ``schemas/LWE_jax.py``)
under a numpy-backed stand-in for the absent ``jax`` package and records their
outputs on seeded inputs as fixtures (``tests/golden/*.npz``).
``tests/test_oracle_golden.py`` checks this module against those fixtures
(bit-exact on the integer stages), and checks the FP64 blind rotation against
the exact integer product.  The reference's only correctness script
(``test_collapse.py:184-191,227-234``) accepts a PBS when the mean decrypted
error is <= 0.5; the tests here require every decrypted message to match.

Keys are generated with numpy's PCG64 from one seed, following the structure
of the reference's key generation (``schemas/RLWE_jax.py:162-197``,
``schemas/LWE_jax.py:86-93``, ``nn_tfhe/activation.py:49-53``).  Keys are
inputs to every path, so the random stream need not match JAX's.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# --------------------------------------------------------------------------
# float64 restatements of schemas/polynomial_jax.py
# --------------------------------------------------------------------------


def centered_mod(x, q):
    """schemas/polynomial_jax.py:7-9  x - q * rint(x / q)  (float64)."""
    x = np.asarray(x, dtype=np.float64)
    return x - q * np.rint(x / q)


def jax_fourier(p):
    """schemas/polynomial_jax.py:11-15: N-point FFT of the twisted polynomial,
    first N/2 outputs = evaluations at exp(-i*pi*(2j+1)/N)."""
    p = np.asarray(p)
    degree = p.shape[-1]
    q_large = np.fft.fft(np.exp(-1j * np.pi * np.arange(degree) / degree) * p, axis=-1)
    return q_large[..., : degree // 2]


def jax_inversefourier(q):
    """schemas/polynomial_jax.py:17-21: Hermitian extension, inverse FFT,
    untwist, real part, round-half-even."""
    q = np.asarray(q)
    q_large = np.concatenate([q, np.flip(np.conj(q), axis=-1)], axis=-1)
    n = 2 * q.shape[-1]
    return np.round(np.real(np.exp(1j * np.pi * np.arange(n) / n) * np.fft.ifft(q_large, axis=-1)))


def decomposition(gamma, beta, l, q):
    """schemas/polynomial_jax.py:90-111: signed gadget digits, most
    significant first, stacked on a new leading axis of length l."""
    x = np.asarray(gamma, dtype=np.float64) / q
    digits = []
    for _ in range(l):
        x_beta = x * beta
        digit = np.round(x_beta)
        x = x_beta - digit
        digits.append(digit)
    return np.stack(digits)


def GLEV_polynomial(x, beta, l, q):
    """schemas/polynomial_jax.py:115-134: x * q/beta^i for i = 1..l."""
    basis = np.array([q / (beta ** i) for i in range(1, l + 1)])[:, None]
    return np.asarray(x, dtype=np.float64) * basis


def coef_rotation(polynomial, alpha):
    """schemas/polynomial_jax.py:150-169: multiply by X^alpha in
    Z[X]/(X^N+1) (roll, sign flip of the wrapped part).  One alpha."""
    polynomial = np.asarray(polynomial, dtype=np.float64)
    n = polynomial.shape[-1]
    alpha = int(alpha)
    rotation = np.roll(polynomial, alpha, axis=-1)
    degree_shift_div = alpha // n
    degree_shift_mod = alpha % n
    rotation = rotation * ((-1.0) ** degree_shift_div)
    mask = (np.arange(n) < degree_shift_mod).astype(np.float64)
    return mask * (-rotation) + (1 - mask) * rotation


def coef_rotation_rows(polys, alphas):
    """Row-wise ``coef_rotation``: polys (..., R, N), alphas (..., R) ints.
    Same result as calling ``coef_rotation`` per row (checked in tests)."""
    polys = np.asarray(polys, dtype=np.float64)
    n = polys.shape[-1]
    alphas = np.asarray(alphas, dtype=np.int64)
    t = np.arange(n)[None, :] - alphas.reshape(-1, 1)
    wraps = np.floor_divide(t, n)
    src = t - wraps * n
    sign = np.where(wraps % 2 == 0, 1.0, -1.0)
    flat = polys.reshape(-1, n)
    out = np.take_along_axis(flat, src, axis=-1) * sign
    return out.reshape(polys.shape)


# --------------------------------------------------------------------------
# schemas/text_jax.py
# --------------------------------------------------------------------------


def sample_extract(ciphertext, alpha):
    """schemas/text_jax.py:191-208: LWE of coefficient alpha of an RLWE.
    ciphertext = (a, b), each (..., N).  Returns (a' (..., N), b' (..., 1))."""
    public_key, b = np.asarray(ciphertext[0]), np.asarray(ciphertext[1])
    degree = public_key.shape[-1]
    j = np.arange(degree)
    src = np.where(j <= alpha, alpha - j, alpha - j + degree)
    sign = np.where(j <= alpha, 1.0, -1.0)
    extracted = np.take(public_key, src, axis=-1) * sign
    return extracted, b[..., alpha:alpha + 1]


def rotate_ciphertext(ciphertext, exponent):
    """schemas/text_jax.py:348-362 (one exponent)."""
    return coef_rotation(ciphertext[0], exponent), coef_rotation(ciphertext[1], exponent)


def all_binary_vectors(m):
    """schemas/text_jax.py:440-454 and cuTFHE/utils.py:5-8: {0,1}^m in
    meshgrid 'ij' order (first coordinate most significant), shape (2^m, m)."""
    values = np.array([0, 1], dtype=np.int32)
    grids = np.meshgrid(*([values] * m), indexing="ij")
    return np.stack(grids, axis=-1).reshape(-1, m)


def rotation_indices(public_key, collapse, degree, q, n_lut):
    """cuTFHE/multiply.py:67-79 (= schemas/text_jax.py:407-414): per group g
    and pattern p, r[g,p] = (round(2N <a_g,p> / (q n_lut)) n_lut) mod 2N.
    public_key (..., n) float64 -> (..., n/collapse, 2^collapse) int32."""
    public_key = np.asarray(public_key, dtype=np.float64)
    n = public_key.shape[-1]
    n_iter = n // collapse
    kron = all_binary_vectors(collapse)
    pk_reshaped = public_key.reshape(*public_key.shape[:-1], n_iter, collapse)
    vals = pk_reshaped @ kron.T.astype(np.float64)
    idx = (np.round(2 * degree * vals / (q * n_lut)) * n_lut).astype(np.int32)
    return np.mod(idx, 2 * degree).astype(np.int32)


def body_rotation(b, degree, q, n_lut):
    """schemas/RLWE_jax.py:295 / text_jax.py:383: b~ = round(2N b/(q n_lut)) n_lut."""
    return np.round(2 * degree * np.asarray(b, dtype=np.float64) / (q * n_lut)) * n_lut


def bsk_reshape(BSK, n_iter, collapse):
    """cuTFHE/multiply.py:81-86: (2,2,L,G*M,d) -> (G, 2 out, L, 2 in, M, d)."""
    shape = list(BSK.shape)
    shape[3] = n_iter
    shape.insert(4, 2 ** collapse)
    return np.transpose(np.asarray(BSK).reshape(shape), (3, 0, 2, 1, 4, 5))


def multiply_seq_monomial(ct_init, public_key, BSK, q, beta, l, degree, collapse,
                          all_rot_fft, n_lut, trace=None):
    """schemas/text_jax.py:390-435 (== cuTFHE/multiply.py:54-92 semantics),
    vectorised over a batch.

    ct_init (B|1, 2, N) float64, public_key (B, n), BSK as the reference's
    ``bsk_ordered`` (2, 2, L, G*M, d) complex128, all_rot_fft (2N, d).
    Returns ACC (B, 2, N) float64 centred.  ``trace`` (list) receives the ACC
    after each group if given."""
    public_key = np.atleast_2d(np.asarray(public_key, dtype=np.float64))
    B = public_key.shape[0]
    n = public_key.shape[-1]
    n_iter = n // collapse
    idx = rotation_indices(public_key, collapse, degree, q, n_lut)      # (B, G, M)
    bskr = bsk_reshape(BSK, n_iter, collapse)                           # (G,2,L,2,M,d)
    ct = np.broadcast_to(np.asarray(ct_init, dtype=np.float64), (B, 2, degree)).copy()
    M = 2 ** collapse
    for g in range(n_iter):
        dec = np.moveaxis(decomposition(ct, beta, l, q), 0, 1)          # (B, L, 2, N)
        dec_fft = jax_fourier(dec)                                      # (B, L, 2, d)
        rot = all_rot_fft[idx[:, g, :]]                                 # (B, M, d)
        chunk = bskr[g]                                                 # (2, L, 2, M, d)
        sum_rgsw = np.zeros((B,) + chunk.shape[:3] + chunk.shape[-1:], dtype=np.complex128)
        for m in range(M):
            sum_rgsw += chunk[None, :, :, :, m, :] * rot[:, None, None, None, m, :]
        prod = np.einsum("kabcd,kbcd->kad", sum_rgsw, dec_fft)
        ct = centered_mod(jax_inversefourier(prod), q)
        if trace is not None:
            trace.append(ct.copy())
    return ct


def blind_rotate(ciphertext_lwe, LUT, BSK, q, beta, l, degree, collapse, all_rot_fft, n_lut):
    """schemas/text_jax.py:365-387: rotate the LUT by -b~ first, then the
    collapsed CMux chain.  Batched: a (B, n), b (B, 1), LUT (B|1, 2, N)."""
    a, b = ciphertext_lwe
    b_ms = body_rotation(np.asarray(b).reshape(-1), degree, q, n_lut)
    lut = np.broadcast_to(np.asarray(LUT, dtype=np.float64), (b_ms.shape[0], 2, degree))
    ct = coef_rotation_rows(lut, -b_ms.astype(np.int64)[:, None].repeat(2, axis=1))
    return multiply_seq_monomial(ct, a, BSK, q, beta, l, degree, collapse, all_rot_fft, n_lut)


def extract_many(acc, n_lut):
    """schemas/RLWE_jax.py:301-303: sample_extract at alpha = 0..n_lut-1.
    acc (B, 2, N) -> (a (B, n_lut, N), b (B, n_lut, 1))."""
    outs = [sample_extract((acc[:, 0], acc[:, 1]), alpha) for alpha in range(n_lut)]
    return np.stack([o[0] for o in outs], axis=1), np.stack([o[1] for o in outs], axis=1)


def bootstrapping(lwe, LUT, BSK, q, beta, l, degree, collapse, all_rot_fft, n_lut=1):
    """schemas/RLWE_jax.py:233-257 (batched)."""
    acc = blind_rotate(lwe, LUT, BSK, q, beta, l, degree, collapse, all_rot_fft, n_lut)
    if n_lut == 1:
        a, b = sample_extract((acc[:, 0], acc[:, 1]), 0)
        return a, b
    return extract_many(acc, n_lut)


def BR(c_lwe_ks, encrypted_LUT, bsk, q, beta, l, degree, collapse, all_rot, n_lut,
       exact_bsk=None):
    """schemas/RLWE_jax.py:305-315: CMux chain from the LUT, THEN rotate by
    -b~ (the rotation comes after the blind rotation on this path).
    encrypted_LUT = [mask (B|1, N), body (B|1, N)].  With ``exact_bsk`` (the
    coefficient-domain key) the external products are exact integers."""
    pk, b = c_lwe_ks
    pk = np.atleast_2d(np.asarray(pk, dtype=np.float64))
    ct_init = np.stack([np.atleast_2d(encrypted_LUT[0]), np.atleast_2d(encrypted_LUT[1])], axis=1)
    if exact_bsk is None:
        acc = multiply_seq_monomial(ct_init, pk, bsk, q, beta, l, degree, collapse, all_rot, n_lut)
    else:
        acc = multiply_seq_monomial_exact(ct_init, pk, exact_bsk, q, beta, l, degree, collapse, n_lut)
    b_ms = body_rotation(np.asarray(b).reshape(-1), degree, q, n_lut).astype(np.int64)
    return coef_rotation_rows(acc, -b_ms[:, None].repeat(2, axis=1))


def cuboot_merge(c_lwe_ks, encrypted_LUT, bsk, q, beta, l, degree, collapse, all_rot, n_lut,
                 exact_bsk=None):
    """schemas/RLWE_jax.py:288-303: BR then many-LUT sample extraction.
    Returns (a (B, n_lut, N), b (B, n_lut, 1))."""
    acc = BR(c_lwe_ks, encrypted_LUT, bsk, q, beta, l, degree, collapse, all_rot, n_lut,
             exact_bsk=exact_bsk)
    return extract_many(acc, n_lut)


# --------------------------------------------------------------------------
# schemas/LWE_jax.py
# --------------------------------------------------------------------------


def gadget_product_LWE(glev, decomp, q):
    """schemas/LWE_jax.py:65-82 (batched over a leading ciphertext axis of
    ``decomp`` (B, l, n_old)).  Exact: partial sums stay below 2^53."""
    glev_pk, glev_b = np.asarray(glev[0], np.float64), np.asarray(glev[1], np.float64)
    l, n_old, n_new = glev_pk.shape
    d2 = decomp.reshape(decomp.shape[0], l * n_old)
    pk_sum = centered_mod(d2 @ glev_pk.reshape(l * n_old, n_new), q)
    b_sum = centered_mod(d2 @ glev_b.reshape(l * n_old, -1), q)
    return pk_sum, b_sum


def key_switch_LWE(key_switching_key, ciphertext, params):
    """schemas/LWE_jax.py:97-117, vmapped over ciphertexts as in
    nn_tfhe/activation.py:150.  ciphertext = (a (B, n_old), b (B, 1))."""
    beta, l, q = params["beta_ks"], params["l_ks"], params["q"]
    a = np.atleast_2d(np.asarray(ciphertext[0], np.float64))
    b = np.asarray(ciphertext[1], np.float64).reshape(a.shape[0], 1)
    dec = np.moveaxis(decomposition(a, beta, l, q), 0, 1)               # (B, l, n_old)
    pk_sum, b_sum = gadget_product_LWE(key_switching_key, dec, q)
    return centered_mod(pk_sum, q), centered_mod(b + b_sum, q)


def decrypt_LWE(ciphertext, sk, params):
    """schemas/LWE_jax.py:30-48 (batched): cmod_t(round((b - <a,s>)/delta))."""
    t, q = params["t"], params["q"]
    delta = q / t
    a, b = np.asarray(ciphertext[0], np.float64), np.asarray(ciphertext[1], np.float64)
    product = a @ np.asarray(sk, np.float64)
    return centered_mod(np.round((b.reshape(product.shape) - product) / delta), t)


def decrypt_LWE_quantization(ciphertext, sk, params, scale=None):
    """schemas/LWE_jax.py:52-62 (batched)."""
    t, q = params["t"], params["q"]
    if scale is None:
        scale = q / t
    a, b = np.asarray(ciphertext[0], np.float64), np.asarray(ciphertext[1], np.float64)
    product = a @ np.asarray(sk, np.float64)
    return centered_mod(b.reshape(product.shape) - product, q) / scale


def get_noise_lwe(ciphertext, sk, q, message):
    """schemas/noise_estimators.py:7-11: cmod_q(b - <a,s> - m)."""
    a, b = np.asarray(ciphertext[0], np.float64), np.asarray(ciphertext[1], np.float64)
    product = a @ np.asarray(sk, np.float64)
    return centered_mod(b.reshape(product.shape) - product - message, q)


# --------------------------------------------------------------------------
# nn_tfhe/utils_spike.py, parameters_crypto.py
# --------------------------------------------------------------------------


def get_plain_LUT(degree_lut, n_lut, index, s, gamma):
    """nn_tfhe/utils_spike.py:72-87: many-LUT step table, sub-LUT ``index``
    on positions base*n_lut + index, then rotated by -N/2."""
    sub_degree = degree_lut // n_lut
    part_lut = np.linspace(-s, s, num=sub_degree, endpoint=False)
    values = np.where(part_lut >= gamma, 1.0, 0.0)
    complete = np.zeros(degree_lut)
    complete[np.arange(sub_degree) * n_lut + index] = values
    return coef_rotation(complete, -degree_lut // 2)


def all_rot_possible_fourier(degree):
    """parameters_crypto.py:86-91: row r = jax_fourier(X^r), r in [0, 2N)."""
    rows = np.zeros((2 * degree, degree))
    rows[:, 0] = 1.0
    idx = np.arange(-degree, degree)
    rows = np.stack([coef_rotation(rows[i], idx[i]) for i in range(2 * degree)])
    rows = np.roll(rows, -degree, axis=0)
    return jax_fourier(rows)


# --------------------------------------------------------------------------
# exact integer arithmetic (the pin for the FFT products)
# --------------------------------------------------------------------------

_LIMB_BITS = 11


def _limbs(x):
    """Split int64 values |x| <= 2^33 into 4 signed limbs of 11 bits (last one
    carries the rest): x = sum_t limb_t 2^(11 t)."""
    x = np.asarray(x, dtype=np.int64)
    out = []
    rest = x.copy()
    for _ in range(3):
        lo = ((rest + (1 << (_LIMB_BITS - 1))) & ((1 << _LIMB_BITS) - 1)) - (1 << (_LIMB_BITS - 1))
        out.append(lo)
        rest = (rest - lo) >> _LIMB_BITS
    out.append(rest)
    return out


def _round_checked(x, what):
    r = np.rint(x)
    err = float(np.max(np.abs(x - r))) if x.size else 0.0
    if err > 1e-2:
        raise ArithmeticError(f"{what}: FFT limb product not integral (max dist {err})")
    return r.astype(np.int64)


def negacyclic_mul_schoolbook(a, b):
    """Exact product in Z[X]/(X^N+1) by the O(N^2) schoolbook with Python
    integers (small N only): the definition every faster route is checked
    against."""
    a = [int(v) for v in np.asarray(a).reshape(-1)]
    b = [int(v) for v in np.asarray(b).reshape(-1)]
    n = len(a)
    out = [0] * n
    for i, ai in enumerate(a):
        if ai == 0:
            continue
        for j, bj in enumerate(b):
            k = i + j
            if k < n:
                out[k] += ai * bj
            else:
                out[k - n] -= ai * bj
    return out


def negacyclic_mul_exact(a, b):
    """Exact negacyclic product of integer polynomials (last axis, broadcast)
    returned modulo 2^64 as int64.  ``b`` is split into 11-bit limbs so each
    FFT product stays below 2^45 and rounds to the exact integer; the
    rounding distance is checked."""
    a = np.asarray(a, dtype=np.int64)
    fa = jax_fourier(a.astype(np.float64))
    total = None
    for t, limb in enumerate(_limbs(b)):
        prod = jax_fourier(limb.astype(np.float64)) * fa
        part = _round_checked(_inverse_unrounded(prod), "negacyclic_mul_exact")
        part = part.astype(np.uint64) << np.uint64(_LIMB_BITS * t)
        total = part if total is None else total + part
    return total.astype(np.int64)


def _inverse_unrounded(q):
    q_large = np.concatenate([q, np.flip(np.conj(q), axis=-1)], axis=-1)
    n = 2 * q.shape[-1]
    return np.real(np.exp(1j * np.pi * np.arange(n) / n) * np.fft.ifft(q_large, axis=-1))


def centered_from_wide(x64, log2_q):
    """Reduce exact integers (given modulo 2^64, int64) the way
    ``centered_mod`` reduces the exact value: result in [-q/2, q/2], with
    q/2 kept positive when floor(x/q) is even and negative when odd
    (rint ties to even).  Needs log2_q <= 62."""
    u = np.asarray(x64).astype(np.uint64)
    q = np.uint64(1) << np.uint64(log2_q)
    half = q >> np.uint64(1)
    r = u & (q - np.uint64(1))
    k_odd = (u >> np.uint64(log2_q)) & np.uint64(1)
    res = r.astype(np.int64)
    res = np.where(r > half, res - np.int64(q), res)
    res = np.where((r == half) & (k_odd == 1), -np.int64(half), res)
    return res.astype(np.float64)


def multiply_seq_monomial_exact(ct_init, public_key, bsk_coeff, q, beta, l, degree, collapse,
                                n_lut, trace=None, fft_trace=None):
    """The collapsed CMux chain of ``multiply_seq_monomial`` with every
    external product computed exactly in integers (then reduced with the
    reference's centred-mod convention).  ``bsk_coeff`` is the
    coefficient-domain key as produced by ``KeySet`` (2 in, 2 out, G*M, L, N).

    The FFT route of ``multiply_seq_monomial`` equals this one bit for bit
    whenever its FFT error stays below 1/2; ``fft_trace`` (list) receives, per
    group, the max |FP64 product - exact product| measured on the same ACC."""
    public_key = np.atleast_2d(np.asarray(public_key, dtype=np.float64))
    B = public_key.shape[0]
    n = public_key.shape[-1]
    n_iter = n // collapse
    M = 2 ** collapse
    log2_q = int(round(math.log2(q)))
    idx = rotation_indices(public_key, collapse, degree, q, n_lut)
    key = bsk_coeff_grouped(bsk_coeff, n_iter, collapse)              # (G,2,L,2,M,N) int64
    key_limbs_f = [jax_fourier(limb.astype(np.float64)) for limb in _limbs(key) if np.any(limb)]
    ct = np.broadcast_to(np.asarray(ct_init, dtype=np.float64), (B, 2, degree)).copy()
    # X^r evaluated at exp(-i pi (2j+1)/N): the rows of parameters_crypto.py:86-91
    ang = np.exp(-1j * np.pi * np.outer(np.arange(2 * degree), 2 * np.arange(degree // 2) + 1) / degree)
    if fft_trace is not None:
        bskr_fft = bsk_reshape(bsk_coeff_fourier_ordered(bsk_coeff), n_iter, collapse)
        all_rot = all_rot_possible_fourier(degree)
    for g in range(n_iter):
        dec = np.moveaxis(decomposition(ct, beta, l, q), 0, 1)       # (B, L, 2, N)
        dec_f = jax_fourier(dec)
        rot = ang[idx[:, g, :]]                                       # (B, M, d)
        total = np.zeros((B, 2, degree), dtype=np.uint64)
        for t, kf in enumerate(key_limbs_f):
            s = np.zeros((B, 2, l, 2, degree // 2), dtype=np.complex128)
            for m in range(M):
                s += kf[g][None, :, :, :, m, :] * rot[:, None, None, None, m, :]
            prod = np.einsum("kabcd,kbcd->kad", s, dec_f)
            part = _round_checked(_inverse_unrounded(prod), "exact external product")
            total += part.astype(np.uint64) << np.uint64(_LIMB_BITS * t)
        wide = total.astype(np.int64)
        exact = centered_from_wide(wide, log2_q)
        if fft_trace is not None:
            # the FP64 route of multiply_seq_monomial on the same ACC
            r = all_rot[idx[:, g, :]]
            s = np.zeros((B, 2, l, 2, degree // 2), dtype=np.complex128)
            for m in range(M):
                s += bskr_fft[g][None, :, :, :, m, :] * r[:, None, None, None, m, :]
            approx = _inverse_unrounded(np.einsum("kabcd,kbcd->kad", s, dec_f))
            fft_trace.append(float(np.max(np.abs(approx - wide.astype(np.float64)))))
        ct = exact
        if trace is not None:
            trace.append(ct.copy())
    return ct


# --------------------------------------------------------------------------
# key generation (structure of the reference; own RNG)
# --------------------------------------------------------------------------


def _randint_torus(rng, shape, q):
    """jax.random.randint(key, shape, -q/2, q/2) * 1. (uniform in [-q/2, q/2))."""
    half = int(q) // 2
    return rng.integers(-half, half, size=shape, dtype=np.int64).astype(np.float64)


def negacyclic_mul_float(a, b):
    """round(fft_polynomial_multiply(a, b)) (schemas/polynomial_jax.py:27-43)
    computed exactly: the reference rounds an FP64 FFT product that is exact
    for its key sizes; here the exact integer product is used directly."""
    return negacyclic_mul_exact(np.asarray(a, np.float64).astype(np.int64),
                                np.asarray(b, np.float64).astype(np.int64)).astype(np.float64)


def encrypt_rlwe(m, sk, q, sigma, rng):
    """schemas/RLWE_jax.py:36-54 (batched over leading axes of m)."""
    m = np.asarray(m, dtype=np.float64)
    degree = m.shape[-1]
    public_key = _randint_torus(rng, m.shape, q)
    e = np.round(rng.standard_normal(m.shape) * sigma)
    product = negacyclic_mul_float(public_key, np.broadcast_to(sk, m.shape))
    b = centered_mod(product + m + e, q)
    return public_key, b


def encrypt_lwe(m, sk, q, sigma, rng):
    """schemas/LWE_jax.py:9-28 (batched over m): the noise is
    round(N(0,1)) * sigma, as in the reference."""
    m = np.asarray(m, dtype=np.float64)
    n = np.asarray(sk).shape[-1]
    public_key = _randint_torus(rng, m.shape + (n,), q)
    e = np.round(rng.standard_normal(m.shape)) * sigma
    product = public_key @ np.asarray(sk, np.float64)
    b = centered_mod(product + m + e, q)
    return public_key, b[..., None]


def get_keyswitch_sk_LWE(new_sk, old_sk, q, beta, l, sigma, rng):
    """schemas/LWE_jax.py:86-93: encryptions of -old_sk * q/beta^j under
    new_sk.  Returns (pk (l, n_old, n_new), b (l, n_old, 1))."""
    glev_old_sk = GLEV_polynomial(old_sk, beta, l, q)                # (l, n_old)
    return encrypt_lwe(-glev_old_sk, new_sk, q, sigma, rng)


def get_boostrapping_key_collapse(sk_poly, sk_lwe, q, beta, l, sigma, collapse, rng):
    """schemas/RLWE_jax.py:162-197: for group g and pattern p, e = [s_g == p];
    'left' rows GLEV(-e * s_glwe), 'right' rows GLEV(e at coefficient 0).
    Returns the coefficient-domain key (2 left/right, 2 pk/b, G*M, L, N)."""
    kron = all_binary_vectors(collapse)
    compare = np.reshape(sk_lwe, (-1, collapse))
    all_eq = np.all(compare[:, None, :] == kron[None, :, :], axis=-1).astype(np.float64).reshape(-1)
    degree = sk_poly.shape[-1]
    left_msg = all_eq[:, None] * (-np.asarray(sk_poly, np.float64))[None, :]      # (GM, N)
    left_glev = centered_mod(np.stack([GLEV_polynomial(r, beta, l, q) for r in left_msg]), q)
    right_poly = np.zeros((all_eq.shape[0], degree))
    right_poly[:, 0] = all_eq
    right_glev = centered_mod(np.stack([GLEV_polynomial(r, beta, l, q) for r in right_poly]), q)
    left = encrypt_rlwe(left_glev, sk_poly, q, sigma, rng)
    right = encrypt_rlwe(right_glev, sk_poly, q, sigma, rng)
    return np.array([[left[0], left[1]], [right[0], right[1]]])


def bsk_coeff_fourier_ordered(bsk_coeff):
    """nn_tfhe/activation.py:49-53: jax_fourier then permute [1,0,3,2,4]
    -> ``bsk_ordered`` (2 pk/b, 2 left/right, L, G*M, d)."""
    return np.transpose(jax_fourier(np.asarray(bsk_coeff, np.float64)), (1, 0, 3, 2, 4))


def bsk_coeff_grouped(bsk_coeff, n_iter, collapse):
    """Coefficient-domain key in the kernel's group order (G, 2 out, L, 2 in,
    M, N) int64: the permutation of activation.py:53 then multiply.py:81-86."""
    ordered = np.transpose(np.asarray(bsk_coeff), (1, 0, 3, 2, 4))
    return bsk_reshape(ordered, n_iter, collapse).astype(np.int64)


@dataclass
class KeySet:
    """Secret and public key material for one parameter set."""
    params: dict
    sk_glwe: np.ndarray          # (N,) binary, also the big LWE key (sk_lut = sk)
    sk_lwe: np.ndarray           # (n,) binary
    ksk: tuple                   # (pk (l_ks, N, n), b (l_ks, N, 1)) float64 centred
    bsk_coeff: np.ndarray        # (2, 2, G*M, L, N) float64 centred
    bsk_ordered: np.ndarray = field(default=None)   # (2, 2, L, G*M, d) complex128
    all_rot: np.ndarray = field(default=None)       # (2N, d) complex128


def keygen(params, seed):
    """Keys for ``params`` (dict with q, N, n, beta_bs, l_bs, collapse,
    beta_ks, l_ks, sigma_glwe, sigma_lwe) from one seed."""
    rng = np.random.default_rng(seed)
    N, n, q = params["N"], params["n"], params["q"]
    sk_glwe = rng.integers(0, 2, size=N).astype(np.float64)
    sk_lwe = rng.integers(0, 2, size=n).astype(np.float64)
    ksk = get_keyswitch_sk_LWE(sk_lwe, sk_glwe, q, params["beta_ks"], params["l_ks"],
                               params["sigma_lwe"], rng)
    bsk = get_boostrapping_key_collapse(sk_glwe, sk_lwe, q, params["beta_bs"], params["l_bs"],
                                        params["sigma_glwe"], params["collapse"], rng)
    ks = KeySet(params=params, sk_glwe=sk_glwe, sk_lwe=sk_lwe, ksk=ksk, bsk_coeff=bsk)
    ks.bsk_ordered = bsk_coeff_fourier_ordered(bsk)
    ks.all_rot = all_rot_possible_fourier(N)
    return ks


def encrypt_inputs(keys, messages, delta, rng):
    """Input LWEs under the GLWE key as in test_collapse.py:111-122: RLWE
    encryption with the message on coefficient 0, then sample_extract(., 0).
    Returns (a (B, N), b (B, 1))."""
    p = keys.params
    B = len(messages)
    polys = np.zeros((B, p["N"]))
    polys[:, 0] = np.asarray(messages, np.float64) * delta
    ct = encrypt_rlwe(polys, keys.sk_glwe, p["q"], p["sigma_glwe"], rng)
    return sample_extract(ct, 0)


def step_lut(N, t_in, threshold, out_scale):
    """Body polynomial of a step LUT for messages m in Z_t_in with a padding
    bit (phase m*q/(2 t_in)): coefficient j holds out_scale * [m(j) >= threshold]
    with m(j) = floor((j + box/2) / box), box = N / t_in; the last half box
    wraps to m = t_in (= -m 0 negacyclically) and holds -out_scale*[0 >= threshold]."""
    box = N // t_in
    j = np.arange(N)
    m = (j + box // 2) // box
    val = (m >= threshold).astype(np.float64) * out_scale
    wrap = m >= t_in
    val[wrap] = -out_scale * float(0 >= threshold)
    return val


# --------------------------------------------------------------------------
# the reference's own torus, q = 2^64 (parameters_crypto.py:6-32)
# --------------------------------------------------------------------------
# At q = 2^64 the reference holds torus values as float64 (53-bit), so its
# arithmetic is no longer exact.  Keys and inputs are made here exactly on
# Z/2^64 (uint64 wrapping) and then handed over as the reference's centred
# float64 values; the float64 functions above then run unchanged at this q.

REF64 = dict(q=2.0 ** 64, N=2048, n=702, beta_bs=2 ** 13, l_bs=2, collapse=3, sigma_glwe=2.0 ** 17)


def negacyclic_mul_binary_q64(a_u64, s):
    """a (..., N) uint64 times a binary polynomial s (N,) in Z/2^64[X]/(X^N+1),
    exactly: a is split into four 16-bit limbs whose products with s
    (|.| < 2^27) are exact integers, recombined with uint64 wrap-around."""
    a = np.asarray(a_u64, dtype=np.uint64)
    s64 = np.broadcast_to(np.asarray(s, dtype=np.int64), a.shape)
    out = np.zeros(a.shape, dtype=np.uint64)
    for t in range(4):
        limb = ((a >> np.uint64(16 * t)) & np.uint64(0xFFFF)).astype(np.int64)
        prod = negacyclic_mul_exact(limb, s64)
        out += prod.astype(np.uint64) << np.uint64(16 * t)
    return out


def u64_to_centred(u):
    """uint64 torus words -> the reference's float64 values in [-q/2, q/2]."""
    return np.asarray(u, dtype=np.uint64).view(np.int64).astype(np.float64)


def keygen_q64(params, seed):
    """Collapsed bootstrapping key at q = 2^64 with the structure of
    get_boostrapping_key_collapse (schemas/RLWE_jax.py:162-197): returns
    (sk_glwe (N,), sk_lwe (n,), bsk_coeff (2, 2, G*M, L, N) float64 centred).
    GLEV rows carry e * q / beta^j (left: times -s_glwe), encrypted with
    Gaussian noise of std sigma_glwe."""
    rng = np.random.default_rng(seed)
    N, n, L, c = params["N"], params["n"], params["l_bs"], params["collapse"]
    log2_beta = int(round(math.log2(params["beta_bs"])))
    sk_glwe = rng.integers(0, 2, size=N).astype(np.int64)
    sk_lwe = rng.integers(0, 2, size=n).astype(np.int64)
    kron = all_binary_vectors(c)
    eq = np.all(sk_lwe.reshape(-1, c)[:, None, :] == kron[None, :, :], axis=-1).reshape(-1).astype(np.uint64)
    gj = np.array([1 << (64 - j * log2_beta) for j in range(1, L + 1)], dtype=np.uint64)
    GM = eq.shape[0]
    left = (np.uint64(0) - eq[:, None, None] * gj[None, :, None]) * sk_glwe.astype(np.uint64)[None, None, :]
    right = np.zeros((GM, L, N), dtype=np.uint64)
    right[:, :, 0] = eq[:, None] * gj[None, :]
    bsk = np.empty((2, 2, GM, L, N), dtype=np.float64)
    for side, msg in enumerate((left, right)):
        mask = rng.integers(0, 2 ** 64, size=msg.shape, dtype=np.uint64)
        e = np.rint(rng.standard_normal(msg.shape) * params["sigma_glwe"]).astype(np.int64).astype(np.uint64)
        body = negacyclic_mul_binary_q64(mask, sk_glwe) + msg + e
        bsk[side, 0], bsk[side, 1] = u64_to_centred(mask), u64_to_centred(body)
    return sk_glwe, sk_lwe, bsk


def encrypt_lwe_q64(messages_u64, sk, sigma, rng):
    """LWE encryptions on Z/2^64 of uint64 messages under a binary key:
    (a (B, n), b (B,)) as centred float64 (the reference's representation)."""
    m = np.asarray(messages_u64, dtype=np.uint64)
    a = rng.integers(0, 2 ** 64, size=m.shape + (len(sk),), dtype=np.uint64)
    dot = (a * np.asarray(sk, dtype=np.uint64)).sum(axis=-1, dtype=np.uint64)
    e = np.rint(rng.standard_normal(m.shape) * sigma).astype(np.int64).astype(np.uint64)
    return u64_to_centred(a), u64_to_centred(dot + m + e)


def phase_q64(a, b, sk):
    """b - <a, s> of float64-held LWEs at q = 2^64, exactly on Z/2^64 after
    reading the float64 values as integers: centred int64."""
    au = np.asarray(a, dtype=np.float64)
    bu = np.asarray(b, dtype=np.float64).reshape(au.shape[:-1])
    to_u = lambda x: np.where(x >= 2.0 ** 63, x - 2.0 ** 64, x).astype(np.int64).astype(np.uint64)
    dot = (to_u(au) * np.asarray(sk, dtype=np.uint64)).sum(axis=-1, dtype=np.uint64)
    return (to_u(bu) - dot).view(np.int64)
