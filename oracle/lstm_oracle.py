"""CPU statement of the encrypted Spike-LSTM timestep (test infrastructure).

ORACLE: used only by tests/ as the checker of the engine's timestep
operators; nothing in the product imports it.

Integers are exact.  Every product of an integer plaintext with a
ciphertext is the exact negacyclic product reduced modulo q = 2^32; the
reference computes it with FP64 FFTs and rounds, which is exact at these
sizes (products stay far below 2^53).  Where the reference keeps values
unreduced (the running sum of pack_lwe_to_rlwe) they stay unreduced here,
because the next gadget decomposition sees the unreduced value.

Functions follow, in order:
  weights_to_polynomial          schemas/polynomial_jax.py:136-148
  linear_kernel_polynomial       nn_tfhe/Spike_LSTM.py:28-41 (set_weights)
  linear                         nn_tfhe/Spike_LSTM.py:48-58 (__call__)
  apply_automorphism             schemas/polynomial_jax.py:171-200
  pack_lwe_to_rlwe               schemas/text_jax.py:173-187, 242-345
  multiply_plaintext_ciphertext  schemas/text_jax.py:58-79
  packing                        schemas/text_jax.py:211-239
  get_plain_LUT                  nn_tfhe/utils_spike.py:72-87
  spike_lstm_step                nn_tfhe/Spike_LSTM.py:103-184 (scan_step)
"""
from __future__ import annotations

import numpy as np

from oracle import tfhe_oracle as O

Q = 2.0 ** 32
LOG2_Q = 32


def cmod_exact(x64):
    """centered_mod of exact integers given modulo 2^64 (int64), with the
    reference's tie rule (rint ties to even)."""
    return O.centered_from_wide(np.asarray(x64, dtype=np.int64), LOG2_Q).astype(np.int64)


def u32(x):
    return (np.asarray(x, dtype=np.int64) & 0xFFFFFFFF).astype(np.uint32)


def negacyclic(p, c):
    """Exact negacyclic product of integer polynomials modulo 2^64 (int64);
    p (..., N) and c (..., N) broadcast."""
    p = np.asarray(p, dtype=np.int64)
    c = np.asarray(c, dtype=np.int64)
    if p.ndim < c.ndim:
        p = np.broadcast_to(p, c.shape)
    if c.ndim < p.ndim:
        c = np.broadcast_to(c, p.shape)
    return O.negacyclic_mul_exact(p, c)


# ---------------------------------------------------------------- linear
def weights_to_polynomial(weights):
    """schemas/polynomial_jax.py:136-148: -flip(w), last coefficient w[0]."""
    w = np.asarray(weights, dtype=np.float64).reshape(-1)
    poly = -np.flip(w)
    poly[-1] = w[0]
    return poly


def linear_kernel_polynomial(W, B, factor, degree):
    """Linear.set_weights (nn_tfhe/Spike_LSTM.py:28-41): W (in, out),
    factor (out,) -> kernel polynomials (out, degree) int64 and bias (out,)."""
    W = np.asarray(W, dtype=np.float64)
    factor = np.asarray(factor, dtype=np.float64)
    wt = W.T
    wp = np.stack([weights_to_polynomial(r) for r in np.round(factor[:, None] * wt)])
    kern = np.zeros((wt.shape[0], degree))
    kern[:, -wt.shape[1] + 1:] = wp[:, :-1]
    kern[:, 0] = wp[:, -1]
    bias = np.round(factor * np.asarray(B, dtype=np.float64))
    return kern.astype(np.int64), bias.astype(np.int64)


def linear(kern, bias, rlwe):
    """Linear.__call__ (nn_tfhe/Spike_LSTM.py:48-58) on one RLWE (a, b)
    (N,) each: W_j * rlwe, sample_extract at 0, + bias_j, centred mod.
    Returns (a (J, N), b (J,)) centred int64."""
    a, b = (np.asarray(v, dtype=np.int64) for v in rlwe)
    pa = negacyclic(kern, a[None])
    pb = negacyclic(kern, b[None])
    N = a.shape[-1]
    ext = np.empty_like(pa)
    ext[:, 0] = pa[:, 0]
    ext[:, 1:] = -pa[:, N - np.arange(1, N)]
    return cmod_exact(ext), cmod_exact(pb[:, 0] + bias)


# ---------------------------------------------------------------- trace
def apply_automorphism(poly, k):
    """schemas/polynomial_jax.py:171-200: X -> X^k on the last axis."""
    poly = np.asarray(poly)
    N = poly.shape[-1]
    idx = (np.arange(N) * k) % (2 * N)
    out = np.zeros_like(poly)
    out[..., idx % N] = np.where(idx >= N, -poly, poly)
    return out


def pack_lwe_to_rlwe(lwe_a, lwe_b, galois, log2_beta, l):
    """pack_lwe_to_rlwe (schemas/text_jax.py:316-345) for LWEs a (R, N),
    b (R,): modulus_switch to q/N (:173-187), trivial_embedding
    (:242-263), then log2 N steps of apply_automorphism_and_keyswitch
    (:265-292) with sums left unreduced.  galois (steps, l, 2, N) integers
    (coefficient domain).  Returns (A, B) (R, N) int64, unreduced."""
    a = np.asarray(lwe_a, dtype=np.float64)
    b = np.asarray(lwe_b, dtype=np.float64).reshape(-1)
    R, N = a.shape
    steps = int(round(np.log2(N)))
    beta = 2.0 ** log2_beta
    a = np.rint(a * (Q / N) / Q)
    b = np.rint(b * (Q / N) / Q)
    A = np.zeros((R, N))
    A[:, 0] = a[:, 0]
    A[:, 1:] = -np.flip(a[:, 1:], axis=-1)
    B = np.zeros((R, N))
    B[:, 0] = b
    galois = np.asarray(galois, dtype=np.int64)
    for i in range(steps):
        k = 2 ** (steps - i) + 1
        Ap = apply_automorphism(A, k)
        Bp = apply_automorphism(B, k)
        dec = np.moveaxis(O.decomposition(Ap, beta, l, Q), 0, 1).astype(np.int64)   # (R, l, N)
        ks_a = np.zeros((R, N), dtype=np.int64)
        ks_b = np.zeros((R, N), dtype=np.int64)
        for j in range(l):
            ks_a = ks_a + negacyclic(dec[:, j], galois[i, j, 0][None])
            ks_b = ks_b + negacyclic(dec[:, j], galois[i, j, 1][None])
        auto_a = cmod_exact(ks_a).astype(np.float64)
        auto_b = cmod_exact(Bp.astype(np.int64) + ks_b).astype(np.float64)
        A = A + auto_a
        B = B + auto_b
    return A.astype(np.int64), B.astype(np.int64)


def multiply_plaintext_ciphertext(p, rlwe):
    """schemas/text_jax.py:58-79 (fft_product_twice, exact): p (..., N)
    times (a, b) -> (p a, p b) modulo 2^64 as int64."""
    a, b = rlwe
    return negacyclic(p, a), negacyclic(p, b)


def packing(lwe_a, lwe_b, ksp_a, ksp_b, log2_beta, l, degree):
    """packing (schemas/text_jax.py:211-239): LWEs a (T, n_dim), b (T,)
    into one RLWE of degree N with the packing key ksp_a / ksp_b
    (n_dim, l, N).  Returns (a, b) (N,) centred int64."""
    lwe_a = np.asarray(lwe_a, dtype=np.float64)
    T, n_dim = lwe_a.shape
    packed_b = np.zeros(degree, dtype=np.int64)
    packed_b[:T] = np.asarray(lwe_b, dtype=np.int64).reshape(-1)
    rows = np.zeros((n_dim, degree))
    rows[:, :T] = lwe_a.T
    dec = np.moveaxis(O.decomposition(rows, 2.0 ** log2_beta, l, Q), 0, 1).astype(np.int64)   # (n_dim, l, N)
    sa = negacyclic(dec, np.asarray(ksp_a, dtype=np.int64)).sum(axis=(0, 1))
    sb = negacyclic(dec, np.asarray(ksp_b, dtype=np.int64)).sum(axis=(0, 1))
    return cmod_exact(-sa), cmod_exact(packed_b - sb)


def sample_extract_many(rlwe, count):
    """sample_extract (schemas/text_jax.py:191-208) at alpha = 0..count-1."""
    a, b = (np.asarray(v, dtype=np.int64) for v in rlwe)
    N = a.shape[-1]
    out_a = np.empty((count, N), dtype=np.int64)
    j = np.arange(N)
    for al in range(count):
        src = np.where(j <= al, al - j, al - j + N)
        sign = np.where(j <= al, 1, -1)
        out_a[al] = a[src] * sign
    return out_a, b[:count].copy()


def rotate(rlwe, alpha):
    """rotate_ciphertext (schemas/text_jax.py:348-362)."""
    return tuple(np.rint(O.coef_rotation(np.asarray(v, dtype=np.float64), alpha)).astype(np.int64) for v in rlwe)


# ---------------------------------------------------------------- LUTs
def get_plain_LUT(degree_lut, n_lut, index, s, gamma):
    """nn_tfhe/utils_spike.py:72-87: sub-LUT `index` of a packed step LUT
    over linspace(-s, s, N/n_lut), value [x >= gamma], rotated by -N/2."""
    sub = degree_lut // n_lut
    part = np.linspace(-s, s, num=sub, endpoint=False)
    values = np.where(part >= gamma, 1.0, 0.0)
    full = np.zeros(degree_lut)
    full[np.arange(sub) * n_lut + index] = values
    return O.coef_rotation(full, -degree_lut // 2)


# ---------------------------------------------------------------- timestep
def cuboot(keys, p, lwe_a, lwe_b, luts_a, luts_b, n_lut):
    """HeavysideBoostrapper.cuboot (nn_tfhe/activation.py:148-162) with the
    FP64 oracle: key switch, cuboot_merge.  Returns (a (B, n_lut, N),
    b (B, n_lut)) centred int64."""
    ka, kb = O.key_switch_LWE(keys.ksk, (np.asarray(lwe_a, np.float64), np.asarray(lwe_b, np.float64)[:, None]),
                              {"beta_ks": p["beta_ks"], "l_ks": p["l_ks"], "q": p["q"]})
    oa, ob = O.cuboot_merge((ka, kb), [np.asarray(luts_a, np.float64), np.asarray(luts_b, np.float64)],
                            keys.bsk_ordered, p["q"], p["beta_bs"], p["l_bs"], p["N"], p["collapse"], keys.all_rot,
                            n_lut)
    return np.rint(oa).astype(np.int64), np.rint(np.asarray(ob)).astype(np.int64).reshape(len(lwe_b), n_lut)


def spike_lstm_step(keys, p, layer, x_t, H, C):
    """scan_step of CipherSpikeLSTM (nn_tfhe/Spike_LSTM.py:103-176) for one
    sequence.  layer: dict with kern_f/i/o, bias_f/i/o, lut_f, lut_o
    (n_lut, H/n_lut, N) ints, lut_i (H/n_lut, N) ints, galois, ksp_a,
    ksp_b, gal_log2_beta, gal_l, pk_log2_beta, pk_l, input_dim, hidden,
    n_lut.  x_t, H, C: RLWEs (a, b) (N,) centred int64.  Returns (H_t, C_t)."""
    hidden, n_lut, N = layer["hidden"], layer["n_lut"], p["N"]
    per = hidden // n_lut
    c_a, c_b = sample_extract_many(C, hidden)
    hx = (cmod_exact(x_t[0] + H[0]), cmod_exact(x_t[1] + H[1]))
    F = linear(layer["kern_f"], layer["bias_f"], hx)
    I = linear(layer["kern_i"], layer["bias_i"], hx)
    Ot = linear(layer["kern_o"], layer["bias_o"], hx)

    def prepare(lwe_a, lwe_b, lut):
        ra, rb = pack_lwe_to_rlwe(lwe_a, lwe_b, layer["galois"], layer["gal_log2_beta"], layer["gal_l"])
        pa, pb = multiply_plaintext_ciphertext(np.asarray(lut, np.int64).reshape(hidden, N), (ra, rb))
        pa = pa.reshape(n_lut, per, N).sum(axis=0)
        pb = pb.reshape(n_lut, per, N).sum(axis=0)
        return cmod_exact(pa), cmod_exact(pb)

    lut_c_a, lut_c_b = prepare(c_a, c_b, layer["lut_f"])
    in_a = np.concatenate([F[0], I[0]])
    in_b = np.concatenate([F[1], I[1]])
    luts_a = np.concatenate([lut_c_a, np.zeros((per, N), np.int64)])
    luts_b = np.concatenate([lut_c_b, np.asarray(layer["lut_i"], np.int64)])
    boot_a, boot_b = cuboot(keys, p, in_a, in_b, luts_a, luts_b, n_lut)          # (2 per, n_lut, N)
    spike_i_a = np.transpose(boot_a[per:], (1, 0, 2)).reshape(-1, N)
    spike_i_b = np.transpose(boot_b[per:], (1, 0)).reshape(-1)
    spike_fc_a = np.transpose(boot_a[:per], (1, 0, 2)).reshape(-1, N)
    spike_fc_b = np.transpose(boot_b[:per], (1, 0)).reshape(-1)
    ct_a = cmod_exact(spike_fc_a + spike_i_a)
    ct_b = cmod_exact(spike_fc_b + spike_i_b)
    lut_h_a, lut_h_b = prepare(ct_a, ct_b, layer["lut_o"])
    h_a, h_b = cuboot(keys, p, Ot[0], Ot[1], lut_h_a, lut_h_b, n_lut)
    h_a = np.transpose(h_a, (1, 0, 2)).reshape(-1, N)
    h_b = np.transpose(h_b, (1, 0)).reshape(-1)
    C_t = packing(ct_a, ct_b, layer["ksp_a"], layer["ksp_b"], layer["pk_log2_beta"], layer["pk_l"], N)
    H_t = packing(h_a, h_b, layer["ksp_a"], layer["ksp_b"], layer["pk_log2_beta"], layer["pk_l"], N)
    H_t = rotate(H_t, layer["input_dim"])
    return H_t, C_t


def relu_lut(degree_lut, s, beta_x):
    """ReluBoostrapper's LUT body (nn_tfhe/activation.py:186-194): a ramp
    over the first N/2 coefficients (arange(0, s, 2s/N) * beta_x), zeros
    after, rounded to integers for the uint32 torus."""
    ramp = np.arange(degree_lut // 2) * (2.0 * s / degree_lut) * beta_x
    return np.rint(np.concatenate([ramp, np.zeros(degree_lut // 2)])).astype(np.int64)


def cipher_mlp(keys, p, head, H):
    """CipherMLP.__call__ (nn_tfhe/Spike_LSTM.py:201-206) on one RLWE:
    linear1, ReLU bootstrap per unit with n_lut = 1 (the reference's
    `bootstrapping` rotates the LUT before the blind rotation, which equals
    cuboot_merge's rotation after it in exact arithmetic), packing,
    linear2.  Returns (a (J2, N), b (J2,))."""
    h1_a, h1_b = linear(head["kern1"], head["bias1"], H)
    J, N = h1_a.shape
    luts_a = np.zeros((J, N), np.int64)
    luts_b = np.asarray(head["relu_luts"], np.int64)
    y_a, y_b = cuboot(keys, p, h1_a, h1_b, luts_a, luts_b, 1)
    h2 = packing(y_a[:, 0], y_b[:, 0], head["ksp_a"], head["ksp_b"], head["pk_log2_beta"], head["pk_l"], N)
    return linear(head["kern2"], head["bias2"], h2)
