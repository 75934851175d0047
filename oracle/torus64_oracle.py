"""CPU statement of the engine's operators on the reference's own torus,
q = 2^64 (test infrastructure).

ORACLE: used only by tests/ as the checker of csrc/torus64.cu and of the
2^64 encrypted Spike-LSTM; nothing in the product imports it.

The reference computes at q = 2^64 in float64 (parameters_crypto.py:6), so
its integer steps round.  The engine makes them exact on Z/2^64; this module
states that exact arithmetic with numpy uint64 (wrap-around = reduction
modulo 2^64):

  decomposition        schemas/polynomial_jax.py:90-111, evaluated exactly
                       (round half to even) on the integer
  key_switch           schemas/LWE_jax.py:65-117
  rotation_indices     cuTFHE/multiply.py:67-79
  rotate_extract       schemas/RLWE_jax.py:295-303 and text_jax.py:191-208
  blind_rotate         schemas/text_jax.py:390-435 with the reference's own
                       float64 steps at q = 2^64 (inexact, as the reference)
  linear               nn_tfhe/Spike_LSTM.py:48-58
  lut_mul_sum          nn_tfhe/activation.py:103-106 + Spike_LSTM.py:129-132
  pack_lwe_to_rlwe     schemas/text_jax.py:173-187, 242-345
  packing              schemas/text_jax.py:211-239
  spike_lstm_step      nn_tfhe/Spike_LSTM.py:103-176 (scan_step)

The parity bar for the GPU is bit-exact on every integer operator; the FP64
blind rotation at q = 2^64 is compared by decryption within a stated noise
bound (its rounding differs between FFTs, in the reference as here).
"""
from __future__ import annotations

import numpy as np

from oracle import tfhe_oracle as O

Q64 = 2.0 ** 64
U1 = np.uint64(1)


def u64(x):
    a = np.asarray(x)
    if a.dtype == np.uint64:
        return a
    return a.astype(np.int64).astype(np.uint64)


def centred(u):
    return np.asarray(u, dtype=np.uint64).view(np.int64)


def rne_shift(x, s):
    """(d, r): d = rne(x / 2^s), r = x - d 2^s for centred int64 x."""
    x = np.asarray(x, dtype=np.int64)
    if s == 0:
        return x.copy(), np.zeros_like(x)
    d = x >> np.int64(s)
    low = x.astype(np.uint64) & ((U1 << np.uint64(s)) - U1)
    half = U1 << np.uint64(s - 1)
    up = (low > half) | ((low == half) & ((d & 1) == 1))
    d = d + up.astype(np.int64)
    rem_up = (low - (U1 << np.uint64(s))).view(np.int64)
    rem = np.where(up, rem_up, low.view(np.int64))
    return d, rem


def decomposition(x_u64, log2_beta, l):
    """Gadget digits (l, ...) int64 of torus words: d_j = rne(r_{j-1} /
    2^(64 - j log2 beta)), r_0 the centred value."""
    r = centred(u64(x_u64))
    out = []
    for j in range(1, l + 1):
        d, r = rne_shift(r, 64 - j * log2_beta)
        out.append(d)
    return np.stack(out)


def _limbs16(x):
    """Signed 16-bit limbs (4, ...) int64 with sum limb_t 2^(16 t) = x mod 2^64."""
    w = u64(x).copy()
    out = []
    for _ in range(4):
        lo = ((w + np.uint64(0x8000)) & np.uint64(0xFFFF)).astype(np.int64) - 0x8000
        out.append(lo)
        w = (w - lo.astype(np.uint64)) >> np.uint64(16)
    return out


def matmul_mod64(D, K):
    """D (R, k) integers, K (k, C) uint64 -> D @ K mod 2^64 (uint64), exact:
    every float64 product of D with a 16-bit limb of K is an integer far below
    2^53 for |D| <= 2^10 and k <= 2^17."""
    D = np.asarray(D, dtype=np.int64)
    assert np.abs(D).max(initial=0) <= 1 << 10 and D.shape[1] <= 1 << 17
    Df = D.astype(np.float64)
    out = np.zeros((D.shape[0], K.shape[1]), dtype=np.uint64)
    for t, limb in enumerate(_limbs16(K)):
        part = np.rint(Df @ limb.astype(np.float64)).astype(np.int64)
        out += part.astype(np.uint64) << np.uint64(16 * t)
    return out


def negacyclic_mod64(x, y):
    """x (..., N) * y (..., N) in Z/2^64[X]/(X^N + 1), both any 64-bit words,
    exactly: 16-bit limb products, each an exact integer product."""
    lx, ly = _limbs16(x), _limbs16(y)
    out = None
    for t1 in range(4):
        for t2 in range(4 - t1):
            if not np.any(ly[t2]) or not np.any(lx[t1]):
                continue
            p = O.negacyclic_mul_exact(lx[t1], ly[t2]).astype(np.uint64) << np.uint64(16 * (t1 + t2))
            out = p if out is None else out + p
    if out is None:
        out = np.zeros(np.broadcast_shapes(np.shape(x), np.shape(y)), dtype=np.uint64)
    return out


# ---------------------------------------------------------------- PBS
def key_switch(ksk, a, b, log2_beta, l):
    """ksk (n_big l, n + 1) uint64 (row i l + j); a (B, n_big), b (B)."""
    a = u64(a)
    B, n_big = a.shape
    dig = np.moveaxis(decomposition(a, log2_beta, l), 0, -1).reshape(B, n_big * l)
    prod = matmul_mod64(dig, ksk)
    return prod[:, :-1], u64(b) + prod[:, -1]


def rotation_indices(a, collapse, N, n_lut):
    """(B, G, M) int32: rne(2N <a_g, p_m> / (q n_lut)) n_lut mod 2N."""
    a = u64(a)
    B, n = a.shape
    G, M = n // collapse, 1 << collapse
    pats = O.all_binary_vectors(collapse).astype(np.uint64)          # (M, c)
    grp = a.reshape(B, G, collapse)
    v = (grp[:, :, None, :] * pats[None, None, :, :]).sum(axis=-1, dtype=np.uint64)
    s = 63 - int(np.log2(N)) + int(np.log2(n_lut))
    d, _ = rne_shift(centred(v), s)
    return ((d * n_lut) % (2 * N)).astype(np.int32)


def blind_rotate(lut, idx, bsk_grouped, rot, log2_beta, l, N):
    """The collapsed CMux chain with the reference's float64 steps at
    q = 2^64 (schemas/text_jax.py:414-433): lut (B|1, 2, N) words, idx
    (B, G, M), bsk_grouped (G, 2, L, 2, M, N/2).  Returns ACC float64."""
    B, G, M = idx.shape
    ct = np.broadcast_to(centred(u64(lut)).astype(np.float64), (B, 2, N)).copy()
    beta = 2.0 ** log2_beta
    for g in range(G):
        dec = np.moveaxis(O.decomposition(ct, beta, l, Q64), 0, 1)    # (B, L, 2, N)
        dec_fft = O.jax_fourier(dec)
        chunk = bsk_grouped[g]                                        # (2, L, 2, M, d)
        rotm = rot[idx[:, g, :]]                                      # (B, M, d)
        sum_rgsw = np.einsum("abcmd,kmd->kabcd", chunk, rotm)
        prod = np.einsum("kabcd,kbcd->kad", sum_rgsw, dec_fft)
        ct = O.centered_mod(O.jax_inversefourier(prod), Q64)
    return ct


def acc_to_words(acc):
    """float64 accumulator in [-q/2, q/2] -> uint64 words (q/2 -> 2^63)."""
    acc = np.asarray(acc, dtype=np.float64)
    hi = acc >= 2.0 ** 63
    v = np.where(hi, acc - Q64, acc).astype(np.int64)
    return v.astype(np.uint64)


def rotate_extract(acc_u64, b, N, n_lut):
    """Rotation by -b~ and sample extraction at 0..n_lut-1: (B, n_lut, N), (B, n_lut)."""
    acc = u64(acc_u64)
    B = acc.shape[0]
    s = 63 - int(np.log2(N)) + int(np.log2(n_lut))
    bt, _ = rne_shift(centred(u64(b)), s)
    bt = bt * n_lut
    out_a = np.empty((B, n_lut, N), dtype=np.uint64)
    out_b = np.empty((B, n_lut), dtype=np.uint64)
    j = np.arange(N)
    neg = lambda v: (~v) + np.uint64(1)                    # 0 - v on uint64 words
    for k in range(B):
        for al in range(n_lut):
            e = (al - j + bt[k]) % (2 * N)
            out_a[k, al] = np.where(e < N, acc[k, 0, e % N], neg(acc[k, 0, e % N]))
            eb = (al + bt[k]) % (2 * N)
            out_b[k, al] = acc[k, 1, eb % N] if eb < N else neg(acc[k, 1, eb % N])
    return out_a, out_b


def pbs(keys, a, b, lut, n_lut):
    """Key switch, blind rotation (float64 at q = 2^64), rotation by -b~,
    extraction.  keys: dict with ksk, bsk_grouped, rot, params (client64.Params64)."""
    p = keys["params"]
    ka, kb = key_switch(keys["ksk"], a, b, p.log2_beta_ks, p.l_ks)
    idx = rotation_indices(ka, p.collapse, p.N, n_lut)
    acc = blind_rotate(lut, idx, keys["bsk_grouped"], keys["rot"], p.log2_beta_bs, p.l_bs, p.N)
    return rotate_extract(acc_to_words(acc), kb, p.N, n_lut)


# ---------------------------------------------------------------- LSTM level
def linear(kern, bias, rlwe):
    """W_j(X) * rlwe, extraction at 0, + bias_j: kern (J, N), bias (J),
    rlwe (a, b) (N,) words -> (J, N), (J,) uint64."""
    a, b = (u64(v) for v in rlwe)
    kern = np.asarray(kern, dtype=np.int64)
    pa = negacyclic_mod64(a[None], kern)
    pb = negacyclic_mod64(b[None], kern)
    N = a.shape[-1]
    ext = np.empty_like(pa)
    ext[:, 0] = pa[:, 0]
    ext[:, 1:] = np.uint64(0) - pa[:, N - np.arange(1, N)]
    return ext, pb[:, 0] + u64(bias)


def lut_mul_sum(luts, rlwe_a, rlwe_b):
    """sum over g of luts[g][k] * (a, b)[g][k]: luts (G, K, N) int,
    rlwe_a / rlwe_b (G, K, N) words -> (K, N), (K, N)."""
    pa = negacyclic_mod64(u64(rlwe_a), np.asarray(luts, dtype=np.int64))
    pb = negacyclic_mod64(u64(rlwe_b), np.asarray(luts, dtype=np.int64))
    return pa.sum(axis=0, dtype=np.uint64), pb.sum(axis=0, dtype=np.uint64)


def automorphism(poly, k):
    poly = u64(poly)
    N = poly.shape[-1]
    idx = (np.arange(N) * k) % (2 * N)
    out = np.zeros_like(poly)
    out[..., idx % N] = np.where(idx >= N, np.uint64(0) - poly, poly)
    return out


def pack_lwe_to_rlwe(a, b, galois, log2_beta, l):
    """a (R, N), b (R) words; galois (log2 N, l, 2, N) uint64 -> (A, B) (R, N)."""
    a = u64(a)
    R, N = a.shape
    steps = int(np.log2(N))
    logn = steps
    ms_a, _ = rne_shift(centred(a), logn)
    ms_b, _ = rne_shift(centred(u64(b)), logn)
    A = np.zeros((R, N), dtype=np.uint64)
    A[:, 0] = u64(ms_a[:, 0])
    A[:, 1:] = np.uint64(0) - u64(np.flip(ms_a[:, 1:], axis=-1))
    Bp = np.zeros((R, N), dtype=np.uint64)
    Bp[:, 0] = u64(ms_b)
    galois = u64(galois)
    for i in range(steps):
        k = 2 ** (steps - i) + 1
        Ap, Bq = automorphism(A, k), automorphism(Bp, k)
        dec = decomposition(Ap, log2_beta, l)                       # (l, R, N)
        ks_a = np.zeros((R, N), dtype=np.uint64)
        ks_b = np.zeros((R, N), dtype=np.uint64)
        for j in range(l):
            ks_a += negacyclic_mod64(galois[i, j, 0][None], dec[j])
            ks_b += negacyclic_mod64(galois[i, j, 1][None], dec[j])
        A = A + ks_a
        Bp = Bp + Bq + ks_b
    return A, Bp


def packing(a, b, ksp, log2_beta, l, N):
    """T LWEs a (T, n_dim), b (T) into one RLWE with ksp (n_dim, l, 2, N)."""
    a = u64(a)
    T, n_dim = a.shape
    dig = np.moveaxis(decomposition(a, log2_beta, l), 0, -1).reshape(T, n_dim * l)      # (T, n_dim l)
    V = matmul_mod64(dig, u64(ksp).reshape(n_dim * l, 2 * N)).reshape(T, 2, N)
    out_a = np.zeros(N, dtype=np.uint64)
    out_b = np.zeros(N, dtype=np.uint64)
    out_b[:T] = u64(b)
    for t in range(T):
        ra = rotate_poly(V[t, 0], t)
        rb = rotate_poly(V[t, 1], t)
        out_a -= ra
        out_b -= rb
    return out_a, out_b


def rotate_poly(p, alpha):
    """X^alpha * p (negacyclic) on words."""
    p = u64(p)
    N = p.shape[-1]
    alpha %= 2 * N
    out = np.empty_like(p)
    j = np.arange(N)
    src = (j - alpha) % (2 * N)
    neg = src >= N
    out[...] = np.where(neg, np.uint64(0) - p[..., src % N], p[..., src % N])
    return out


def sample_extract_many(a, b, count):
    a, b = u64(a), u64(b)
    N = a.shape[-1]
    out_a = np.empty((count, N), dtype=np.uint64)
    j = np.arange(N)
    for al in range(count):
        src = np.where(j <= al, al - j, al - j + N)
        out_a[al] = np.where(j <= al, a[src], np.uint64(0) - a[src])
    return out_a, b[:count].copy()


def spike_lstm_step(keys, layer, x_t, H, C):
    """scan_step (nn_tfhe/Spike_LSTM.py:103-176) on Z/2^64 for one sequence.
    layer: dict with kern_f/i/o, bias_f/i/o, lut_f, lut_o (n_lut, per, N),
    lut_i (per, N), galois, gal_log2_beta, gal_l, ksp, pk_log2_beta, pk_l,
    input_dim, hidden, n_lut.  x_t, H, C: (a, b) (N,) words."""
    hidden, n_lut = layer["hidden"], layer["n_lut"]
    N = u64(x_t[0]).shape[-1]
    per = hidden // n_lut
    c_a, c_b = sample_extract_many(C[0], C[1], hidden)
    hx = (u64(x_t[0]) + u64(H[0]), u64(x_t[1]) + u64(H[1]))
    F = linear(layer["kern_f"], layer["bias_f"], hx)
    I = linear(layer["kern_i"], layer["bias_i"], hx)
    Ot = linear(layer["kern_o"], layer["bias_o"], hx)

    def prepare(lwe_a, lwe_b, lut):
        ra, rb = pack_lwe_to_rlwe(lwe_a, lwe_b, layer["galois"], layer["gal_log2_beta"], layer["gal_l"])
        return lut_mul_sum(np.asarray(lut, np.int64), ra.reshape(n_lut, per, N), rb.reshape(n_lut, per, N))

    lut_c_a, lut_c_b = prepare(c_a, c_b, layer["lut_f"])
    in_a = np.concatenate([F[0], I[0]])
    in_b = np.concatenate([F[1], I[1]])
    luts = np.zeros((2 * per, 2, N), dtype=np.uint64)
    luts[:per, 0], luts[:per, 1] = lut_c_a, lut_c_b
    luts[per:, 1] = u64(layer["lut_i"])
    boot_a, boot_b = pbs(keys, in_a, in_b, luts, n_lut)                         # (2 per, n_lut, N)
    spike_i_a = np.transpose(boot_a[per:], (1, 0, 2)).reshape(-1, N)
    spike_i_b = np.transpose(boot_b[per:], (1, 0)).reshape(-1)
    spike_fc_a = np.transpose(boot_a[:per], (1, 0, 2)).reshape(-1, N)
    spike_fc_b = np.transpose(boot_b[:per], (1, 0)).reshape(-1)
    ct_a, ct_b = spike_fc_a + spike_i_a, spike_fc_b + spike_i_b
    lut_h_a, lut_h_b = prepare(ct_a, ct_b, layer["lut_o"])
    luts_h = np.stack([lut_h_a, lut_h_b], axis=1)
    h_a, h_b = pbs(keys, Ot[0], Ot[1], luts_h, n_lut)
    h_a = np.transpose(h_a, (1, 0, 2)).reshape(-1, N)
    h_b = np.transpose(h_b, (1, 0)).reshape(-1)
    C_t = packing(ct_a, ct_b, layer["ksp"], layer["pk_log2_beta"], layer["pk_l"], N)
    H_p = packing(h_a, h_b, layer["ksp"], layer["pk_log2_beta"], layer["pk_l"], N)
    H_t = (rotate_poly(H_p[0], layer["input_dim"]), rotate_poly(H_p[1], layer["input_dim"]))
    return H_t, C_t
