"""The 2^64-torus Spike-LSTM oracle against fixtures recorded from the
reference's own code at its own modulus and parameters
(tests/golden/make_lstm64_golden.py; q = 2^64 in float64, N = 2048,
n = 702, gadget 2^13 x 2, collapse 3; hidden 128, 4 packed LUTs).

The reference rounds at q = 2^64 (float64 FFT products, unreduced float64
trace sums), so the bar is a stated distance, not bit equality:
  - Linear: ciphertext words within 2^24 of the reference's (measured 2^19.1);
  - packing: within 2^36 (measured 2^31.7);
  - prepare_LUT: the reference keeps the trace sums unreduced, so its
    ciphertexts are other representatives of the same phases: phases within
    2^48 (measured 2^42.1; a z unit of the LUTs is 2^54).
The reference's own timestep decrypts to the plaintext recurrence up to
spikes flipped by its blind rotation's rounding (one eta <= 1 per flip);
CPU only."""
import os

import numpy as np

import lstm_golden_cases as GC
from oracle import lstm_oracle as LO
from oracle import torus64_oracle as T64
from tfhe_b200 import client64 as C64

FX = np.load(os.path.join(os.path.dirname(__file__), "golden", "lstm64_golden.npz"))
LIN_TOL, PACK_TOL, PREP_PHASE_TOL = 2.0 ** 24, 2.0 ** 36, 2.0 ** 48


def test_linear64_within_rounding_of_reference():
    c = GC.cfg4_q64_case()
    cfg = c["cfg"]
    per = cfg.hidden // cfg.n_lut
    x0 = (c["xs"][0, 0, 0], c["xs"][0, 0, 1])
    for g in "fio":
        kern, bias = LO.linear_kernel_polynomial(c["W"][g], c["B"][g], np.ones(per), cfg.pbs.N)
        a, b = T64.linear(kern, bias, x0)
        assert GC.torus_dist64(a[:4], FX[f"lin_{g}_a_rows"]).max() <= LIN_TOL
        assert GC.torus_dist64(b, FX[f"lin_{g}_b"]).max() <= LIN_TOL


def test_packing64_within_rounding_of_reference():
    c = GC.cfg4_q64_case()
    cfg = c["cfg"]
    ops = GC.q64_op_inputs(c)
    qa, qb = T64.packing(ops["pack_a"], ops["pack_b"], c["model"].ksp, cfg.pk_log2_beta, cfg.pk_l, cfg.pbs.N)
    assert GC.torus_dist64(qa, FX["pack_a"]).max() <= PACK_TOL
    assert GC.torus_dist64(qb, FX["pack_b"]).max() <= PACK_TOL


def test_prepare_lut64_phases_match_reference():
    c = GC.cfg4_q64_case()
    cfg = c["cfg"]
    N, per = cfg.pbs.N, cfg.hidden // cfg.n_lut
    ops = GC.q64_op_inputs(c)
    model = c["model"]
    ra, rb = T64.pack_lwe_to_rlwe(ops["prep_a"][:, :4].reshape(-1, N), ops["prep_b"][:, :4].reshape(-1),
                                  model.galois, cfg.gal_log2_beta, cfg.gal_l)
    pa, pb = T64.lut_mul_sum(np.asarray(c["lut_f"], np.int64)[:, :4], ra.reshape(cfg.n_lut, 4, N),
                             rb.reshape(cfg.n_lut, 4, N))
    sk = model.keys.sk_glwe
    d = C64.rlwe_phase(pa, pb, sk) - C64.rlwe_phase(FX["prep_a_rows"], FX["prep_b_rows"], sk)
    assert np.abs(d.astype(np.float64)).max() <= PREP_PHASE_TOL


def test_reference_step_at_q64_tracks_plaintext():
    """The fixture itself: the reference's encrypted timestep decrypts to the
    plaintext recurrence on all but a few units (flipped spikes)."""
    c = GC.cfg4_q64_case()
    cfg, model = c["cfg"], c["model"]
    sk = model.keys.sk_glwe
    cc, hh = plaintext_step(c)
    phC = C64.rlwe_phase(FX["C_a"][0], FX["C_b"][0], sk)[: cfg.hidden] / cfg.beta_x
    phH = C64.rlwe_phase(FX["H_a"][0], FX["H_b"][0], sk)[cfg.emb_dim: cfg.emb_dim + cfg.hidden] / cfg.beta_x
    assert np.mean(np.abs(phC - cc) < 0.05) >= 0.9
    assert np.mean(np.abs(phH - hh) < 0.05) >= 0.9
    assert np.abs(phC - cc).max() <= 1.0 and np.abs(phH - hh).max() <= 1.0


def plaintext_step(c):
    """First timestep of the plaintext spiking recurrence with the encrypted
    layer's quantisation (LUT grid of N / n_lut entries over z / 256)."""
    cfg, model = c["cfg"], c["model"]
    L = model.layers[0]
    N = cfg.pbs.N
    scale = 4.0 * cfg.beta_x / 2.0 ** 64
    sub = N // cfg.n_lut

    def spike(z, gamma):
        g = np.clip(np.rint(z * scale * sub / 2) * 2 / sub, -1.0, 1.0 - 2.0 / sub)
        return np.concatenate([(g >= gamma[i]).astype(np.float64) for i in range(cfg.n_lut)])

    x = model.embedding[c["tokens"][0, 0]].astype(np.float64)
    hx = np.concatenate([x, np.zeros(cfg.hidden)])
    z = {g: hx @ L.W[g] + L.B[g] for g in "fio"}
    cc = spike(z["i"], L.gamma["i"]) * np.concatenate([L.eta[k] for k in range(cfg.n_lut)])
    return cc, spike(z["o"], L.gamma["o"]) * cc
