"""Golden fixtures of the encrypted Spike-LSTM on the reference's OWN torus
and parameters (q = 2^64 held in float64, N = 2048, n = 702, gadget
2^13 x 2, collapse 3; parameters_crypto.py:6-32), recorded by running the
reference's code under the jax / flax stand-ins (see refenv.py):

  Linear.__call__                      nn_tfhe/Spike_LSTM.py:48-58
  HeavysideBoostrapper.prepare_LUT     nn_tfhe/activation.py:103-106
  HeavysideBoostrapper.packing         nn_tfhe/activation.py:109-115
  CipherSpikeLSTM.__call__ (one step)  nn_tfhe/Spike_LSTM.py:103-184
  CipherMLP + ReluBoostrapper          nn_tfhe/Spike_LSTM.py:187-206

on the layer of tests/lstm_golden_cases.cfg4_q64_case (keys and inputs from
fixed seeds, handed to the reference as its centred float64 values).  The
reference rounds at q = 2^64, so these are its own float64 results: tests
compare ciphertext words within a stated distance and states / logits by
decryption.  Outputs as uint64 words in tests/golden/lstm64_golden.npz.
Run from the repository root:

    REFERENCE_ROOT=<path to the reference checkout> python tests/golden/make_lstm64_golden.py
"""
from __future__ import annotations

import os
import sys
import time

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import refenv  # noqa: E402

refenv.setup()

import numpy as np  # noqa: E402

import nn_tfhe.activation as RA  # noqa: E402  (the reference)
import nn_tfhe.Spike_LSTM as RS  # noqa: E402
from schemas import polynomial_jax as PJ  # noqa: E402
from jax import vmap  # noqa: E402
from schemas import text_jax as TJ  # noqa: E402

import lstm_golden_cases as GC  # noqa: E402
from oracle import tfhe_oracle as O  # noqa: E402

Q = 2.0 ** 64


def f64(u):
    return np.asarray(u, dtype=np.uint64).view(np.int64).astype(np.float64)


def words(x):
    """the reference's float64 values (centred, possibly +-q/2) -> uint64 words"""
    x = np.asarray(x, dtype=np.float64)
    x = np.where(x >= 2.0 ** 63, x - Q, x)
    x = np.where(x < -2.0 ** 63, x + Q, x)
    return x.astype(np.int64).astype(np.uint64)


def main():
    t0 = time.time()
    c = GC.cfg4_q64_case()
    cfg, model = c["cfg"], c["model"]
    p, N = cfg.pbs, cfg.pbs.N
    per = cfg.hidden // cfg.n_lut
    k = model.keys
    # keys as the reference holds them (float64 centred)
    ksk = k.ksk.reshape(p.big, p.l_ks, p.n + 1)
    ksk_ref = (np.transpose(f64(ksk[:, :, :p.n]), (1, 0, 2)), np.transpose(f64(ksk[:, :, p.n:]), (1, 0, 2)))
    bsk_ordered = O.bsk_coeff_fourier_ordered(f64(k.bsk))
    all_rot = O.all_rot_possible_fourier(N)
    dict_params = {"t": N, "degree": N, "q": Q, "beta_ks": 2.0 ** cfg.pk_log2_beta, "l_ks": cfg.pk_l,
                   "beta_bs": 2.0 ** p.log2_beta_bs, "l_bs": p.l_bs}
    dict_params_lut = {"t": N, "degree": N, "q": Q, "beta_bs": 2.0 ** p.log2_beta_bs, "l_bs": p.l_bs,
                       "beta_ks": 2.0 ** cfg.pk_log2_beta, "l_ks": cfg.pk_l, "collapse": p.collapse}
    dict_params_ks = {"t": N, "degree": p.n, "q": Q, "beta_ks": 2.0 ** p.log2_beta_ks, "l_ks": p.l_ks}
    dict_params_packing = {"t": N, "degree": N, "q": Q, "beta_ks": 2.0 ** cfg.gal_log2_beta, "l_ks": cfg.gal_l}
    galois_fourier = PJ.jax_fourier(f64(model.galois))
    ksp = (f64(model.ksp[:, :, 0]), f64(model.ksp[:, :, 1]))
    hbs = RA.HeavysideBoostrapper(bsk_ordered, ksk_ref, ksp, galois_fourier, dict_params, dict_params_lut,
                                  dict_params_ks, dict_params_packing, p.collapse, all_rot, cfg.n_lut)
    lins = {}
    for g in "fio":
        lin = RS.Linear(per, dict_params, np.ones(per))
        lin.set_weights(np.asarray(c["W"][g], np.float64), np.asarray(c["B"][g], np.float64))
        lins[g] = lin
    out = {}
    x0 = (f64(c["xs"][0, 0, 0]), f64(c["xs"][0, 0, 1]))
    hx = TJ.sum_ciphertext_ciphertext(x0, (np.zeros(N), np.zeros(N)), Q)
    for g in "fio":
        la, lb = lins[g](hx)
        out[f"lin_{g}_a_rows"] = words(np.asarray(la)[:4])
        out[f"lin_{g}_b"] = words(np.asarray(lb).reshape(-1))
    ops = GC.q64_op_inputs(c)
    lwe = (f64(ops["prep_a"]), f64(ops["prep_b"])[..., None])
    prod = vmap(vmap(hbs.prepare_LUT, (0, 0)), (0, 0))(lwe, np.asarray(c["lut_f"], np.float64))
    pa, pb = TJ.centered_mod_ciphertext((np.sum(prod[0], axis=0), np.sum(prod[1], axis=0)), Q)
    out["prep_a_rows"], out["prep_b_rows"] = words(np.asarray(pa)[:4]), words(np.asarray(pb)[:4])
    qa, qb = hbs.packing((f64(ops["pack_a"]), f64(ops["pack_b"])[:, None]))
    out["pack_a"], out["pack_b"] = words(qa), words(qb)
    t1 = time.time()
    lut_i = [np.zeros((per, N)), np.asarray(c["lut_i"], np.float64)]
    model_ref = RS.CipherSpikeLSTM(dict_params, dict_params_lut, cfg.emb_dim, cfg.hidden, 1, lins["f"], lins["i"],
                                   lins["o"], hbs, cfg.n_lut, np.asarray(c["lut_f"], np.float64), lut_i,
                                   np.asarray(c["lut_o"], np.float64), float(cfg.beta_x))
    _, (Hs, Cs) = model_ref([f64(c["xs"][:, 0, 0]), f64(c["xs"][:, 0, 1])], 1)
    out["H_a"], out["H_b"] = words(Hs[0]), words(Hs[1])
    out["C_a"], out["C_b"] = words(Cs[0]), words(Cs[1])
    t2 = time.time()
    relu = RA.ReluBoostrapper(bsk_ordered, ksk_ref, ksp, dict_params, dict_params_lut, dict_params_ks,
                              dict_params_packing, p.collapse, all_rot, float(cfg.beta_x), c["s_head"])
    h1 = RS.Linear(c["head_W1"].shape[1], dict_params, np.ones(c["head_W1"].shape[1]))
    h1.set_weights(np.asarray(c["head_W1"], np.float64), np.asarray(c["head_B1"], np.float64))
    h2 = RS.Linear(1, dict_params, np.ones(1))
    h2.set_weights(np.asarray(c["head_W2"], np.float64), np.asarray(c["head_B2"], np.float64))
    head = RS.CipherMLP(dict_params, dict_params_lut, cfg.hidden, h1, h2, relu)
    ya, yb = head((f64(c["head_x"][0]), f64(c["head_x"][1])))
    out["head_a"], out["head_b"] = words(ya), words(np.asarray(yb).reshape(-1))
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lstm64_golden.npz")
    np.savez_compressed(path, **out)
    print(f"operators {t1 - t0:.1f} s, recurrence {t2 - t1:.1f} s, head {time.time() - t2:.1f} s; wrote {path} "
          f"{os.path.getsize(path)} bytes")


if __name__ == "__main__":
    main()
