"""Generate the golden fixtures of the encrypted Spike-LSTM operators by
running the REFERENCE's own code (AMIAD-Research/Blind-Spiking-LSTM) under
the jax / flax stand-ins (see refenv.py):

  Linear.set_weights / Linear.__call__      nn_tfhe/Spike_LSTM.py:28-58
  HeavysideBoostrapper.prepare_LUT          nn_tfhe/activation.py:103-106
    (pack_lwe_to_rlwe, schemas/text_jax.py:316-345, times the plain LUT)
  pack_lwe_to_rlwe                          schemas/text_jax.py:316-345
  HeavysideBoostrapper.packing              nn_tfhe/activation.py:109-115
    (packing, schemas/text_jax.py:211-239)
  CipherSpikeLSTM.__call__ (lax.scan of scan_step)
                                            nn_tfhe/Spike_LSTM.py:103-184
  CipherMLP with ReluBoostrapper            nn_tfhe/Spike_LSTM.py:187-206,
                                            nn_tfhe/activation.py:166-237

on the layers of tests/lstm_golden_cases.py (torus q = 2^32, keys and
inputs from fixed seeds).  Outputs are stored as uint32 torus words in
tests/golden/lstm_golden.npz (large arrays as a SHA-256 digest plus their
first row).  Run from the repository root:

    REFERENCE_ROOT=<path to the reference checkout> python tests/golden/make_lstm_golden.py
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
from schemas import text_jax as TJ  # noqa: E402
from jax import vmap  # noqa: E402

import lstm_golden_cases as GC  # noqa: E402

Q = 2.0 ** 32


def f64(u):
    return GC.cen(u).astype(np.float64)


def reference_objects(c: GC.Case):
    """The reference's HeavysideBoostrapper, Linears and CipherSpikeLSTM for
    a case, with its dict_params as parameters_crypto.py lays them out."""
    p, N = c.p, c.N
    dict_params = {"t": N, "degree": N, "q": Q, "beta_ks": 2.0 ** c.pk_log2_beta, "l_ks": c.pk_l,
                   "beta_bs": p["beta_bs"], "l_bs": p["l_bs"]}
    dict_params_lut = {"t": N, "degree": N, "q": Q, "beta_bs": p["beta_bs"], "l_bs": p["l_bs"],
                       "beta_ks": 2.0 ** c.pk_log2_beta, "l_ks": c.pk_l, "collapse": p["collapse"]}
    dict_params_ks = {"t": N, "degree": p["n"], "q": Q, "beta_ks": p["beta_ks"], "l_ks": p["l_ks"]}
    dict_params_packing = {"t": N, "degree": N, "q": Q, "beta_ks": 2.0 ** c.gal_log2_beta, "l_ks": c.gal_l}
    galois_fourier = PJ.jax_fourier(f64(c.galois))                  # (log2 N, l, 2, N/2), as get_galois_key
    ksp = (f64(c.ksp[:, :, 0]), f64(c.ksp[:, :, 1]))                 # KSP of get_packing_KSK
    hbs = RA.HeavysideBoostrapper(c.keys.bsk_ordered, c.keys.ksk, ksp, galois_fourier, dict_params,
                                  dict_params_lut, dict_params_ks, dict_params_packing, p["collapse"],
                                  c.keys.all_rot, c.n_lut)
    lins = {}
    for g in "fio":
        lin = RS.Linear(c.per, dict_params, np.ones(c.per))
        lin.set_weights(np.asarray(c.W[g], np.float64), np.asarray(c.B[g], np.float64))
        lins[g] = lin
    lut_i = [np.zeros((c.per, N)), np.asarray(c.lut_i, np.float64)]
    model = RS.CipherSpikeLSTM(dict_params, dict_params_lut, c.input_dim, c.hidden, c.xs.shape[0],
                               lins["f"], lins["i"], lins["o"], hbs, c.n_lut,
                               np.asarray(c.lut_f, np.float64), lut_i, np.asarray(c.lut_o, np.float64),
                               float(c.beta_x))
    relu = RA.ReluBoostrapper(c.keys.bsk_ordered, c.keys.ksk, ksp, dict_params, dict_params_lut, dict_params_ks,
                              dict_params_packing, p["collapse"], c.keys.all_rot, float(c.beta_x), c.s_head)
    h1 = RS.Linear(c.head_W1.shape[1], dict_params, np.ones(c.head_W1.shape[1]))
    h1.set_weights(np.asarray(c.head_W1, np.float64), np.asarray(c.head_B1, np.float64))
    h2 = RS.Linear(c.head_W2.shape[1], dict_params, np.ones(c.head_W2.shape[1]))
    h2.set_weights(np.asarray(c.head_W2, np.float64), np.asarray(c.head_B2, np.float64))
    head = RS.CipherMLP(dict_params, dict_params_lut, c.hidden, h1, h2, relu)
    return dict(params=dict_params, packing=dict_params_packing, hbs=hbs, lins=lins, model=model, head=head,
                galois_fourier=galois_fourier)


def gen_case(c: GC.Case, out):
    t0 = time.time()
    ref = reference_objects(c)
    pre = c.name + "_"
    N = c.N
    for g in "fio":
        out[pre + f"kern_{g}"] = np.asarray(ref["lins"][g].kernel_polynomial).astype(np.int16)
    # Linear.__call__ on HX of the first timestep (H = 0: HX = x_0)
    x0 = (f64(c.xs[0, 0, 0]), f64(c.xs[0, 0, 1]))
    hx = TJ.sum_ciphertext_ciphertext(x0, (np.zeros(N), np.zeros(N)), Q)
    for g in "fio":
        la, lb = ref["lins"][g](hx)
        GC.put(out, pre + f"lin_{g}_a", np.asarray(la))
        GC.put(out, pre + f"lin_{g}_b", np.asarray(lb).reshape(-1))
    ops = GC.op_inputs(c)
    # pack_lwe_to_rlwe on two LWEs (sums left unreduced by the reference)
    pk = ref["packing"]
    for r in range(2):
        A, B = TJ.pack_lwe_to_rlwe((f64(ops["r2r_a"][r]), f64(ops["r2r_b"][r:r + 1])), ref["galois_fourier"],
                                   pk["beta_ks"], pk["l_ks"], pk["q"], pk["degree"])
        out[pre + f"r2r{r}_A"] = np.asarray(A).astype(np.int64)
        out[pre + f"r2r{r}_B"] = np.asarray(B).astype(np.int64)
    # prepare_LUT over (n_lut, per) LWEs with lut_f, summed over the packed
    # LUTs and reduced as in scan_step (nn_tfhe/Spike_LSTM.py:129-132)
    lwe = (f64(ops["prep_a"]), f64(ops["prep_b"])[..., None])
    prod = vmap(vmap(ref["hbs"].prepare_LUT, (0, 0)), (0, 0))(lwe, np.asarray(c.lut_f, np.float64))
    pa, pb = TJ.centered_mod_ciphertext((np.sum(prod[0], axis=0), np.sum(prod[1], axis=0)), Q)
    GC.put(out, pre + "prep_a", np.asarray(pa))
    GC.put(out, pre + "prep_b", np.asarray(pb))
    # packing of `hidden` LWEs into one RLWE
    qa, qb = ref["hbs"].packing((f64(ops["pack_a"]), f64(ops["pack_b"])[:, None]))
    GC.put(out, pre + "pack_a", np.asarray(qa))
    GC.put(out, pre + "pack_b", np.asarray(qb))
    t1 = time.time()
    # the recurrence: lax.scan of scan_step over all timesteps of sequence 0
    xs = [f64(c.xs[:, 0, 0]), f64(c.xs[:, 0, 1])]
    _, (Hs, Cs) = ref["model"](xs, c.xs.shape[0])
    GC.put(out, pre + "H_a", np.asarray(Hs[0]))
    GC.put(out, pre + "H_b", np.asarray(Hs[1]))
    GC.put(out, pre + "C_a", np.asarray(Cs[0]))
    GC.put(out, pre + "C_b", np.asarray(Cs[1]))
    t2 = time.time()
    ya, yb = ref["head"]((f64(c.head_x[0]), f64(c.head_x[1])))
    GC.put(out, pre + "head_a", np.asarray(ya))
    GC.put(out, pre + "head_b", np.asarray(yb).reshape(-1))
    print(f"{c.name}: operators {t1 - t0:.1f} s, recurrence {t2 - t1:.1f} s, head {time.time() - t2:.1f} s")


def main():
    out = {}
    names = sys.argv[1:] or list(GC.CASES)
    for name in names:
        gen_case(GC.CASES[name](), out)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lstm_golden.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes,", len(out), "arrays")


if __name__ == "__main__":
    main()
