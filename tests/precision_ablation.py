"""Precision ablation of the external product (test infrastructure).

Parameters: n=630, N=1024, gadget 2^7 x 3, collapse 3, key switch 2^3 x 5,
4 LUTs packed per blind rotation (n_lut=4), messages in Z_4 with a padding
bit, outputs in Z_4 at scale q/8.

Forms of the per-group external product ACC <- sum_in DEC_F[in] *
sum_p BSK[g, p] X^{r_p}, all run on the same keys, inputs and accumulators:

  exact    the integer product (the oracle's 11-bit-limb route, every limb
           product checked integral): the reference value
  fp64     the FP64 FFT product of schemas/text_jax.py:390-435 (the
           engine's form)
  fp32xK   FFT, pointwise products and inverse FFT in FP32 with every key
           coefficient split into K signed limbs of ceil(32/K) bits; each
           limb's product is rounded to an integer and the limbs are
           recombined exactly modulo 2^32

Reported per form:
  per-group error   (form's product - exact product) on the torus, on the
                    same accumulator, over every coefficient of every group
  final difference  the GLWE phase b - a s of the form's own accumulator
                    chain after all groups minus the exact chain's, per
                    coefficient (the added noise)
  output noise      phase of the 4 extracted LWEs minus the table value,
                    and decryption failures of the sample; the Gaussian tail
                    at q/16 gives the expected failures in 10^6 PBS

FP32 arithmetic is numpy/scipy single precision (pocketfft computes in
complex64 for complex64 inputs); a GPU FP32 FFT rounds differently in
detail but with the same 2^-24 unit roundoff and log N growth.

Run ``python tests/precision_ablation.py --samples 16`` for the table;
``test_precision_ablation.py`` runs a small case.
"""
from __future__ import annotations

import argparse
import math
import os
import sys
import time

import numpy as np
import scipy.fft

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for _p in (ROOT, HERE, os.path.join(ROOT, "blind-spiking-lstm_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

from oracle import tfhe_oracle as O  # noqa: E402
from pbs_cases import PARAMS, canon, keys as case_keys, ks_params  # noqa: E402
from tfhe_b200 import client  # noqa: E402

Q = 2.0 ** 32
N_LUT = 4
T_IN = 8          # Z_4 messages with a padding bit: phase m q / 8
T_OUT = 8         # outputs in Z_4 at scale q / 8
FORMS = ("fp64", "fp32x2", "fp32x3", "fp32x4")


def split_limbs(x, count):
    """Signed balanced limbs of width w = ceil(32 / count) of int64 values in
    [-2^31, 2^31): x = sum_i limb_i 2^(w i); the top limb carries the rest."""
    w = -(-32 // count)
    rest = np.asarray(x, dtype=np.int64).copy()
    out = []
    for i in range(count - 1):
        lo = ((rest + (1 << (w - 1))) & ((1 << w) - 1)) - (1 << (w - 1))
        out.append((lo, w * i))
        rest = (rest - lo) >> w
    out.append((rest, w * (count - 1)))
    return out


def fourier32(p):
    """jax_fourier in single precision."""
    p = np.asarray(p, dtype=np.float32)
    n = p.shape[-1]
    tw = np.exp(-1j * np.pi * np.arange(n) / n).astype(np.complex64)
    return scipy.fft.fft(tw * p, axis=-1)[..., : n // 2].astype(np.complex64)


def inverse32(P):
    """jax_inversefourier without the rounding, in single precision."""
    P = np.asarray(P, dtype=np.complex64)
    full = np.concatenate([P, np.flip(np.conj(P), axis=-1)], axis=-1)
    n = full.shape[-1]
    tw = np.exp(1j * np.pi * np.arange(n) / n).astype(np.complex64)
    return np.real(tw * scipy.fft.ifft(full, axis=-1).astype(np.complex64)).astype(np.float32)


def torus(x64):
    """int64 values (exact integers modulo 2^64) -> centred int64 mod 2^32."""
    return (((np.asarray(x64, dtype=np.int64) + 2 ** 31) & 0xFFFFFFFF) - 2 ** 31).astype(np.int64)


class Study:
    """One sample of ciphertexts with every form's chain."""

    def __init__(self, samples, seed=0, groups=None, name="cfg1", n_lut=N_LUT, t_in=T_IN, t_out=T_OUT,
                 fp32=True):
        p = PARAMS[name]
        self.n_lut, self.t_in, self.t_out = n_lut, t_in, t_out
        self.p = p
        self.k = case_keys(name)
        N, n, c = p["N"], p["n"], p["collapse"]
        self.N, self.L, self.beta = N, p["l_bs"], p["beta_bs"]
        self.G = n // c if groups is None else groups
        self.M = 2 ** c
        rng = np.random.default_rng(1000 + seed)
        self.msgs = rng.integers(0, t_in // 2, size=samples)
        a, b = O.encrypt_inputs(self.k, self.msgs, Q / t_in, rng)
        a, b = canon(a), canon(b)
        ka, kb = O.key_switch_LWE(self.k.ksk, (a, b), ks_params(name))
        self.ka, self.kb = ka, np.asarray(kb).reshape(-1)
        self.idx = O.rotation_indices(self.ka, c, N, Q, n_lut)                 # (B, G, M)
        self.tables = rng.integers(0, t_out // 2, size=(n_lut, t_in // 2))
        self.expect = self.tables[:, self.msgs].T                              # (B, n_lut)
        body = client.packed_table_lut(N, self.tables, t_out)
        self.acc0 = np.zeros((samples, 2, N))
        self.acc0[:, 1] = canon(body.view(np.int32).astype(np.float64))
        # keys in every form
        key = O.bsk_coeff_grouped(self.k.bsk_coeff, n // c, c)                  # (G,2,L,2,M,N) int64
        self.exact_limbs = [(O.jax_fourier(lb.astype(np.float64)), 11 * t)
                            for t, lb in enumerate(O._limbs(key)) if np.any(lb)]
        self.fp64_key = O.bsk_reshape(self.k.bsk_ordered, n // c, c)
        self.fp32_keys = {cnt: [(O.jax_fourier(lb.astype(np.float64)).astype(np.complex64), s)
                                for lb, s in split_limbs(key, cnt)] for cnt in (2, 3, 4)} if fp32 else {}
        self.ang64 = np.exp(-1j * np.pi * np.outer(np.arange(2 * N), 2 * np.arange(N // 2) + 1) / N)
        self.ang32 = self.ang64.astype(np.complex64)
        self.rot64 = O.all_rot_possible_fourier(N)

    # ------------------------------------------------------------ products
    def _summed(self, kf, rot, g):
        s = kf[g][None, :, :, :, 0, :] * rot[:, None, None, None, 0, :]
        for m in range(1, self.M):
            s = s + kf[g][None, :, :, :, m, :] * rot[:, None, None, None, m, :]
        return s

    def product(self, form, acc, g):
        """The form's external product of group g on accumulator acc (B, 2, N)
        as centred int64 on the torus."""
        dec = np.moveaxis(O.decomposition(acc, self.beta, self.L, Q), 0, 1)      # (B, L, 2, N)
        idx = self.idx[:, g, :]
        if form == "exact":
            dec_f = O.jax_fourier(dec)
            rot = self.ang64[idx]
            total = np.zeros(acc.shape, dtype=np.uint64)
            for kf, shift in self.exact_limbs:
                prod = np.einsum("kabcd,kbcd->kad", self._summed(kf, rot, g), dec_f)
                part = O._round_checked(O._inverse_unrounded(prod), "exact product")
                total += part.astype(np.uint64) << np.uint64(shift)
            return torus(total.astype(np.int64))
        if form == "fp64":
            dec_f = O.jax_fourier(dec)
            rot = self.rot64[idx]
            prod = np.einsum("kabcd,kbcd->kad", self._summed(self.fp64_key, rot, g), dec_f)
            return torus(np.rint(O._inverse_unrounded(prod)).astype(np.int64))
        cnt = int(form.split("x")[1])
        dec_f = fourier32(dec)
        rot = self.ang32[idx]
        total = np.zeros(acc.shape, dtype=np.uint64)
        for kf, shift in self.fp32_keys[cnt]:
            prod = np.einsum("kabcd,kbcd->kad", self._summed(kf, rot, g), dec_f).astype(np.complex64)
            part = np.rint(inverse32(prod).astype(np.float64)).astype(np.int64)
            total += part.astype(np.uint64) << np.uint64(shift)
        return torus(total.astype(np.int64))

    def glwe_phase(self, acc):
        """b(X) - a(X) s(X) mod X^N + 1 of accumulators (B, 2, N), centred
        int64: two chains that differ only by rounding have unrelated masks,
        so they are compared through their phases."""
        a = np.rint(acc[:, 0]).astype(np.int64)
        b = np.rint(acc[:, 1]).astype(np.int64)
        s = self.k.sk_glwe.astype(np.int64)
        return torus(b - O.negacyclic_mul_exact(a, s))

    # ------------------------------------------------------------ chains
    def run(self, forms=FORMS):
        res = {}
        accs = {f: self.acc0.copy() for f in ("exact",) + tuple(forms)}
        per_group = {f: [0.0, 0.0, 0] for f in forms}       # max |e|, sum e^2, count
        for g in range(self.G):
            for f in ("exact",) + tuple(forms):
                acc = accs[f]
                mine = self.product(f, acc, g)
                if f != "exact":
                    ref = self.product("exact", acc, g)
                    e = torus(mine - ref).astype(np.float64)
                    st = per_group[f]
                    st[0] = max(st[0], float(np.max(np.abs(e))))
                    st[1] += float(np.sum(e * e))
                    st[2] += e.size
                accs[f] = mine.astype(np.float64)
        b_rot = O.body_rotation(self.kb, self.N, Q, self.n_lut)
        for f in ("exact",) + tuple(forms):
            alphas = np.repeat(-b_rot.astype(np.int64)[:, None], 2, axis=1)
            rotated = O.coef_rotation_rows(accs[f], alphas)
            a_out, b_out = O.extract_many(rotated, self.n_lut)
            a_out = np.asarray(a_out).reshape(-1, self.N)
            b_out = np.asarray(b_out).reshape(-1)
            phase = torus(np.rint(b_out).astype(np.int64) -
                          np.rint(a_out @ self.k.sk_glwe).astype(np.int64))
            want = self.expect.reshape(-1) * (2 ** 32 // self.t_out)
            noise = torus(phase - want).astype(np.float64)
            dec = np.mod(np.rint(phase / (2.0 ** 32 / self.t_out)), self.t_out).astype(np.int64)
            fails = int(np.sum(dec != self.expect.reshape(-1)))
            entry = {"output_noise_std": float(np.std(noise)), "output_noise_max": float(np.max(np.abs(noise))),
                     "failures": fails, "outputs": int(noise.size)}
            if f != "exact":
                d = torus(self.glwe_phase(accs[f]) - self.glwe_phase(accs["exact"])).astype(np.float64)
                mx, s2, cnt = per_group[f]
                entry.update({"group_err_max": mx, "group_err_var": s2 / max(cnt, 1),
                              "final_diff_max": float(np.max(np.abs(d))), "final_diff_var": float(np.mean(d * d))})
            sigma = entry["output_noise_std"]
            thr = 2.0 ** 32 / (2 * self.t_out)
            p_fail = math.erfc(thr / (sigma * math.sqrt(2))) if sigma > 0 else 0.0
            entry["expected_failures_per_1e6_pbs"] = p_fail * 1e6 * self.n_lut
            res[f] = entry
        return res


def _fmt(x):
    if x == 0:
        return "0"
    return f"2^{math.log2(abs(x)):.2f}"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--samples", type=int, default=16)
    ap.add_argument("--groups", type=int, default=None)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--params", choices=["cfg1", "cfg2"], default="cfg1",
                    help="cfg1: 4 LUTs, Z_4, every form; cfg2 (gadget 2^15 x 2): 1 LUT, Z_8 inputs, FP64 only")
    args = ap.parse_args()
    t0 = time.time()
    if args.params == "cfg1":
        st = Study(args.samples, args.seed, args.groups)
        forms = FORMS
    else:
        st = Study(args.samples, args.seed, args.groups, name="cfg2", n_lut=1, t_in=16, t_out=8, fp32=False)
        forms = ("fp64",)
    res = st.run(forms)
    print(f"# {args.params}: {args.samples} PBS x {st.n_lut} outputs, {st.G} groups, {time.time() - t0:.0f} s")
    print("| form | per-group error max | per-group error var | final phase diff max | final phase diff var | "
          "output noise std | failures (sample) | expected failures / 10^6 PBS |")
    print("|---|---:|---:|---:|---:|---:|---:|---:|")
    for f in ("exact",) + tuple(forms):
        e = res[f]
        print(f"| {f} | {_fmt(e.get('group_err_max', 0))} | {_fmt(e.get('group_err_var', 0))} | "
              f"{_fmt(e.get('final_diff_max', 0))} | {_fmt(e.get('final_diff_var', 0))} | "
              f"{_fmt(e['output_noise_std'])} | {e['failures']}/{e['outputs']} | "
              f"{e['expected_failures_per_1e6_pbs']:.3g} |")


if __name__ == "__main__":
    main()
