"""Precision ablation of the external product on the GPU (the config-3
workload): n = 630, N = 1024, gadget 2^7 x 3, collapse 3, 4 packed LUTs per
blind rotation over Z_4 messages with a padding bit (outputs in Z_4 at
q/8, a decryption fails beyond q/16 = 2^28).

Forms, all on the same keys and inputs:
  fp64     the engine (FP64 folded FFT, tfhe_cuboot_merge)
  fp32 xP  the split-limb form (FP32 FFT, key in P = 2, 3, 4 signed limbs
           recombined exactly, tfhe_fp32_cuboot_merge)
and the exact integer product (oracle) for the per-group error.

Per form: the per-coefficient error of one CMux group against the exact
product (max, variance; 64 random accumulators and masks), and over
`--pbs` bootstraps: decryption failures of the 4 outputs, the output noise
std, its variance relative to FP64's, and the blind rotation's PBS/s.

    python tests/precision_ablation_gpu.py [--pbs 1000000] [--json out.json]
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
for p in (os.path.dirname(HERE), os.path.join(os.path.dirname(HERE), "blind-spiking-lstm_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

from oracle import tfhe_oracle as O  # noqa: E402
from tfhe_b200 import client  # noqa: E402
from tfhe_b200.engine import FP32Keys, Keys  # noqa: E402
from tfhe_b200.params import CONFIG3, ParamSet  # noqa: E402

N_LUT, T_IN, T_OUT = 4, 8, 8
CHUNK = 16384
FORMS = ("fp64", "fp32x2", "fp32x3", "fp32x4")


def _torus(x):
    return ((x + 2 ** 31) & 0xFFFFFFFF) - 2 ** 31


def one_group_errors(p, keys, forms, samples=64, seed=11):
    """Each form's accumulator after the first CMux group against the exact
    integer product: per-coefficient error (torus units) max and variance."""
    rng = np.random.default_rng(seed)
    c, M, L, N = p.collapse, p.M, p.l_bs, p.N
    p1 = ParamSet(p.name + "_g1", N=N, n=c, log2_beta_bs=p.log2_beta_bs, l_bs=L, collapse=c,
                  log2_beta_ks=p.log2_beta_ks, l_ks=p.l_ks, sigma_glwe=p.sigma_glwe, sigma_lwe=p.sigma_lwe, n_big=N)
    bsk1 = keys.bsk.reshape(2, 2, p.G, M, L, N)[:, :, :1].reshape(2, 2, M, L, N)
    acc0 = rng.integers(0, 2 ** 32, size=(samples, 2, N), dtype=np.uint64).astype(np.uint32)
    pk = rng.integers(0, 2 ** 32, size=(samples, c), dtype=np.uint64).astype(np.uint32)
    cen = lambda u: u.view(np.int32).astype(np.float64)
    exact = O.multiply_seq_monomial_exact(cen(acc0), cen(pk), cen(bsk1).reshape(2, 2, M, L, N).astype(np.float64),
                                          2.0 ** 32, 2 ** p.log2_beta_bs, L, N, c, 1)
    exact = (np.rint(exact).astype(np.int64) & 0xFFFFFFFF).astype(np.uint32)
    dev = torch.device("cuda", 0)
    i32 = lambda x: torch.from_numpy(np.ascontiguousarray(x).view(np.int32)).to(dev)
    lut, a = i32(acc0), i32(pk)
    out = {}
    for f in forms:
        if f == "fp64":
            ksk_a = np.zeros((p1.l_ks, p1.big, p1.n), np.uint32)
            ksk_b = np.zeros((p1.l_ks, p1.big), np.uint32)
            e = Keys.create(p1, bsk1, ksk_a, ksk_b)
            got = e.blind_rotate(a, torch.zeros(samples, dtype=torch.int32, device=dev), lut, 1)
            e.close()
        else:
            k = FP32Keys(p1, bsk1, int(f[-1]))
            got = k.chain(a, lut, 1)
            k.close()
        g = got.cpu().numpy().view(np.uint32)
        err = ((g.astype(np.int64) - exact.astype(np.int64) + 2 ** 31) % 2 ** 32) - 2 ** 31
        out[f] = {"group_err_max_log2": float(np.log2(np.abs(err).max() + 1)),
                  "group_err_var": float(np.var(err.astype(np.float64))),
                  "group_exact_fraction": float(np.mean(err == 0))}
    return out


def run(total=1_000_000, forms=FORMS, seed=303):
    p = CONFIG3
    dev = torch.device("cuda", 0)
    keys = client.keygen(p, seed)
    eng = Keys.create(p, keys.bsk, keys.ksk_a, keys.ksk_b)
    f32 = {f: FP32Keys(p, keys.bsk, int(f[-1])) for f in forms if f != "fp64"}
    rng = np.random.default_rng(seed + 1)
    tables = rng.integers(0, T_OUT // 2, size=(N_LUT, T_IN // 2))
    body = client.packed_table_lut(p.N, tables, T_OUT)
    lut = torch.zeros((1, 2, p.N), dtype=torch.int32, device=dev)
    lut[0, 1] = torch.from_numpy(body.view(np.int32)).to(dev)
    s = torch.from_numpy(keys.sk_glwe.astype(np.float64)).to(dev)
    tab = torch.from_numpy(tables).to(dev)
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed + 2)
    stats = {f: {"failures": 0, "noise_sq": 0.0, "noise_max": 0, "ms": 0.0} for f in forms}
    done = 0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    while done < total:
        B = min(CHUNK, total - done)
        m = torch.randint(0, T_IN // 2, (B,), device=dev, generator=gen)
        a = torch.randint(-2 ** 31, 2 ** 31, (B, p.N), device=dev, generator=gen, dtype=torch.int64)
        e = torch.round(torch.randn((B,), device=dev, generator=gen, dtype=torch.float64) * p.sigma_glwe)
        b = _torus((a.to(torch.float64) @ s).to(torch.int64) + m * (2 ** 32 // T_IN) + e.to(torch.int64))
        ka, kb = eng.keyswitch(a.to(torch.int32), b.to(torch.int32))
        want = tab[:, m].T
        for f in forms:
            e0.record()
            if f == "fp64":
                oa, ob = eng.cuboot_merge(ka, kb, lut, N_LUT)
            else:
                oa, ob = f32[f].cuboot_merge(ka, kb, lut, N_LUT)
            e1.record()
            torch.cuda.synchronize()
            st = stats[f]
            st["ms"] += e0.elapsed_time(e1)
            phase = _torus(ob.to(torch.int64) - (oa.to(torch.float64) @ s).to(torch.int64))
            noise = _torus(phase - want * (2 ** 32 // T_OUT))
            dec = torch.remainder(torch.round(phase.to(torch.float64) / (2 ** 32 / T_OUT)), T_OUT).to(torch.int64)
            st["failures"] += int((dec != want).sum())
            st["noise_max"] = max(st["noise_max"], int(noise.abs().max()))
            st["noise_sq"] += float((noise.to(torch.float64) ** 2).sum())
        done += B
    eng.close()
    for k in f32.values():
        k.close()
    groups = one_group_errors(p, keys, forms)
    outs = done * N_LUT
    var64 = stats["fp64"]["noise_sq"] / outs if "fp64" in stats else None
    rows = []
    for f in forms:
        st = stats[f]
        var = st["noise_sq"] / outs
        rows.append(dict(form=f, pbs=done, outputs=outs, failures=st["failures"],
                         noise_std_log2=float(np.log2(np.sqrt(var))),
                         noise_max_log2=float(np.log2(st["noise_max"] + 1)),
                         noise_var_vs_fp64=(var / var64) if var64 else None,
                         br_pbs_per_s=done / (st["ms"] * 1e-3), **groups[f]))
    return rows


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--pbs", type=int, default=1_000_000)
    ap.add_argument("--json", default=None)
    args = ap.parse_args()
    rows = run(args.pbs)
    for r in rows:
        print(json.dumps(r))
    if args.json:
        with open(args.json, "w") as fh:
            json.dump(rows, fh, indent=1)


if __name__ == "__main__":
    main()
