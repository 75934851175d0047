"""10^6 programmable bootstraps with 4 packed LUTs each at n=630, N=1024,
gadget 2^7 x 3, collapse 3 (Z_4 messages with a padding bit, outputs in Z_4
at scale q/8): every one of the 4 x 10^6 outputs is decrypted and must be
right.  Encryption and decryption run on the GPU in float64 (sums of at
most 1024 products of 32-bit values by bits stay below 2^53, so they are
exact)."""
import json
import os

import numpy as np
import pytest
import torch

from tfhe_b200 import client
from tfhe_b200.engine import Keys
from tfhe_b200.params import CONFIG3

pytestmark = pytest.mark.gpu

TOTAL = 1_000_000
CHUNK = 16384
N_LUT = 4
T_IN = 8
T_OUT = 8


def _torus(x):
    """int64 -> centred int64 modulo 2^32"""
    return ((x + 2 ** 31) & 0xFFFFFFFF) - 2 ** 31


def test_million_pbs_four_luts_zero_failures():
    p = CONFIG3
    dev = torch.device("cuda", 0)
    keys = client.keygen(p, 303)
    eng = Keys.create(p, keys.bsk, keys.ksk_a, keys.ksk_b)
    rng = np.random.default_rng(304)
    tables = rng.integers(0, T_OUT // 2, size=(N_LUT, T_IN // 2))
    body = client.packed_table_lut(p.N, tables, T_OUT)
    lut = torch.zeros((1, 2, p.N), dtype=torch.int32, device=dev)
    lut[0, 1] = torch.from_numpy(body.view(np.int32)).to(dev)
    s = torch.from_numpy(keys.sk_glwe.astype(np.float64)).to(dev)
    tab = torch.from_numpy(tables).to(dev)
    gen = torch.Generator(device=dev)
    gen.manual_seed(305)
    done = failures = 0
    noise_max = 0
    noise_sq = 0.0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    pbs_ms = 0.0
    while done < TOTAL:
        B = CHUNK
        m = torch.randint(0, T_IN // 2, (B,), device=dev, generator=gen)
        a = torch.randint(-2 ** 31, 2 ** 31, (B, p.N), device=dev, generator=gen, dtype=torch.int64)
        e = torch.round(torch.randn((B,), device=dev, generator=gen, dtype=torch.float64) * p.sigma_glwe)
        dot = (a.to(torch.float64) @ s).to(torch.int64)
        b = _torus(dot + m * (2 ** 32 // T_IN) + e.to(torch.int64))
        a32 = a.to(torch.int32)
        b32 = b.to(torch.int32)
        e0.record()
        oa, ob = eng.pbs(a32, b32, lut, N_LUT)
        e1.record()
        torch.cuda.synchronize()
        pbs_ms += e0.elapsed_time(e1)
        phase = _torus(ob.to(torch.int64) - (oa.to(torch.float64) @ s).to(torch.int64))      # (B, n_lut)
        want = tab[:, m].T                                                                    # (B, n_lut)
        noise = _torus(phase - want * (2 ** 32 // T_OUT))
        dec = torch.remainder(torch.round(phase.to(torch.float64) / (2 ** 32 / T_OUT)), T_OUT).to(torch.int64)
        failures += int((dec != want).sum())
        noise_max = max(noise_max, int(noise.abs().max()))
        noise_sq += float((noise.to(torch.float64) ** 2).sum())
        done += B
    eng.close()
    summary = {"pbs": done, "outputs": done * N_LUT, "failures": failures,
               "output_noise_std_log2": float(np.log2(np.sqrt(noise_sq / (done * N_LUT)))),
               "output_noise_max_log2": float(np.log2(max(noise_max, 1))),
               "threshold_log2": float(np.log2(2 ** 32 / (2 * T_OUT))),
               "pbs_per_s": done / (pbs_ms * 1e-3)}
    out_path = os.environ.get("TFHE_CONFIG3_SUMMARY")   # optional: where to keep the summary
    if out_path:
        with open(out_path, "w") as fh:
            json.dump(summary, fh)
    print(summary)
    assert failures == 0, summary
