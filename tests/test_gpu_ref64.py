"""The mul_bootstrap drop-in (tfhe_mul_bootstrap through ops.py) at the
reference's own parameter set: q = 2^64 held in float64, N = 2048, n = 702,
gadget 2^13 x 2, collapse 3 (parameters_crypto.py:6-32), against fixtures
recorded from the reference's code (tests/golden/make_ref64_golden.py).

The reference's float64 arithmetic is inexact at q = 2^64, and the engine's
FP64 FFT rounds differently from the one the fixtures were recorded with, so
the bar is the rounding bound of test_ref64.py:
  - one CMux group: |engine - reference| <= 2^36 per coefficient;
  - the 234-group chain (cuboot_merge: chain, rotation by -b~, extraction):
    every output decrypts to the LUT's value with noise <= 2^50
    (a decryption fails at 2^59)."""
import os

import numpy as np
import pytest
import torch

import ref64_cases as RC
from oracle import tfhe_oracle as O

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU runs deselect -m gpu
    pytest.skip("needs a CUDA device", allow_module_level=True)

from tfhe_b200 import ops  # noqa: E402

FX = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref64_golden.npz"))
ONE_GROUP_TOL = 2.0 ** 36
NOISE_TOL = 2.0 ** 50
DELTA = 2.0 ** 60


def cuda(x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def test_dropin_one_group_at_q64_within_rounding_of_reference():
    c = RC.case()
    p = O.REF64
    g1 = RC.one_group_inputs(c)
    got = ops.multiply_seq_monomial(cuda(g1["acc"]), cuda(g1["pk"]), cuda(g1["bsk1"]), 64, 13, p["l_bs"], p["N"],
                                    p["collapse"], cuda(c["all_rot"]), 1).cpu().numpy()
    d = np.abs(O.centered_mod(got - FX["group1_acc"], p["q"]))
    print(f"q=2^64 one group: max |engine - reference| = 2^{np.log2(d.max() + 1):.2f}")
    assert d.max() <= ONE_GROUP_TOL


def test_dropin_chain_at_q64_decrypts_like_reference():
    c = RC.case()
    p = O.REF64
    bsk = cuda(c["bsk_ordered"])
    ma, mb = ops.cuboot_merge((cuda(c["lwe_a"]), cuda(c["lwe_b"][:, None])),
                              [cuda(c["luts"][0]), cuda(c["luts"][1])], bsk, p["q"], p["beta_bs"], p["l_bs"],
                              p["N"], p["collapse"], cuda(c["all_rot"]), 1)
    ma, mb = ma.cpu().numpy(), mb.cpu().numpy()
    ph = O.phase_q64(ma[:, 0], mb[:, 0, 0], c["sk_glwe"]).astype(np.float64)
    ph_ref = O.phase_q64(FX["merge_a"][:, 0], FX["merge_b"][:, 0, 0], c["sk_glwe"]).astype(np.float64)
    want = (c["msgs"] >= 4).astype(np.float64)
    noise = np.abs(ph - want * DELTA)
    print(f"q=2^64 chain: engine noise 2^{np.log2(noise.max() + 1):.2f}, reference noise "
          f"2^{np.log2(np.abs(ph_ref - want * DELTA).max() + 1):.2f}")
    assert np.array_equal(np.rint(ph / DELTA), want)
    assert noise.max() <= NOISE_TOL
