"""The oracle at the reference's own parameter set (q = 2^64 held in
float64, N = 2048, n = 702, gadget 2^13 x 2, collapse 3) against fixtures
recorded from the reference's code (tests/golden/make_ref64_golden.py).

At q = 2^64 the reference's float64 arithmetic rounds, so two statements of
it that only sum in a different order (here: the oracle's einsum loop
against the reference's einsum, both with numpy's FFT) agree within a
rounding bound rather than bit for bit:
  - one CMux group: |difference| <= 2^36 per coefficient (measured 2^31.7);
  - the 234-group chain: the digit sequences part after the first rounding
    difference, so the outputs are compared as decryptions: every output
    decrypts to the LUT's value, with noise (phase - m q/16) <= 2^50
    (measured 2^44-2^46; a decryption fails at 2^59).
CPU only."""
import os

import numpy as np

import ref64_cases as RC
from oracle import tfhe_oracle as O

FX = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref64_golden.npz"))
ONE_GROUP_TOL = 2.0 ** 36
NOISE_TOL = 2.0 ** 50
DELTA = 2.0 ** 60


def check_outputs(a, b, c):
    """a (B, N), b (B,) float64 LWEs under the GLWE key: decrypt to the step
    LUT's value with noise within NOISE_TOL."""
    ph = O.phase_q64(a, b, c["sk_glwe"]).astype(np.float64)
    want = (c["msgs"] >= 4).astype(np.float64)
    assert np.array_equal(np.rint(ph / DELTA), want), ph / DELTA
    assert np.abs(ph - want * DELTA).max() <= NOISE_TOL


def test_ref64_fixture_decrypts():
    c = RC.case()
    check_outputs(FX["merge_a"][:, 0], FX["merge_b"][:, 0, 0], c)


def test_oracle_one_group_within_rounding_of_reference():
    c = RC.case()
    p = O.REF64
    g1 = RC.one_group_inputs(c)
    got = O.multiply_seq_monomial(g1["acc"], g1["pk"], g1["bsk1"], p["q"], p["beta_bs"], p["l_bs"], p["N"],
                                  p["collapse"], c["all_rot"], 1)
    d = O.centered_mod(got - FX["group1_acc"], p["q"])
    assert np.abs(d).max() <= ONE_GROUP_TOL


def test_oracle_chain_decrypts_like_reference():
    c = RC.case()
    p = O.REF64
    ma, mb = O.cuboot_merge((c["lwe_a"], c["lwe_b"][:, None]), c["luts"], c["bsk_ordered"], p["q"], p["beta_bs"],
                            p["l_bs"], p["N"], p["collapse"], c["all_rot"], 1)
    check_outputs(ma[:, 0], mb[:, 0, 0], c)
