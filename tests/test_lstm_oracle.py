"""CPU checks of the Spike-LSTM operator statements: each one decrypts to
the plaintext computation it stands for."""
import numpy as np

from lstm_cases import BETA_X, GAL_L, GAL_LOG2_BETA, PK_L, PK_LOG2_BETA, cen, layer_material
from oracle import lstm_oracle as LO
from tfhe_b200 import client


def _centred(x):
    return ((np.asarray(x, dtype=np.int64) + 2 ** 31) % 2 ** 32) - 2 ** 31


def test_automorphism_statements_agree():
    rng = np.random.default_rng(0)
    poly = rng.integers(-100, 100, size=(3, 64))
    for k in (3, 5, 65, 127):
        assert np.array_equal(LO.apply_automorphism(poly, k), client.automorphism(poly, k))


def test_linear_decrypts_to_inner_product():
    m = layer_material()
    sk, N = m["sk"], m["p"]["N"]
    rng = np.random.default_rng(1)
    msg = np.zeros(N, dtype=np.int64)
    msg[:12] = rng.integers(-2, 3, size=12)
    a, b = client.encrypt_rlwe(msg * int(BETA_X), sk, 1.0, rng)
    W = rng.integers(-7, 8, size=(12, 5))
    B = rng.integers(-3, 4, size=5) * int(BETA_X)
    kern, bias = LO.linear_kernel_polynomial(W, B, np.ones(5), N)
    la, lb = LO.linear(kern, bias, (cen(a), cen(b)))
    phase = _centred(lb - la @ sk)
    want = (W.T @ msg[:12]) * int(BETA_X) + B
    assert np.max(np.abs(_centred(phase - want))) < 2 ** 12


def test_trace_decrypts_to_constant_polynomial():
    m = layer_material()
    sk, N = m["sk"], m["p"]["N"]
    rng = np.random.default_rng(2)
    vals = rng.integers(-3, 4, size=4) * int(BETA_X)
    a, b = client._lwe_encrypt(vals, sk, 1.0, rng)
    A, B = LO.pack_lwe_to_rlwe(cen(a), cen(b), cen(m["galois"]), GAL_LOG2_BETA, GAL_L)
    phase = client.rlwe_phase(A & 0xFFFFFFFF, B & 0xFFFFFFFF, sk)
    want = np.zeros((4, N), dtype=np.int64)
    want[:, 0] = vals
    assert np.max(np.abs(_centred(phase - want))) < 2 ** 17


def test_packing_decrypts_to_coefficients():
    m = layer_material()
    sk, N = m["sk"], m["p"]["N"]
    rng = np.random.default_rng(3)
    T = 10
    vals = rng.integers(-3, 4, size=T) * int(BETA_X)
    a, b = client._lwe_encrypt(vals, sk, 1.0, rng)
    pa, pb = LO.packing(cen(a), cen(b), m["layer"]["ksp_a"], m["layer"]["ksp_b"], PK_LOG2_BETA, PK_L, N)
    phase = client.rlwe_phase(pa & 0xFFFFFFFF, pb & 0xFFFFFFFF, sk)
    want = np.zeros(N, dtype=np.int64)
    want[:T] = vals
    assert np.max(np.abs(_centred(phase - want))) < 2 ** 18


def test_plain_lut_is_packed_step():
    N, n_lut = 256, 2
    lut = LO.get_plain_LUT(N, n_lut, 1, 1.0, 0.25)
    unrot = LO.O.coef_rotation(lut, N // 2)
    assert np.all(unrot[0::2] == 0)
    part = np.linspace(-1.0, 1.0, N // 2, endpoint=False)
    assert np.array_equal(unrot[1::2], (part >= 0.25).astype(float))
