"""Host-side logic of the reference-surface mirror, checked on the CPU
against the oracle: rotation indices (cuTFHE/multiply.py:67-79), pattern
order, BSK reshape/permute, torus conversions and parameter sets."""
import numpy as np
import pytest
import torch

from oracle import tfhe_oracle as O
from tfhe_b200 import ops
from tfhe_b200.engine import centred, to_u32, u32_as_i32
from tfhe_b200.params import ALL, CONFIG1, CONFIG2


def test_binary_vectors_match_reference_order():
    for c in (1, 2, 3, 4):
        assert np.array_equal(ops.all_binary_vectors(c).numpy(), O.all_binary_vectors(c))


@pytest.mark.parametrize("collapse,degree,n_lut", [(3, 1024, 1), (3, 1024, 4), (2, 2048, 1), (1, 256, 2),
                                                   (4, 4096, 8)])
def test_rotation_indices_match_oracle(collapse, degree, n_lut):
    rng = np.random.default_rng(collapse * 100 + n_lut)
    q = 2.0 ** 32
    pk = rng.integers(-2 ** 31, 2 ** 31, size=(7, 12 * collapse)).astype(np.float64)
    pk[0, :collapse] = 2.0 ** 31                      # the +q/2 representative
    pk[1, :collapse] = -2.0 ** 31
    pk[2, 0] = q / (4 * degree) * n_lut                # exact rounding ties
    pk[3, 0] = 3 * q / (4 * degree) * n_lut
    want = O.rotation_indices(pk, collapse, degree, q, n_lut)
    got = ops.rotation_indices(torch.from_numpy(pk), collapse, degree, q, n_lut).numpy()
    assert np.array_equal(got, want)


def test_torus_conversions():
    x = np.array([0.0, 1.0, -1.0, 2.0 ** 31, -2.0 ** 31, 2.0 ** 31 - 1, 5 * 2.0 ** 32 + 3])
    u = to_u32(x)
    assert list(u) == [0, 1, 0xFFFFFFFF, 0x80000000, 0x80000000, 0x7FFFFFFF, 3]
    assert list(centred(u)) == [0, 1, -1, -2 ** 31, -2 ** 31, 2 ** 31 - 1, 3]
    assert np.array_equal(u32_as_i32(u).view(np.uint32), u)


def test_param_sets():
    assert CONFIG1.G == 210 and CONFIG1.M == 8 and CONFIG1.big == 1024
    assert CONFIG2.G == 371 and CONFIG2.M == 4 and CONFIG2.big == 2048
    assert CONFIG1.bsk_bytes_fp64() == 165_150_720
    assert CONFIG2.bsk_bytes_fp64() == 194_510_848
    for p in ALL.values():
        assert p.n % p.collapse == 0
        d = p.oracle_dict()
        assert d["beta_bs"] == 2 ** p.log2_beta_bs and d["q"] == 2.0 ** 32


def test_bsk_permutation_matches_reference_reshape():
    """The mirror's reshape/permute of bsk_ordered equals multiply.py:81-86."""
    rng = np.random.default_rng(0)
    G, M, L, d = 5, 4, 2, 8
    bo = rng.standard_normal((2, 2, L, G * M, d)) + 1j * rng.standard_normal((2, 2, L, G * M, d))
    want = O.bsk_reshape(bo, G, 2)
    t = torch.from_numpy(bo)
    shape = list(t.shape)
    shape[3] = G
    shape.insert(4, M)
    got = t.reshape(shape).permute(3, 0, 2, 1, 4, 5).contiguous().numpy()
    assert np.array_equal(got, want)
