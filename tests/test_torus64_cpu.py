"""The 2^64-torus client and oracle on CPU: exact encryption, exact gadget
digits against Python integers, key switching, pack_lwe_to_rlwe, packing
and the blind rotation checked by decryption on small parameters."""
import numpy as np
import pytest

from oracle import torus64_oracle as T64
from tfhe_b200 import client64 as C64

SMALL = C64.Params64("small64", N=256, n=12, log2_beta_bs=13, l_bs=2, collapse=3, log2_beta_ks=4, l_ks=5,
                     sigma_glwe=2.0 ** 17, sigma_lwe=2.0 ** 40)


def test_rne_shift_matches_python_integers():
    rng = np.random.default_rng(1)
    xs = np.concatenate([rng.integers(-2 ** 63, 2 ** 63, size=2000, dtype=np.int64),
                         np.array([-2 ** 63, 2 ** 63 - 1, 0, 1, -1, 2 ** 51, -2 ** 51, 3 * 2 ** 50, -3 * 2 ** 50,
                                   2 ** 50, 5 * 2 ** 50], dtype=np.int64)])
    for s in (1, 4, 13, 51, 60, 63):
        d, r = T64.rne_shift(xs, s)
        for x, dd, rr in zip(xs.tolist(), d.tolist(), r.tolist()):
            q, rem = divmod(x, 1 << s)
            half = 1 << (s - 1)
            if rem > half or (rem == half and q % 2 == 1):
                q, rem = q + 1, rem - (1 << s)
            assert (dd, rr) == (q, rem), (x, s)


def test_decomposition_reconstructs_top_bits():
    rng = np.random.default_rng(2)
    x = rng.integers(0, 2 ** 64, size=500, dtype=np.uint64)
    for lb, l in ((4, 5), (8, 4), (13, 2)):
        d = T64.decomposition(x, lb, l)
        assert np.abs(d).max() <= 2 ** (lb - 1)
        rec = sum(d[j].astype(np.uint64) << np.uint64(64 - (j + 1) * lb) for j in range(l))
        err = T64.centred(x - rec)
        assert np.abs(err.astype(np.float64)).max() <= 2.0 ** (64 - l * lb - 1)


def test_client_encryptions_decrypt_exactly():
    rng = np.random.default_rng(3)
    sk = rng.integers(0, 2, size=256)
    m = rng.integers(-2 ** 62, 2 ** 62, size=(3, 256))
    a, b = C64.encrypt_rlwe(m, sk, 2.0 ** 17, rng)
    ph = C64.rlwe_phase(a, b, sk)
    assert np.abs((ph - m).astype(np.float64)).max() < 2 ** 21
    msg = rng.integers(-2 ** 62, 2 ** 62, size=7)
    a, b = C64.encrypt_lwe(msg, sk, 2.0 ** 20, rng)
    assert np.abs((C64.phase(a, b, sk) - msg).astype(np.float64)).max() < 2 ** 24
    # the 16-bit limb product against a schoolbook product on Python integers
    x = rng.integers(0, 2 ** 64, size=(2, 16), dtype=np.uint64)
    s = rng.integers(0, 2, size=16)
    got = C64.negacyclic_mul_binary(x, s)
    for r in range(2):
        want = [0] * 16
        for i in range(16):
            for j in range(16):
                if s[j]:
                    k = i + j
                    if k >= 16:
                        want[k - 16] -= int(x[r, i])
                    else:
                        want[k] += int(x[r, i])
        assert [w % 2 ** 64 for w in want] == [int(v) for v in got[r]]


def test_negacyclic_mod64_matches_schoolbook():
    rng = np.random.default_rng(4)
    x = rng.integers(0, 2 ** 64, size=16, dtype=np.uint64)
    y = rng.integers(-2 ** 60, 2 ** 60, size=16)
    got = T64.negacyclic_mod64(x, y)
    want = [0] * 16
    for i in range(16):
        for j in range(16):
            k = i + j
            v = int(x[i]) * int(y[j])
            if k >= 16:
                want[k - 16] -= v
            else:
                want[k] += v
    assert [w % 2 ** 64 for w in want] == [int(v) for v in got]


@pytest.fixture(scope="module")
def small_keys():
    return C64.keygen(SMALL, 5)


def test_key_switch_keeps_the_phase(small_keys):
    k = small_keys
    rng = np.random.default_rng(6)
    msg = (rng.integers(0, 8, size=9).astype(np.uint64) << np.uint64(60))
    a, b = C64.encrypt_lwe(msg, k.sk_glwe, 2.0 ** 20, rng)
    ka, kb = T64.key_switch(k.ksk, a, b, SMALL.log2_beta_ks, SMALL.l_ks)
    err = (C64.phase(ka, kb, k.sk_lwe) - C64.phase(a, b, k.sk_glwe)).astype(np.float64)
    assert np.abs(err).max() < 2.0 ** 52


def test_pbs_evaluates_the_lut(small_keys):
    k = small_keys
    p = SMALL
    rng = np.random.default_rng(7)
    msgs = rng.integers(0, 8, size=6)
    a, b = C64.encrypt_lwe(msgs.astype(np.uint64) << np.uint64(60), k.sk_glwe, 2.0 ** 20, rng)
    from oracle import tfhe_oracle as O
    body = O.step_lut(p.N, 8, 4, 2.0 ** 60).astype(np.int64)
    lut = np.stack([np.zeros(p.N, np.int64), body])[None]
    keys = {"params": p, "ksk": k.ksk, "bsk_grouped": C64.bsk_fourier_grouped(k.bsk, p), "rot": C64.monomial_fourier(p.N)}
    oa, ob = T64.pbs(keys, a, b, lut, 1)
    ph = C64.phase(oa[:, 0], ob[:, 0], k.sk_glwe).astype(np.float64)
    assert np.array_equal(np.rint(ph / 2.0 ** 60), (msgs >= 4).astype(float))


def test_trace_and_packing_keep_phases():
    rng = np.random.default_rng(8)
    N = 256
    sk = rng.integers(0, 2, size=N)
    gal = C64.galois_keys(sk, 8, 5, 2.0 ** 17, rng)
    msg = rng.integers(-2 ** 50, 2 ** 50, size=3) << 8
    a, b = C64.encrypt_lwe(msg, sk, 2.0 ** 17, rng)
    A, B = T64.pack_lwe_to_rlwe(a, b, gal, 8, 5)
    ph = C64.rlwe_phase(A, B, sk)
    # the trace multiplies by N what the modulus switch divided by N; the
    # gadget's dropped 24 bits enter every step and double at coefficient 0
    # in each later step (expected ~2^34 here)
    assert np.abs((ph[:, 0] - msg).astype(np.float64)).max() < 2.0 ** 38
    ksp = C64.packing_key(sk, sk, 8, 4, 2.0 ** 17, rng)
    T = 5
    msg2 = rng.integers(-2 ** 60, 2 ** 60, size=T)
    a2, b2 = C64.encrypt_lwe(msg2, sk, 2.0 ** 17, rng)
    pa, pb = T64.packing(a2, b2, ksp, 8, 4, N)
    ph2 = C64.rlwe_phase(pa, pb, sk)
    assert np.abs((ph2[:T] - msg2).astype(np.float64)).max() < 2.0 ** 45
