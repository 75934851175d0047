"""Pin the CPU oracle against golden fixtures recorded from the reference's
own Python code (tests/golden/make_golden.py), and against exact integer
arithmetic.  CPU only."""
import os

import numpy as np
import pytest

from oracle import tfhe_oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
G = np.load(os.path.join(HERE, "golden", "pbs_golden.npz"))
Q = 2.0 ** 32

# must match tests/golden/make_golden.py
PARAMS = {
    "tiny_c3": dict(q=Q, N=256, n=24, beta_bs=2 ** 7, l_bs=3, collapse=3, beta_ks=2 ** 3, l_ks=5,
                    sigma_glwe=2.0 ** 7, sigma_lwe=2.0 ** 17),
    "tiny_c2": dict(q=Q, N=512, n=16, beta_bs=2 ** 15, l_bs=2, collapse=2, beta_ks=2 ** 4, l_ks=5,
                    sigma_glwe=1.0, sigma_lwe=2.0 ** 15),
    "cfg1": dict(q=Q, N=1024, n=630, beta_bs=2 ** 7, l_bs=3, collapse=3, beta_ks=2 ** 3, l_ks=5,
                 sigma_glwe=2.0 ** 7, sigma_lwe=2.0 ** 17),
}
KEY_SEED = {"tiny_c3": 11, "tiny_c2": 12, "cfg1": 13}
INPUT_SEED = {"tiny_c3": 21, "tiny_c2": 22, "cfg1": 23}
_KEYS = {}


def keys(name):
    if name not in _KEYS:
        _KEYS[name] = O.keygen(PARAMS[name], KEY_SEED[name])
    return _KEYS[name]


def test_decomposition_golden():
    x = G["poly_x"]
    for beta, l in [(2 ** 7, 3), (2 ** 15, 2), (2 ** 3, 5), (2 ** 4, 5), (2 ** 13, 2)]:
        got = O.decomposition(x, beta, l, Q)
        assert np.array_equal(got, G[f"poly_dec_b{beta}_l{l}"]), (beta, l)


def test_decomposition_ties_half_even():
    # gamma = 2^24 at beta=2^7, l=3: x*beta hits exactly .5 at level 2, and
    # half-to-even gives [0, 64, 0] (an offset/half-up scheme gives [1,-64,0])
    d = O.decomposition(np.array([2.0 ** 24]), 2 ** 7, 3, Q)[:, 0]
    assert list(d) == [0.0, 64.0, 0.0]
    # q/2 and -q/2 keep their sign through the digits
    assert list(O.decomposition(np.array([2.0 ** 31]), 2 ** 7, 3, Q)[:, 0]) == [64.0, 0.0, 0.0]
    assert list(O.decomposition(np.array([-2.0 ** 31]), 2 ** 7, 3, Q)[:, 0]) == [-64.0, 0.0, 0.0]


def test_centered_mod_golden():
    x = G["poly_x"]
    assert np.array_equal(O.centered_mod(x * 3.0 + 2 ** 31, Q), G["poly_cmod"])


def test_fourier_golden():
    small = G["poly_small"]
    np.testing.assert_allclose(O.jax_fourier(small), G["poly_fourier"], rtol=0, atol=1e-9)
    assert np.array_equal(O.jax_inversefourier(O.jax_fourier(small)), G["poly_inverse"])
    assert np.array_equal(G["poly_inverse"], small)


def test_rotation_and_extract_golden():
    small = G["poly_small"]
    for a, row in zip(G["rot_alphas"], G["rot_out"]):
        assert np.array_equal(O.coef_rotation(small[0], a), row), a
        assert np.array_equal(O.coef_rotation_rows(small[0][None], [a])[0], row), a
    for a, row in zip(G["extract_alphas"], G["extract_out"]):
        ea, eb = O.sample_extract((small[1], small[2]), int(a))
        assert np.array_equal(np.concatenate([ea, eb]), row), a


def test_binary_vectors_and_plain_lut_golden():
    for c in (1, 2, 3, 4):
        assert np.array_equal(O.all_binary_vectors(c), G[f"binvec_{c}"])
    lut = np.stack([O.get_plain_LUT(256, 4, i, 4.0, g) for i, g in enumerate([-1.5, -0.5, 0.5, 1.5])])
    assert np.array_equal(lut, G["plain_lut_n4"])


def _inputs(name, batch):
    p = PARAMS[name]
    k = keys(name)
    rng = np.random.default_rng(INPUT_SEED[name])
    msgs = rng.integers(0, 16, size=batch)
    a, b = O.encrypt_inputs(k, msgs, p["q"] / 32, rng)
    return msgs, a, b


@pytest.mark.parametrize("name,batch,luts", [("tiny_c3", 6, (1, 4)), ("tiny_c2", 6, (1, 2)),
                                             ("cfg1", 4, (1, 4))])
def test_pbs_golden(name, batch, luts):
    p = PARAMS[name]
    k = keys(name)
    msgs, a, b = _inputs(name, batch)
    assert np.array_equal(msgs, G[f"{name}_msgs"])
    assert np.array_equal(a, G[f"{name}_in_a"]) and np.array_equal(b, G[f"{name}_in_b"])
    ksp = {"beta_ks": p["beta_ks"], "l_ks": p["l_ks"], "q": p["q"]}
    ca, cb = O.key_switch_LWE(k.ksk, (a, b), ksp)
    assert np.array_equal(ca, G[f"{name}_ks_a"]) and np.array_equal(cb, G[f"{name}_ks_b"])
    N = p["N"]
    for n_lut in luts:
        body = G[f"{name}_lut{n_lut}"]
        enc = [np.zeros((batch, N)), np.broadcast_to(body, (batch, N))]
        acc = O.BR((ca, cb), enc, k.bsk_ordered, p["q"], p["beta_bs"], p["l_bs"], N, p["collapse"],
                   k.all_rot, n_lut)
        ra, rb = O.extract_many(acc, n_lut)
        if p["beta_bs"] <= 2 ** 7:
            # FP64 products are exact here: bit-identical to the reference
            # BR returns the reference tuple (mask, body): stored as (2, B, N)
            assert np.array_equal(acc, np.moveaxis(G[f"{name}_br{n_lut}"], 0, 1))
            assert np.array_equal(ra, G[f"{name}_merge{n_lut}_a"])
            assert np.array_equal(rb, G[f"{name}_merge{n_lut}_b"])
        else:
            # FP64 rounding decides some coefficients: same pocketfft in
            # both, so still identical, but only decryption is the contract
            dec_ref = O.decrypt_LWE((G[f"{name}_merge{n_lut}_a"][:, 0], G[f"{name}_merge{n_lut}_b"][:, 0]),
                                    k.sk_glwe, {"t": 32, "q": p["q"]})
            dec = O.decrypt_LWE((ra[:, 0], rb[:, 0]), k.sk_glwe, {"t": 32, "q": p["q"]})
            assert np.array_equal(dec, dec_ref)
    body = G[f"{name}_lut1"]
    enc = [np.zeros((batch, N)), np.broadcast_to(body, (batch, N))]
    ba, bb = O.bootstrapping((ca, cb), np.stack(enc, axis=1), k.bsk_ordered, p["q"], p["beta_bs"],
                             p["l_bs"], N, p["collapse"], k.all_rot, 1)
    if p["beta_bs"] <= 2 ** 7:
        assert np.array_equal(ba, G[f"{name}_boot_a"]) and np.array_equal(bb, G[f"{name}_boot_b"])


@pytest.mark.parametrize("name", ["tiny_c3", "cfg1"])
def test_pbs_decrypts_to_step(name):
    p = PARAMS[name]
    k = keys(name)
    msgs, a, b = _inputs(name, 4 if name == "cfg1" else 6)
    ksp = {"beta_ks": p["beta_ks"], "l_ks": p["l_ks"], "q": p["q"]}
    ca, cb = O.key_switch_LWE(k.ksk, (a, b), ksp)
    assert np.array_equal(O.decrypt_LWE((ca, cb), k.sk_lwe, {"t": 32, "q": p["q"]}) % 32, msgs % 32)
    ra, rb = G[f"{name}_merge1_a"][:, 0], G[f"{name}_merge1_b"][:, 0]
    out = O.decrypt_LWE((ra, rb), k.sk_glwe, {"t": 32, "q": p["q"]})
    assert np.array_equal(out, (msgs >= 8).astype(float))


def test_fp64_br_equals_exact_at_beta_2_7():
    """The exact-integer route reproduces the reference fixture bit for bit
    when the FP64 error is below 1/2 (beta = 2^7, N = 256)."""
    name = "tiny_c3"
    p = PARAMS[name]
    k = keys(name)
    ca, cb = G[f"{name}_ks_a"], G[f"{name}_ks_b"]
    N = p["N"]
    body = G[f"{name}_lut1"]
    enc = [np.zeros((6, N)), np.broadcast_to(body, (6, N))]
    trace = []
    acc = O.BR((ca, cb), enc, k.bsk_ordered, p["q"], p["beta_bs"], p["l_bs"], N, p["collapse"],
               k.all_rot, 1, exact_bsk=k.bsk_coeff)
    assert np.array_equal(acc, np.moveaxis(G[f"{name}_br1"], 0, 1))
    ct_init = np.stack(enc, axis=1)
    O.multiply_seq_monomial_exact(ct_init, ca, k.bsk_coeff, p["q"], p["beta_bs"], p["l_bs"], N,
                                  p["collapse"], 1, fft_trace=trace)
    assert max(trace) < 0.1


def test_exact_product_matches_schoolbook():
    rng = np.random.default_rng(3)
    for n in (8, 64):
        a = rng.integers(-2 ** 14, 2 ** 14, n)
        b = rng.integers(-2 ** 31, 2 ** 31, n)
        want = np.array([v % (1 << 64) for v in O.negacyclic_mul_schoolbook(a, b)], dtype=np.uint64)
        got = O.negacyclic_mul_exact(a, b).astype(np.uint64)
        assert np.array_equal(got, want)


def test_centered_from_wide_tie_rule():
    q = 2.0 ** 32
    for x in [2 ** 31, 2 ** 31 + 2 ** 32, -2 ** 31, -2 ** 31 - 2 ** 32, 5, -5, 2 ** 32 + 7]:
        want = O.centered_mod(np.array([float(x)]), q)[0]
        got = O.centered_from_wide(np.array([x], dtype=np.int64), 32)[0]
        assert got == want, x


def test_all_rot_table_matches_reference_digest():
    import hashlib
    arr = np.ascontiguousarray(O.all_rot_possible_fourier(2048))
    np.testing.assert_array_equal(arr[[0, 1, 2047, 2048, 4095]], G["allrot2048_rows"])
    digest = np.frombuffer(hashlib.sha256(arr.tobytes()).digest(), dtype=np.uint8)
    assert np.array_equal(digest, G["allrot2048_sha256"])


G2 = np.load(os.path.join(HERE, "golden", "pbs_cfg2_golden.npz"))
CFG2 = dict(q=Q, N=2048, n=742, beta_bs=2 ** 15, l_bs=2, collapse=2, beta_ks=2 ** 4, l_ks=5,
            sigma_glwe=1.0, sigma_lwe=2.0 ** 15)


def test_pbs_golden_cfg2():
    """Config 2 (n=742, N=2048, gadget 2^15 x 2, collapse 2) against the
    reference's own key switch and cuboot_merge (tests/golden/make_golden.py
    cfg2): the key switch bit for bit; the bootstrap, where gadget 2^15
    makes both FP64 chains round, by decryption (Z_8 inputs at q/16, the step
    LUT's output at q/8) and by phase: each output within 2^27 of its value
    (the decision margin is q/16 = 2^28; measured noise ~2^25)."""
    from pbs_cases import keys as case_keys
    p = CFG2
    k = case_keys("cfg2")
    q, N = p["q"], p["N"]
    rng = np.random.default_rng(24)
    msgs = rng.integers(0, 8, size=4)
    a, b = O.encrypt_inputs(k, msgs, q / 16, rng)
    assert np.array_equal(msgs, G2["cfg2_msgs"])
    assert np.array_equal(a, G2["cfg2_in_a"]) and np.array_equal(b, G2["cfg2_in_b"])
    ca, cb = O.key_switch_LWE(k.ksk, (a, b), {"beta_ks": p["beta_ks"], "l_ks": p["l_ks"], "q": q})
    assert np.array_equal(ca, G2["cfg2_ks_a"]) and np.array_equal(cb, G2["cfg2_ks_b"])
    body = G2["cfg2_lut1"]
    enc = [np.zeros((4, N)), np.broadcast_to(body, (4, N))]
    acc = O.BR((ca, cb), enc, k.bsk_ordered, q, p["beta_bs"], p["l_bs"], N, p["collapse"], k.all_rot, 1)
    ra, rb = O.extract_many(acc, 1)
    want = (msgs >= 4).astype(np.float64)
    sk = k.sk_glwe.astype(np.float64)
    for oa, ob in ((ra, rb), (G2["cfg2_merge1_a"], G2["cfg2_merge1_b"])):
        assert np.array_equal(O.decrypt_LWE((oa[:, 0], ob[:, 0]), k.sk_glwe, {"t": 8, "q": q}), want)
        ph = np.mod(np.asarray(ob[:, 0, 0], np.float64) - np.asarray(oa[:, 0], np.float64) @ sk + q / 2, q) - q / 2
        assert np.abs(ph - want * q / 8).max() <= 2.0 ** 27
