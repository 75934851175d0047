"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Integer stages (key switching, digits, rotation indices, rotations,
extraction) must be bit-exact.  The FP64 external product is bit-exact
against the oracle whenever its rounding error stays below 1/2 (beta <= 2^7
here: measured max error 0.03); with beta = 2^15 it is compared with the
exact integer product within a stated bound, and by decryption."""
import numpy as np
import pytest
import torch

from oracle import tfhe_oracle as O
from pbs_cases import PARAMS, canon, inputs, keys, ks_params, many_lut_body, step_body

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU runs deselect -m gpu
    pytest.skip("needs a CUDA device", allow_module_level=True)

from tfhe_b200 import TFHEError, ops  # noqa: E402
from tfhe_b200.engine import Keys, centred, device_u32, sample_extract  # noqa: E402
from tfhe_b200.params import ParamSet  # noqa: E402

# FFT rounding bound used where the FP64 product is not exact (beta = 2^15):
# |engine - exact| <= FFT_TOL units of q/2^32 per coefficient
FFT_TOL = 64


def pset(name):
    p = PARAMS[name]
    lg = lambda v: int(round(np.log2(v)))
    return ParamSet(name, N=p["N"], n=p["n"], log2_beta_bs=lg(p["beta_bs"]), l_bs=p["l_bs"],
                    collapse=p["collapse"], log2_beta_ks=lg(p["beta_ks"]), l_ks=p["l_ks"],
                    sigma_glwe=p["sigma_glwe"], sigma_lwe=p["sigma_lwe"])


_ENG = {}


def engine(name):
    if name not in _ENG:
        k = keys(name)
        _ENG[name] = Keys.create(pset(name), k.bsk_coeff, k.ksk[0], k.ksk[1].reshape(k.ksk[1].shape[:2]))
    return _ENG[name]


def u32(x):
    return (np.rint(np.asarray(x, dtype=np.float64)).astype(np.int64) & 0xFFFFFFFF).astype(np.uint32)


def host_u32(t):
    return t.cpu().numpy().view(np.uint32)


def torus_dist(a, b):
    """|a - b| on Z/2^32 (elementwise, as int64)"""
    d = (u32(a).astype(np.int64) - u32(b).astype(np.int64)) & 0xFFFFFFFF
    return np.minimum(d, 2 ** 32 - d)


@pytest.mark.parametrize("name", ["tiny_c3", "tiny_c2", "cfg1", "cfg2"])
def test_keyswitch_bit_exact(name):
    k = keys(name)
    msgs, a, b = inputs(name, 37)
    ra, rb = O.key_switch_LWE(k.ksk, (a, b), ks_params(name))
    ea, eb = engine(name).keyswitch(device_u32(a), device_u32(b.reshape(-1)))
    assert np.array_equal(host_u32(ea), u32(ra))
    assert np.array_equal(host_u32(eb), u32(rb.reshape(-1)))


@pytest.mark.parametrize("name,batch,n_lut", [("tiny_c3", 9, 1), ("tiny_c3", 5, 4), ("cfg1", 6, 1),
                                              ("cfg1", 5, 4)])
def test_blind_rotate_bit_exact(name, batch, n_lut):
    """BR (schemas/RLWE_jax.py:305-315) at beta = 2^7: bit-exact."""
    p = PARAMS[name]
    k = keys(name)
    msgs, a, b = inputs(name, batch)
    ca, cb = O.key_switch_LWE(k.ksk, (a, b), ks_params(name))
    body = step_body(name) if n_lut == 1 else many_lut_body(name, n_lut)
    enc = [np.zeros((batch, p["N"])), np.broadcast_to(body, (batch, p["N"]))]
    want = O.BR((ca, cb), enc, k.bsk_ordered, p["q"], p["beta_bs"], p["l_bs"], p["N"], p["collapse"],
                k.all_rot, n_lut)
    lut = device_u32(np.stack([np.zeros(p["N"]), body])[None])
    acc = engine(name).blind_rotate(device_u32(ca), device_u32(cb.reshape(-1)), lut, n_lut=n_lut)
    assert np.array_equal(host_u32(acc), u32(want))


@pytest.mark.parametrize("name,batch", [("tiny_c3", 7), ("cfg1", 12)])
def test_pbs_bit_exact_and_decrypts(name, batch):
    """tfhe_pbs = cuboot_merge(key_switch_LWE(h)) (activation.py:148-162)."""
    p = PARAMS[name]
    k = keys(name)
    msgs, a, b = inputs(name, batch)
    ca, cb = O.key_switch_LWE(k.ksk, (a, b), ks_params(name))
    body = step_body(name)
    enc = [np.zeros((batch, p["N"])), np.broadcast_to(body, (batch, p["N"]))]
    wa, wb = O.cuboot_merge((ca, cb), enc, k.bsk_ordered, p["q"], p["beta_bs"], p["l_bs"], p["N"],
                            p["collapse"], k.all_rot, 1)
    lut = device_u32(np.stack([np.zeros(p["N"]), body])[None])
    oa, ob = engine(name).pbs(device_u32(a), device_u32(b.reshape(-1)), lut, n_lut=1)
    assert np.array_equal(host_u32(oa), u32(wa))
    assert np.array_equal(host_u32(ob), u32(wb[..., 0]))
    dec = O.decrypt_LWE((centred(host_u32(oa)[:, 0]), centred(host_u32(ob)[:, 0])), k.sk_glwe,
                        {"t": 32, "q": p["q"]})
    want = O.decrypt_LWE((wa[:, 0], wb[:, 0]), k.sk_glwe, {"t": 32, "q": p["q"]})
    assert np.array_equal(dec, want)


def test_pbs_per_ciphertext_luts_and_ragged_batches():
    """lut_count == batch, batch sizes around the CTA width, batch 1 and 0."""
    name = "tiny_c3"
    p = PARAMS[name]
    k = keys(name)
    eng = engine(name)
    rng = np.random.default_rng(7)
    for batch in (1, 2, 15, 16, 17, 33):
        msgs, a, b = inputs(name, batch, seed_offset=batch)
        bodies = canon(rng.integers(-2 ** 31, 2 ** 31, size=(batch, p["N"])))
        masks = canon(rng.integers(-2 ** 31, 2 ** 31, size=(batch, p["N"])))
        ca, cb = O.key_switch_LWE(k.ksk, (a, b), ks_params(name))
        wa, wb = O.cuboot_merge((ca, cb), [masks, bodies], k.bsk_ordered, p["q"], p["beta_bs"], p["l_bs"],
                                p["N"], p["collapse"], k.all_rot, 2)
        lut = device_u32(np.stack([masks, bodies], axis=1))
        oa, ob = eng.pbs(device_u32(a), device_u32(b.reshape(-1)), lut, n_lut=2)
        assert np.array_equal(host_u32(oa), u32(wa)), batch
        assert np.array_equal(host_u32(ob), u32(wb[..., 0])), batch
    empty = torch.empty((0, p["N"]), dtype=torch.int32, device="cuda")
    oa, ob = eng.pbs(empty, torch.empty((0,), dtype=torch.int32, device="cuda"),
                     device_u32(np.zeros((1, 2, p["N"]))), n_lut=1)
    assert oa.shape == (0, 1, p["N"]) and ob.shape == (0, 1)


@pytest.mark.parametrize("name,batch", [("tiny_c2", 6), ("cfg2", 3)])
def test_beta15_against_exact_product(name, batch):
    """beta = 2^15: the FP64 product is not exact; compare with the exact
    integer chain and with the decryptions."""
    p = PARAMS[name]
    k = keys(name)
    msgs, a, b = inputs(name, batch, t=16)
    ca, cb = O.key_switch_LWE(k.ksk, (a, b), ks_params(name))
    body = step_body(name, t=16)
    enc = [np.zeros((batch, p["N"])), np.broadcast_to(body, (batch, p["N"]))]
    exact = O.BR((ca, cb), enc, k.bsk_ordered, p["q"], p["beta_bs"], p["l_bs"], p["N"], p["collapse"],
                 k.all_rot, 1, exact_bsk=k.bsk_coeff)
    lut = device_u32(np.stack([np.zeros(p["N"]), body])[None])
    acc = host_u32(engine(name).blind_rotate(device_u32(ca), device_u32(cb.reshape(-1)), lut))
    # a single-group error feeds later digits, so compare phases: decrypt
    # the extracted LWEs of both and compare messages and noise
    ea, eb = O.extract_many(centred(acc).astype(np.float64), 1)
    xa, xb = O.extract_many(exact, 1)
    sk = k.sk_glwe
    dec_e = O.decrypt_LWE((ea[:, 0], eb[:, 0]), sk, {"t": 16, "q": p["q"]})
    dec_x = O.decrypt_LWE((xa[:, 0], xb[:, 0]), sk, {"t": 16, "q": p["q"]})
    assert np.array_equal(dec_e, dec_x)
    assert np.array_equal(dec_x, (msgs >= 4).astype(float))


@pytest.mark.parametrize("name", ["tiny_c3", "tiny_c2", "c1_N128", "c4_N4096", "cfg1", "cfg2"])
def test_one_group_against_exact(name):
    """One CMux group through tfhe_mul_bootstrap (reference layout) against
    the exact integer product: max error bounded, bit-exact when beta <= 2^8."""
    p = PARAMS[name]
    k = keys(name)
    c = p["collapse"]
    batch = 4
    rng = np.random.default_rng(99)
    acc0 = canon(rng.integers(-2 ** 31, 2 ** 31, size=(batch, 2, p["N"])))
    pk = canon(rng.integers(-2 ** 31, 2 ** 31, size=(batch, c)))
    # keys restricted to the first group
    G = p["n"] // c
    M = 2 ** c
    bsk1 = k.bsk_ordered.reshape(2, 2, p["l_bs"], G, M, p["N"] // 2)[:, :, :, :1].reshape(
        2, 2, p["l_bs"], M, p["N"] // 2)
    coeff1 = k.bsk_coeff.reshape(2, 2, G, M, p["l_bs"], p["N"])[:, :, :1].reshape(2, 2, M, p["l_bs"], p["N"])
    exact = O.multiply_seq_monomial_exact(acc0, pk, coeff1, p["q"], p["beta_bs"], p["l_bs"], p["N"], c, 1)
    got = ops.multiply_seq_monomial(torch.from_numpy(acc0).cuda(), torch.from_numpy(pk).cuda(),
                                    torch.from_numpy(bsk1).cuda(), 32, int(np.log2(p["beta_bs"])), p["l_bs"],
                                    p["N"], c, torch.from_numpy(k.all_rot).cuda(), 1).cpu().numpy()
    err = torus_dist(got, exact)
    if p["beta_bs"] <= 2 ** 8:
        assert err.max() == 0
        assert np.array_equal(got, exact)          # incl. the +-q/2 representative
    assert err.max() <= FFT_TOL, err.max()


@pytest.mark.parametrize("name,batch", [("tiny_c3", 5), ("cfg1", 3)])
def test_mul_bootstrap_dropin_matches_reference_path(name, batch):
    """tfhe_mul_bootstrap on reference buffers == multiply_seq_monomial of
    the oracle (float64 values, +-q/2 representatives included)."""
    p = PARAMS[name]
    k = keys(name)
    msgs, a, b = inputs(name, batch)
    ca, cb = O.key_switch_LWE(k.ksk, (a, b), ks_params(name))
    body = step_body(name)
    ct = np.stack([np.zeros((batch, p["N"])), np.broadcast_to(body, (batch, p["N"]))], axis=1)
    want = O.multiply_seq_monomial(ct, ca, k.bsk_ordered, p["q"], p["beta_bs"], p["l_bs"], p["N"],
                                   p["collapse"], k.all_rot, 1)
    got = ops.multiply_seq_monomial(torch.from_numpy(ct).cuda(), torch.from_numpy(ca).cuda(),
                                    torch.from_numpy(k.bsk_ordered).cuda(), 32, int(np.log2(p["beta_bs"])),
                                    p["l_bs"], p["N"], p["collapse"], torch.from_numpy(k.all_rot).cuda(), 1)
    assert np.array_equal(got.cpu().numpy(), want)
    # broadcast ACC (ct_init of 2N elements, stride 0)
    got1 = ops.multiply_seq_monomial(torch.from_numpy(ct[:1]).cuda(), torch.from_numpy(ca).cuda(),
                                     torch.from_numpy(k.bsk_ordered).cuda(), 32, int(np.log2(p["beta_bs"])),
                                     p["l_bs"], p["N"], p["collapse"], torch.from_numpy(k.all_rot).cuda(), 1)
    assert np.array_equal(got1.cpu().numpy(), want)


@pytest.mark.parametrize("name", ["tiny_c3", "cfg1", "cfg2"])
def test_key_ring_and_plain_paths_agree(name, monkeypatch):
    """The key-ring kernel (keys in the chunked layout, bulk copies) and the
    plain kernel give identical outputs."""
    p = PARAMS[name]
    k = keys(name)
    t = 32 if p["beta_bs"] <= 2 ** 7 else 16
    msgs, a, b = inputs(name, 5, t=t)
    lut = device_u32(np.stack([np.zeros(p["N"]), step_body(name, t=t)])[None])
    outs = []
    for ring in ("1", "0"):
        monkeypatch.setenv("TFHE_B200_KEY_RING", ring)   # read when the keys are created
        e = Keys.create(pset(name), k.bsk_coeff, k.ksk[0], k.ksk[1].reshape(k.ksk[1].shape[:2]))
        outs.append(e.pbs(device_u32(a), device_u32(b.reshape(-1)), lut))
        e.close()
    if p["beta_bs"] <= 2 ** 7:
        assert torch.equal(outs[0][0], outs[1][0]) and torch.equal(outs[0][1], outs[1][1])
    else:
        # beta = 2^15: FFT rounding may differ in the last unit; decryptions agree
        for oa, ob in outs:
            dec = O.decrypt_LWE((centred(host_u32(oa)[:, 0]), centred(host_u32(ob)[:, 0])), k.sk_glwe,
                                {"t": t, "q": p["q"]})
            assert np.array_equal(dec, (msgs >= t // 4).astype(float))


def test_fourier_key_upload_equals_coefficient_upload():
    name = "tiny_c3"
    k = keys(name)
    e2 = Keys.create_fourier(pset(name), k.bsk_ordered, k.ksk[0], k.ksk[1].reshape(k.ksk[1].shape[:2]))
    msgs, a, b = inputs(name, 8)
    lut = device_u32(np.stack([np.zeros(PARAMS[name]["N"]), step_body(name)])[None])
    o1 = engine(name).pbs(device_u32(a), device_u32(b.reshape(-1)), lut)
    o2 = e2.pbs(device_u32(a), device_u32(b.reshape(-1)), lut)
    assert torch.equal(o1[0], o2[0]) and torch.equal(o1[1], o2[1])
    e2.close()


def test_standalone_extract_and_rotate_ops():
    rng = np.random.default_rng(5)
    N = 256
    acc = canon(rng.integers(-2 ** 31, 2 ** 31, size=(3, 2, N)))
    oa, ob = sample_extract(device_u32(acc), n_lut=5)
    wa, wb = O.extract_many(acc, 5)
    assert np.array_equal(host_u32(oa), u32(wa)) and np.array_equal(host_u32(ob), u32(wb[..., 0]))
    for alpha in (0, 1, 100, 255):
        ga, gb = ops.sample_extract((torch.from_numpy(acc[0, 0]).cuda(), torch.from_numpy(acc[0, 1]).cuda()), alpha)
        ra, rb = O.sample_extract((acc[0, 0], acc[0, 1]), alpha)
        assert np.array_equal(ga.cpu().numpy(), ra) and np.array_equal(gb.cpu().numpy(), rb)
    for e in (0, 1, -1, 255, 256, 257, -256, -300, 511, 512, 700, -700):
        ga, gb = ops.rotate_ciphertext((torch.from_numpy(acc[1, 0]).cuda(), torch.from_numpy(acc[1, 1]).cuda()), e)
        ra, rb = O.rotate_ciphertext((acc[1, 0], acc[1, 1]), e)
        assert np.array_equal(ga.cpu().numpy(), ra) and np.array_equal(gb.cpu().numpy(), rb), e


def test_repeat_runs_identical():
    """Any run-to-run difference would flag a race on shared memory."""
    name = "cfg1"
    msgs, a, b = inputs(name, 9)
    lut = device_u32(np.stack([np.zeros(PARAMS[name]["N"]), step_body(name)])[None])
    first = engine(name).pbs(device_u32(a), device_u32(b.reshape(-1)), lut)
    for _ in range(2):
        again = engine(name).pbs(device_u32(a), device_u32(b.reshape(-1)), lut)
        assert torch.equal(first[0], again[0]) and torch.equal(first[1], again[1])


def test_invalid_arguments_raise():
    eng = engine("tiny_c3")
    N = PARAMS["tiny_c3"]["N"]
    a = torch.zeros((4, N), dtype=torch.int32, device="cuda")
    b = torch.zeros((4,), dtype=torch.int32, device="cuda")
    lut3 = torch.zeros((3, 2, N), dtype=torch.int32, device="cuda")
    with pytest.raises(TFHEError, match="INVALID_ARGUMENT"):
        eng.pbs(a, b, lut3)
    with pytest.raises(TFHEError, match="INVALID_ARGUMENT"):
        eng.pbs(a, b, lut3[:1], n_lut=0)
    bad = pset("tiny_c3").with_(N=300)
    k = keys("tiny_c3")
    with pytest.raises((TFHEError, ValueError)):
        Keys.create(bad, k.bsk_coeff, k.ksk[0], k.ksk[1])


@pytest.mark.parametrize("name,batch,n_lut", [("tiny_c3", 6, 1), ("tiny_c3", 6, 4), ("cfg1", 4, 1),
                                              ("cfg1", 4, 4)])
def test_reference_golden_fixtures(name, batch, n_lut):
    """The engine reproduces the outputs recorded from the reference's own
    Python code (tests/golden/make_golden.py)."""
    import os
    G = np.load(os.path.join(os.path.dirname(__file__), "golden", "pbs_golden.npz"))
    p = PARAMS[name]
    k = O.keygen(p, {"tiny_c3": 11, "cfg1": 13}[name])
    if np.any(np.abs(k.bsk_coeff) == 2 ** 31) or np.any(np.abs(k.ksk[0]) == 2 ** 31):
        pytest.skip("key holds +-q/2: the uint32 view changes the reference's representative")
    ks = ParamSet(name, N=p["N"], n=p["n"], log2_beta_bs=7, l_bs=p["l_bs"], collapse=p["collapse"],
                  log2_beta_ks=3, l_ks=p["l_ks"], sigma_glwe=p["sigma_glwe"], sigma_lwe=p["sigma_lwe"])
    eng = Keys.create(ks, k.bsk_coeff, k.ksk[0], k.ksk[1].reshape(k.ksk[1].shape[:2]))
    a, b = G[f"{name}_in_a"], G[f"{name}_in_b"]
    ka, kb = eng.keyswitch(device_u32(a), device_u32(b.reshape(-1)))
    assert np.array_equal(host_u32(ka), u32(G[f"{name}_ks_a"]))
    assert np.array_equal(host_u32(kb), u32(G[f"{name}_ks_b"].reshape(-1)))
    body = G[f"{name}_lut{n_lut}"]
    lut = device_u32(np.stack([np.zeros(p["N"]), body])[None])
    oa, ob = eng.pbs(device_u32(a), device_u32(b.reshape(-1)), lut, n_lut=n_lut)
    assert np.array_equal(host_u32(oa), u32(G[f"{name}_merge{n_lut}_a"]))
    assert np.array_equal(host_u32(ob), u32(G[f"{name}_merge{n_lut}_b"][..., 0]))
    # the reference-surface mirror on the reference's float64 buffers
    ga, gb = ops.cuboot_merge((torch.from_numpy(G[f"{name}_ks_a"]).cuda(), torch.from_numpy(G[f"{name}_ks_b"]).cuda()),
                              [torch.zeros((batch, p["N"]), dtype=torch.float64),
                               torch.from_numpy(np.broadcast_to(body, (batch, p["N"])).copy())],
                              torch.from_numpy(k.bsk_ordered).cuda(), p["q"], p["beta_bs"], p["l_bs"], p["N"],
                              p["collapse"], torch.from_numpy(k.all_rot).cuda(), n_lut)
    assert np.array_equal(ga.cpu().numpy(), G[f"{name}_merge{n_lut}_a"])
    assert np.array_equal(gb.cpu().numpy(), G[f"{name}_merge{n_lut}_b"])
    kk = ops.key_switch_LWE((torch.from_numpy(k.ksk[0]).cuda(), torch.from_numpy(k.ksk[1]).cuda()),
                            (torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()), ks_params(name))
    assert np.array_equal(u32(kk[0].cpu().numpy()), u32(G[f"{name}_ks_a"]))
    assert np.array_equal(u32(kk[1].cpu().numpy()), u32(G[f"{name}_ks_b"]))
    eng.close()


def test_bounded_wait_gives_up_and_reports():
    """A wait that nothing completes returns after its limit and sets the
    device status word; the context stays usable."""
    import ctypes
    from tfhe_b200 import _lib
    lib = _lib.load()
    st = ctypes.c_int32()
    _lib.check(lib.tfhe_device_status(ctypes.byref(st), 1))
    waited = ctypes.c_int32(-1)
    _lib.check(lib.tfhe_probe_wait_timeout(2_000_000, ctypes.byref(waited)))
    assert waited.value == 0
    _lib.check(lib.tfhe_device_status(ctypes.byref(st), 1))
    assert st.value == 1
    _lib.check(lib.tfhe_device_status(ctypes.byref(st), 0))
    assert st.value == 0
    # the device still runs the engine afterwards
    test_standalone_extract_and_rotate_ops()


def test_no_wait_timeouts_recorded():
    import ctypes
    from tfhe_b200 import _lib
    st = ctypes.c_int32()
    _lib.check(_lib.load().tfhe_device_status(ctypes.byref(st), 0))
    assert st.value == 0


def test_two_cta_layout_matches_one_cta_layout_at_cfg1():
    """At config 1, 1184 ciphertexts (two waves of two per CTA) run two CTAs
    per SM: root table in global memory in rotation order, twist factors
    derived from one read.  One ciphertext per CTA runs the shared-memory
    layout that the oracle tests above pin bit for bit; the two layouts must
    agree bit for bit."""
    name = "cfg1"
    p = PARAMS[name]
    eng = engine(name)
    batch = 1184
    msgs, a, b = inputs(name, batch)
    k, threads, smem = eng.launch_shape(batch)
    # two CTAs per SM: K = 2 and no 8 KB root table in shared memory
    assert k == 2 and threads == 2 * k * p["N"] // 16 and smem < 110 * 1024
    lut = device_u32(np.stack([np.zeros(p["N"]), step_body(name)])[None])
    two = eng.pbs(device_u32(a), device_u32(b.reshape(-1)), lut)
    eng.set_tuning(ciphertexts_per_cta=1)
    try:
        assert eng.launch_shape(batch)[0] == 1
        one = eng.pbs(device_u32(a), device_u32(b.reshape(-1)), lut)
    finally:
        eng.set_tuning()
    assert torch.equal(two[0], one[0]) and torch.equal(two[1], one[1])
    # and the first ciphertexts against the oracle directly
    k4 = keys(name)
    ca, cb = O.key_switch_LWE(k4.ksk, (a[:4], b[:4]), ks_params(name))
    enc = [np.zeros((4, p["N"])), np.broadcast_to(step_body(name), (4, p["N"]))]
    wa, wb = O.cuboot_merge((ca, cb), enc, k4.bsk_ordered, p["q"], p["beta_bs"], p["l_bs"], p["N"],
                            p["collapse"], k4.all_rot, 1)
    assert np.array_equal(host_u32(two[0])[:4], u32(wa))
    assert np.array_equal(host_u32(two[1])[:4], u32(wb[..., 0]))


def test_partial_last_round_runs_as_its_own_launch():
    """n=742 N=2048, 396 ciphertexts: two full rounds of K = 2 on 148 CTAs,
    then the last 100 as a second launch of one ciphertext per CTA; the
    outputs equal one launch of the requested K = 2 bit for bit, and the
    library's launch counter sees the two launches."""
    from tfhe_b200.engine import launch_count
    name = "cfg2"
    p = PARAMS[name]
    eng = engine(name)
    batch = 396
    msgs, a, b = inputs(name, batch, t=16)
    lut = device_u32(np.stack([np.zeros(p["N"]), step_body(name, t=16)])[None])
    ka, kb = eng.keyswitch(device_u32(a), device_u32(b.reshape(-1)))
    n0 = launch_count()
    split = eng.blind_rotate(ka, kb, lut)
    n_split = launch_count() - n0
    eng.set_tuning(ciphertexts_per_cta=2)
    try:
        n0 = launch_count()
        one = eng.blind_rotate(ka, kb, lut)
        n_one = launch_count() - n0
    finally:
        eng.set_tuning()
    assert torch.equal(split, one)
    assert n_split == n_one + 1


@pytest.mark.parametrize("name", ["cfg1", "cfg2"])
def test_small_batches_get_512_threads(name):
    """Under one wave, a CTA holds K < max ciphertexts but still 512 threads:
    2K N/16 own the register-resident butterflies, the rest share the
    shared-memory stages (the bit-exact tests above run these shapes)."""
    p = PARAMS[name]
    eng = engine(name)
    for batch in (1, 100):
        k, threads, smem = eng.launch_shape(batch)
        assert k == 1 and threads == 512 and 2 * k * p["N"] // 16 < threads
    k, threads, smem = eng.launch_shape(16384)
    assert threads == 2 * k * p["N"] // 16


def test_tuning_changes_speed_not_results(tmp_path):
    """Every launch shape gives identical outputs; the autotuner picks one,
    caches it and the cache is applied on the next call."""
    from tfhe_b200.autotune import autotune, candidates
    name = "tiny_c3"
    N = PARAMS[name]["N"]
    eng = engine(name)
    msgs, a, b = inputs(name, 21)
    lut = device_u32(np.stack([np.zeros(N), step_body(name)])[None])
    want = eng.pbs(device_u32(a), device_u32(b.reshape(-1)), lut)
    for shape in candidates(eng, 21):
        eng.set_tuning(*shape)
        got = eng.pbs(device_u32(a), device_u32(b.reshape(-1)), lut)
        assert torch.equal(got[0], want[0]) and torch.equal(got[1], want[1]), shape
    path = str(tmp_path / "tune.json")
    best, times = autotune(eng, 21, path=path, reps=1)
    assert best in times
    again, times2 = autotune(eng, 21, path=path)
    assert again == best and times2 == {}
    eng.set_tuning()                     # back to automatic for the other tests


def test_cuda_graph_replay_matches_direct_calls():
    from tfhe_b200.engine import PBSGraph
    name = "tiny_c3"
    N = PARAMS[name]["N"]
    eng = engine(name)
    lut = device_u32(np.stack([np.zeros(N), step_body(name)])[None])
    graph = PBSGraph(eng, 13, n_lut=1)
    for seed in (1, 2):
        msgs, a, b = inputs(name, 13, seed_offset=seed)
        want = eng.pbs(device_u32(a), device_u32(b.reshape(-1)), lut)
        got = graph(device_u32(a), device_u32(b.reshape(-1)), lut)
        torch.cuda.synchronize()
        assert torch.equal(got[0], want[0]) and torch.equal(got[1], want[1])


@pytest.mark.parametrize("chunk,shared_lut", [(10, False), (10, True), (0, False), (37, True)])
def test_pbs_from_host_buffers_matches_device_pbs(chunk, shared_lut):
    """tfhe_pbs_host (chunked, copies overlapped) gives tfhe_pbs's outputs."""
    name = "tiny_c3"
    N = PARAMS[name]["N"]
    eng = engine(name)
    msgs, a, b = inputs(name, 37)
    rng = np.random.default_rng(5)
    luts = u32(np.stack([np.zeros((37, N)), rng.integers(0, 2 ** 32, size=(37, N))], axis=1))
    if shared_lut:
        luts = luts[:1]
    a_h = torch.from_numpy(u32(a).view(np.int32)).pin_memory()
    b_h = torch.from_numpy(u32(b.reshape(-1)).view(np.int32)).pin_memory()
    lut_h = torch.from_numpy(np.ascontiguousarray(luts).view(np.int32)).pin_memory()
    got_a, got_b = eng.pbs_host(a_h, b_h, lut_h, 2, chunk=chunk)
    torch.cuda.synchronize()
    want_a, want_b = eng.pbs(a_h.cuda(), b_h.cuda(), lut_h.cuda(), 2)
    assert torch.equal(got_a, want_a.cpu()) and torch.equal(got_b, want_b.cpu())


@pytest.mark.parametrize("name", ["tiny_c3", "tiny_c2", "cfg1", "cfg2", "c1_N128", "c4_N4096"])
def test_keyswitch_tensor_cores_bit_exact(name):
    """The tcgen05 int8 key switch equals the CUDA-core one and the oracle,
    over partial and several 128-ciphertext tiles."""
    k = keys(name)
    eng = engine(name)
    for batch in (37, 300):
        msgs, a, b = inputs(name, batch, seed_offset=batch)
        ra, rb = O.key_switch_LWE(k.ksk, (a, b), ks_params(name))
        out = {}
        for tc in (1, 0):
            eng.set_tuning(ks_tensor_cores=tc)
            out[tc] = eng.keyswitch(device_u32(a), device_u32(b.reshape(-1)))
        eng.set_tuning()
        assert torch.equal(out[1][0], out[0][0]) and torch.equal(out[1][1], out[0][1])
        assert np.array_equal(host_u32(out[1][0]), u32(ra))
        assert np.array_equal(host_u32(out[1][1]), u32(rb.reshape(-1)))


def test_keyswitch_unaligned_input_uses_cuda_cores():
    """An input not 16-byte aligned takes the CUDA-core kernel (the
    tensor-core kernel loads 16-byte vectors) and is still exact."""
    name = "tiny_c3"
    k = keys(name)
    eng = engine(name)
    msgs, a, b = inputs(name, 9)
    big = torch.zeros((9 * a.shape[1] + 1,), dtype=torch.int32, device="cuda")
    big[1:] = device_u32(a).reshape(-1)
    a_view = big[1:].view(9, a.shape[1])
    assert a_view.data_ptr() % 16 != 0
    ga, gb = eng.keyswitch(a_view, device_u32(b.reshape(-1)))
    ra, rb = O.key_switch_LWE(k.ksk, (a, b), ks_params(name))
    assert np.array_equal(host_u32(ga), u32(ra)) and np.array_equal(host_u32(gb), u32(rb.reshape(-1)))


def small_batch_cluster(name):
    """CTAs per ciphertext of this set's smallest batches: eight at N = 2048
    and at N = 1024 with four or eight patterns, four at N = 1024 with two
    (collapse <= 3), else two"""
    p = PARAMS[name]
    if p["l_bs"] <= 3 and 2 ** p["collapse"] <= 8 and p["N"] in (1024, 2048):
        return 4 if (p["N"] == 1024 and p["collapse"] == 1) else 8
    return 2


@pytest.mark.parametrize("name", ["tiny_c3", "tiny_c2", "cfg1", "cfg2", "c1_N128", "c4_N4096", "c1_N1024_l1",
                                  "c3_N2048_l3"])
def test_cluster_kernels_match_one_cta_kernel(name):
    """Small batches run one ciphertext on a cluster of eight or four CTAs
    (N = 1024 and 2048, collapse <= 3: each CTA owns one ACC polynomial and a
    quarter or half of the spectrum) or of two (each owns one ACC
    polynomial); the outputs are bit-identical to the one-CTA kernel's
    (requested shape K = 1), at every parameter set, for the extraction
    (n_lut 1 and 4) and for the rotated accumulator."""
    p = PARAMS[name]
    N = p["N"]
    eng = engine(name)
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    for batch, n_lut in ((1, 1), (5, 4), (sms // 4, 1), (sms // 2, 1)):
        msgs, a, b = inputs(name, batch, seed_offset=batch)
        body = step_body(name) if n_lut == 1 else many_lut_body(name, n_lut)
        lut = device_u32(np.stack([np.zeros(N), body])[None])
        a_d, b_d = device_u32(a), device_u32(b.reshape(-1))
        eng.set_tuning()
        cs = eng.cluster_size(batch)
        if batch <= 5:
            assert cs == small_batch_cluster(name), (batch, cs)
        elif batch == sms // 2:
            assert cs == 2, (batch, cs)
        else:
            assert cs in (2, 4), (batch, cs)
        got = eng.pbs(a_d, b_d, lut, n_lut=n_lut)
        ka, kb = eng.keyswitch(a_d, b_d)
        acc = eng.blind_rotate(ka, kb, lut, n_lut=n_lut)
        eng.set_tuning(ciphertexts_per_cta=1)
        assert eng.cluster_size(batch) == 1
        want = eng.pbs(a_d, b_d, lut, n_lut=n_lut)
        acc1 = eng.blind_rotate(ka, kb, lut, n_lut=n_lut)
        eng.set_tuning()
        assert torch.equal(got[0], want[0]) and torch.equal(got[1], want[1]), (batch, n_lut, cs)
        assert torch.equal(acc, acc1), (batch, n_lut, cs)
    assert eng.cluster_size(sms // 2 + 1) == 1


def test_cfg2_against_reference_golden():
    """Config 2 through the engine against the reference's own key switch
    and cuboot_merge (tests/golden/pbs_cfg2_golden.npz, generated by
    make_golden.py cfg2): the key switch bit for bit; the bootstrap by
    decryption and by phase, each output within 2^27 of its value (decision
    margin q/16 = 2^28), on the one-CTA and the cluster-pair kernels."""
    import os
    G2 = np.load(os.path.join(os.path.dirname(__file__), "golden", "pbs_cfg2_golden.npz"))
    name = "cfg2"
    p = PARAMS[name]
    q, N = p["q"], p["N"]
    k = keys(name)
    eng = engine(name)
    a_d, b_d = device_u32(G2["cfg2_in_a"]), device_u32(G2["cfg2_in_b"].reshape(-1))
    ka, kb = eng.keyswitch(a_d, b_d)
    assert np.array_equal(host_u32(ka), u32(G2["cfg2_ks_a"]))
    assert np.array_equal(host_u32(kb), u32(G2["cfg2_ks_b"].reshape(-1)))
    lut = device_u32(np.stack([np.zeros(N), G2["cfg2_lut1"]])[None])
    want = (G2["cfg2_msgs"] >= 4).astype(np.float64)
    sk = k.sk_glwe.astype(np.float64)
    for cpc in (0, 1):                     # automatic (cluster pair at this batch), one CTA per ciphertext
        eng.set_tuning(ciphertexts_per_cta=cpc)
        oa, ob = eng.pbs(a_d, b_d, lut)
        oa = centred(host_u32(oa))[:, 0].astype(np.float64)
        ob = centred(host_u32(ob))[:, 0].astype(np.float64)
        ph = np.mod(ob - oa @ sk + q / 2, q) - q / 2
        assert np.array_equal(np.rint(ph / (q / 8)), want), cpc
        assert np.abs(ph - want * q / 8).max() <= 2.0 ** 27, cpc
    eng.set_tuning()


def test_tensor_memory_kernel_matches_two_per_cta():
    """Three ciphertexts per CTA with the accumulators in tensor memory
    (ciphertexts_per_cta = 3, N = 2048) give the outputs of the two-per-CTA
    kernel bit for bit; the batch leaves a remainder after the whole rounds
    of 3 x SMs, which runs on the other shapes."""
    name = "cfg2"
    p = PARAMS[name]
    N = p["N"]
    eng = engine(name)
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    batch = 3 * sms + 37
    msgs, a, b = inputs(name, batch, seed_offset=7)
    lut = device_u32(np.stack([np.zeros(N), many_lut_body(name, 2)])[None])
    a_d, b_d = device_u32(a), device_u32(b.reshape(-1))
    ka, kb = eng.keyswitch(a_d, b_d)
    eng.set_tuning(ciphertexts_per_cta=3)
    got = eng.pbs(a_d, b_d, lut, n_lut=2)
    acc = eng.blind_rotate(ka, kb, lut, n_lut=2)
    eng.set_tuning(ciphertexts_per_cta=2)
    want = eng.pbs(a_d, b_d, lut, n_lut=2)
    acc2 = eng.blind_rotate(ka, kb, lut, n_lut=2)
    eng.set_tuning()
    assert torch.equal(got[0], want[0]) and torch.equal(got[1], want[1])
    assert torch.equal(acc, acc2)
