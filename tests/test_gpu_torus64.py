"""The 2^64-torus operators on the GPU against the oracle
(oracle/torus64_oracle.py): bit for bit on every integer operator (key
switch, rotation indices, rotation + extraction, linear, LUT products, trace
packing, packing, rotate/add, extraction); the FP64 blind rotation at
q = 2^64 (the native one-kernel cuboot_merge and the reference-layout chain)
within the float64 rounding of the oracle's chain and by decryption; whole
Spike-LSTM timesteps on the reference's parameter set against the oracle by
decryption and against the plaintext recurrence."""
import numpy as np
import pytest
import torch

from oracle import tfhe_oracle as O
from oracle import torus64_oracle as T64

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU runs deselect -m gpu
    pytest.skip("needs a CUDA device", allow_module_level=True)

from tfhe_b200 import client64 as C64  # noqa: E402
from tfhe_b200 import torus64 as D64  # noqa: E402

SMALL = C64.Params64("small64", N=256, n=12, log2_beta_bs=13, l_bs=2, collapse=3, log2_beta_ks=4, l_ks=5,
                     sigma_glwe=2.0 ** 17, sigma_lwe=2.0 ** 40)
# one CMux group at the reference's degree and gadget (G = 1)
ONE64 = C64.Params64("one64", N=2048, n=3, log2_beta_bs=13, l_bs=2, collapse=3, log2_beta_ks=4, l_ks=5,
                     sigma_glwe=2.0 ** 17, sigma_lwe=2.0 ** 40)
DELTA = 2.0 ** 60
# float64 rounding of one group at q = 2^64, N = 2048 (test_gpu_ref64.py's bound)
ONE_GROUP_TOL = 2.0 ** 36
_KEYS = {}


def keys_for(p):
    if p.name not in _KEYS:
        ck = C64.keygen(p, 5)
        _KEYS[p.name] = (ck, D64.Keys64(ck, reflayout=True), {"params": p, "ksk": ck.ksk, "rot": C64.monomial_fourier(p.N),
                                               "bsk_grouped": C64.bsk_fourier_grouped(ck.bsk, p)})
    return _KEYS[p.name]


def rnd(rng, *shape):
    return rng.integers(0, 2 ** 64, size=shape, dtype=np.uint64)


def d64(x):
    return D64.device_u64(x)


def h64(t):
    return D64.host_u64(t)


@pytest.mark.parametrize("p", [SMALL, C64.REF64], ids=lambda p: p.name)
def test_keyswitch64_bit_exact(p):
    ck, dk, ok = keys_for(p)
    rng = np.random.default_rng(1)
    a, b = rnd(rng, 33, p.N), rnd(rng, 33)
    a_d, b_d = d64(a), d64(b)
    wa, wb = T64.key_switch(ck.ksk, a, b, p.log2_beta_ks, p.l_ks)
    assert dk.ksk_limbs is not None                      # base 2^4: the tensor-core path
    for tc in (1, 0):                                    # tcgen05 int8 limbs, CUDA cores
        ga, gb = dk.keyswitch(a_d, b_d, tensor_cores=tc)
        assert np.array_equal(h64(ga), wa) and np.array_equal(h64(gb), wb), tc


@pytest.mark.parametrize("n_lut", [1, 4])
def test_indices_and_rotate_extract64_bit_exact(n_lut):
    from tfhe_b200 import _lib
    from tfhe_b200.engine import _ptr, _stream
    rng = np.random.default_rng(2)
    N, n, c, B = 2048, 702, 3, 5
    a = rnd(rng, B, n)
    a[0, :6] = [0, 1 << 63, (1 << 63) - 1, 1 << 52, 3 << 51, (1 << 64) - (1 << 51)]
    idx = torch.empty((B, n // c, 1 << c), dtype=torch.int32, device="cuda")
    a_d = d64(a)                       # device buffers stay referenced until the kernels have run
    _lib.check(_lib.load().tfhe64_rotation_indices(_ptr(a_d), n, c, N, n_lut, _ptr(idx), B, _stream()))
    assert np.array_equal(idx.cpu().numpy(), T64.rotation_indices(a, c, N, n_lut))
    acc = rnd(rng, B, 2, N)
    b = rnd(rng, B)
    b[0] = 1 << 63
    oa = torch.empty((B, n_lut, N), dtype=torch.int64, device="cuda")
    ob = torch.empty((B, n_lut), dtype=torch.int64, device="cuda")
    acc_d, b_d = d64(acc), d64(b)
    _lib.check(_lib.load().tfhe64_rotate_extract(_ptr(acc_d), _ptr(b_d), N, n_lut, _ptr(oa), _ptr(ob), B,
                                                 _stream()))
    wa, wb = T64.rotate_extract(acc, b, N, n_lut)
    assert np.array_equal(h64(oa), wa) and np.array_equal(h64(ob), wb)


def _cdiff(x, y):
    """|x - y| of uint64 words, centred mod 2^64, as float64."""
    return np.abs((np.asarray(x, np.uint64) - np.asarray(y, np.uint64)).view(np.int64).astype(np.float64))


@pytest.mark.parametrize("batch", [1, 7, 300])
@pytest.mark.parametrize("n_lut", [1, 4])
def test_native_blind_rotation64_one_group_within_rounding_of_oracle(batch, n_lut):
    """tfhe64_blind_rotate / tfhe64_cuboot_merge (indices from the masks,
    chain, rotation by -b~, extraction) against the oracle's float64 chain
    and exact rotation/extraction, one group at N = 2048, random full-range
    accumulators and masks (300 ciphertexts: several per CTA and the
    one-per-SM last round)."""
    p = ONE64
    ck, dk, ok = keys_for(p)
    rng = np.random.default_rng(40 + batch + n_lut)
    lut = rnd(rng, batch, 2, p.N)
    a = rnd(rng, batch, p.n)
    a[0, :3] = [1 << 63, (1 << 63) - 1, 3 << 51]
    b = rnd(rng, batch)
    lut_d, a_d, b_d = d64(lut), d64(a), d64(b)
    idx = T64.rotation_indices(a, p.collapse, p.N, n_lut)
    acc = T64.acc_to_words(T64.blind_rotate(lut, idx, ok["bsk_grouped"], ok["rot"], p.log2_beta_bs, p.l_bs, p.N))
    zero = d64(np.zeros(batch, np.uint64))
    got = h64(dk.blind_rotate(a_d, zero, lut_d, n_lut))
    d = _cdiff(got, acc)
    print(f"one group, native: max |engine - oracle| = 2^{np.log2(d.max() + 1):.2f}")
    assert d.max() <= ONE_GROUP_TOL
    ga, gb = dk.cuboot_merge(a_d, b_d, lut_d, n_lut)
    wa, wb = T64.rotate_extract(acc, b, p.N, n_lut)
    assert _cdiff(h64(ga), wa).max() <= ONE_GROUP_TOL and _cdiff(h64(gb), wb).max() <= ONE_GROUP_TOL


def test_native_and_reference_layout_chains_agree64():
    """The native kernel and tfhe_mul_bootstrap on the reference's key layout
    compute the same chain over all 234 groups.  From the second group on,
    the two FFTs' rounding moves some gadget digits by one, and each such
    digit adds a different key row (a fresh RLWE with a uniform mask): the
    raw words part, so the accumulators are compared by their phases under
    the GLWE key.  There the two chains differ by independent decomposition
    remainders of their (by then unrelated) masks: |r| <= 2^37 times the
    binary key over N/2 terms, about 2^41.7 rms per group for the
    difference, 2^45.6 rms after 234 groups, about 2^47.6 at the maximum
    over 4 x 2048 coefficients (measured 2^47.7); the bound is the
    decryption-noise bound of the drop-in tests, 2^50 (a decryption fails
    at 2^59)."""
    p = C64.REF64
    ck, dk, ok = keys_for(p)
    rng = np.random.default_rng(44)
    B = 4
    lut = rnd(rng, B, 2, p.N)
    a = rnd(rng, B, p.n)
    lut_d, a_d, z_d = d64(lut), d64(a), d64(np.zeros(B, np.uint64))
    native = h64(dk.blind_rotate(a_d, z_d, lut_d, 1))
    ref = h64(dk.blind_rotate_reflayout(a_d, lut_d, 1))
    ph_n = C64.rlwe_phase(native[:, 0], native[:, 1], ck.sk_glwe)
    ph_r = C64.rlwe_phase(ref[:, 0], ref[:, 1], ck.sk_glwe)
    d = _cdiff(ph_n.view(np.uint64), ph_r.view(np.uint64))
    print(f"234 groups: max |phase(native) - phase(reference layout)| = 2^{np.log2(d.max() + 1):.2f}")
    assert d.max() <= 2.0 ** 50


def test_cluster_kernels_match_one_cta_kernel64():
    """Small batches on clusters of eight CTAs (up to an eighth of the SM
    count), of four (up to a quarter) and of two give the one-CTA kernel's
    outputs bit for bit on the 64-bit torus (reference parameters, n_lut 1
    and 4)."""
    p = C64.REF64
    ck, dk, ok = keys_for(p)
    rng = np.random.default_rng(45)
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    for B, n_lut in ((1, 1), (6, 4), (sms // 4, 1), (sms // 2, 1)):
        lut_d, a_d, b_d = d64(rnd(rng, B, 2, p.N)), d64(rnd(rng, B, p.n)), d64(rnd(rng, B))
        dk.set_tuning()
        cs = dk.cluster_size(B)
        if B <= 6:
            assert cs == 8, (B, cs)
        elif B == sms // 2:
            assert cs == 2, (B, cs)
        else:
            assert cs in (2, 4), (B, cs)
        got = dk.cuboot_merge(a_d, b_d, lut_d, n_lut)
        acc = dk.blind_rotate(a_d, b_d, lut_d, n_lut)
        dk.set_tuning(ciphertexts_per_cta=1)
        assert dk.cluster_size(B) == 1
        want = dk.cuboot_merge(a_d, b_d, lut_d, n_lut)
        acc1 = dk.blind_rotate(a_d, b_d, lut_d, n_lut)
        dk.set_tuning()
        assert torch.equal(got[0], want[0]) and torch.equal(got[1], want[1]), (B, n_lut, cs)
        assert torch.equal(acc, acc1), (B, n_lut, cs)


@pytest.mark.parametrize("N,bound,density", [(2048, 1, 0.5), (2048, 256, 1.0), (1024, 255, 0.3), (256, 3, 0.9),
                                             (2048, 257, 0.2)])
def test_lut_products_in_the_fourier_domain_are_exact64(N, bound, density):
    """tfhe64_lut_mul_sum multiplies LUTs with |entries| <= 2^8 in the
    Fourier domain (16-bit limbs of the ciphertext words) and larger ones by
    direct sums: exact modulo 2^64 either way, including dense LUTs at the
    2^8 bound and one entry past it."""
    rng = np.random.default_rng(N + bound)
    G, K, S = 4, 5, 2
    luts = rng.integers(-bound, bound + 1, size=(G, K, N)) * (rng.random((G, K, N)) < density)
    luts[:, :, 0] = bound                             # the extreme value in every LUT
    rl = rnd(rng, S, G, K, 2, N)
    rl[0, 0, 0, 0, :4] = [0, 1 << 63, (1 << 64) - 1, 1 << 32]
    got = D64.lut_mul_sum(torch.from_numpy(luts).cuda(), d64(rl))
    for s in range(S):
        pa, pb = T64.lut_mul_sum(luts, rl[s, :, :, 0], rl[s, :, :, 1])
        assert np.array_equal(h64(got[s, :, 0]), pa) and np.array_equal(h64(got[s, :, 1]), pb)


def test_tensor_memory_kernel_matches_two_per_cta64():
    """The tensor-memory kernel (three ciphertexts per CTA) on the 64-bit
    torus at the reference's parameters: bit-identical to two per CTA."""
    p = C64.REF64
    ck, dk, ok = keys_for(p)
    rng = np.random.default_rng(46)
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    B = 3 * sms + 11
    lut_d, a_d, b_d = d64(rnd(rng, B, 2, p.N)), d64(rnd(rng, B, p.n)), d64(rnd(rng, B))
    dk.set_tuning(ciphertexts_per_cta=3)
    got = dk.cuboot_merge(a_d, b_d, lut_d, 4)
    dk.set_tuning(ciphertexts_per_cta=2)
    want = dk.cuboot_merge(a_d, b_d, lut_d, 4)
    dk.set_tuning()
    assert torch.equal(got[0], want[0]) and torch.equal(got[1], want[1])


def test_64bit_keys_refuse_32bit_entry_points():
    from tfhe_b200 import _lib
    ck, dk, ok = keys_for(SMALL)
    lib = _lib.load()
    x = torch.zeros(64, dtype=torch.int64, device="cuda")
    rc = lib.tfhe_cuboot_merge(dk.handle, x.data_ptr(), x.data_ptr(), x.data_ptr(), 1, 1, x.data_ptr(),
                               x.data_ptr(), 1, None)
    assert rc != 0 and b"2^64" in lib.tfhe_last_error()
    rc = lib.tfhe64_cuboot_merge(dk.handle, x.data_ptr(), x.data_ptr(), x.data_ptr(), 1, 3, x.data_ptr(),
                                 x.data_ptr(), 1, None)
    assert rc != 0 and b"power of two" in lib.tfhe_last_error()


@pytest.mark.parametrize("reflayout", [False, True], ids=["native", "reflayout"])
@pytest.mark.parametrize("p,batch", [(SMALL, 9), (C64.REF64, 6)], ids=["small64", "ref64"])
def test_pbs64_decrypts_like_oracle(p, batch, reflayout):
    ck, dk, ok = keys_for(p)
    rng = np.random.default_rng(3)
    msgs = rng.integers(0, 8, size=batch)
    a, b = C64.encrypt_lwe(msgs.astype(np.uint64) << np.uint64(60), ck.sk_glwe, 2.0 ** 20, rng)
    body = O.step_lut(p.N, 8, 4, DELTA).astype(np.int64)
    lut = np.stack([np.zeros(p.N, np.int64), body])[None]
    a_d, b_d, lut_d = d64(a), d64(b), d64(lut)
    ga, gb = dk.pbs(a_d, b_d, lut_d, 1, reflayout=reflayout)
    wa, wb = T64.pbs(ok, a, b, lut, 1)
    want = (msgs >= 4).astype(np.float64)
    for oa, ob in ((h64(ga), h64(gb)), (wa, wb)):
        ph = C64.phase(oa[:, 0], ob[:, 0], ck.sk_glwe).astype(np.float64)
        assert np.array_equal(np.rint(ph / DELTA), want)
        assert np.abs(ph - want * DELTA).max() < 2.0 ** 50


def test_linear_lut_rotate_add_extract64_bit_exact():
    rng = np.random.default_rng(4)
    N, S, J = 2048, 2, 5
    ct = rnd(rng, S, 2, N)
    kern = rng.integers(-7, 8, size=(J, N)) * (rng.random((J, N)) < 0.1)
    bias = rng.integers(-2 ** 62, 2 ** 62, size=J)
    ga, gb = D64.linear_extract(torch.from_numpy(kern.astype(np.int32)).cuda(), torch.from_numpy(bias).cuda(), d64(ct))
    for s in range(S):
        wa, wb = T64.linear(kern, bias, (ct[s, 0], ct[s, 1]))
        assert np.array_equal(h64(ga[s]), wa) and np.array_equal(h64(gb[s]), wb)
    G, K = 4, 3
    luts = rng.integers(-1, 2, size=(G, K, N)) * (rng.random((G, K, N)) < 0.2)
    luts[0, 0] = rng.integers(-2 ** 54, 2 ** 54, size=N)
    rl = rnd(rng, S, G, K, 2, N)
    got = D64.lut_mul_sum(torch.from_numpy(luts).cuda(), d64(rl))
    for s in range(S):
        pa, pb = T64.lut_mul_sum(luts, rl[s, :, :, 0], rl[s, :, :, 1])
        assert np.array_equal(h64(got[s, :, 0]), pa) and np.array_equal(h64(got[s, :, 1]), pb)
    x, y = rnd(rng, S, 2, N), rnd(rng, S, 2, N)
    for rot in (0, 7, 2047, 2048, 3000, -5):
        got = D64.rlwe_rotate_add(d64(x), rot, d64(y))
        for s in range(S):
            for c in range(2):
                assert np.array_equal(h64(got[s, c]), T64.rotate_poly(x[s, c], rot) + y[s, c])
    assert np.array_equal(h64(D64.add(d64(x), d64(y))), x + y)
    ea, eb = D64.sample_extract(d64(x), 130)
    for s in range(S):
        wa, wb = T64.sample_extract_many(x[s, 0], x[s, 1], 130)
        assert np.array_equal(h64(ea[s]), wa) and np.array_equal(h64(eb[s]), wb)


@pytest.mark.parametrize("N,l", [(256, 5), (2048, 5)])
def test_trace_pack_lwe_to_rlwe64_bit_exact(N, l):
    rng = np.random.default_rng(5 + N)
    sk = rng.integers(0, 2, size=N)
    gal = C64.galois_keys(sk, 8, l, 2.0 ** 17, rng)
    gk = D64.GaloisKeys64(gal, 8, l)
    R = 3
    a, b = rnd(rng, R, N), rnd(rng, R)
    got = gk.pack_lwe_to_rlwe(d64(a), d64(b))
    A, B = T64.pack_lwe_to_rlwe(a, b, gal, 8, l)
    assert np.array_equal(h64(got[:, 0]), A) and np.array_equal(h64(got[:, 1]), B)
    gk.close()


@pytest.mark.parametrize("N,T,lb,l", [(256, 7, 8, 4), (2048, 128, 8, 4), (256, 7, 7, 5), (2048, 128, 7, 5)])
def test_packing64_bit_exact(N, T, lb, l):
    """Base 2^8 (digits up to 128) packs on CUDA cores; base 2^7 also on the
    tensor cores (8-bit limbs of the 64-bit key), with the same result."""
    rng = np.random.default_rng(6 + T + lb)
    sk = rng.integers(0, 2, size=N)
    ksp = C64.packing_key(sk, sk, lb, l, 2.0 ** 17, rng)
    key = D64.PackingKey64(ksp, lb, l)
    assert key.tensor_cores == (lb <= 7)
    S = 2
    a, b = rnd(rng, S, T, N), rnd(rng, S, T)
    a_d, b_d = d64(a), d64(b)
    for tc in ((1, 0) if key.tensor_cores else (0,)):
        got = key.pack(a_d, b_d, tensor_cores=tc)
        for s in range(S):
            pa, pb = T64.packing(a[s], b[s], ksp, lb, l, N)
            assert np.array_equal(h64(got[s, 0]), pa) and np.array_equal(h64(got[s, 1]), pb), (tc, s)


def _model64(hidden, emb_dim, seed):
    from tfhe_b200 import spike_model as SM
    cfg = SM.config_q64(hidden=hidden, emb_dim=emb_dim)
    return cfg, SM.build_model(cfg, seed)


def test_spike_lstm64_timesteps_track_oracle_and_plaintext():
    """Three timesteps of a hidden-16 layer on the reference's parameter set:
    the GPU's and the oracle's encrypted cell / hidden states decrypt to the
    plaintext recurrence within 0.05 (units of beta_x) on all units but the
    spikes that the blind rotation's rounding of the phase flips next to a
    threshold (at most one eta <= 1 per flipped spike)."""
    from oracle import lstm_oracle as LO
    from tfhe_b200 import spike_model as SM
    cfg, model = _model64(16, 8, 7)
    dm = SM.to_device(model)
    p = cfg.pbs
    N = p.N
    L = model.layers[0]
    per = cfg.hidden // cfg.n_lut
    lut_f, lut_i, lut_o = SM.layer_luts(cfg, L)
    layer = {"hidden": cfg.hidden, "n_lut": cfg.n_lut, "input_dim": cfg.emb_dim, "galois": model.galois,
             "gal_log2_beta": cfg.gal_log2_beta, "gal_l": cfg.gal_l, "ksp": model.ksp,
             "pk_log2_beta": cfg.pk_log2_beta, "pk_l": cfg.pk_l, "lut_f": lut_f, "lut_i": lut_i, "lut_o": lut_o}
    for g in "fio":
        layer[f"kern_{g}"], layer[f"bias_{g}"] = LO.linear_kernel_polynomial(L.W[g], L.B[g] * cfg.beta_x,
                                                                             np.ones(per), N)
    okeys = {"params": p, "ksk": model.keys.ksk, "bsk_grouped": C64.bsk_fourier_grouped(model.keys.bsk, p),
             "rot": C64.monomial_fourier(N)}
    rng = np.random.default_rng(3)
    T = 3
    tokens = SM.sample_tokens(rng, 1, T, cfg.vocab, cfg.zipf)
    xs = SM.encrypt_tokens(model, tokens, rng)
    xs_d = SM.encrypted_words(model, xs).cuda()
    H = torch.zeros((1, 2, N), dtype=torch.int64, device="cuda")
    C = torch.zeros_like(H)
    oH = (np.zeros(N, np.uint64), np.zeros(N, np.uint64))
    oC = (np.zeros(N, np.uint64), np.zeros(N, np.uint64))
    scale = 4.0 * cfg.beta_x / 2.0 ** 64
    sub = N // cfg.n_lut

    def spike(z, gamma):
        g = np.clip(np.rint(z * scale * sub / 2) * 2 / sub, -1.0, 1.0 - 2.0 / sub)
        return np.concatenate([(g >= gamma[i]).astype(np.float64) for i in range(cfg.n_lut)])

    def plain_step(t, h, c):
        x = model.embedding[tokens[0, t]].astype(np.float64)
        z = {g: np.concatenate([x, h]) @ L.W[g] + L.B[g] for g in "fio"}
        i_g = spike(z["i"], L.gamma["i"]) * np.concatenate([L.eta[k] for k in range(cfg.n_lut)])
        c = spike(z["f"], L.gamma["f"]) * c + i_g
        return spike(z["o"], L.gamma["o"]) * c, c

    sk = model.keys.sk_glwe
    hs = slice(cfg.emb_dim, cfg.emb_dim + cfg.hidden)
    # each chain is compared with the plaintext step taken from its own
    # decrypted previous state, so that one flipped spike does not carry over
    prev = {"gpu": (np.zeros(cfg.hidden), np.zeros(cfg.hidden)), "oracle": (np.zeros(cfg.hidden), np.zeros(cfg.hidden))}
    for t in range(T):
        H, C = dm.layers[0].step(xs_d[t], H, C)
        oH, oC = T64.spike_lstm_step(okeys, layer, (xs[t, 0, 0], xs[t, 0, 1]), oH, oC)
        for name, (Hs, Cs) in (("gpu", (D64.host_u64(H[0]), D64.host_u64(C[0]))),
                               ("oracle", (np.stack(oH), np.stack(oC)))):
            h, c = plain_step(t, *prev[name])
            phC = C64.rlwe_phase(Cs[0], Cs[1], sk)[: cfg.hidden] / cfg.beta_x
            phH = C64.rlwe_phase(Hs[0], Hs[1], sk)[hs] / cfg.beta_x
            for got, want in ((phC, c), (phH, h)):
                assert np.mean(np.abs(got - want) < 0.05) >= 0.85, (name, t, got, want)
                assert np.abs(got - want).max() <= 1.0, (name, t, got, want)
            prev[name] = (phH, phC)


# ---------------------------------------------------------------- reference fixtures at q = 2^64
def _fx64():
    import os
    return np.load(os.path.join(os.path.dirname(__file__), "golden", "lstm64_golden.npz"))


_DEV64 = {}


def _device_case64():
    if "c" not in _DEV64:
        import lstm_golden_cases as GC
        from tfhe_b200 import spike_model as SM
        c = GC.cfg4_q64_case()
        _DEV64["c"] = (c, SM.to_device(c["model"]))
    return _DEV64["c"]


def test_gpu_lstm64_operators_within_rounding_of_reference():
    """Linear, packing and prepare_LUT on the GPU at the reference's own
    parameters against the reference's float64 results (the tolerances of
    tests/test_lstm64_golden.py)."""
    import lstm_golden_cases as GC
    from test_lstm64_golden import LIN_TOL, PACK_TOL, PREP_PHASE_TOL
    fx = _fx64()
    c, dm = _device_case64()
    cfg, model = c["cfg"], c["model"]
    N, per = cfg.pbs.N, cfg.hidden // cfg.n_lut
    layer = dm.layers[0]
    x0 = d64(c["xs"][0])
    for g, lin in zip("fio", (layer.W_f, layer.W_i, layer.W_o)):
        a, b = lin(x0)
        assert GC.torus_dist64(h64(a[0, :4]), fx[f"lin_{g}_a_rows"]).max() <= LIN_TOL
        assert GC.torus_dist64(h64(b[0]), fx[f"lin_{g}_b"]).max() <= LIN_TOL
    ops = GC.q64_op_inputs(c)
    got = dm.keys.packing.pack(d64(ops["pack_a"])[None], d64(ops["pack_b"])[None])
    assert GC.torus_dist64(h64(got[0, 0]), fx["pack_a"]).max() <= PACK_TOL
    assert GC.torus_dist64(h64(got[0, 1]), fx["pack_b"]).max() <= PACK_TOL
    prep = layer._encrypted_luts(d64(ops["prep_a"]).reshape(1, cfg.hidden, N),
                                 d64(ops["prep_b"]).reshape(1, cfg.hidden), layer.lut_f)
    sk = model.keys.sk_glwe
    d = C64.rlwe_phase(h64(prep[0, :4, 0]), h64(prep[0, :4, 1]), sk) - \
        C64.rlwe_phase(fx["prep_a_rows"], fx["prep_b_rows"], sk)
    assert np.abs(d.astype(np.float64)).max() <= PREP_PHASE_TOL


def test_gpu_lstm64_step_decrypts_like_reference():
    """One timestep of the one-layer workload on the GPU at q = 2^64: the
    cell and hidden states decrypt to the plaintext recurrence and to the
    reference's own encrypted step on >= 90% of units within 0.05 beta_x
    (the rest: spikes flipped by blind-rotation rounding, one eta <= 1 each)."""
    from test_lstm64_golden import plaintext_step
    fx = _fx64()
    c, dm = _device_case64()
    cfg, model = c["cfg"], c["model"]
    N = cfg.pbs.N
    H = torch.zeros((1, 2, N), dtype=torch.int64, device="cuda")
    H, C = dm.layers[0].step(d64(c["xs"][0]), H, torch.zeros_like(H))
    sk = model.keys.sk_glwe
    hs = slice(cfg.emb_dim, cfg.emb_dim + cfg.hidden)
    phC = C64.rlwe_phase(h64(C[0, 0]), h64(C[0, 1]), sk)[: cfg.hidden] / cfg.beta_x
    phH = C64.rlwe_phase(h64(H[0, 0]), h64(H[0, 1]), sk)[hs] / cfg.beta_x
    rC = C64.rlwe_phase(fx["C_a"][0], fx["C_b"][0], sk)[: cfg.hidden] / cfg.beta_x
    rH = C64.rlwe_phase(fx["H_a"][0], fx["H_b"][0], sk)[hs] / cfg.beta_x
    cc, hh = plaintext_step(c)
    print(f"q=2^64 step: |C - plain| max {np.abs(phC - cc).max():.3f}, |C - ref| max {np.abs(phC - rC).max():.3f}, "
          f"units within 0.05 of plain {np.mean(np.abs(phC - cc) < 0.05):.3f}")
    for got, want in ((phC, cc), (phH, hh), (phC, rC), (phH, rH)):
        assert np.mean(np.abs(got - want) < 0.05) >= 0.9
        assert np.abs(got - want).max() <= 1.0


def test_gpu_lstm64_head_decrypts_like_reference():
    fx = _fx64()
    c, dm = _device_case64()
    cfg, model = c["cfg"], c["model"]
    from tfhe_b200.lstm import CipherMLP, Linear
    from tfhe_b200 import spike_model as SM
    lin1, lin2 = Linear(cfg.hidden, cfg.pbs.N, 1.0), Linear(1, cfg.pbs.N, 1.0)
    lin1.set_weights(c["head_W1"], c["head_B1"])
    lin2.set_weights(c["head_W2"], c["head_B2"])
    relu = np.stack([SM.relu_lut(cfg.pbs.N, s, cfg.beta_x) for s in c["s_head"]])
    head = CipherMLP(dm.keys, lin1, lin2, relu)
    ya, yb = head(d64(c["head_x"])[None])
    sk = model.keys.sk_glwe
    got = C64.phase(h64(ya[0]), h64(yb[0]), sk)[0] / cfg.beta_x
    ref = C64.phase(fx["head_a"], fx["head_b"], sk)[0] / cfg.beta_x
    print(f"q=2^64 head logit: engine {got:.4f}, reference {ref:.4f}")
    assert abs(got - ref) < 0.25
