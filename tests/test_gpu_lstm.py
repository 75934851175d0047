"""Spike-LSTM operators on the GPU against the oracle, bit for bit: linear
+ extraction, pack_lwe_to_rlwe, LUT products, packing, rotation, and whole
timesteps of CipherSpikeLSTM and the CipherMLP head."""
import numpy as np
import pytest
import torch

from lstm_cases import (GAL_L, GAL_LOG2_BETA, HIDDEN, INPUT_DIM, N_LUT, NAME, PK_L, PK_LOG2_BETA, cen,
                        encrypt_inputs, layer_material)
from oracle import lstm_oracle as LO
from pbs_cases import PARAMS

pytestmark = pytest.mark.gpu

DEV = torch.device("cuda", 0) if torch.cuda.is_available() else None


def d32(x):
    return torch.from_numpy(np.ascontiguousarray((np.asarray(x, dtype=np.int64) & 0xFFFFFFFF).astype(np.uint32))
                            .view(np.int32)).to(DEV)


def h64(t):
    return t.cpu().numpy().view(np.uint32).astype(np.int64)


def u(x):
    return np.asarray(x, dtype=np.int64) & 0xFFFFFFFF


def rnd(rng, shape):
    return rng.integers(0, 2 ** 32, size=shape, dtype=np.uint64).astype(np.int64) - 2 ** 31


_DEV_LAYER = {}


def device_layer():
    if "x" in _DEV_LAYER:
        return _DEV_LAYER["x"]
    from tfhe_b200.engine import Keys
    from tfhe_b200.lstm import CipherSpikeLSTM, GaloisKeys, LayerKeys, Linear
    from tfhe_b200.params import TINY_C3
    m = layer_material()
    k = m["keys"]
    pbs = Keys.create(TINY_C3, k.bsk_coeff, k.ksk[0], k.ksk[1].reshape(k.ksk[1].shape[:2]))
    gk = GaloisKeys(m["galois"], GAL_LOG2_BETA, GAL_L, DEV)
    ksp = torch.from_numpy(np.ascontiguousarray(m["ksp"]).view(np.int32)).to(DEV)
    keys = LayerKeys(pbs, gk, ksp, PK_LOG2_BETA, PK_L)
    N = PARAMS[NAME]["N"]
    per = HIDDEN // N_LUT
    lins = []
    for g in "fio":
        lin = Linear(per, N, 1.0, DEV)
        lin.set_weights(m["mats"][g], m["biases"][g])
        assert np.array_equal(lin.kernel_np, m["layer"][f"kern_{g}"])
        lins.append(lin)
    L = m["layer"]
    layer = CipherSpikeLSTM(keys, INPUT_DIM, HIDDEN, N_LUT, *lins, L["lut_f"], L["lut_i"], L["lut_o"])
    _DEV_LAYER["x"] = (m, keys, layer)
    return _DEV_LAYER["x"]


def test_linear_extract_matches_oracle():
    from tfhe_b200.lstm import linear_extract
    rng = np.random.default_rng(10)
    N = 256
    for J, S, density in ((5, 3, 0.05), (9, 2, 1.0)):
        kern = rng.integers(-7, 8, size=(J, N)) * (rng.random((J, N)) < density)
        bias = rng.integers(-2 ** 31, 2 ** 31, size=J)
        ct = rnd(rng, (S, 2, N))
        ga, gb = linear_extract(d32(kern), d32(bias), d32(ct))
        for s in range(S):
            wa, wb = LO.linear(kern, bias, (ct[s, 0], ct[s, 1]))
            assert np.array_equal(h64(ga[s]), u(wa))
            assert np.array_equal(h64(gb[s]), u(wb))


@pytest.mark.parametrize("N,l,log2_beta", [(256, 6, 4), (512, 4, 6)])
def test_pack_lwe_to_rlwe_matches_oracle(N, l, log2_beta):
    from tfhe_b200 import client
    from tfhe_b200.lstm import GaloisKeys
    rng = np.random.default_rng(N + l)
    sk = rng.integers(0, 2, size=N)
    gal = client.galois_keys(sk, log2_beta, l, 1.0, rng)
    gk = GaloisKeys(gal, log2_beta, l, DEV)
    R = 5
    a = rnd(rng, (R, N))
    b = rnd(rng, (R,))
    got = gk.pack_lwe_to_rlwe(d32(a), d32(b))
    A, B = LO.pack_lwe_to_rlwe(a, b, cen(gal), log2_beta, l)
    assert np.array_equal(h64(got[:, 0]), u(A))
    assert np.array_equal(h64(got[:, 1]), u(B))
    gk.close()


def test_lut_mul_sum_matches_oracle():
    from tfhe_b200.lstm import lut_mul_sum
    rng = np.random.default_rng(11)
    N, G, K, S = 256, 2, 3, 2
    luts = rng.integers(-1, 2, size=(G, K, N)) * (rng.random((G, K, N)) < 0.3)
    luts[0, 0] = rng.integers(-2 ** 20, 2 ** 20, size=N)            # a dense row with large values
    ct = rnd(rng, (S, G, K, 2, N))
    got = lut_mul_sum(d32(luts), d32(ct))
    for s in range(S):
        pa, pb = LO.multiply_plaintext_ciphertext(luts, (ct[s, :, :, 0], ct[s, :, :, 1]))
        assert np.array_equal(h64(got[s, :, 0]), u(pa.sum(axis=0)))
        assert np.array_equal(h64(got[s, :, 1]), u(pb.sum(axis=0)))


@pytest.mark.parametrize("T", [1, 10, 256])
def test_pack_lwes_matches_oracle(T):
    from tfhe_b200.lstm import pack_lwes
    m = layer_material()
    rng = np.random.default_rng(12 + T)
    N = 256
    S = 2
    a = rnd(rng, (S, T, N))
    b = rnd(rng, (S, T))
    ksp = torch.from_numpy(np.ascontiguousarray(m["ksp"]).view(np.int32)).to(DEV)
    got = pack_lwes(ksp, PK_LOG2_BETA, PK_L, d32(a), d32(b))
    for s in range(S):
        pa, pb = LO.packing(a[s], b[s], m["layer"]["ksp_a"], m["layer"]["ksp_b"], PK_LOG2_BETA, PK_L, N)
        assert np.array_equal(h64(got[s, 0]), u(pa))
        assert np.array_equal(h64(got[s, 1]), u(pb))


def test_rotate_add_matches_oracle():
    from tfhe_b200.lstm import rlwe_rotate_add
    rng = np.random.default_rng(13)
    N, S = 256, 3
    x = rnd(rng, (S, 2, N))
    y = rnd(rng, (S, 2, N))
    for rot in (0, 5, 255, 256, 300, 511, -7):
        got = rlwe_rotate_add(d32(x), rot, d32(y))
        for s in range(S):
            ra, rb = LO.rotate((x[s, 0], x[s, 1]), rot)
            assert np.array_equal(h64(got[s, 0]), u(ra + y[s, 0]))
            assert np.array_equal(h64(got[s, 1]), u(rb + y[s, 1]))


def test_spike_lstm_timesteps_match_oracle():
    m, keys, layer = device_layer()
    p = m["p"]
    N = p["N"]
    T, S = 2, 2
    xs, _ = encrypt_inputs(m["sk"], T, S, N)
    H = torch.zeros((S, 2, N), dtype=torch.int32, device=DEV)
    C = torch.zeros_like(H)
    oh = [(np.zeros(N, np.int64), np.zeros(N, np.int64)) for _ in range(S)]
    oc = [(np.zeros(N, np.int64), np.zeros(N, np.int64)) for _ in range(S)]
    for t in range(T):
        H, C = layer.step(d32(xs[t]), H, C)
        for s in range(S):
            x_t = (cen(xs[t, s, 0]), cen(xs[t, s, 1]))
            oh[s], oc[s] = LO.spike_lstm_step(m["keys"], p, m["layer"], x_t, oh[s], oc[s])
            assert np.array_equal(h64(H[s, 0]), u(oh[s][0])), (t, s)
            assert np.array_equal(h64(H[s, 1]), u(oh[s][1])), (t, s)
            assert np.array_equal(h64(C[s, 0]), u(oc[s][0])), (t, s)
            assert np.array_equal(h64(C[s, 1]), u(oc[s][1])), (t, s)


def test_sequences_alone_equal_sequences_batched():
    m, keys, layer = device_layer()
    N = m["p"]["N"]
    xs, _ = encrypt_inputs(m["sk"], 2, 3, N, seed=21)
    xs_d = d32(xs)
    (Hb, Cb), _ = layer(xs_d)
    for s in range(3):
        (Hs, Cs), _ = layer(xs_d[:, s:s + 1].contiguous())
        assert torch.equal(Hs[0], Hb[s]) and torch.equal(Cs[0], Cb[s])


def test_cipher_mlp_head_matches_oracle():
    from tfhe_b200.lstm import CipherMLP, Linear
    m, keys, layer = device_layer()
    p = m["p"]
    N = p["N"]
    rng = np.random.default_rng(31)
    W1 = rng.integers(-7, 8, size=(INPUT_DIM + HIDDEN, 6))
    B1 = rng.integers(-2, 3, size=6) * 2 ** 22
    W2 = rng.integers(-7, 8, size=(6, 1))
    B2 = rng.integers(-2, 3, size=1) * 2 ** 22
    lin1, lin2 = Linear(6, N, 1.0, DEV), Linear(1, N, 1.0, DEV)
    lin1.set_weights(W1, B1)
    lin2.set_weights(W2, B2)
    s_head = rng.uniform(0.5, 2.0, size=6)
    relu = np.stack([LO.relu_lut(N, s, 2.0 ** 22) for s in s_head])
    head_dev = CipherMLP(keys, lin1, lin2, relu)
    xs, _ = encrypt_inputs(m["sk"], 1, 2, N, seed=33)
    got_a, got_b = head_dev(d32(xs[0]))
    head = {"kern1": lin1.kernel_np, "bias1": lin1.bias_np, "kern2": lin2.kernel_np, "bias2": lin2.bias_np,
            "relu_luts": relu, "ksp_a": m["layer"]["ksp_a"], "ksp_b": m["layer"]["ksp_b"],
            "pk_log2_beta": PK_LOG2_BETA, "pk_l": PK_L}
    for s in range(2):
        wa, wb = LO.cipher_mlp(m["keys"], p, head, (cen(xs[0, s, 0]), cen(xs[0, s, 1])))
        assert np.array_equal(h64(got_a[s]), u(wa))
        assert np.array_equal(h64(got_b[s]), u(wb))


@pytest.mark.parametrize("T", [1, 10, 256])
def test_packing_key_tensor_cores_match_oracle(T):
    """Packing on the tcgen05 tensor cores (base 2^7, 4 levels: int8 digits)
    equals the CUDA-core packing and the oracle."""
    from tfhe_b200 import client
    from tfhe_b200.lstm import PackingKey
    m = layer_material()
    rng = np.random.default_rng(40 + T)
    N, S = 256, 2
    ksp = client.packing_key(m["sk"], m["sk"], 7, 4, 1.0, rng)
    key = PackingKey(ksp, 7, 4, DEV)
    assert key.tensor_cores
    a = rnd(rng, (S, T, N))
    b = rnd(rng, (S, T))
    got_tc = key.pack(d32(a), d32(b), tensor_cores=1)
    got_cc = key.pack(d32(a), d32(b), tensor_cores=0)
    assert torch.equal(got_tc, got_cc)
    for s in range(S):
        pa, pb = LO.packing(a[s], b[s], cen(ksp[:, :, 0]), cen(ksp[:, :, 1]), 7, 4, N)
        assert np.array_equal(h64(got_tc[s, 0]), u(pa))
        assert np.array_equal(h64(got_tc[s, 1]), u(pb))
    key.close()


def test_packing_key_with_wide_digits_stays_on_cuda_cores():
    from tfhe_b200.lstm import PackingKey
    m = layer_material()
    key = PackingKey(m["ksp"], PK_LOG2_BETA, PK_L, DEV)       # base 2^8: digits reach 128
    assert not key.tensor_cores
    rng = np.random.default_rng(50)
    a = rnd(rng, (1, 5, 256))
    b = rnd(rng, (1, 5))
    got = key.pack(d32(a), d32(b))
    pa, pb = LO.packing(a[0], b[0], m["layer"]["ksp_a"], m["layer"]["ksp_b"], PK_LOG2_BETA, PK_L, 256)
    assert np.array_equal(h64(got[0, 0]), u(pa)) and np.array_equal(h64(got[0, 1]), u(pb))
    key.close()


def test_timestep_with_tensor_core_packing_matches_oracle():
    from tfhe_b200 import client
    from tfhe_b200.lstm import CipherSpikeLSTM, LayerKeys, PackingKey
    m, keys, layer = device_layer()
    rng = np.random.default_rng(60)
    ksp = client.packing_key(m["sk"], m["sk"], 7, 4, 1.0, rng)
    lk = LayerKeys(keys.pbs, keys.galois, torch.from_numpy(ksp.view(np.int32)).to(DEV), 7, 4,
                   PackingKey(ksp, 7, 4, DEV))
    L = m["layer"]
    tc_layer = CipherSpikeLSTM(lk, INPUT_DIM, HIDDEN, N_LUT, layer.W_f, layer.W_i, layer.W_o,
                               L["lut_f"], L["lut_i"], L["lut_o"])
    oracle_layer = dict(L, ksp_a=cen(ksp[:, :, 0]), ksp_b=cen(ksp[:, :, 1]), pk_log2_beta=7, pk_l=4)
    N = m["p"]["N"]
    xs, _ = encrypt_inputs(m["sk"], 2, 2, N, seed=61)
    H = torch.zeros((2, 2, N), dtype=torch.int32, device=DEV)
    C = torch.zeros_like(H)
    oh = [(np.zeros(N, np.int64), np.zeros(N, np.int64)) for _ in range(2)]
    oc = [(np.zeros(N, np.int64), np.zeros(N, np.int64)) for _ in range(2)]
    for t in range(2):
        H, C = tc_layer.step(d32(xs[t]), H, C)
        for s in range(2):
            oh[s], oc[s] = LO.spike_lstm_step(m["keys"], m["p"], oracle_layer, (cen(xs[t, s, 0]), cen(xs[t, s, 1])),
                                              oh[s], oc[s])
            assert np.array_equal(h64(H[s, 0]), u(oh[s][0])) and np.array_equal(h64(H[s, 1]), u(oh[s][1]))
            assert np.array_equal(h64(C[s, 0]), u(oc[s][0])) and np.array_equal(h64(C[s, 1]), u(oc[s][1]))


def test_timestep_graph_replay_equals_direct_steps():
    """The CUDA-graph timestep (StepGraph) reproduces direct steps bit for bit."""
    from tfhe_b200.lstm import StepGraph
    m, keys, layer = device_layer()
    N = m["p"]["N"]
    xs, _ = encrypt_inputs(m["sk"], 3, 2, N, seed=71)
    xs_d = d32(xs)
    g = StepGraph(layer, 2)
    Hg, Cg = g.run(xs_d)
    H = torch.zeros((2, 2, N), dtype=torch.int32, device=DEV)
    C = torch.zeros_like(H)
    for t in range(3):
        H, C = layer.step(xs_d[t], H, C)
    assert torch.equal(Hg, H) and torch.equal(Cg, C)


def test_packing_key_unaligned_input_uses_cuda_cores():
    """LWE masks that are not 16-byte aligned take the CUDA-core packing (the
    tensor-core kernel loads 16-byte vectors) with the same result."""
    from tfhe_b200 import client
    from tfhe_b200.lstm import PackingKey
    m = layer_material()
    rng = np.random.default_rng(80)
    ksp = client.packing_key(m["sk"], m["sk"], 7, 4, 1.0, rng)
    key = PackingKey(ksp, 7, 4, DEV)
    a = rnd(rng, (1, 6, 256))
    b = rnd(rng, (1, 6))
    big = torch.zeros((a.size + 1,), dtype=torch.int32, device=DEV)
    big[1:] = d32(a).reshape(-1)
    a_view = big[1:].view(1, 6, 256)
    assert a_view.data_ptr() % 16 != 0
    got = key.pack(a_view, d32(b))
    pa, pb = LO.packing(a[0], b[0], cen(ksp[:, :, 0]), cen(ksp[:, :, 1]), 7, 4, 256)
    assert np.array_equal(h64(got[0, 0]), u(pa)) and np.array_equal(h64(got[0, 1]), u(pb))
    key.close()
