"""The GPU Spike-LSTM path against golden fixtures recorded from the
reference's own code (tests/golden/make_lstm_golden.py), bit for bit:
Linear, pack_lwe_to_rlwe, prepare_LUT (+ the sub-LUT sum), packing on CUDA
cores and on the tcgen05 tensor cores, the scan_step recurrence and the
CipherMLP head, at the small layer (N = 256, hidden 8) and at the one-layer
workload shape (PBS n = 630, N = 1024; hidden 128, embedding 64, 4 packed
LUTs)."""
import os

import numpy as np
import pytest
import torch

import lstm_golden_cases as GC

pytestmark = pytest.mark.gpu

FX = np.load(os.path.join(os.path.dirname(__file__), "golden", "lstm_golden.npz"))
DEV = torch.device("cuda", 0) if torch.cuda.is_available() else None
_BUILT = {}


def d32(x):
    return torch.from_numpy(np.ascontiguousarray((np.asarray(x, dtype=np.int64) & 0xFFFFFFFF).astype(np.uint32))
                            .view(np.int32)).to(DEV)


def host(t):
    return t.cpu().numpy().view(np.uint32)


def device_case(name):
    """The case's layer, head and keys on the GPU (built once per case)."""
    if name in _BUILT:
        return _BUILT[name]
    from tfhe_b200.engine import Keys
    from tfhe_b200.lstm import CipherMLP, CipherSpikeLSTM, GaloisKeys, LayerKeys, Linear, PackingKey
    from tfhe_b200.params import CONFIG1, TINY_C3
    c = GC.CASES[name]()
    if name == "tiny":
        k = c.keys
        pbs = Keys.create(TINY_C3, k.bsk_coeff, k.ksk[0], k.ksk[1].reshape(k.ksk[1].shape[:2]))
    else:
        ck = c.client_keys
        pbs = Keys.create(CONFIG1, ck.bsk, ck.ksk_a, ck.ksk_b)
    gk = GaloisKeys(c.galois, c.gal_log2_beta, c.gal_l, DEV)
    ksp = torch.from_numpy(np.ascontiguousarray(c.ksp).view(np.int32)).to(DEV)
    pkey = PackingKey(c.ksp, c.pk_log2_beta, c.pk_l, DEV)
    keys = LayerKeys(pbs, gk, ksp, c.pk_log2_beta, c.pk_l, pkey)
    lins = {}
    for g in "fio":
        lin = Linear(c.per, c.N, 1.0, DEV)
        lin.set_weights(c.W[g], c.B[g])
        lins[g] = lin
    layer = CipherSpikeLSTM(keys, c.input_dim, c.hidden, c.n_lut, lins["f"], lins["i"], lins["o"], c.lut_f,
                            c.lut_i, c.lut_o)
    h1, h2 = Linear(c.head_W1.shape[1], c.N, 1.0, DEV), Linear(1, c.N, 1.0, DEV)
    h1.set_weights(c.head_W1, c.head_B1)
    h2.set_weights(c.head_W2, c.head_B2)
    head = CipherMLP(keys, h1, h2, c.relu_luts())
    _BUILT[name] = (c, keys, lins, layer, head)
    return _BUILT[name]


CASES = ["tiny", "cfg4"]


@pytest.mark.parametrize("name", CASES)
def test_gpu_linear_matches_reference(name):
    c, keys, lins, layer, head = device_case(name)
    x0 = d32(c.xs[0])                                           # (1, 2, N); HX = x_0 + 0
    for g in "fio":
        assert np.array_equal(lins[g].kernel_np, FX[f"{name}_kern_{g}"].astype(np.int64)), g
        a, b = lins[g](x0)
        assert GC.matches(FX, f"{name}_lin_{g}_a", host(a[0])), g
        assert GC.matches(FX, f"{name}_lin_{g}_b", host(b[0])), g


@pytest.mark.parametrize("name", CASES)
def test_gpu_pack_lwe_to_rlwe_matches_reference(name):
    c, keys, lins, layer, head = device_case(name)
    ops = GC.op_inputs(c)
    got = keys.galois.pack_lwe_to_rlwe(d32(ops["r2r_a"]), d32(ops["r2r_b"]))
    for r in range(2):
        # the reference leaves the trace sums unreduced; the engine reduces mod 2^32
        assert np.array_equal(host(got[r, 0]), (FX[f"{name}_r2r{r}_A"] & 0xFFFFFFFF).astype(np.uint32))
        assert np.array_equal(host(got[r, 1]), (FX[f"{name}_r2r{r}_B"] & 0xFFFFFFFF).astype(np.uint32))


@pytest.mark.parametrize("name", CASES)
def test_gpu_prepare_lut_matches_reference(name):
    c, keys, lins, layer, head = device_case(name)
    ops = GC.op_inputs(c)
    a = d32(ops["prep_a"]).reshape(1, c.hidden, c.N)
    b = d32(ops["prep_b"]).reshape(1, c.hidden)
    got = layer._encrypted_luts(a, b, layer.lut_f)              # (1, per, 2, N)
    assert GC.matches(FX, f"{name}_prep_a", host(got[0, :, 0]))
    assert GC.matches(FX, f"{name}_prep_b", host(got[0, :, 1]))


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("tensor_cores", [0, 1])
def test_gpu_packing_matches_reference(name, tensor_cores):
    c, keys, lins, layer, head = device_case(name)
    if tensor_cores and not keys.packing.tensor_cores:
        pytest.skip("this packing key's digits do not fit int8")
    ops = GC.op_inputs(c)
    got = keys.packing.pack(d32(ops["pack_a"])[None], d32(ops["pack_b"])[None], tensor_cores=tensor_cores)
    assert GC.matches(FX, f"{name}_pack_a", host(got[0, 0]))
    assert GC.matches(FX, f"{name}_pack_b", host(got[0, 1]))


@pytest.mark.parametrize("name", CASES)
def test_gpu_recurrence_matches_reference(name):
    c, keys, lins, layer, head = device_case(name)
    (_, _), _ = layer(d32(c.xs))                                 # warm-up pass, results discarded
    H = torch.zeros((1, 2, c.N), dtype=torch.int32, device=DEV)
    C = torch.zeros_like(H)
    hs, cs = [], []
    for t in range(c.xs.shape[0]):
        H, C = layer.step(d32(c.xs[t]), H, C)
        hs.append(host(H[0]))
        cs.append(host(C[0]))
    hs, cs = np.stack(hs), np.stack(cs)
    assert GC.matches(FX, f"{name}_H_a", hs[:, 0])
    assert GC.matches(FX, f"{name}_H_b", hs[:, 1])
    assert GC.matches(FX, f"{name}_C_a", cs[:, 0])
    assert GC.matches(FX, f"{name}_C_b", cs[:, 1])


@pytest.mark.parametrize("name", CASES)
def test_gpu_head_matches_reference(name):
    c, keys, lins, layer, head = device_case(name)
    ya, yb = head(d32(c.head_x)[None])
    assert GC.matches(FX, f"{name}_head_a", host(ya[0]))
    assert GC.matches(FX, f"{name}_head_b", host(yb[0]))
