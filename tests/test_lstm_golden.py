"""The Spike-LSTM oracle against golden fixtures recorded from the
reference's own code (tests/golden/make_lstm_golden.py): Linear,
pack_lwe_to_rlwe, prepare_LUT, packing, the scan_step recurrence and the
CipherMLP head, bit for bit, at the small layer and at the one-layer
workload shape (N = 1024, hidden 128, 4 packed LUTs).  CPU only."""
import os

import numpy as np
import pytest

import lstm_golden_cases as GC
from oracle import lstm_oracle as LO

FX = np.load(os.path.join(os.path.dirname(__file__), "golden", "lstm_golden.npz"))


def _case(name):
    if name + "_H_a" not in FX and name + "_H_a_sha256" not in FX:
        pytest.skip(f"no fixtures for {name}")
    return GC.CASES[name]()


def _x(u, i):
    return GC.cen(u[i])


@pytest.mark.parametrize("name", ["tiny", "cfg4"])
def test_linear_matches_reference(name):
    c = _case(name)
    layer = c.oracle_layer()
    x0 = (GC.cen(c.xs[0, 0, 0]), GC.cen(c.xs[0, 0, 1]))
    for g in "fio":
        assert np.array_equal(layer[f"kern_{g}"], FX[f"{name}_kern_{g}"].astype(np.int64)), g
        a, b = LO.linear(layer[f"kern_{g}"], layer[f"bias_{g}"], x0)
        assert GC.matches(FX, f"{name}_lin_{g}_a", a), g
        assert GC.matches(FX, f"{name}_lin_{g}_b", b), g


@pytest.mark.parametrize("name", ["tiny", "cfg4"])
def test_pack_lwe_to_rlwe_matches_reference(name):
    c = _case(name)
    ops = GC.op_inputs(c)
    A, B = LO.pack_lwe_to_rlwe(GC.cen(ops["r2r_a"]), GC.cen(ops["r2r_b"]), GC.cen(c.galois), c.gal_log2_beta,
                               c.gal_l)
    for r in range(2):
        assert np.array_equal(A[r], FX[f"{name}_r2r{r}_A"])
        assert np.array_equal(B[r], FX[f"{name}_r2r{r}_B"])


@pytest.mark.parametrize("name", ["tiny", "cfg4"])
def test_prepare_lut_matches_reference(name):
    c = _case(name)
    ops = GC.op_inputs(c)
    a = GC.cen(ops["prep_a"]).reshape(c.hidden, c.N)
    b = GC.cen(ops["prep_b"]).reshape(c.hidden)
    ra, rb = LO.pack_lwe_to_rlwe(a, b, GC.cen(c.galois), c.gal_log2_beta, c.gal_l)
    pa, pb = LO.multiply_plaintext_ciphertext(np.asarray(c.lut_f, np.int64).reshape(c.hidden, c.N), (ra, rb))
    pa = LO.cmod_exact(pa.reshape(c.n_lut, c.per, c.N).sum(axis=0))
    pb = LO.cmod_exact(pb.reshape(c.n_lut, c.per, c.N).sum(axis=0))
    assert GC.matches(FX, f"{name}_prep_a", pa)
    assert GC.matches(FX, f"{name}_prep_b", pb)


@pytest.mark.parametrize("name", ["tiny", "cfg4"])
def test_packing_matches_reference(name):
    c = _case(name)
    ops = GC.op_inputs(c)
    layer = c.oracle_layer()
    pa, pb = LO.packing(GC.cen(ops["pack_a"]), GC.cen(ops["pack_b"]), layer["ksp_a"], layer["ksp_b"],
                        c.pk_log2_beta, c.pk_l, c.N)
    assert GC.matches(FX, f"{name}_pack_a", pa)
    assert GC.matches(FX, f"{name}_pack_b", pb)


@pytest.mark.parametrize("name", ["tiny", "cfg4"])
def test_recurrence_matches_reference(name):
    c = _case(name)
    layer = c.oracle_layer()
    N = c.N
    H = (np.zeros(N, np.int64), np.zeros(N, np.int64))
    C = (np.zeros(N, np.int64), np.zeros(N, np.int64))
    hs_a, hs_b, cs_a, cs_b = [], [], [], []
    for t in range(c.xs.shape[0]):
        x_t = (GC.cen(c.xs[t, 0, 0]), GC.cen(c.xs[t, 0, 1]))
        H, C = LO.spike_lstm_step(c.keys, c.p, layer, x_t, H, C)
        hs_a.append(H[0]), hs_b.append(H[1]), cs_a.append(C[0]), cs_b.append(C[1])
    assert GC.matches(FX, f"{name}_H_a", np.stack(hs_a))
    assert GC.matches(FX, f"{name}_H_b", np.stack(hs_b))
    assert GC.matches(FX, f"{name}_C_a", np.stack(cs_a))
    assert GC.matches(FX, f"{name}_C_b", np.stack(cs_b))


@pytest.mark.parametrize("name", ["tiny", "cfg4"])
def test_head_matches_reference(name):
    c = _case(name)
    wa, wb = LO.cipher_mlp(c.keys, c.p, c.oracle_head(), (GC.cen(c.head_x[0]), GC.cen(c.head_x[1])))
    assert GC.matches(FX, f"{name}_head_a", wa)
    assert GC.matches(FX, f"{name}_head_b", wb)
