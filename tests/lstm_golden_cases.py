"""Inputs of the Spike-LSTM golden fixtures (tests/golden/lstm_golden.npz).

Two layers, both rebuilt here from fixed seeds so that the fixtures hold
outputs only:

  tiny  the small layer of lstm_cases (N = 256 bootstrapping parameters,
        hidden 8, input 4, 2 packed LUTs, Galois key 2^4 x 6, packing key
        2^8 x 3), two timesteps of one sequence;
  cfg4  the one-layer encrypted Spike-LSTM workload: PBS at n = 630,
        N = 1024, gadget 2^7 x 3, collapse 3; hidden 128, embedding dim 64,
        4 packed LUTs, weights in [-7, 7], Galois key 2^4 x 6, packing key
        2^7 x 4 (the tensor-core packing); one timestep of one sequence of
        Zipf(1.1) tokens over a vocabulary of 8192.

Each case also carries a CipherMLP head (linear, ReLU bootstrap per unit,
packing, linear).  Its ReLU ramps use dyadic slopes so that the reference's
float ramp (nn_tfhe/activation.py:186-194) is made of exact integers.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from oracle import lstm_oracle as LO
from oracle import tfhe_oracle as O

Q = 2.0 ** 32


def cen(u):
    """uint32 torus words -> centred int64."""
    return np.asarray(u, dtype=np.uint32).view(np.int32).astype(np.int64)


@dataclass
class Case:
    name: str
    p: dict                 # bootstrapping parameters (oracle dict)
    keys: O.KeySet          # PBS keys in the oracle's (reference's) layout
    sk: np.ndarray          # GLWE secret (N,)
    input_dim: int
    hidden: int
    n_lut: int
    gal_log2_beta: int
    gal_l: int
    pk_log2_beta: int
    pk_l: int
    beta_x: int
    galois: np.ndarray      # (log2 N, gal_l, 2, N) uint32
    ksp: np.ndarray         # (N, pk_l, 2, N) uint32
    W: dict                 # gate -> (input_dim + hidden, hidden / n_lut) int
    B: dict                 # gate -> (hidden / n_lut,) int, absolute (torus units)
    lut_f: np.ndarray       # (n_lut, per, N) int
    lut_i: np.ndarray       # (per, N) int
    lut_o: np.ndarray       # (n_lut, per, N) int
    xs: np.ndarray          # (T, 1, 2, N) uint32 input RLWEs
    head_W1: np.ndarray
    head_B1: np.ndarray
    head_W2: np.ndarray
    head_B2: np.ndarray
    s_head: np.ndarray      # dyadic ReLU slopes
    head_x: np.ndarray      # (2, N) uint32 RLWE fed to the head

    @property
    def N(self):
        return self.p["N"]

    @property
    def per(self):
        return self.hidden // self.n_lut

    def oracle_layer(self):
        """The layer as lstm_oracle.spike_lstm_step takes it."""
        layer = {"input_dim": self.input_dim, "hidden": self.hidden, "n_lut": self.n_lut,
                 "galois": cen(self.galois), "gal_log2_beta": self.gal_log2_beta, "gal_l": self.gal_l,
                 "ksp_a": cen(self.ksp[:, :, 0]), "ksp_b": cen(self.ksp[:, :, 1]),
                 "pk_log2_beta": self.pk_log2_beta, "pk_l": self.pk_l,
                 "lut_f": self.lut_f, "lut_o": self.lut_o, "lut_i": self.lut_i}
        for g in "fio":
            kern, bias = LO.linear_kernel_polynomial(self.W[g], self.B[g], np.ones(self.per), self.N)
            layer[f"kern_{g}"], layer[f"bias_{g}"] = kern, bias
        return layer

    def relu_luts(self):
        return np.stack([LO.relu_lut(self.N, s, float(self.beta_x)) for s in self.s_head])

    def oracle_head(self):
        k1, b1 = LO.linear_kernel_polynomial(self.head_W1, self.head_B1, np.ones(self.head_W1.shape[1]), self.N)
        k2, b2 = LO.linear_kernel_polynomial(self.head_W2, self.head_B2, np.ones(self.head_W2.shape[1]), self.N)
        return {"kern1": k1, "bias1": b1, "kern2": k2, "bias2": b2, "relu_luts": self.relu_luts(),
                "ksp_a": cen(self.ksp[:, :, 0]), "ksp_b": cen(self.ksp[:, :, 1]),
                "pk_log2_beta": self.pk_log2_beta, "pk_l": self.pk_l}


def _dyadic_slopes(rng, count):
    return rng.choice(np.array([0.5, 0.625, 0.75, 0.875, 1.0]), size=count)


def _head(rng, in_dim, hidden, J, beta_x):
    W1 = np.zeros((in_dim + hidden, J), dtype=np.int64)
    W1[in_dim:] = rng.integers(-7, 8, size=(hidden, J))
    B1 = rng.integers(-3, 4, size=J) * beta_x
    W2 = rng.integers(-7, 8, size=(J, 1))
    B2 = rng.integers(-3, 4, size=1) * beta_x
    return W1, B1, W2, B2, _dyadic_slopes(rng, J)


def tiny_case() -> Case:
    import lstm_cases as LC
    from tfhe_b200 import client
    m = LC.layer_material()
    L = m["layer"]
    N = m["p"]["N"]
    xs, _ = LC.encrypt_inputs(m["sk"], 2, 1, N, seed=91)
    rng = np.random.default_rng(92)
    W1, B1, W2, B2, s_head = _head(rng, LC.INPUT_DIM, LC.HIDDEN, 6, int(LC.BETA_X))
    hx = np.zeros(N, dtype=np.int64)
    hx[LC.INPUT_DIM:LC.INPUT_DIM + LC.HIDDEN] = rng.integers(0, 2, size=LC.HIDDEN) * int(LC.BETA_X)
    ha, hb = client.encrypt_rlwe(hx, m["sk"], 1.0, rng)
    return Case("tiny", m["p"], m["keys"], m["sk"], LC.INPUT_DIM, LC.HIDDEN, LC.N_LUT, LC.GAL_LOG2_BETA,
                LC.GAL_L, LC.PK_LOG2_BETA, LC.PK_L, int(LC.BETA_X), m["galois"], m["ksp"], m["mats"],
                m["biases"], L["lut_f"], L["lut_i"], L["lut_o"], xs, W1, B1, W2, B2, s_head,
                np.stack([ha, hb]))


def oracle_keyset(ck) -> O.KeySet:
    """client.ClientKeys -> the oracle's key layout (float64 centred)."""
    p = ck.params
    d = p.oracle_dict()
    ksk = (cen(ck.ksk_a).astype(np.float64), cen(ck.ksk_b).astype(np.float64)[..., None])
    ks = O.KeySet(params=d, sk_glwe=ck.sk_glwe.astype(np.float64), sk_lwe=ck.sk_lwe.astype(np.float64), ksk=ksk,
                  bsk_coeff=cen(ck.bsk).astype(np.float64))
    ks.bsk_ordered = O.bsk_coeff_fourier_ordered(ks.bsk_coeff)
    ks.all_rot = O.all_rot_possible_fourier(p.N)
    return ks


_CFG4 = {}


def cfg4_case() -> Case:
    if "case" in _CFG4:
        return _CFG4["case"]
    from tfhe_b200 import client
    from tfhe_b200.spike_model import SpikeModelConfig, build_model, encrypt_tokens, layer_luts, sample_tokens
    cfg = SpikeModelConfig()
    model = build_model(cfg, seed=41)
    rng = np.random.default_rng(42)
    tokens = sample_tokens(rng, 1, 1, cfg.vocab, cfg.zipf)
    xs = encrypt_tokens(model, tokens, rng)                     # (1, 1, 2, N)
    L = model.layers[0]
    lut_f, lut_i, lut_o = layer_luts(cfg, L)
    B = {g: L.B[g] * cfg.beta_x for g in "fio"}
    W1, B1, W2, B2, s_head = _head(rng, cfg.emb_dim, cfg.hidden, cfg.hidden, cfg.beta_x)
    N = cfg.pbs.N
    hx = np.zeros(N, dtype=np.int64)
    hx[cfg.emb_dim:cfg.emb_dim + cfg.hidden] = rng.integers(0, 2, size=cfg.hidden) * cfg.beta_x
    ha, hb = client.encrypt_rlwe(hx, model.keys.sk_glwe, cfg.sigma_rlwe, rng)
    case = Case("cfg4", cfg.pbs.oracle_dict(), oracle_keyset(model.keys), model.keys.sk_glwe.astype(np.int64),
                cfg.emb_dim, cfg.hidden, cfg.n_lut, cfg.gal_log2_beta, cfg.gal_l, cfg.pk_log2_beta, cfg.pk_l,
                cfg.beta_x, model.galois, model.ksp, L.W, B, lut_f, lut_i, lut_o, xs, W1, B1, W2, B2, s_head,
                np.stack([ha, hb]))
    case.client_keys = model.keys
    _CFG4["case"] = case
    return case


CASES = {"tiny": tiny_case, "cfg4": cfg4_case}


def op_inputs(case: Case):
    """Seeded operator-level inputs (uint32): R LWEs for pack_lwe_to_rlwe,
    the (n_lut, per) LWEs whose encrypted LUTs prepare_LUT builds, and the
    hidden LWEs packed into one RLWE."""
    rng = np.random.default_rng({"tiny": 201, "cfg4": 202}[case.name])
    N = case.N
    u = lambda *shape: rng.integers(0, 2 ** 32, size=shape, dtype=np.uint64).astype(np.uint32)
    return {"r2r_a": u(2, N), "r2r_b": u(2),
            "prep_a": u(case.n_lut, case.per, N), "prep_b": u(case.n_lut, case.per),
            "pack_a": u(case.hidden, N), "pack_b": u(case.hidden)}


FULL_LIMIT = 64 * 1024      # arrays above this many bytes are kept as a digest + first row


def put(out, key, arr):
    """Store a torus array (uint32 words) in a fixture dict."""
    import hashlib
    a = np.ascontiguousarray(np.asarray(arr, dtype=np.int64) & 0xFFFFFFFF).astype(np.uint32)
    if a.nbytes <= FULL_LIMIT:
        out[key] = a
    else:
        out[key + "_sha256"] = np.frombuffer(hashlib.sha256(a.tobytes()).digest(), dtype=np.uint8)
        out[key + "_shape"] = np.array(a.shape, dtype=np.int64)
        out[key + "_row0"] = a.reshape(a.shape[0], -1)[0]


def matches(fx, key, got):
    """True when `got` (torus words, any integer dtype) equals the fixture."""
    import hashlib
    g = np.ascontiguousarray(np.asarray(got, dtype=np.int64) & 0xFFFFFFFF).astype(np.uint32)
    if key in fx:
        return g.shape == fx[key].shape and np.array_equal(g, fx[key])
    if tuple(fx[key + "_shape"]) != g.shape:
        return False
    if not np.array_equal(g.reshape(g.shape[0], -1)[0], fx[key + "_row0"]):
        return False
    return hashlib.sha256(g.tobytes()).digest() == fx[key + "_sha256"].tobytes()


# ---------------------------------------------------------------- q = 2^64
_Q64 = {}


def cfg4_q64_case():
    """The one-layer workload on the reference's own torus and bootstrapping
    parameters (q = 2^64, N = 2048, n = 702, gadget 2^13 x 2, collapse 3),
    one timestep of one sequence, and its head."""
    if "case" in _Q64:
        return _Q64["case"]
    from tfhe_b200 import client64
    from tfhe_b200.spike_model import build_model, config_q64, encrypt_tokens, layer_luts, sample_tokens
    cfg = config_q64()
    model = build_model(cfg, seed=43)
    rng = np.random.default_rng(44)
    tokens = sample_tokens(rng, 1, 1, cfg.vocab, cfg.zipf)
    xs = encrypt_tokens(model, tokens, rng)                     # (1, 1, 2, N) uint64
    L = model.layers[0]
    lut_f, lut_i, lut_o = layer_luts(cfg, L)
    W1, B1, W2, B2, s_head = _head(rng, cfg.emb_dim, cfg.hidden, cfg.hidden, cfg.beta_x)
    N = cfg.pbs.N
    hx = np.zeros(N, dtype=np.int64)
    hx[cfg.emb_dim:cfg.emb_dim + cfg.hidden] = rng.integers(0, 2, size=cfg.hidden) * cfg.beta_x
    ha, hb = client64.encrypt_rlwe(hx, model.keys.sk_glwe, cfg.sigma_rlwe, rng)
    c = dict(cfg=cfg, model=model, tokens=tokens, xs=xs, lut_f=lut_f, lut_i=lut_i, lut_o=lut_o,
             W={g: L.W[g] for g in "fio"}, B={g: L.B[g] * cfg.beta_x for g in "fio"}, gamma=L.gamma, eta=L.eta,
             head_W1=W1, head_B1=B1, head_W2=W2, head_B2=B2, s_head=s_head, head_x=np.stack([ha, hb]),
             hx_plain=hx)
    _Q64["case"] = c
    return c


def q64_op_inputs(c):
    """Seeded uint64 inputs of the operator fixtures at q = 2^64."""
    rng = np.random.default_rng(203)
    N, hid, n_lut = c["cfg"].pbs.N, c["cfg"].hidden, c["cfg"].n_lut
    u = lambda *shape: rng.integers(0, 2 ** 64, size=shape, dtype=np.uint64)
    return {"prep_a": u(n_lut, hid // n_lut, N), "prep_b": u(n_lut, hid // n_lut),
            "pack_a": u(hid, N), "pack_b": u(hid)}


def torus_dist64(x, y):
    """|x - y| on Z/2^64 as float64 (x, y uint64 words)."""
    d = (np.asarray(x, dtype=np.uint64) - np.asarray(y, dtype=np.uint64)).view(np.int64)
    return np.abs(d.astype(np.float64))
