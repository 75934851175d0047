"""Synthetic encrypted Spike-LSTM models on the engine: random integer
weights, thresholds and embeddings of a given shape (the reference's GLUE
data, HF embeddings and trained checkpoints are not available), client key
material, encryption of token sequences, decryption of logits, and a
plaintext mirror of the spiking recurrence.

Encoding: inputs x, spikes h and cell values c sit at scale beta_x on the
torus; a pre-activation z (integer units) is read by the packed step LUTs
over linspace(-1, 1) at z * 4 beta_x / q (get_plain_LUT with s = 1,
nn_tfhe/utils_spike.py:72-87); the head's ReLU LUT covers [0, s_head) the
same way.  Two tori: q = 2^32 with the config-1 bootstrapping parameters
(beta_x = 2^22), and the reference's own q = 2^64 with its bootstrapping
parameters (parameters_crypto.py:6-32; beta_x = 2^54, so z reads the LUTs at
the same z / 256 on both).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import torch

from . import client
from . import client64
from .engine import Keys
from .lstm import CipherMLP, CipherSpikeLSTM, GaloisKeys, LayerKeys, Linear, PackingKey
from .params import CONFIG1, ParamSet


@dataclass
class SpikeModelConfig:
    vocab: int = 8192
    zipf: float = 1.1
    emb_dim: int = 64
    hidden: int = 128
    layers: int = 1
    n_lut: int = 4
    weight_max: int = 7
    emb_max: int = 2
    log2_beta_x: int = 22
    gal_log2_beta: int = 4
    gal_l: int = 6
    pk_log2_beta: int = 7          # digits in int8: the packing runs on the tensor cores
    pk_l: int = 4
    sigma_rlwe: float = 1.0
    pbs: ParamSet = field(default_factory=lambda: CONFIG1)
    torus_bits: int = 32

    @property
    def beta_x(self) -> int:
        return 1 << self.log2_beta_x


def config_q64(**kw) -> SpikeModelConfig:
    """The layer on the reference's torus q = 2^64 with its bootstrapping
    parameters (N = 2048, n = 702, gadget 2^13 x 2, collapse 3, sigma 2^17),
    Galois key 2^8 x 5 (the reference's 40 bits, 2^2 x 20), packing key
    2^7 x 5 (35 bits where the reference keeps 32, parameters_crypto.py:18-20;
    base 2^7 keeps the digits in int8, so the packing runs on the tensor
    cores), inputs at beta_x = 2^54."""
    base = dict(log2_beta_x=54, gal_log2_beta=8, gal_l=5, pk_log2_beta=7, pk_l=5, sigma_rlwe=2.0 ** 17,
                pbs=client64.REF64, torus_bits=64)
    base.update(kw)
    return SpikeModelConfig(**base)


def plain_lut(N, n_lut, index, gamma):
    """get_plain_LUT with s = 1 (nn_tfhe/utils_spike.py:72-87) as integers."""
    sub = N // n_lut
    part = np.linspace(-1.0, 1.0, num=sub, endpoint=False)
    full = np.zeros(N, dtype=np.int64)
    full[np.arange(sub) * n_lut + index] = (part >= gamma).astype(np.int64)
    return np.concatenate([full[N // 2:], -full[: N // 2]])        # X^(-N/2)


def relu_lut(N, s, beta_x):
    """ReluBoostrapper's ramp LUT (nn_tfhe/activation.py:186-194), rounded."""
    ramp = np.arange(N // 2) * (2.0 * s / N) * beta_x
    return np.rint(np.concatenate([ramp, np.zeros(N // 2)])).astype(np.int64)


@dataclass
class PlainLayer:
    W: dict            # gate -> (in_dim + hidden, hidden / n_lut) int
    B: dict            # gate -> (hidden / n_lut,) int (units of beta_x)
    gamma: dict        # gate -> (n_lut, hidden / n_lut)
    eta: np.ndarray    # (n_lut, hidden / n_lut)
    in_dim: int


@dataclass
class SpikeModel:
    cfg: SpikeModelConfig
    keys: client.ClientKeys
    galois: np.ndarray
    ksp: np.ndarray
    embedding: np.ndarray            # (vocab, emb_dim) int
    layers: list                     # PlainLayer per layer
    head_W1: np.ndarray
    head_B1: np.ndarray
    head_W2: np.ndarray
    head_B2: np.ndarray
    s_head: np.ndarray


def build_model(cfg: SpikeModelConfig, seed: int = 0) -> SpikeModel:
    rng = np.random.default_rng(seed)
    cl = client64 if cfg.torus_bits == 64 else client
    keys = cl.keygen(cfg.pbs, seed + 1)
    sk = keys.sk_glwe
    galois = cl.galois_keys(sk, cfg.gal_log2_beta, cfg.gal_l, cfg.sigma_rlwe, rng)
    ksp = cl.packing_key(sk, sk, cfg.pk_log2_beta, cfg.pk_l, cfg.sigma_rlwe, rng)
    per = cfg.hidden // cfg.n_lut
    layers = []
    in_dim = cfg.emb_dim
    for _ in range(cfg.layers):
        dim = in_dim + cfg.hidden
        W = {g: rng.integers(-cfg.weight_max, cfg.weight_max + 1, size=(dim, per)) for g in "fio"}
        B = {g: rng.integers(-3, 4, size=per) for g in "fio"}
        gamma = {g: rng.uniform(-0.5, 0.5, size=(cfg.n_lut, per)) for g in "fio"}
        eta = rng.uniform(0.25, 1.0, size=(cfg.n_lut, per))
        layers.append(PlainLayer(W, B, gamma, eta, in_dim))
        in_dim = cfg.hidden
    J = cfg.hidden
    last_in = layers[-1].in_dim
    head_W1 = np.zeros((last_in + cfg.hidden, J), dtype=np.int64)
    head_W1[last_in:] = rng.integers(-cfg.weight_max, cfg.weight_max + 1, size=(cfg.hidden, J))
    head_B1 = rng.integers(-3, 4, size=J)
    head_W2 = rng.integers(-cfg.weight_max, cfg.weight_max + 1, size=(J, 1))
    head_B2 = rng.integers(-3, 4, size=1)
    s_head = rng.uniform(0.5, 1.0, size=J)
    emb = rng.integers(-cfg.emb_max, cfg.emb_max + 1, size=(cfg.vocab, cfg.emb_dim))
    return SpikeModel(cfg, keys, galois, ksp, emb, layers, head_W1, head_B1, head_W2, head_B2, s_head)


def sample_tokens(rng, count, length, vocab, a):
    """Token ids from a Zipf(a) law truncated to the vocabulary."""
    w = 1.0 / np.arange(1, vocab + 1) ** a
    return rng.choice(vocab, size=(count, length), p=w / w.sum())


def encrypt_tokens(model: SpikeModel, tokens, rng):
    """(S, T) token ids -> (T, S, 2, N) RLWEs (uint32, or uint64 on the 2^64
    torus) of the embeddings at coefficients [0, emb_dim), scale beta_x."""
    cfg = model.cfg
    N = cfg.pbs.N
    S, T = tokens.shape
    poly = np.zeros((T, S, N), dtype=np.int64)
    poly[..., : cfg.emb_dim] = model.embedding[tokens.T] * cfg.beta_x
    cl = client64 if cfg.torus_bits == 64 else client
    a, b = cl.encrypt_rlwe(poly, model.keys.sk_glwe, cfg.sigma_rlwe, rng)
    return np.stack([a, b], axis=2)


def encrypted_words(model: SpikeModel, x) -> torch.Tensor:
    """Host torus words -> the torch dtype of the model's torus (int32 /
    int64 bit patterns), on the host."""
    dt = np.int64 if model.cfg.torus_bits == 64 else np.int32
    return torch.from_numpy(np.ascontiguousarray(x).view(dt))


def layer_luts(cfg: SpikeModelConfig, L: PlainLayer):
    """The layer's packed step LUTs as integer polynomials: lut_f and lut_o
    (n_lut, hidden / n_lut, N) read the forget / output pre-activations
    (values 0/1), lut_i (hidden / n_lut, N) the input gate, its n_lut
    sub-LUTs weighted by eta at scale beta_x (the lut_f / lut_i / lut_o of
    CipherSpikeLSTM, nn_tfhe/Spike_LSTM.py:73-100)."""
    N = cfg.pbs.N
    per = cfg.hidden // cfg.n_lut
    lut = {g: np.stack([np.stack([plain_lut(N, cfg.n_lut, i, L.gamma[g][i, kk]) for kk in range(per)])
                        for i in range(cfg.n_lut)]) for g in "fo"}
    lut_i = np.zeros((per, N), dtype=np.int64)
    for i in range(cfg.n_lut):
        for kk in range(per):
            lut_i[kk] += np.rint(plain_lut(N, cfg.n_lut, i, L.gamma["i"][i, kk]) * L.eta[i, kk]
                                 * cfg.beta_x).astype(np.int64)
    return lut["f"], lut_i, lut["o"]


@dataclass
class DeviceModel:
    layers: list                     # CipherSpikeLSTM per layer
    head: CipherMLP
    keys: LayerKeys


def to_device(model: SpikeModel, device=None) -> DeviceModel:
    cfg = model.cfg
    dev = device or torch.device("cuda", torch.cuda.current_device())
    N = cfg.pbs.N
    k = model.keys
    if cfg.torus_bits == 64:
        from .torus64 import GaloisKeys64, Keys64, PackingKey64
        pbs = Keys64(k, dev)
        gk = GaloisKeys64(model.galois, cfg.gal_log2_beta, cfg.gal_l, dev)
        pk = PackingKey64(model.ksp, cfg.pk_log2_beta, cfg.pk_l, dev)
        lk = LayerKeys(pbs, gk, pk.ksp, cfg.pk_log2_beta, cfg.pk_l, pk)
    else:
        pbs = Keys.create(cfg.pbs, k.bsk, k.ksk_a, k.ksk_b)
        gk = GaloisKeys(model.galois, cfg.gal_log2_beta, cfg.gal_l, dev)
        ksp = torch.from_numpy(np.ascontiguousarray(model.ksp).view(np.int32)).to(dev)
        lk = LayerKeys(pbs, gk, ksp, cfg.pk_log2_beta, cfg.pk_l,
                       PackingKey(model.ksp, cfg.pk_log2_beta, cfg.pk_l, dev))
    per = cfg.hidden // cfg.n_lut
    layers = []
    for L in model.layers:
        lins = []
        for g in "fio":
            lin = Linear(per, N, 1.0, dev)
            lin.set_weights(L.W[g], L.B[g] * cfg.beta_x)
            lins.append(lin)
        lut_f, lut_i, lut_o = layer_luts(cfg, L)
        layers.append(CipherSpikeLSTM(lk, L.in_dim, cfg.hidden, cfg.n_lut, *lins, lut_f, lut_i, lut_o))
    lin1 = Linear(cfg.hidden, N, 1.0, dev)
    lin1.set_weights(model.head_W1, model.head_B1 * cfg.beta_x)
    lin2 = Linear(1, N, 1.0, dev)
    lin2.set_weights(model.head_W2, model.head_B2 * cfg.beta_x)
    relu = np.stack([relu_lut(N, s, cfg.beta_x) for s in model.s_head])
    return DeviceModel(layers, CipherMLP(lk, lin1, lin2, relu), lk)


def run_layers(dm: DeviceModel, xs, states=None, stream=None, per_gate=False):
    """All layers over T timesteps for S sequences: xs (T, S, 2, N).  Layer
    l + 1 reads layer l's hidden spikes moved to coefficients [0, hidden).
    Returns the final hidden RLWE of the last layer and the per-layer
    states [(H, C)].  per_gate=True launches one bootstrap per gate and
    sequence (the plain per-gate form)."""
    from .lstm import rlwe_rotate_add
    T, S = xs.shape[0], xs.shape[1]
    N = xs.shape[-1]
    if states is None:
        states = [(torch.zeros((S, 2, N), dtype=xs.dtype, device=xs.device),
                   torch.zeros((S, 2, N), dtype=xs.dtype, device=xs.device)) for _ in dm.layers]
    for t in range(T):
        x = xs[t]
        for li, layer in enumerate(dm.layers):
            H, C = layer.step(x, *states[li], stream, per_gate)
            states[li] = (H, C)
            x = rlwe_rotate_add(H, -layer.input_dim, stream=stream)
    return states[-1][0], states


def decrypt_logits(model: SpikeModel, out_a, out_b):
    """LWE logits (S, 1, N) / (S, 1) -> decrypted values in units of beta_x."""
    if model.cfg.torus_bits == 64:
        a = out_a.cpu().numpy().view(np.uint64).reshape(out_a.shape[0], -1)
        b = out_b.cpu().numpy().view(np.uint64).reshape(-1)
        return client64.phase(a, b, model.keys.sk_glwe).astype(np.float64) / model.cfg.beta_x
    a = out_a.cpu().numpy().view(np.uint32).reshape(out_a.shape[0], -1)
    b = out_b.cpu().numpy().view(np.uint32).reshape(-1)
    ph = client.phase(a, b, model.keys.sk_glwe)
    return ph / model.cfg.beta_x


def plain_forward(model: SpikeModel, tokens):
    """The spiking recurrence and head in plaintext with the encrypted
    model's quantisation (nn_jax/Spike_LSTM.py semantics with the LUT
    thresholds read at z * 4 beta_x / q): returns logits (S,) in units of
    beta_x and the final hidden spikes (S, hidden)."""
    cfg = model.cfg
    S, T = tokens.shape
    scale = 4.0 * cfg.beta_x / 2.0 ** cfg.torus_bits
    per = cfg.hidden // cfg.n_lut
    sub = cfg.pbs.N // cfg.n_lut
    # the bootstrap reads sub-LUT entry rint(z * scale * sub / 2) of linspace(-1, 1, sub)
    grid = lambda z: np.clip(np.rint(z * scale * sub / 2) * 2 / sub, -1.0, 1.0 - 2.0 / sub)

    def spike(z, gamma):            # (S, per), (n_lut, per) -> (S, n_lut * per) in cell order
        g = grid(z)
        return np.concatenate([(g >= gamma[i]).astype(np.float64) for i in range(cfg.n_lut)], axis=1)

    x_all = model.embedding[tokens].astype(np.float64)           # (S, T, emb)
    states = [(np.zeros((S, cfg.hidden)), np.zeros((S, cfg.hidden))) for _ in model.layers]
    for t in range(T):
        x = x_all[:, t]
        for li, L in enumerate(model.layers):
            h, c = states[li]
            hx = np.concatenate([x, h], axis=1)
            z = {g: hx @ L.W[g] + L.B[g] for g in "fio"}
            f = spike(z["f"], L.gamma["f"])
            i = spike(z["i"], L.gamma["i"]) * np.concatenate([L.eta[k] for k in range(cfg.n_lut)])[None]
            c = f * c + i
            o = spike(z["o"], L.gamma["o"])
            h = o * c
            states[li] = (h, c)
            x = h
    h = states[-1][0]
    h_in = np.concatenate([np.zeros((S, model.layers[-1].in_dim)), h], axis=1)
    z1 = h_in @ model.head_W1 + model.head_B1
    u = z1 * scale                   # ReLU ramp over phases [0, q/4), zero above and below
    y1 = np.where((u > 0) & (u < 1), u * model.s_head[None], 0.0)
    return (y1 @ model.head_W2 + model.head_B2)[:, 0], h
