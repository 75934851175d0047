"""Encrypted Spike-LSTM layer on the engine: the reference's CipherSpikeLSTM,
Linear and CipherMLP (nn_tfhe/Spike_LSTM.py) with every operator on the
GPU through the C ABI, batched over the sequences in flight.

State layout per sequence (nn_tfhe/Spike_LSTM.py:103-184):
  x_t  RLWE, the encrypted input at coefficients [0, input_dim)
  H    RLWE, the hidden spikes at coefficients [input_dim, input_dim + hidden)
  C    RLWE, the cell state at coefficients [0, hidden)
Each timestep runs three linears (hidden / n_lut outputs each), two
encrypted-LUT preparations (pack_lwe_to_rlwe x plaintext sub-LUTs, summed
over the n_lut packed sub-LUTs), two programmable bootstraps with n_lut
outputs, the sum f*C + i, and two LWE -> RLWE packings.

Values are uint32 torus words (q = 2^32) held in int32 tensors, or, with
keys of the reference's own modulus (torus64.Keys64), uint64 words (q = 2^64)
held in int64 tensors; every operator picks its kernels by the tensors' dtype.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from .engine import Keys, _need, _ptr, _stream


# ---------------------------------------------------------------- operators
def _t64():
    from . import torus64
    return torus64


def linear_extract(weights, bias, rlwe, out_a=None, out_b=None, stream=None):
    """Linear.__call__ for S ciphertexts: weights (J, N), bias (J) int32,
    rlwe (S, 2, N) -> (S, J, N), (S, J)."""
    if rlwe.dtype == torch.int64:
        return _t64().linear_extract(weights, bias, rlwe, out_a, out_b, stream)
    J, N = weights.shape
    S = rlwe.shape[0]
    _need(weights, torch.int32, (J, N), "weights")
    _need(bias, torch.int32, (J,), "bias")
    _need(rlwe, torch.int32, (S, 2, N), "rlwe")
    out_a = out_a if out_a is not None else torch.empty((S, J, N), dtype=torch.int32, device=rlwe.device)
    out_b = out_b if out_b is not None else torch.empty((S, J), dtype=torch.int32, device=rlwe.device)
    _need(out_a, torch.int32, (S, J, N), "out_a")
    _need(out_b, torch.int32, (S, J), "out_b")
    _lib.check(_lib.load().tfhe_linear_extract(_ptr(weights), _ptr(bias), J, _ptr(rlwe), S, N, _ptr(out_a),
                                               _ptr(out_b), _stream(stream)))
    return out_a, out_b


def lut_mul_sum(luts, rlwe, out=None, stream=None):
    """sum over g of luts[g][k] * rlwe[s][g][k]: luts (G, K, N) int32,
    rlwe (S, G, K, 2, N) -> (S, K, 2, N)."""
    if rlwe.dtype == torch.int64:
        return _t64().lut_mul_sum(luts, rlwe, out, stream)
    G, K, N = luts.shape
    S = rlwe.shape[0]
    _need(luts, torch.int32, (G, K, N), "luts")
    _need(rlwe, torch.int32, (S, G, K, 2, N), "rlwe")
    out = out if out is not None else torch.empty((S, K, 2, N), dtype=torch.int32, device=rlwe.device)
    _need(out, torch.int32, (S, K, 2, N), "out")
    _lib.check(_lib.load().tfhe_lut_mul_sum(_ptr(luts), G, K, _ptr(rlwe), S, N, _ptr(out), _stream(stream)))
    return out


class GaloisKeys:
    """Device Galois keys of pack_lwe_to_rlwe (FP64 Fourier domain)."""

    def __init__(self, keys_u32: np.ndarray, log2_beta: int, l: int, device=None, stream=None):
        steps, l2, two, N = keys_u32.shape
        if l2 != l or two != 2 or (1 << steps) != N:
            raise ValueError("galois keys must be (log2 N, l, 2, N)")
        dev = device or torch.device("cuda", torch.cuda.current_device())
        src = torch.from_numpy(np.ascontiguousarray(keys_u32).view(np.int32)).to(dev)
        h = ctypes.c_void_p()
        _lib.check(_lib.load().tfhe_galois_keys_create(N, log2_beta, l, _ptr(src), _stream(stream), ctypes.byref(h)))
        self._h, self.N, self.log2_beta, self.l = h, N, log2_beta, l

    def close(self):
        if self._h:
            _lib.load().tfhe_galois_keys_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def pack_lwe_to_rlwe(self, lwe_a, lwe_b, out=None, stream=None):
        """lwe_a (R, N), lwe_b (R) -> (R, 2, N)."""
        R, N = lwe_a.shape
        _need(lwe_a, torch.int32, (R, self.N), "lwe_a")
        _need(lwe_b, torch.int32, (R,), "lwe_b")
        out = out if out is not None else torch.empty((R, 2, N), dtype=torch.int32, device=lwe_a.device)
        _need(out, torch.int32, (R, 2, N), "out")
        _lib.check(_lib.load().tfhe_pack_lwe_to_rlwe(self._h, _ptr(lwe_a), _ptr(lwe_b), R, _ptr(out),
                                                     _stream(stream)))
        return out


def pack_lwes(ksp, log2_beta, l, lwe_a, lwe_b, out=None, stream=None):
    """packing: lwe_a (S, T, n_dim), lwe_b (S, T) with ksp (n_dim, l, 2, N)
    -> (S, 2, N)."""
    n_dim, l2, two, N = ksp.shape
    S, T, nd = lwe_a.shape
    if l2 != l or two != 2 or nd != n_dim:
        raise ValueError("packing key / LWE shapes disagree")
    _need(ksp, torch.int32, (n_dim, l, 2, N), "ksp")
    _need(lwe_a, torch.int32, (S, T, n_dim), "lwe_a")
    _need(lwe_b, torch.int32, (S, T), "lwe_b")
    out = out if out is not None else torch.empty((S, 2, N), dtype=torch.int32, device=lwe_a.device)
    _need(out, torch.int32, (S, 2, N), "out")
    _lib.check(_lib.load().tfhe_pack_lwes(_ptr(ksp), n_dim, N, log2_beta, l, _ptr(lwe_a), _ptr(lwe_b), T, S,
                                          _ptr(out), _stream(stream)))
    return out


class PackingKey:
    """Device packing key (tfhe_packing_key_create): packs T LWEs per RLWE on
    the tcgen05 tensor cores where the key allows, else on CUDA cores."""

    def __init__(self, ksp_u32: np.ndarray, log2_beta: int, l: int, device=None, stream=None):
        n_dim, l2, two, N = ksp_u32.shape
        if l2 != l or two != 2:
            raise ValueError("packing key must be (n_dim, l, 2, N)")
        dev = device or torch.device("cuda", torch.cuda.current_device())
        src = torch.from_numpy(np.ascontiguousarray(ksp_u32).view(np.int32)).to(dev)
        h = ctypes.c_void_p()
        _lib.check(_lib.load().tfhe_packing_key_create(_ptr(src), n_dim, N, log2_beta, l, _stream(stream),
                                                       ctypes.byref(h)))
        self._h, self.n_dim, self.N, self.log2_beta, self.l = h, n_dim, N, log2_beta, l

    @property
    def tensor_cores(self) -> bool:
        return bool(_lib.load().tfhe_packing_key_uses_tensor_cores(self._h))

    def close(self):
        if self._h:
            _lib.load().tfhe_packing_key_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def pack(self, lwe_a, lwe_b, out=None, tensor_cores=-1, stream=None):
        """lwe_a (S, T, n_dim), lwe_b (S, T) -> (S, 2, N)."""
        S, T, nd = lwe_a.shape
        _need(lwe_a, torch.int32, (S, T, self.n_dim), "lwe_a")
        _need(lwe_b, torch.int32, (S, T), "lwe_b")
        out = out if out is not None else torch.empty((S, 2, self.N), dtype=torch.int32, device=lwe_a.device)
        _need(out, torch.int32, (S, 2, self.N), "out")
        _lib.check(_lib.load().tfhe_pack_lwes_with_key(self._h, _ptr(lwe_a), _ptr(lwe_b), T, S, _ptr(out),
                                                       int(tensor_cores), _stream(stream)))
        return out


def rlwe_rotate_add(x, rot, y=None, out=None, stream=None):
    """X^rot * x + y for RLWEs (S, 2, N)."""
    if x.dtype == torch.int64:
        return _t64().rlwe_rotate_add(x, rot, y, out, stream)
    S, two, N = x.shape
    _need(x, torch.int32, (S, 2, N), "x")
    if y is not None:
        _need(y, torch.int32, (S, 2, N), "y")
    out = out if out is not None else torch.empty_like(x)
    _need(out, torch.int32, (S, 2, N), "out")
    _lib.check(_lib.load().tfhe_rlwe_rotate_add(_ptr(x), int(rot), _ptr(y) if y is not None else None, S, N,
                                                _ptr(out), _stream(stream)))
    return out


def u32_add(x, y, out=None, stream=None):
    """x + y on the torus of the tensors' dtype."""
    if x.dtype == torch.int64:
        return _t64().add(x, y, out, stream)
    if x.shape != y.shape:
        raise ValueError("add: shapes differ")
    _need(x, torch.int32, tuple(x.shape), "x")
    _need(y, torch.int32, tuple(y.shape), "y")
    out = out if out is not None else torch.empty_like(x)
    _lib.check(_lib.load().tfhe_u32_add(_ptr(x), _ptr(y), x.numel(), _ptr(out), _stream(stream)))
    return out


# ---------------------------------------------------------------- layers
def weights_to_polynomial(weights: np.ndarray) -> np.ndarray:
    """schemas/polynomial_jax.py:136-148."""
    poly = -np.flip(np.asarray(weights, dtype=np.float64).reshape(-1))
    poly[-1] = np.asarray(weights).reshape(-1)[0]
    return poly


class Linear:
    """Linear (nn_tfhe/Spike_LSTM.py:15-58): integer weight polynomials in
    the layout of set_weights, applied to an RLWE and extracted at 0."""

    def __init__(self, output_dim: int, degree: int, factor, device=None):
        self.degree = degree
        self.factor = np.broadcast_to(np.asarray(factor, dtype=np.float64), (output_dim,)).copy()
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        self.kernel_polynomial = None
        self.bias = None

    def set_weights(self, W, B):
        """W (in, out) and B (out) plaintext; weights are round(factor * W)."""
        W = np.asarray(W, dtype=np.float64)
        wt = W.T
        if wt.shape[0] != self.factor.shape[0]:
            self.factor = np.broadcast_to(self.factor[:1], (wt.shape[0],)).copy()
        wp = np.stack([weights_to_polynomial(r) for r in np.round(self.factor[:, None] * wt)])
        kern = np.zeros((wt.shape[0], self.degree))
        kern[:, -wt.shape[1] + 1:] = wp[:, :-1]
        kern[:, 0] = wp[:, -1]
        bias = np.round(self.factor * np.asarray(B, dtype=np.float64))
        self.kernel_np = kern.astype(np.int64)
        self.bias_np = bias.astype(np.int64)
        self.kernel_polynomial = torch.from_numpy(kern.astype(np.int64).astype(np.int32)).to(self.device)
        self.bias = torch.from_numpy(bias.astype(np.int64).astype(np.int32)).to(self.device)
        self.bias64 = torch.from_numpy(bias.astype(np.int64)).to(self.device)

    def __call__(self, rlwe, stream=None):
        bias = self.bias64 if rlwe.dtype == torch.int64 else self.bias
        return linear_extract(self.kernel_polynomial, bias, rlwe, stream=stream)


@dataclass
class LayerKeys:
    """Everything a layer needs on the device."""
    pbs: Keys                 # bootstrapping + key-switching keys (engine.Keys)
    galois: GaloisKeys        # pack_lwe_to_rlwe
    ksp: torch.Tensor         # packing key (N, l, 2, N) int32
    pk_log2_beta: int
    pk_l: int
    packing: "PackingKey" = None   # device packing key (tensor cores where possible)

    @property
    def torus_bits(self) -> int:
        """64 with keys of the 2^64 torus (torus64.Keys64), else 32."""
        return 64 if self.ksp.dtype == torch.int64 else 32

    def pack(self, lwe_a, lwe_b, stream=None):
        if self.packing is not None:
            return self.packing.pack(lwe_a, lwe_b, stream=stream)
        return pack_lwes(self.ksp, self.pk_log2_beta, self.pk_l, lwe_a, lwe_b, stream=stream)


class CipherSpikeLSTM:
    """CipherSpikeLSTM (nn_tfhe/Spike_LSTM.py:62-184) for S sequences at
    once.  lut_f, lut_o: (n_lut, hidden / n_lut, N) plaintext sub-LUTs;
    lut_i: (hidden / n_lut, N) plaintext LUT bodies (the reference's lut_i[1];
    its mask lut_i[0] is zero)."""

    def __init__(self, keys: LayerKeys, input_dim: int, hidden_dim: int, n_lut: int,
                 linear_f: Linear, linear_i: Linear, linear_o: Linear, lut_f, lut_i, lut_o):
        self.keys = keys
        self.N = keys.galois.N
        self.input_dim, self.hidden_dim, self.n_lut = input_dim, hidden_dim, n_lut
        if hidden_dim % n_lut or input_dim + hidden_dim > self.N:
            raise ValueError("need n_lut | hidden and input_dim + hidden <= N")
        self.per = hidden_dim // n_lut
        self.W_f, self.W_i, self.W_o = linear_f, linear_i, linear_o
        dev = linear_f.device
        self.dtype = torch.int64 if keys.torus_bits == 64 else torch.int32
        np_dt = np.int64 if keys.torus_bits == 64 else np.int32
        word = lambda x: torch.from_numpy(np.ascontiguousarray(np.asarray(x, dtype=np.int64)).astype(np_dt)).to(dev)
        self.lut_f = word(lut_f).reshape(n_lut, self.per, self.N)
        self.lut_o = word(lut_o).reshape(n_lut, self.per, self.N)
        self.lut_i = word(lut_i).reshape(self.per, self.N)
        self.device = dev

    # prepare_LUT (nn_tfhe/activation.py:103-106) of every cell LWE, summed
    # over the packed sub-LUTs
    def _encrypted_luts(self, lwe_a, lwe_b, luts, stream=None):
        S = lwe_a.shape[0]
        rl = self.keys.galois.pack_lwe_to_rlwe(lwe_a.reshape(-1, self.N), lwe_b.reshape(-1), stream=stream)
        return lut_mul_sum(luts, rl.reshape(S, self.n_lut, self.per, 2, self.N), stream=stream)

    def _spikes(self, boot_a, boot_b, S):
        """(S * per, n_lut, N) bootstrap outputs -> cell order (S, hidden, N):
        cell i * per + k holds sub-LUT i of pre-activation k."""
        a = boot_a.reshape(S, self.per, self.n_lut, self.N).permute(0, 2, 1, 3).reshape(S, self.hidden_dim, self.N)
        b = boot_b.reshape(S, self.per, self.n_lut).permute(0, 2, 1).reshape(S, self.hidden_dim)
        return a.contiguous(), b.contiguous()

    def step_phases(self, x_t, H, C, stream=None):
        """One timestep for S sequences as a generator over its two
        bootstraps: it yields (lwe_a, lwe_b, luts) for each bootstrap, is sent
        the bootstrap's (out_a, out_b), and returns (H_t, C_t).  Drivers can
        merge the bootstraps of several layers into one launch."""
        S, N, per, hid = x_t.shape[0], self.N, self.per, self.hidden_dim
        if x_t.dtype == torch.int64:
            c_a, c_b = _t64().sample_extract(C, hid, stream)
        else:
            c_a = torch.empty((S, hid, N), dtype=torch.int32, device=x_t.device)
            c_b = torch.empty((S, hid), dtype=torch.int32, device=x_t.device)
            _lib.check(_lib.load().tfhe_sample_extract(_ptr(C), N, hid, _ptr(c_a), _ptr(c_b), S, _stream(stream)))
        hx = rlwe_rotate_add(H, 0, x_t, stream=stream)
        f_a, f_b = self.W_f(hx, stream)
        i_a, i_b = self.W_i(hx, stream)
        o_a, o_b = self.W_o(hx, stream)
        lut_c = self._encrypted_luts(c_a, c_b, self.lut_f, stream)                     # (S, per, 2, N)
        # first bootstrap: [F, I] against [encrypted LUT of C, plaintext lut_i]
        in_a = torch.cat([f_a, i_a], dim=1).reshape(S * 2 * per, N)
        in_b = torch.cat([f_b, i_b], dim=1).reshape(S * 2 * per)
        luts = torch.zeros((S, 2 * per, 2, N), dtype=x_t.dtype, device=x_t.device)
        luts[:, :per] = lut_c
        luts[:, per:, 1] = self.lut_i
        boot_a, boot_b = yield in_a, in_b, luts.reshape(S * 2 * per, 2, N)
        boot_a = boot_a.reshape(S, 2 * per, self.n_lut, N)
        boot_b = boot_b.reshape(S, 2 * per, self.n_lut)
        fc_a, fc_b = self._spikes(boot_a[:, :per], boot_b[:, :per], S)
        si_a, si_b = self._spikes(boot_a[:, per:], boot_b[:, per:], S)
        ct_a = u32_add(fc_a, si_a, stream=stream)
        ct_b = u32_add(fc_b, si_b, stream=stream)
        # second bootstrap: O against the encrypted LUT of C_t
        lut_h = self._encrypted_luts(ct_a, ct_b, self.lut_o, stream)
        h_a, h_b = yield o_a.reshape(S * per, N), o_b.reshape(S * per), lut_h.reshape(S * per, 2, N)
        h_a, h_b = self._spikes(h_a, h_b, S)
        k = self.keys
        C_t = k.pack(ct_a, ct_b, stream=stream)
        H_p = k.pack(h_a, h_b, stream=stream)
        H_t = rlwe_rotate_add(H_p, self.input_dim, stream=stream)
        return H_t, C_t

    def step(self, x_t, H, C, stream=None, per_gate=False):
        """One timestep for S sequences: x_t, H, C (S, 2, N) -> (H_t, C_t)."""
        return step_merged([(self, x_t, H, C)], stream, per_gate)[0]

    def __call__(self, xs, stream=None):
        """xs (T, S, 2, N): the encrypted inputs of T timesteps.  Returns the
        final (H, C) and the per-step H (T, S, 2, N) (jax.lax.scan of the
        reference)."""
        T, S = xs.shape[0], xs.shape[1]
        H = torch.zeros((S, 2, self.N), dtype=xs.dtype, device=xs.device)
        C = torch.zeros_like(H)
        hs = []
        for t in range(T):
            H, C = self.step(xs[t], H, C, stream)
            hs.append(H)
        return (H, C), torch.stack(hs)


def step_merged(items, stream=None, per_gate=False):
    """One timestep of several layers at once: items [(layer, x_t, H, C)]
    over any numbers of sequences.  The layers' bootstraps run as one
    launch per phase (all layers share the bootstrapping key and n_lut);
    returns [(H_t, C_t)] in the order of items.  per_gate=True instead
    launches one bootstrap per gate of each sequence (hidden / n_lut
    ciphertexts), the way the reference's timestep issues them."""
    gens, reqs, results = [], [], [None] * len(items)
    for i, (layer, x, H, C) in enumerate(items):
        g = layer.step_phases(x, H, C, stream)
        gens.append((i, layer, g))
        reqs.append(next(g))
    while gens:
        keys = gens[0][1].keys.pbs
        n_lut = gens[0][1].n_lut
        if any(l.keys.pbs is not keys or l.n_lut != n_lut for _, l, _ in gens):
            raise ValueError("merged layers must share the bootstrapping key and n_lut")
        counts = [r[0].shape[0] for r in reqs]
        if len(reqs) == 1:
            a, b, lut = reqs[0]
        else:
            a = torch.cat([r[0] for r in reqs])
            b = torch.cat([r[1] for r in reqs])
            lut = torch.cat([r[2] for r in reqs])
        if per_gate:
            per = gens[0][1].per
            N = a.shape[-1]
            out_a = torch.empty((a.shape[0], n_lut, N), dtype=a.dtype, device=a.device)
            out_b = torch.empty((a.shape[0], n_lut), dtype=a.dtype, device=a.device)
            for o in range(0, a.shape[0], per):
                keys.pbs(a[o:o + per], b[o:o + per], lut[o:o + per], n_lut, out_a[o:o + per], out_b[o:o + per],
                         stream=stream)
        else:
            out_a, out_b = keys.pbs(a, b, lut, n_lut, stream=stream)
        nxt_gens, nxt_reqs, off = [], [], 0
        for (i, layer, g), c in zip(gens, counts):
            try:
                nxt_reqs.append(g.send((out_a[off:off + c], out_b[off:off + c])))
                nxt_gens.append((i, layer, g))
            except StopIteration as stop:
                results[i] = stop.value
            off += c
        gens, reqs = nxt_gens, nxt_reqs
    return results


class StepGraph:
    """One CipherSpikeLSTM timestep for S sequences captured in a CUDA graph
    on fixed device buffers (x, H, C -> H_out, C_out); run() replays it once
    per timestep, so a sequence costs one graph launch per token instead of
    the step's ~25 kernel launches and their host work."""

    def __init__(self, layer: "CipherSpikeLSTM", S: int, stream=None):
        dev = layer.device
        N = layer.N
        self.layer = layer
        self.x = torch.zeros((S, 2, N), dtype=layer.dtype, device=dev)
        self.H = torch.zeros_like(self.x)
        self.C = torch.zeros_like(self.x)
        layer.step(self.x, self.H, self.C)        # uncaptured: kernel attributes, status word, allocator
        torch.cuda.synchronize()
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self.H_out, self.C_out = layer.step(self.x, self.H, self.C)

    def step(self, x_t, H, C):
        """(S, 2, N) inputs -> graph-owned (H_t, C_t), valid until the next replay."""
        self.x.copy_(x_t)
        self.H.copy_(H)
        self.C.copy_(C)
        self.graph.replay()
        return self.H_out, self.C_out

    def run(self, xs):
        """xs (T, S, 2, N) from zero state -> final (H, C) (copies)."""
        self.H.zero_()
        self.C.zero_()
        for t in range(xs.shape[0]):
            self.x.copy_(xs[t])
            self.graph.replay()
            self.H.copy_(self.H_out)
            self.C.copy_(self.C_out)
        return self.H.clone(), self.C.clone()


class CipherMLP:
    """CipherMLP (nn_tfhe/Spike_LSTM.py:187-206) with the ReLU bootstrap of
    ReluBoostrapper (nn_tfhe/activation.py:166-237): linear1, one bootstrap
    per unit with its own ramp LUT, packing, linear2."""

    def __init__(self, keys: LayerKeys, linear1: Linear, linear2: Linear, relu_luts):
        self.keys, self.linear1, self.linear2 = keys, linear1, linear2
        dev = linear1.device
        np_dt = np.int64 if keys.torus_bits == 64 else np.int32
        self.relu_luts = torch.from_numpy(np.asarray(relu_luts, dtype=np.int64).astype(np_dt)).to(dev)

    def __call__(self, H, stream=None):
        S, _, N = H.shape
        h1_a, h1_b = self.linear1(H, stream)                               # (S, J, N)
        J = h1_a.shape[1]
        luts = torch.zeros((S, J, 2, N), dtype=H.dtype, device=H.device)
        luts[:, :, 1] = self.relu_luts
        y_a, y_b = self.keys.pbs.pbs(h1_a.reshape(S * J, N), h1_b.reshape(S * J), luts.reshape(S * J, 2, N), 1,
                                     stream=stream)
        k = self.keys
        h2 = k.pack(y_a.reshape(S, J, N), y_b.reshape(S, J), stream=stream)
        return self.linear2(h2, stream)
