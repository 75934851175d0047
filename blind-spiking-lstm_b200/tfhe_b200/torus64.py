"""The engine on the reference's own torus, q = 2^64 (parameters_crypto.py:6),
for the encrypted Spike-LSTM at the reference's parameters.  Torus values are
uint64 bit patterns held in torch.int64 CUDA tensors; all arithmetic runs in
libtfhe_b200.so (csrc/torus64.cu and the FP64 blind rotation at q = 2^64).

  Keys64        device bootstrapping + key-switching keys; pbs() =
                HeavysideBoostrapper.cuboot (nn_tfhe/activation.py:148-162):
                the key switch, then one kernel for the rotation indices, the
                blind rotation, the rotation by -b~ and the many-LUT extraction
                (tfhe64_cuboot_merge); blind_rotate_reflayout() is the same
                chain through tfhe_mul_bootstrap on the reference's key layout
  GaloisKeys64  pack_lwe_to_rlwe (schemas/text_jax.py:316-345)
  PackingKey64  packing (schemas/text_jax.py:211-239)
  linear_extract / lut_mul_sum / rlwe_rotate_add / add / sample_extract
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from . import client64 as C64
from .engine import _need, _ptr, _stream

I64 = torch.int64


def device_u64(x, device=None) -> torch.Tensor:
    """Host uint64 words (or integers) -> int64 CUDA tensor of the same bits."""
    return torch.from_numpy(np.ascontiguousarray(C64.u64(x)).view(np.int64)).to(device or "cuda")


def host_u64(t: torch.Tensor) -> np.ndarray:
    return t.cpu().numpy().view(np.uint64)


class Keys64:
    """Device key material of one 64-bit parameter set."""

    def __init__(self, keys: C64.ClientKeys64, device=None, reflayout=False, stream=None):
        p = keys.params
        dev = device or torch.device("cuda", torch.cuda.current_device())
        self.params, self.device = p, dev
        lib = _lib.load()
        prm = _lib.TfheParams(p.N, p.n, p.big, p.log2_beta_bs, p.l_bs, p.collapse, p.log2_beta_ks, p.l_ks, 64)
        bsk = np.ascontiguousarray(C64.u64(keys.bsk))                                   # (2, 2, G M, L, N)
        h = ctypes.c_void_p()
        with torch.cuda.device(dev):
            _lib.check(lib.tfhe64_keys_create(ctypes.byref(prm), bsk.ctypes.data, _stream(stream), ctypes.byref(h)))
        self.handle = h
        self.ksk = device_u64(keys.ksk, dev)                                            # (n_big l, n + 1)
        # the reference's key layout for tfhe_mul_bootstrap, on request
        self.bsk = self.rot = self.bsk_dims = None
        if reflayout:
            self.bsk = torch.from_numpy(C64.bsk_fourier_grouped(keys.bsk, p)).to(dev)  # (G, 2, L, 2, M, d)
            self.rot = torch.from_numpy(C64.monomial_fourier(p.N)).to(dev)             # (2N, d)
            self.bsk_dims = (ctypes.c_int64 * 6)(*self.bsk.shape)
        # the key switch on the tensor cores where its digits fit 8 bits
        self.ksk_limbs = _limbs(self.ksk, p.big * p.l_ks, p.n + 1) if _tc_ok(p.big, p.l_ks, p.log2_beta_ks) else None
        self.ks_tensor_cores = -1

    def keyswitch(self, a, b, out_a=None, out_b=None, tensor_cores=-1, stream=None):
        """key_switch_LWE: on the tensor cores when the key has limbs and a is
        16-byte aligned (tensor_cores -1 / 1), else on CUDA cores; same result."""
        p = self.params
        B = a.shape[0]
        _need(a, I64, (B, p.big), "a")
        _need(b, I64, (B,), "b")
        out_a = out_a if out_a is not None else torch.empty((B, p.n), dtype=I64, device=a.device)
        out_b = out_b if out_b is not None else torch.empty((B,), dtype=I64, device=a.device)
        lib = _lib.load()
        if tensor_cores < 0:
            tensor_cores = self.ks_tensor_cores
        if self.ksk_limbs is not None and tensor_cores != 0 and a.data_ptr() % 16 == 0:
            _lib.check(lib.tfhe64_keyswitch_tc(_ptr(self.ksk_limbs), p.big, p.n, p.l_ks, p.log2_beta_ks, _ptr(a),
                                               _ptr(b), _ptr(out_a), _ptr(out_b), B, _stream(stream)))
        else:
            _lib.check(lib.tfhe64_keyswitch(_ptr(self.ksk), p.big, p.n, p.l_ks, p.log2_beta_ks, _ptr(a), _ptr(b),
                                            _ptr(out_a), _ptr(out_b), B, _stream(stream)))
        return out_a, out_b

    def set_tuning(self, ciphertexts_per_cta=0, prefetch=-1, persistent=-1, ks_tensor_cores=-1,
                   l2_prefetch=-1) -> None:
        """Launch shapes (speed only; 0 / -1: automatic), as Keys.set_tuning:
        the blind rotation's ciphertexts per CTA, L1 prefetch, persistent
        CTAs, L2 prefetch, and whether the key switch uses the tensor cores."""
        t = _lib.TfheTuning(int(ciphertexts_per_cta), int(prefetch), int(persistent), int(ks_tensor_cores),
                            int(l2_prefetch))
        _lib.check(_lib.load().tfhe_keys_set_tuning(self.handle, ctypes.byref(t)))
        self.ks_tensor_cores = int(ks_tensor_cores)

    def cluster_size(self, batch: int) -> int:
        """CTAs per ciphertext of a batch's blind rotation (8, 4 or 2: one
        ciphertext per cluster of that many CTAs; 1: several per CTA)."""
        return int(_lib.load().tfhe_keys_cluster_size(self.handle, int(batch)))

    def close(self):
        if getattr(self, "handle", None):
            _lib.load().tfhe_keys_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check_lut(self, lut, B):
        if lut.shape[0] not in (1, B):
            raise ValueError("lut must hold 1 or B polynomial pairs")
        _need(lut, I64, (lut.shape[0], 2, self.params.N), "lut")

    def blind_rotate(self, lwe_a, lwe_b, lut, n_lut=1, out=None, stream=None):
        """The collapsed CMux chain of multiply_seq_monomial (cuTFHE/
        multiply.py:54-92) from key-switched LWEs, then the rotation by
        X^(-b~) (schemas/RLWE_jax.py:295-297): ACC (B, 2, N) int64."""
        p = self.params
        B = lwe_a.shape[0]
        _need(lwe_a, I64, (B, p.n), "lwe_a")
        _need(lwe_b, I64, (B,), "lwe_b")
        self._check_lut(lut, B)
        out = out if out is not None else torch.empty((B, 2, p.N), dtype=I64, device=lwe_a.device)
        _need(out, I64, (B, 2, p.N), "out")
        _lib.check(_lib.load().tfhe64_blind_rotate(self.handle, _ptr(lwe_a), _ptr(lwe_b), _ptr(lut), lut.shape[0],
                                                   int(n_lut), _ptr(out), B, _stream(stream)))
        return out

    def cuboot_merge(self, lwe_a, lwe_b, lut, n_lut=1, out_a=None, out_b=None, stream=None):
        """cuboot_merge (schemas/RLWE_jax.py:281-303) in one kernel:
        (B, n), (B) -> (B, n_lut, N), (B, n_lut)."""
        p = self.params
        B = lwe_a.shape[0]
        _need(lwe_a, I64, (B, p.n), "lwe_a")
        _need(lwe_b, I64, (B,), "lwe_b")
        self._check_lut(lut, B)
        out_a = out_a if out_a is not None else torch.empty((B, n_lut, p.N), dtype=I64, device=lwe_a.device)
        out_b = out_b if out_b is not None else torch.empty((B, n_lut), dtype=I64, device=lwe_a.device)
        _need(out_a, I64, (B, n_lut, p.N), "out_a")
        _need(out_b, I64, (B, n_lut), "out_b")
        _lib.check(_lib.load().tfhe64_cuboot_merge(self.handle, _ptr(lwe_a), _ptr(lwe_b), _ptr(lut), lut.shape[0],
                                                   int(n_lut), _ptr(out_a), _ptr(out_b), B, _stream(stream)))
        return out_a, out_b

    def blind_rotate_reflayout(self, lwe_a, lut, n_lut, stream=None):
        """The chain through tfhe_mul_bootstrap on the reference's key layout
        (keys made with reflayout=True): ACC (B, 2, N) int64, not rotated."""
        if self.bsk is None:
            raise ValueError("these keys hold no reference-layout key (Keys64(..., reflayout=True))")
        p = self.params
        B = lwe_a.shape[0]
        _need(lwe_a, I64, (B, p.n), "lwe_a")
        self._check_lut(lut, B)
        idx = torch.empty((B, p.G, p.M), dtype=torch.int32, device=lwe_a.device)
        st = _stream(stream)
        lib = _lib.load()
        _lib.check(lib.tfhe64_rotation_indices(_ptr(lwe_a), p.n, p.collapse, p.N, int(n_lut), _ptr(idx), B, st))
        acc = torch.empty((B, 2, p.N), dtype=I64, device=lwe_a.device)
        _lib.check(lib.tfhe_mul_bootstrap(st, _ptr(lut), lut.numel(), _ptr(self.bsk), self.bsk_dims, _ptr(self.rot),
                                          self.rot.shape[0], _ptr(idx), p.log2_beta_bs, 64, p.l_bs, p.N, _ptr(acc), B))
        return acc

    def pbs(self, a, b, lut, n_lut=1, out_a=None, out_b=None, reflayout=False, stream=None):
        """Key switch, blind rotation, rotation by -b~ and many-LUT
        extraction: a (B, N), b (B), lut (1|B, 2, N) -> (B, n_lut, N), (B, n_lut).
        reflayout: the chain through tfhe_mul_bootstrap (rotation indices,
        chain, then rotation + extraction as separate kernels)."""
        ka, kb = self.keyswitch(a, b, stream=stream)
        if not reflayout:
            return self.cuboot_merge(ka, kb, lut, n_lut, out_a, out_b, stream)
        p = self.params
        B = a.shape[0]
        acc = self.blind_rotate_reflayout(ka, lut, n_lut, stream)
        out_a = out_a if out_a is not None else torch.empty((B, n_lut, p.N), dtype=I64, device=a.device)
        out_b = out_b if out_b is not None else torch.empty((B, n_lut), dtype=I64, device=a.device)
        _need(out_a, I64, (B, n_lut, p.N), "out_a")
        _need(out_b, I64, (B, n_lut), "out_b")
        _lib.check(_lib.load().tfhe64_rotate_extract(_ptr(acc), _ptr(kb), p.N, int(n_lut), _ptr(out_a), _ptr(out_b),
                                                     B, _stream(stream)))
        return out_a, out_b


class GaloisKeys64:
    """Device Galois keys of pack_lwe_to_rlwe on Z/2^64: the Fourier
    transforms of the four 16-bit limbs of every key polynomial."""

    def __init__(self, keys_u64: np.ndarray, log2_beta: int, l: int, device=None, stream=None):
        steps, l2, two, N = keys_u64.shape
        if l2 != l or two != 2 or (1 << steps) != N:
            raise ValueError("galois keys must be (log2 N, l, 2, N)")
        dev = device or torch.device("cuda", torch.cuda.current_device())
        src = device_u64(keys_u64, dev)
        h = ctypes.c_void_p()
        _lib.check(_lib.load().tfhe64_galois_keys_create(N, log2_beta, l, _ptr(src), _stream(stream), ctypes.byref(h)))
        self._h, self.N, self.log2_beta, self.l = h, N, log2_beta, l

    def close(self):
        if self._h:
            _lib.load().tfhe64_galois_keys_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def pack_lwe_to_rlwe(self, lwe_a, lwe_b, out=None, stream=None):
        """lwe_a (R, N), lwe_b (R) -> (R, 2, N)."""
        R = lwe_a.shape[0]
        _need(lwe_a, I64, (R, self.N), "lwe_a")
        _need(lwe_b, I64, (R,), "lwe_b")
        out = out if out is not None else torch.empty((R, 2, self.N), dtype=I64, device=lwe_a.device)
        _need(out, I64, (R, 2, self.N), "out")
        _lib.check(_lib.load().tfhe64_pack_lwe_to_rlwe(self._h, _ptr(lwe_a), _ptr(lwe_b), R, _ptr(out),
                                                       _stream(stream)))
        return out


class PackingKey64:
    """Device packing key (n_dim, l, 2, N) on Z/2^64; packs on the tcgen05
    tensor cores (8-bit limbs of the key) where the digits fit 8 bits."""

    def __init__(self, ksp_u64: np.ndarray, log2_beta: int, l: int, device=None):
        n_dim, l2, two, N = ksp_u64.shape
        if l2 != l or two != 2:
            raise ValueError("packing key must be (n_dim, l, 2, N)")
        dev = device or torch.device("cuda", torch.cuda.current_device())
        self.ksp = device_u64(ksp_u64, dev)
        self.n_dim, self.N, self.log2_beta, self.l = n_dim, N, log2_beta, l
        self.limbs = _limbs(self.ksp, n_dim * l, 2 * N) if _tc_ok(n_dim, l, log2_beta) else None
        self.tensor_cores = self.limbs is not None

    def pack(self, lwe_a, lwe_b, out=None, tensor_cores=-1, stream=None):
        """lwe_a (S, T, n_dim), lwe_b (S, T) -> (S, 2, N); tensor_cores -1 / 1
        use the limbs when the key has them and lwe_a is 16-byte aligned."""
        S, T, nd = lwe_a.shape
        _need(lwe_a, I64, (S, T, self.n_dim), "lwe_a")
        _need(lwe_b, I64, (S, T), "lwe_b")
        out = out if out is not None else torch.empty((S, 2, self.N), dtype=I64, device=lwe_a.device)
        _need(out, I64, (S, 2, self.N), "out")
        lib = _lib.load()
        if self.limbs is not None and tensor_cores != 0 and lwe_a.data_ptr() % 16 == 0:
            _lib.check(lib.tfhe64_pack_lwes_tc(_ptr(self.limbs), self.n_dim, self.N, self.log2_beta, self.l,
                                               _ptr(lwe_a), _ptr(lwe_b), T, S, _ptr(out), _stream(stream)))
        else:
            _lib.check(lib.tfhe64_pack_lwes(_ptr(self.ksp), self.n_dim, self.N, self.log2_beta, self.l,
                                            _ptr(lwe_a), _ptr(lwe_b), T, S, _ptr(out), _stream(stream)))
        return out

    def close(self):
        self.ksp = None


def _tc_ok(K_rows: int, l: int, log2_beta: int) -> bool:
    """The tensor-core contraction takes the digits as int8 and sums K
    products in int32: log2_beta <= 7, K multiple of 32, no overflow."""
    K = K_rows * l
    return 1 <= log2_beta <= 7 and K_rows % 32 == 0 and K * (1 << (log2_beta - 1)) * 128 < (1 << 31)


def _limbs(key_dev, K: int, cols: int):
    """int8 limb matrix (rows, K) of a (K, cols) 64-bit key on the device."""
    rows = int(_lib.load().tfhe64_tc_limb_rows(cols))
    limbs = torch.empty((rows, K), dtype=torch.int8, device=key_dev.device)
    _lib.check(_lib.load().tfhe64_tc_limbs(_ptr(key_dev), K, cols, _ptr(limbs), _stream()))
    return limbs


def linear_extract(weights, bias, rlwe, out_a=None, out_b=None, stream=None):
    """Linear.__call__ on Z/2^64: weights (J, N) int32, bias (J) int64,
    rlwe (S, 2, N) -> (S, J, N), (S, J)."""
    J, N = weights.shape
    S = rlwe.shape[0]
    _need(weights, torch.int32, (J, N), "weights")
    _need(bias, I64, (J,), "bias")
    _need(rlwe, I64, (S, 2, N), "rlwe")
    out_a = out_a if out_a is not None else torch.empty((S, J, N), dtype=I64, device=rlwe.device)
    out_b = out_b if out_b is not None else torch.empty((S, J), dtype=I64, device=rlwe.device)
    _lib.check(_lib.load().tfhe64_linear_extract(_ptr(weights), _ptr(bias), J, _ptr(rlwe), S, N, _ptr(out_a),
                                                 _ptr(out_b), _stream(stream)))
    return out_a, out_b


def lut_mul_sum(luts, rlwe, out=None, stream=None):
    """sum over g of luts[g][k] * rlwe[s][g][k]: luts (G, K, N) int64,
    rlwe (S, G, K, 2, N) -> (S, K, 2, N)."""
    G, K, N = luts.shape
    S = rlwe.shape[0]
    _need(luts, I64, (G, K, N), "luts")
    _need(rlwe, I64, (S, G, K, 2, N), "rlwe")
    out = out if out is not None else torch.empty((S, K, 2, N), dtype=I64, device=rlwe.device)
    _lib.check(_lib.load().tfhe64_lut_mul_sum(_ptr(luts), G, K, _ptr(rlwe), S, N, _ptr(out), _stream(stream)))
    return out


def rlwe_rotate_add(x, rot, y=None, out=None, stream=None):
    """X^rot * x + y for RLWEs (S, 2, N) on Z/2^64."""
    S, two, N = x.shape
    _need(x, I64, (S, 2, N), "x")
    if y is not None:
        _need(y, I64, (S, 2, N), "y")
    out = out if out is not None else torch.empty_like(x)
    _lib.check(_lib.load().tfhe64_rlwe_rotate_add(_ptr(x), int(rot), _ptr(y) if y is not None else None, S, N,
                                                  _ptr(out), _stream(stream)))
    return out


def add(x, y, out=None, stream=None):
    if x.shape != y.shape:
        raise ValueError("add: shapes differ")
    _need(x, I64, tuple(x.shape), "x")
    _need(y, I64, tuple(y.shape), "y")
    out = out if out is not None else torch.empty_like(x)
    _lib.check(_lib.load().tfhe64_add(_ptr(x), _ptr(y), x.numel(), _ptr(out), _stream(stream)))
    return out


def sample_extract(rlwe, count, stream=None):
    """LWEs of coefficients 0 .. count-1 of RLWEs (S, 2, N) -> (S, count, N), (S, count)."""
    S, two, N = rlwe.shape
    _need(rlwe, I64, (S, 2, N), "rlwe")
    out_a = torch.empty((S, count, N), dtype=I64, device=rlwe.device)
    out_b = torch.empty((S, count), dtype=I64, device=rlwe.device)
    _lib.check(_lib.load().tfhe64_sample_extract(_ptr(rlwe), N, count, _ptr(out_a), _ptr(out_b), S,
                                                 _stream(stream)))
    return out_a, out_b
