"""The reference's PBS-path operator surface on the B200 engine.

Same names, argument order and meaning as the reference's operators, taking
torch CUDA tensors in the reference's layouts (float64 centred integers,
complex128 Fourier keys) and returning the same shapes:

  multiply_seq_monomial  cuTFHE/multiply.py:54-92 (batched as
                         cutfhe_multiply_merge, schemas/RLWE_jax.py:269-274)
  cuboot_merge, BR       schemas/RLWE_jax.py:288-315
  key_switch_LWE         schemas/LWE_jax.py:97-117 (batched as
                         nn_tfhe/activation.py:150)
  sample_extract         schemas/text_jax.py:191-208
  rotate_ciphertext      schemas/text_jax.py:348-362
  HeavysideBoostrapper   nn_tfhe/activation.py:70-162 (cuboot)

Every value is computed by libtfhe_b200.so: the blind rotation by
tfhe_mul_bootstrap (the drop-in of the reference's "mul_bootstrap" FFI
target), rotation/extraction by tfhe_rotate_extract_i64, key switching by
tfhe_keyswitch_ref.  torch only holds the buffers and evaluates the
reference's host-side index arithmetic (multiply.py:70-86) on the device.
Unsupported parameters raise (the reference's handler returns
InvalidArgument for unsupported degree / l).
"""
from __future__ import annotations

import ctypes
import math

import torch

from . import _lib
from .engine import _ptr, _stream


def _as_cuda(x, dtype):
    t = x if isinstance(x, torch.Tensor) else torch.as_tensor(x)
    if not t.is_cuda:
        t = t.to("cuda")
    return t.to(dtype).contiguous()


def _u32_bits(x: torch.Tensor) -> torch.Tensor:
    """centred float64 / int64 torus values -> int32 tensor of uint32 bits"""
    if x.dtype.is_floating_point:
        x = torch.round(x)
    return (x.to(torch.int64) & 0xFFFFFFFF).to(torch.int32).contiguous()


def all_binary_vectors(m: int, device=None) -> torch.Tensor:
    """cuTFHE/utils.py:5-8: {0,1}^m in meshgrid 'ij' order, (2^m, m) int32."""
    values = torch.tensor([0, 1], dtype=torch.int32, device=device)
    grids = torch.meshgrid(*([values] * m), indexing="ij")
    return torch.stack(grids, dim=-1).reshape(-1, m)


def rotation_indices(public_key: torch.Tensor, collapse: int, degree: int, q: float, n_lut: int) -> torch.Tensor:
    """cuTFHE/multiply.py:67-79 on the device (float64, exact for q <= 2^53)."""
    n = public_key.shape[-1]
    n_iter = n // collapse
    kron = all_binary_vectors(collapse, device=public_key.device).to(torch.float64)
    pk = public_key.reshape(*public_key.shape[:-1], n_iter, collapse)
    vals = pk @ kron.T
    idx = (torch.round(2 * degree * vals / (q * n_lut)) * n_lut).to(torch.int32)
    return torch.remainder(idx, 2 * degree).to(torch.int32)


def _mul_bootstrap_i64(ct_init, public_key, BSK, log_q, log_beta, l, degree, collapse, all_rot_fft, n_lut):
    pk = _as_cuda(public_key, torch.float64)
    if pk.dim() == 1:
        pk = pk.unsqueeze(0)
    B, n = pk.shape
    if n % collapse:
        raise ValueError(f"public key length {n} is not a multiple of collapse {collapse}")
    n_iter = n // collapse
    if isinstance(ct_init, (tuple, list)):
        ct_init = torch.stack([_as_cuda(c, torch.float64) for c in ct_init])
    ct = _as_cuda(ct_init, torch.float64)
    if torch.is_floating_point(ct):
        ct = torch.round(ct)
    ct = ct.to(torch.int64).contiguous()
    if ct.numel() not in (2 * degree, 2 * degree * B):
        raise ValueError(f"ciphertext must hold 2*degree or batch*2*degree values, got {tuple(ct.shape)}")
    q = 2.0 ** log_q
    idx = rotation_indices(pk, collapse, degree, q, n_lut).contiguous()
    bsk = _as_cuda(BSK, torch.complex128)
    shape = list(bsk.shape)
    if len(shape) != 5 or shape[3] != n_iter * 2 ** collapse:
        raise ValueError(f"BSK must be bsk_ordered (2, 2, l, n/collapse * 2^collapse, degree/2), got {shape}")
    shape[3] = n_iter
    shape.insert(4, 2 ** collapse)
    bsk_r = bsk.reshape(shape).permute(3, 0, 2, 1, 4, 5).contiguous()        # multiply.py:81-86
    rot = _as_cuda(all_rot_fft, torch.complex128)
    out = torch.empty((B, 2, degree), dtype=torch.int64, device=pk.device)
    dims = (ctypes.c_int64 * 6)(*bsk_r.shape)
    _lib.check(_lib.load().tfhe_mul_bootstrap(_stream(), _ptr(ct), ct.numel(), _ptr(bsk_r), dims, _ptr(rot),
                                              rot.shape[0], _ptr(idx), int(log_beta), int(log_q), int(l),
                                              int(degree), _ptr(out), B))
    return out


def multiply_seq_monomial(ciphertext, public_key, BSK, log_q: int, log_beta: int, l: int, degree: int,
                          collapse: int, all_rot_fft, n_lut: int):
    """cuTFHE/multiply.py:54-92: ACC <- X^{sum a_i s_i} ACC through the
    collapsed CMux chain.  ciphertext (2, N) / (B|1, 2, N) / (mask, body);
    public_key (n,) or (B, n).  Returns float64 (2, N) or (B, 2, N)."""
    single = torch.as_tensor(public_key).dim() == 1 if not isinstance(public_key, torch.Tensor) \
        else public_key.dim() == 1
    out = _mul_bootstrap_i64(ciphertext, public_key, BSK, log_q, log_beta, l, degree, collapse,
                             all_rot_fft, n_lut).to(torch.float64)
    return out[0] if single else out


def _rotate_extract(acc_i64, b, degree, n_lut, log_q, want_acc, want_lwe):
    B = acc_i64.shape[0]
    bb = _as_cuda(b, torch.float64).reshape(B).contiguous()
    out_acc = torch.empty((B, 2, degree), dtype=torch.int64, device=acc_i64.device) if want_acc else None
    out_a = torch.empty((B, n_lut, degree), dtype=torch.int64, device=acc_i64.device) if want_lwe else None
    out_b = torch.empty((B, n_lut), dtype=torch.int64, device=acc_i64.device) if want_lwe else None
    _lib.check(_lib.load().tfhe_rotate_extract_i64(_ptr(acc_i64), _ptr(bb), degree, n_lut, int(log_q),
                                                   _ptr(out_acc), _ptr(out_a), _ptr(out_b), B, _stream()))
    return out_acc, out_a, out_b


def _log2_exact(v, what):
    lg = int(math.log2(v) + 1e-6)
    if 2 ** lg != v:
        raise ValueError(f"{what} must be a power of two, got {v}")
    return lg


def cuboot_merge(c_lwe_ks, encrypted_LUT, bsk, q, beta, l, degree, collapse, all_rot_possible_fourier, n_lut):
    """schemas/RLWE_jax.py:288-303: blind rotation from the LUT, rotation by
    -b~ after it, many-LUT extraction.  Returns (a (B, n_lut, N),
    b (B, n_lut, 1)) float64."""
    pk, b = c_lwe_ks
    ct = torch.stack([_as_cuda(encrypted_LUT[0], torch.float64), _as_cuda(encrypted_LUT[1], torch.float64)], dim=1)
    log_q = int(math.log2(q))
    acc = _mul_bootstrap_i64(ct, pk, bsk, log_q, int(math.log2(beta) + 1e-6), l, degree, collapse,
                             all_rot_possible_fourier, n_lut)
    _, out_a, out_b = _rotate_extract(acc, b, degree, n_lut, log_q, False, True)
    return out_a.to(torch.float64), out_b.to(torch.float64).unsqueeze(-1)


def BR(c_lwe_ks, encrypted_LUT, bsk, q, beta, l, degree, collapse, all_rot_possible_fourier, n_lut):
    """schemas/RLWE_jax.py:305-315: the rotated accumulator (mask (B, N),
    body (B, N)) float64."""
    pk, b = c_lwe_ks
    ct = torch.stack([_as_cuda(encrypted_LUT[0], torch.float64), _as_cuda(encrypted_LUT[1], torch.float64)], dim=1)
    log_q = int(math.log2(q))
    acc = _mul_bootstrap_i64(ct, pk, bsk, log_q, int(math.log2(beta) + 1e-6), l, degree, collapse,
                             all_rot_possible_fourier, n_lut)
    out_acc, _, _ = _rotate_extract(acc, b, degree, n_lut, log_q, True, False)
    out = out_acc.to(torch.float64)
    return out[:, 0], out[:, 1]


def key_switch_LWE(key_switching_key, ciphertext, dict_params):
    """schemas/LWE_jax.py:97-117 over a batch (nn_tfhe/activation.py:150):
    key (pk (l_ks, n_big, n), b (l_ks, n_big, 1)), ciphertext (a (B, n_big),
    b (B, 1)) -> (a (B, n), b (B, 1)) float64 centred in [-q/2, q/2)."""
    q = float(dict_params["q"])
    if q != 2.0 ** 32:
        raise ValueError("tfhe_b200 key switching runs on the 2^32 torus (dict_params['q'] == 2**32)")
    log2_beta = _log2_exact(dict_params["beta_ks"], "beta_ks")
    l_ks = int(dict_params["l_ks"])
    kpk = _u32_bits(_as_cuda(key_switching_key[0], torch.float64))
    kb = _u32_bits(_as_cuda(key_switching_key[1], torch.float64))
    if kpk.dim() != 3 or kpk.shape[0] != l_ks:
        raise ValueError(f"key switching key mask must be (l_ks, n_big, n), got {tuple(kpk.shape)}")
    _, n_big, n = kpk.shape
    a = _as_cuda(ciphertext[0], torch.float64)
    single = a.dim() == 1
    a = a.reshape(-1, n_big)
    B = a.shape[0]
    b = _as_cuda(ciphertext[1], torch.float64).reshape(B)
    a32, b32 = _u32_bits(a), _u32_bits(b)
    a_out = torch.empty((B, n), dtype=torch.int32, device=a.device)
    b_out = torch.empty((B,), dtype=torch.int32, device=a.device)
    _lib.check(_lib.load().tfhe_keyswitch_ref(_ptr(a32), _ptr(b32), _ptr(kpk), _ptr(kb.reshape(l_ks, n_big)),
                                              n_big, n, l_ks, log2_beta, _ptr(a_out), _ptr(b_out), B, _stream()))
    ra, rb = a_out.to(torch.float64), b_out.to(torch.float64).unsqueeze(-1)
    return (ra[0], rb[0]) if single else (ra, rb)


def sample_extract(ciphertext, alpha: int):
    """schemas/text_jax.py:191-208: LWE of coefficient alpha.  ciphertext
    (a, b) with a, b of shape (N,) or (B, N)."""
    a = _as_cuda(ciphertext[0], torch.float64)
    single = a.dim() == 1
    a = a.reshape(-1, a.shape[-1])
    N = a.shape[-1]
    body = _as_cuda(ciphertext[1], torch.float64).reshape(-1, N)
    acc = torch.round(torch.stack([a, body], dim=1)).to(torch.int64).contiguous()
    zero = torch.zeros(acc.shape[0], dtype=torch.float64, device=acc.device)
    _, out_a, out_b = _rotate_extract(acc, zero, N, int(alpha) + 1, 64, False, True)
    ra, rb = out_a[:, alpha].to(torch.float64), out_b[:, alpha:alpha + 1].to(torch.float64)
    return (ra[0], rb[0]) if single else (ra, rb)


def rotate_ciphertext(ciphertext, exponent):
    """schemas/text_jax.py:348-362: (a, b) -> (X^e a, X^e b); e scalar or
    one per row."""
    a = _as_cuda(ciphertext[0], torch.float64)
    single = a.dim() == 1
    a = a.reshape(-1, a.shape[-1])
    N = a.shape[-1]
    body = _as_cuda(ciphertext[1], torch.float64).reshape(-1, N)
    B = a.shape[0]
    acc = torch.round(torch.stack([a, body], dim=1)).to(torch.int64).contiguous()
    e = _as_cuda(exponent, torch.float64).reshape(-1).expand(B).contiguous()
    # rotate_extract applies X^(-b~) with b~ = round(2N b / q): b = -e q / 2N
    q = 2.0 ** 32
    b = -e * (q / (2 * N))
    out_acc, _, _ = _rotate_extract(acc, b, N, 1, 32, True, False)
    out = out_acc.to(torch.float64)
    return (out[0, 0], out[0, 1]) if single else (out[:, 0], out[:, 1])


class HeavysideBoostrapper:
    """nn_tfhe/activation.py:70-162 (the GPU path, ``cuboot``)."""

    def __init__(self, bootstrapping_key, key_switching_key_bs, ksk_packing, galois_key, dict_params,
                 dict_params_lut, dict_params_ks_LWE, dict_params_packing, collapse, all_rot_possible_fourier,
                 n_lut):
        self.bootstrapping_key = bootstrapping_key
        self.key_switching_key_bs = key_switching_key_bs
        self.ksk_packing = ksk_packing
        self.galois_key = galois_key
        self.dict_params = dict_params
        self.dict_params_lut = dict_params_lut
        self.dict_params_ks_LWE = dict_params_ks_LWE
        self.dict_params_packing = dict_params_packing
        self.collapse = collapse
        self.all_rot_possible_fourier = all_rot_possible_fourier
        self.log2q = int(math.log2(self.dict_params_lut["q"]))
        self.log2beta = int(math.log2(self.dict_params_lut["beta_bs"]) + 1e-6)
        self.n_lut = n_lut

    def cuboot(self, h, encrypted_LUT):
        c_lwe_ks = key_switch_LWE(self.key_switching_key_bs, h, self.dict_params_ks_LWE)
        return cuboot_merge(c_lwe_ks, encrypted_LUT, self.bootstrapping_key, self.dict_params_lut["q"],
                            self.dict_params_lut["beta_bs"], self.dict_params_lut["l_bs"],
                            self.dict_params_lut["degree"], self.collapse, self.all_rot_possible_fourier,
                            self.n_lut)
