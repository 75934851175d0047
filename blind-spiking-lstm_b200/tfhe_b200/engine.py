"""Native engine: device-resident keys and batched PBS stages on torch CUDA
tensors.  Torus values are uint32 bit patterns held in torch.int32 tensors
(the reference's centred float64 values reduced modulo 2^32).  torch is used
for device memory and streams only; all arithmetic runs in libtfhe_b200.so.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .params import ParamSet


def _ptr(t) -> int:
    return 0 if t is None else int(t.data_ptr())


def _stream(stream=None) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


def _need(t, dtype, shape, name):
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"{name} must be a torch tensor")
    if not t.is_cuda:
        raise ValueError(f"{name} must live on a CUDA device")
    if t.dtype != dtype:
        raise TypeError(f"{name} must be {dtype}, got {t.dtype}")
    if tuple(t.shape) != tuple(shape):
        raise ValueError(f"{name} must have shape {tuple(shape)}, got {tuple(t.shape)}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")


# ---------------------------------------------------------------- torus views
def to_u32(x) -> np.ndarray:
    """Centred integers (float64/int64, any range) -> uint32 modulo 2^32."""
    a = np.asarray(x)
    if a.dtype.kind == "f":
        a = np.rint(a)
    return (a.astype(np.int64) & 0xFFFFFFFF).astype(np.uint32)


def u32_as_i32(x: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(x, dtype=np.uint32)).view(np.int32)


def centred(x) -> np.ndarray:
    """uint32 / int32 bit patterns -> centred int64 in [-2^31, 2^31)."""
    a = np.asarray(x)
    return a.astype(np.uint32).view(np.int32).astype(np.int64)


def device_u32(x, device=None) -> torch.Tensor:
    """Host torus values -> int32 CUDA tensor of uint32 bit patterns."""
    return torch.from_numpy(u32_as_i32(to_u32(x))).to(device or "cuda")


# ---------------------------------------------------------------- keys
class Keys:
    """Device-resident bootstrapping and key-switching keys (tfhe_keys)."""

    def __init__(self, params: ParamSet, handle: int, device: int):
        self.params = params
        self._h = ctypes.c_void_p(handle)
        self.device = device

    @classmethod
    def create(cls, params: ParamSet, bsk_coeff, ksk_a, ksk_b, stream=None) -> "Keys":
        """From the coefficient-domain key (2, 2, G*M, l_bs, N) and the
        key-switching key (l_ks, n_big, n) / (l_ks, n_big), host arrays of
        torus values (centred floats or unsigned)."""
        lib = _lib.load()
        p = params
        bsk = np.ascontiguousarray(to_u32(bsk_coeff).reshape(2, 2, p.G * p.M, p.l_bs, p.N))
        ka = np.ascontiguousarray(to_u32(ksk_a).reshape(p.l_ks, p.big, p.n))
        kb = np.ascontiguousarray(to_u32(ksk_b).reshape(p.l_ks, p.big))
        cp = p.ctypes()
        out = ctypes.c_void_p()
        _lib.check(lib.tfhe_keys_create(ctypes.byref(cp), bsk.ctypes.data, ka.ctypes.data, kb.ctypes.data,
                                        _stream(stream), ctypes.byref(out)))
        return cls(params, out.value, torch.cuda.current_device())

    @classmethod
    def create_fourier(cls, params: ParamSet, bsk_ordered, ksk_a, ksk_b, stream=None) -> "Keys":
        """From the reference's Fourier key ``bsk_ordered`` (complex128
        (2, 2, l_bs, G*M, N/2), nn_tfhe/activation.py:49-53)."""
        lib = _lib.load()
        p = params
        bo = np.ascontiguousarray(np.asarray(bsk_ordered, dtype=np.complex128)
                                  .reshape(2, 2, p.l_bs, p.G * p.M, p.N // 2))
        ka = np.ascontiguousarray(to_u32(ksk_a).reshape(p.l_ks, p.big, p.n))
        kb = np.ascontiguousarray(to_u32(ksk_b).reshape(p.l_ks, p.big))
        cp = p.ctypes()
        out = ctypes.c_void_p()
        _lib.check(lib.tfhe_keys_create_fourier(ctypes.byref(cp), bo.ctypes.data, ka.ctypes.data,
                                                kb.ctypes.data, _stream(stream), ctypes.byref(out)))
        return cls(params, out.value, torch.cuda.current_device())

    @property
    def handle(self) -> ctypes.c_void_p:
        if not self._h or not self._h.value:
            raise RuntimeError("keys have been released")
        return self._h

    def pbs_host(self, a, b, lut, n_lut=1, out_a=None, out_b=None, chunk=0, stream=None):
        """pbs from host (CPU, ideally pinned) tensors with the copies
        overlapped chunk by chunk (tfhe_pbs_host); outputs are host tensors,
        valid once the stream has synchronised."""
        p = self.params
        B = a.shape[0]
        for t, name in ((a, "a"), (b, "b"), (lut, "lut")):
            if t.device.type != "cpu" or t.dtype != torch.int32 or not t.is_contiguous():
                raise ValueError(f"{name}: contiguous int32 host tensor required")
        if tuple(a.shape) != (B, p.big) or tuple(b.shape) != (B,) or tuple(lut.shape[1:]) != (2, p.N):
            raise ValueError("pbs_host: shapes (B, n_big), (B), (1|B, 2, N) required")
        out_a = out_a if out_a is not None else torch.empty((B, n_lut, p.N), dtype=torch.int32).pin_memory()
        out_b = out_b if out_b is not None else torch.empty((B, n_lut), dtype=torch.int32).pin_memory()
        for t, name in ((out_a, "out_a"), (out_b, "out_b")):
            if t.device.type != "cpu" or t.dtype != torch.int32 or not t.is_contiguous():
                raise ValueError(f"{name}: contiguous int32 host tensor required")
        if tuple(out_a.shape) != (B, n_lut, p.N) or tuple(out_b.shape) != (B, n_lut):
            raise ValueError("pbs_host: outputs (B, n_lut, N), (B, n_lut) required")
        _lib.check(_lib.load().tfhe_pbs_host(self.handle, a.data_ptr(), b.data_ptr(), lut.data_ptr(), lut.shape[0],
                                             n_lut, out_a.data_ptr(), out_b.data_ptr(), B, int(chunk),
                                             _stream(stream)))
        return out_a, out_b

    def set_tuning(self, ciphertexts_per_cta=0, prefetch=-1, persistent=-1, ks_tensor_cores=-1,
                   l2_prefetch=-1) -> None:
        """Launch shapes of this key set (speed only; 0 / -1 mean automatic):
        the blind rotation's ciphertexts per CTA, L1 prefetch, persistent
        CTAs and the L2 prefetch of the next group's key block, and whether
        the key switch runs on the tensor cores.  tfhe_keys_set_tuning."""
        t = _lib.TfheTuning(int(ciphertexts_per_cta), int(prefetch), int(persistent), int(ks_tensor_cores),
                            int(l2_prefetch))
        _lib.check(_lib.load().tfhe_keys_set_tuning(self.handle, ctypes.byref(t)))
        self.tuning = (int(ciphertexts_per_cta), int(prefetch), int(persistent))

    def launch_shape(self, batch: int):
        """(ciphertexts per CTA, threads per CTA, shared bytes) a batch gets."""
        k, nt, sm = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int64()
        _lib.check(_lib.load().tfhe_keys_launch_shape(self.handle, int(batch), ctypes.byref(k), ctypes.byref(nt),
                                                      ctypes.byref(sm)))
        return k.value, nt.value, sm.value

    def cluster_size(self, batch: int) -> int:
        """CTAs per ciphertext of a batch's blind rotation: 8, 4 or 2 where
        one ciphertext runs on a cluster of that many CTAs (small batches),
        else 1."""
        return int(_lib.load().tfhe_keys_cluster_size(self.handle, int(batch)))

    def device_bytes(self) -> int:
        return int(_lib.load().tfhe_keys_device_bytes(self.handle))

    def close(self) -> None:
        if self._h and self._h.value:
            _lib.load().tfhe_keys_destroy(self._h)
            self._h = ctypes.c_void_p(0)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------ stages
    def keyswitch(self, a, b, a_out=None, b_out=None, stream=None):
        """key_switch_LWE over a batch: a (B, n_big), b (B) -> (B, n), (B)."""
        p = self.params
        B = a.shape[0]
        _need(a, torch.int32, (B, p.big), "a")
        _need(b, torch.int32, (B,), "b")
        a_out = a_out if a_out is not None else torch.empty((B, p.n), dtype=torch.int32, device=a.device)
        b_out = b_out if b_out is not None else torch.empty((B,), dtype=torch.int32, device=a.device)
        _need(a_out, torch.int32, (B, p.n), "a_out")
        _need(b_out, torch.int32, (B,), "b_out")
        _lib.check(_lib.load().tfhe_keyswitch(self.handle, _ptr(a), _ptr(b), _ptr(a_out), _ptr(b_out), B,
                                              _stream(stream)))
        return a_out, b_out

    def blind_rotate(self, lwe_a, lwe_b, lut, n_lut=1, acc_out=None, stream=None):
        """BR: lwe (B, n) / (B), lut (1|B, 2, N) -> ACC (B, 2, N)."""
        p = self.params
        B = lwe_a.shape[0]
        _need(lwe_a, torch.int32, (B, p.n), "lwe_a")
        _need(lwe_b, torch.int32, (B,), "lwe_b")
        _need(lut, torch.int32, (lut.shape[0], 2, p.N), "lut")
        acc_out = acc_out if acc_out is not None else torch.empty((B, 2, p.N), dtype=torch.int32,
                                                                  device=lwe_a.device)
        _need(acc_out, torch.int32, (B, 2, p.N), "acc_out")
        _lib.check(_lib.load().tfhe_blind_rotate(self.handle, _ptr(lwe_a), _ptr(lwe_b), _ptr(lut), lut.shape[0],
                                                 n_lut, _ptr(acc_out), B, _stream(stream)))
        return acc_out

    def cuboot_merge(self, lwe_a, lwe_b, lut, n_lut=1, out_a=None, out_b=None, stream=None):
        """cuboot_merge from key-switched LWEs: lwe (B, n) / (B), lut
        (1|B, 2, N) -> out_a (B, n_lut, N), out_b (B, n_lut)."""
        p = self.params
        B = lwe_a.shape[0]
        _need(lwe_a, torch.int32, (B, p.n), "lwe_a")
        _need(lwe_b, torch.int32, (B,), "lwe_b")
        _need(lut, torch.int32, (lut.shape[0], 2, p.N), "lut")
        out_a = out_a if out_a is not None else torch.empty((B, n_lut, p.N), dtype=torch.int32, device=lwe_a.device)
        out_b = out_b if out_b is not None else torch.empty((B, n_lut), dtype=torch.int32, device=lwe_a.device)
        _need(out_a, torch.int32, (B, n_lut, p.N), "out_a")
        _need(out_b, torch.int32, (B, n_lut), "out_b")
        _lib.check(_lib.load().tfhe_cuboot_merge(self.handle, _ptr(lwe_a), _ptr(lwe_b), _ptr(lut), lut.shape[0],
                                                 n_lut, _ptr(out_a), _ptr(out_b), B, _stream(stream)))
        return out_a, out_b

    def pbs(self, a, b, lut, n_lut=1, out_a=None, out_b=None, stream=None):
        """Key switch + blind rotation + many-LUT extraction
        (HeavysideBoostrapper.cuboot): a (B, n_big), b (B), lut (1|B, 2, N)
        -> out_a (B, n_lut, N), out_b (B, n_lut)."""
        p = self.params
        B = a.shape[0]
        _need(a, torch.int32, (B, p.big), "a")
        _need(b, torch.int32, (B,), "b")
        _need(lut, torch.int32, (lut.shape[0], 2, p.N), "lut")
        out_a = out_a if out_a is not None else torch.empty((B, n_lut, p.N), dtype=torch.int32, device=a.device)
        out_b = out_b if out_b is not None else torch.empty((B, n_lut), dtype=torch.int32, device=a.device)
        _need(out_a, torch.int32, (B, n_lut, p.N), "out_a")
        _need(out_b, torch.int32, (B, n_lut), "out_b")
        _lib.check(_lib.load().tfhe_pbs(self.handle, _ptr(a), _ptr(b), _ptr(lut), lut.shape[0], n_lut,
                                        _ptr(out_a), _ptr(out_b), B, _stream(stream)))
        return out_a, out_b


def sample_extract(acc, n_lut=1, out_a=None, out_b=None, stream=None):
    """Many-LUT sample extraction: acc (B, 2, N) -> (B, n_lut, N), (B, n_lut)."""
    B, two, N = acc.shape
    _need(acc, torch.int32, (B, 2, N), "acc")
    out_a = out_a if out_a is not None else torch.empty((B, n_lut, N), dtype=torch.int32, device=acc.device)
    out_b = out_b if out_b is not None else torch.empty((B, n_lut), dtype=torch.int32, device=acc.device)
    _lib.check(_lib.load().tfhe_sample_extract(_ptr(acc), N, n_lut, _ptr(out_a), _ptr(out_b), B,
                                               _stream(stream)))
    return out_a, out_b


def launch_count() -> int:
    """Kernels the library has launched in this process (tfhe_launch_count);
    the difference across a region of calls counts that region's launches."""
    return int(_lib.load().tfhe_launch_count())


def probe_fp64_peak(iters=4096, reps=5) -> float:
    """Measured FP64 FMA throughput of the current device in TFLOP/s (best
    of ``reps`` launches of 8 independent FMA chains per thread, 8 CTAs of
    512 threads per SM)."""
    dev = torch.cuda.current_device()
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    scratch = torch.zeros(1, dtype=torch.float64, device="cuda")
    flops = ctypes.c_double()
    lib = _lib.load()
    s = _stream()
    best = 0.0
    for i in range(reps + 1):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        _lib.check(lib.tfhe_probe_fp64_fma(sms * 8, 512, iters, _ptr(scratch), ctypes.byref(flops), s))
        e1.record()
        torch.cuda.synchronize()
        if i:
            best = max(best, flops.value / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    return best


class PBSGraph:
    """One programmable bootstrap of a fixed batch captured in a CUDA graph:
    the key switch and the blind rotation / extraction launches on fixed
    device buffers, replayed per call (inputs are copied into the captured
    buffers).  Removes the per-call host work of small batches."""

    def __init__(self, keys: Keys, batch: int, n_lut: int = 1, lut_count: int = 1):
        p = keys.params
        dev = torch.device("cuda", torch.cuda.current_device())
        self.keys, self.batch, self.n_lut = keys, batch, n_lut
        i32 = dict(dtype=torch.int32, device=dev)
        self.a = torch.zeros((batch, p.big), **i32)
        self.b = torch.zeros((batch,), **i32)
        self.lut = torch.zeros((lut_count, 2, p.N), **i32)
        self.ka = torch.empty((batch, p.n), **i32)
        self.kb = torch.empty((batch,), **i32)
        self.out_a = torch.empty((batch, n_lut, p.N), **i32)
        self.out_b = torch.empty((batch, n_lut), **i32)
        self._step()                      # uncaptured: sets kernel attributes
        torch.cuda.synchronize()
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self._step()

    def _step(self):
        self.keys.keyswitch(self.a, self.b, self.ka, self.kb)
        self.keys.cuboot_merge(self.ka, self.kb, self.lut, self.n_lut, self.out_a, self.out_b)

    def __call__(self, a, b, lut=None):
        self.a.copy_(a, non_blocking=True)
        self.b.copy_(b, non_blocking=True)
        if lut is not None:
            self.lut.copy_(lut, non_blocking=True)
        self.graph.replay()
        return self.out_a, self.out_b


class FP32Keys:
    """The FP32 split-limb blind rotation (tfhe_fp32_*): every FFT in FP32,
    the bootstrapping key split into `limbs` signed limbs whose FP32 products
    are rounded and recombined exactly modulo 2^32.  The precision ablation
    of the external product against the FP64 engine (Keys)."""

    def __init__(self, params: ParamSet, bsk_coeff, limbs: int, stream=None):
        p = params
        bsk = np.ascontiguousarray(to_u32(bsk_coeff).reshape(2, 2, p.G * p.M, p.l_bs, p.N))
        cp = p.ctypes()
        out = ctypes.c_void_p()
        _lib.check(_lib.load().tfhe_fp32_keys_create(ctypes.byref(cp), bsk.ctypes.data, int(limbs), _stream(stream),
                                                     ctypes.byref(out)))
        self.params, self.limbs, self._h = p, int(limbs), out

    def close(self) -> None:
        if self._h and self._h.value:
            _lib.load().tfhe_fp32_keys_destroy(self._h)
            self._h = ctypes.c_void_p(0)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def cuboot_merge(self, lwe_a, lwe_b, lut, n_lut=1, out_a=None, out_b=None, ciphertexts_per_cta=0, stream=None):
        """lwe (B, n) / (B), lut (1|B, 2, N) -> out_a (B, n_lut, N), out_b (B, n_lut)."""
        p = self.params
        B = lwe_a.shape[0]
        _need(lwe_a, torch.int32, (B, p.n), "lwe_a")
        _need(lwe_b, torch.int32, (B,), "lwe_b")
        _need(lut, torch.int32, (lut.shape[0], 2, p.N), "lut")
        out_a = out_a if out_a is not None else torch.empty((B, n_lut, p.N), dtype=torch.int32, device=lwe_a.device)
        out_b = out_b if out_b is not None else torch.empty((B, n_lut), dtype=torch.int32, device=lwe_a.device)
        _lib.check(_lib.load().tfhe_fp32_cuboot_merge(self._h, _ptr(lwe_a), _ptr(lwe_b), _ptr(lut), lut.shape[0],
                                                      n_lut, _ptr(out_a), _ptr(out_b), None, B,
                                                      int(ciphertexts_per_cta), _stream(stream)))
        return out_a, out_b

    def chain(self, lwe_a, lut, n_lut=1, stream=None):
        """The accumulator after the CMux chain (B, 2, N), not rotated."""
        p = self.params
        B = lwe_a.shape[0]
        _need(lwe_a, torch.int32, (B, p.n), "lwe_a")
        _need(lut, torch.int32, (lut.shape[0], 2, p.N), "lut")
        acc = torch.empty((B, 2, p.N), dtype=torch.int32, device=lwe_a.device)
        b = torch.zeros((B,), dtype=torch.int32, device=lwe_a.device)
        _lib.check(_lib.load().tfhe_fp32_cuboot_merge(self._h, _ptr(lwe_a), _ptr(b), _ptr(lut), lut.shape[0], n_lut,
                                                      None, None, _ptr(acc), B, 0, _stream(stream)))
        return acc
