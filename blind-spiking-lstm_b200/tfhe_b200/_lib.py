"""ctypes binding of libtfhe_b200.so (the C ABI declared in
include/tfhe_b200.h).  The library is built in-tree by
``blind-spiking-lstm_b200/build.py``; there is no fallback when it is
missing: every entry point raises."""
from __future__ import annotations

import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libtfhe_b200.so")

STATUS = {0: "OK", 1: "INVALID_ARGUMENT", 2: "INTERNAL", 3: "OUT_OF_MEMORY", 4: "NO_DEVICE"}


class TFHEError(RuntimeError):
    """A non-zero status from the C ABI, with tfhe_last_error()'s message."""

    def __init__(self, status: int, message: str):
        self.status = status
        self.status_name = STATUS.get(status, str(status))
        super().__init__(f"{self.status_name}: {message}")


class TfheTuning(ctypes.Structure):
    _fields_ = [("ciphertexts_per_cta", ctypes.c_int32), ("prefetch", ctypes.c_int32),
                ("persistent", ctypes.c_int32), ("ks_tensor_cores", ctypes.c_int32),
                ("l2_prefetch", ctypes.c_int32)]


class TfheParams(ctypes.Structure):
    _fields_ = [(name, ctypes.c_int32) for name in
                ("N", "n", "n_big", "log2_beta_bs", "l_bs", "collapse", "log2_beta_ks", "l_ks", "log2_q")]


_P = ctypes.c_void_p
_I32 = ctypes.c_int32
_I64 = ctypes.c_int64

# name -> (restype, argtypes); every function declared in include/tfhe_b200.h
SIGNATURES = {
    "tfhe_version": (ctypes.c_char_p, []),
    "tfhe_last_error": (ctypes.c_char_p, []),
    "tfhe_mul_bootstrap": (ctypes.c_int, [_P, _P, _I64, _P, _P, _P, _I64, _P, _I64, _I64, _I64, _I64, _P, _I64]),
    "tfhe_keys_create": (ctypes.c_int, [ctypes.POINTER(TfheParams), _P, _P, _P, _P, ctypes.POINTER(_P)]),
    "tfhe_keys_create_fourier": (ctypes.c_int, [ctypes.POINTER(TfheParams), _P, _P, _P, _P, ctypes.POINTER(_P)]),
    "tfhe_keys_destroy": (None, [_P]),
    "tfhe_keys_set_tuning": (ctypes.c_int, [_P, ctypes.POINTER(TfheTuning)]),
    "tfhe_keys_cluster_size": (ctypes.c_int32, [_P, _I64]),
    "tfhe_keys_launch_shape": (ctypes.c_int, [_P, _I64, ctypes.POINTER(_I32), ctypes.POINTER(_I32),
                                              ctypes.POINTER(_I64)]),
    "tfhe_keys_device_bytes": (_I64, [_P]),
    "tfhe_keyswitch": (ctypes.c_int, [_P, _P, _P, _P, _P, _I64, _P]),
    "tfhe_blind_rotate": (ctypes.c_int, [_P, _P, _P, _P, _I64, _I32, _P, _I64, _P]),
    "tfhe_sample_extract": (ctypes.c_int, [_P, _I32, _I32, _P, _P, _I64, _P]),
    "tfhe_pbs": (ctypes.c_int, [_P, _P, _P, _P, _I64, _I32, _P, _P, _I64, _P]),
    "tfhe_pbs_noalloc": (ctypes.c_int, [_P, _P, _P, _P, _I64, _I32, _P, _P, _I64, _P]),
    "tfhe_cuboot_merge": (ctypes.c_int, [_P, _P, _P, _P, _I64, _I32, _P, _P, _I64, _P]),
    "tfhe_probe_fp64_fma": (ctypes.c_int, [_I32, _I32, _I32, _P, ctypes.POINTER(ctypes.c_double), _P]),
    "tfhe_device_status": (ctypes.c_int, [ctypes.POINTER(_I32), _I32]),
    "tfhe_launch_count": (ctypes.c_int64, []),
    "tfhe_probe_wait_timeout": (ctypes.c_int, [_I64, ctypes.POINTER(_I32)]),
    "tfhe_keyswitch_ref": (ctypes.c_int, [_P, _P, _P, _P, _I32, _I32, _I32, _I32, _P, _P, _I64, _P]),
    "tfhe_pbs_host": (ctypes.c_int, [_P, _P, _P, _P, _I64, _I32, _P, _P, _I64, _I64, _P]),
    "tfhe_linear_extract": (ctypes.c_int, [_P, _P, _I32, _P, _I64, _I32, _P, _P, _P]),
    "tfhe_lut_mul_sum": (ctypes.c_int, [_P, _I32, _I32, _P, _I64, _I32, _P, _P]),
    "tfhe_galois_keys_create": (ctypes.c_int, [_I32, _I32, _I32, _P, _P, ctypes.POINTER(_P)]),
    "tfhe_galois_keys_destroy": (ctypes.c_int, [_P]),
    "tfhe_pack_lwe_to_rlwe": (ctypes.c_int, [_P, _P, _P, _I64, _P, _P]),
    "tfhe_pack_lwes": (ctypes.c_int, [_P, _I32, _I32, _I32, _I32, _P, _P, _I32, _I64, _P, _P]),
    "tfhe_packing_key_create": (ctypes.c_int, [_P, _I32, _I32, _I32, _I32, _P, ctypes.POINTER(_P)]),
    "tfhe_packing_key_destroy": (ctypes.c_int, [_P]),
    "tfhe_packing_key_uses_tensor_cores": (ctypes.c_int, [_P]),
    "tfhe_pack_lwes_with_key": (ctypes.c_int, [_P, _P, _P, _I32, _I64, _P, _I32, _P]),
    "tfhe_rlwe_rotate_add": (ctypes.c_int, [_P, _I32, _P, _I64, _I32, _P, _P]),
    "tfhe_u32_add": (ctypes.c_int, [_P, _P, _I64, _P, _P]),
    "tfhe_rotate_extract_i64": (ctypes.c_int, [_P, _P, _I32, _I32, _I64, _P, _P, _P, _I64, _P]),
    # the FP32 split-limb blind rotation (br_fp32.cu)
    "tfhe_fp32_keys_create": (ctypes.c_int, [_P, _P, _I32, _P, ctypes.POINTER(_P)]),
    "tfhe_fp32_keys_destroy": (None, [_P]),
    "tfhe_fp32_cuboot_merge": (ctypes.c_int, [_P, _P, _P, _P, _I64, _I32, _P, _P, _P, _I64, _I32, _P]),
    # the 64-bit torus (torus64.cu)
    "tfhe64_keys_create": (ctypes.c_int, [ctypes.POINTER(TfheParams), _P, _P, ctypes.POINTER(_P)]),
    "tfhe64_cuboot_merge": (ctypes.c_int, [_P, _P, _P, _P, _I64, _I32, _P, _P, _I64, _P]),
    "tfhe64_blind_rotate": (ctypes.c_int, [_P, _P, _P, _P, _I64, _I32, _P, _I64, _P]),
    "tfhe64_keyswitch": (ctypes.c_int, [_P, _I32, _I32, _I32, _I32, _P, _P, _P, _P, _I64, _P]),
    "tfhe64_rotation_indices": (ctypes.c_int, [_P, _I32, _I32, _I32, _I32, _P, _I64, _P]),
    "tfhe64_rotate_extract": (ctypes.c_int, [_P, _P, _I32, _I32, _P, _P, _I64, _P]),
    "tfhe64_linear_extract": (ctypes.c_int, [_P, _P, _I32, _P, _I64, _I32, _P, _P, _P]),
    "tfhe64_lut_mul_sum": (ctypes.c_int, [_P, _I32, _I32, _P, _I64, _I32, _P, _P]),
    "tfhe64_galois_keys_create": (ctypes.c_int, [_I32, _I32, _I32, _P, _P, ctypes.POINTER(_P)]),
    "tfhe64_galois_keys_destroy": (ctypes.c_int, [_P]),
    "tfhe64_pack_lwe_to_rlwe": (ctypes.c_int, [_P, _P, _P, _I64, _P, _P]),
    "tfhe64_pack_lwes": (ctypes.c_int, [_P, _I32, _I32, _I32, _I32, _P, _P, _I32, _I64, _P, _P]),
    "tfhe64_tc_limb_rows": (ctypes.c_int64, [_I32]),
    "tfhe64_tc_limbs": (ctypes.c_int, [_P, _I64, _I32, _P, _P]),
    "tfhe64_keyswitch_tc": (ctypes.c_int, [_P, _I32, _I32, _I32, _I32, _P, _P, _P, _P, _I64, _P]),
    "tfhe64_pack_lwes_tc": (ctypes.c_int, [_P, _I32, _I32, _I32, _I32, _P, _P, _I32, _I64, _P, _P]),
    "tfhe64_rlwe_rotate_add": (ctypes.c_int, [_P, _I32, _P, _I64, _I32, _P, _P]),
    "tfhe64_add": (ctypes.c_int, [_P, _P, _I64, _P, _P]),
    "tfhe64_sample_extract": (ctypes.c_int, [_P, _I32, _I32, _P, _P, _I64, _P]),
}

_lock = threading.Lock()
_lib = None


def load() -> ctypes.CDLL:
    """Load the library once; raise if it has not been built."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    f"{LIB_PATH} is missing: build it with `python blind-spiking-lstm_b200/build.py` "
                    "(the engine has no CPU fallback)")
            lib = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


def check(status: int) -> None:
    if status != 0:
        msg = load().tfhe_last_error()
        raise TFHEError(int(status), msg.decode() if msg else "")


def version() -> str:
    return load().tfhe_version().decode()
