"""The C-ABI library loads without a GPU, exports every symbol that
include/tfhe_b200.h declares, and rejects invalid arguments before touching
the device (the reference's handler returns InvalidArgument for an
unsupported degree or l, csrc/mul_bootstrap.cuh:211-223)."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "tfhe_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tfhe(?:64)?_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from tfhe_b200 import _lib
    return _lib.load()


def test_header_lists_the_abi():
    names = declared_functions()
    assert "tfhe_mul_bootstrap" in names and "tfhe_pbs" in names
    from tfhe_b200 import _lib
    assert set(names) == set(_lib.SIGNATURES), "ctypes binding and header disagree"


def test_library_exports_every_declared_symbol(lib):
    from tfhe_b200 import _lib
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], stdout=subprocess.PIPE,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\sT\s(tfhe(?:64)?_\w+)", out))
    missing = set(declared_functions()) - exported
    assert not missing, missing
    for name in declared_functions():
        assert getattr(lib, name) is not None


def test_version_and_last_error(lib):
    from tfhe_b200 import version
    assert "sm_100a" in version()
    assert isinstance(lib.tfhe_last_error(), bytes)


def _mul_bootstrap(lib, degree=1024, l=3, dims=None, rot_rows=None, ct_elems=None, batch=1, log2_q=32):
    dims = dims or (210, 2, l, 2, 8, degree // 2)
    arr = (ctypes.c_int64 * 6)(*dims)
    return lib.tfhe_mul_bootstrap(None, ctypes.c_void_p(1), ct_elems or 2 * degree, ctypes.c_void_p(1), arr,
                                  ctypes.c_void_p(1), rot_rows or 2 * degree, ctypes.c_void_p(1), 7, log2_q, l,
                                  degree, ctypes.c_void_p(1), batch)


def test_mul_bootstrap_rejects_like_the_reference(lib):
    assert _mul_bootstrap(lib, degree=1000, dims=(210, 2, 3, 2, 8, 500)) == 1
    assert b"Unsupported degree" in lib.tfhe_last_error()
    assert _mul_bootstrap(lib, l=5, dims=(210, 2, 5, 2, 8, 512)) == 1
    assert b"Unsupported l" in lib.tfhe_last_error()
    # shape checks the reference does not make
    assert _mul_bootstrap(lib, dims=(210, 2, 2, 2, 8, 512)) == 1          # bsk levels != l
    assert _mul_bootstrap(lib, dims=(210, 2, 3, 2, 6, 512)) == 1          # M not a power of two
    assert _mul_bootstrap(lib, rot_rows=100) == 1
    assert _mul_bootstrap(lib, ct_elems=3) == 1
    assert _mul_bootstrap(lib, log2_q=65) == 1
    # batch 0 is a no-op that needs no device
    assert _mul_bootstrap(lib, batch=0) == 0


def test_keys_create_validates_params(lib):
    from tfhe_b200 import _lib
    from tfhe_b200.params import CONFIG1
    out = ctypes.c_void_p()
    for bad in (CONFIG1.with_(N=1000), CONFIG1.with_(l_bs=5), CONFIG1.with_(n=631),
                CONFIG1.with_(log2_q=64), CONFIG1.with_(l_ks=9), CONFIG1.with_(collapse=5)):
        p = bad.ctypes()
        rc = lib.tfhe_keys_create(ctypes.byref(p), ctypes.c_void_p(1), ctypes.c_void_p(1), ctypes.c_void_p(1),
                                  None, ctypes.byref(out))
        assert rc == 1, bad
        with pytest.raises(_lib.TFHEError, match="INVALID_ARGUMENT"):
            _lib.check(rc)


def test_stateless_entry_points_validate(lib):
    assert lib.tfhe_sample_extract(ctypes.c_void_p(1), 1000, 1, ctypes.c_void_p(1), ctypes.c_void_p(1), 4,
                                   None) == 1
    assert lib.tfhe_sample_extract(ctypes.c_void_p(1), 1024, 0, ctypes.c_void_p(1), ctypes.c_void_p(1), 4,
                                   None) == 1
    assert lib.tfhe_keyswitch_ref(ctypes.c_void_p(1), ctypes.c_void_p(1), ctypes.c_void_p(1), ctypes.c_void_p(1),
                                  1024, 630, 9, 3, ctypes.c_void_p(1), ctypes.c_void_p(1), 4, None) == 1
    assert lib.tfhe_rotate_extract_i64(ctypes.c_void_p(1), ctypes.c_void_p(1), 1024, 2, 32, None, None, None, 4,
                                       None) == 1
    assert lib.tfhe_keys_device_bytes(None) == 0
    lib.tfhe_keys_destroy(None)
