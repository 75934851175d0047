"""tfhe_pbs_noalloc: the programmable bootstrap for callers that must not
allocate device memory (an XLA custom call inside a runtime that has
preallocated the GPU, a serving loop that keeps allocation off its latency
path, code under an external memory manager).  It keeps the key-switched
intermediate in a static device array of the library instead of allocating
it, so its results must equal tfhe_pbs's, call after call, and batches that
do not fit the array must be refused with a clear error.

This file is collected last so that a run stopping at the first failure has
already run every other test; it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU runs deselect -m gpu
    pytest.skip("needs a CUDA device", allow_module_level=True)

from pbs_cases import PARAMS, inputs, keys, step_body  # noqa: E402
from tfhe_b200 import _lib  # noqa: E402
from tfhe_b200.engine import Keys, _ptr, _stream, device_u32  # noqa: E402
from tfhe_b200.params import ParamSet  # noqa: E402


def _engine(name):
    p = PARAMS[name]
    k = keys(name)
    lg = lambda v: int(round(np.log2(v)))
    ps = ParamSet(name, N=p["N"], n=p["n"], log2_beta_bs=lg(p["beta_bs"]), l_bs=p["l_bs"],
                  collapse=p["collapse"], log2_beta_ks=lg(p["beta_ks"]), l_ks=p["l_ks"],
                  sigma_glwe=p["sigma_glwe"], sigma_lwe=p["sigma_lwe"])
    return ps, Keys.create(ps, k.bsk_coeff, k.ksk[0], k.ksk[1].reshape(k.ksk[1].shape[:2]))


def _noalloc(eng, a, b, lut, n_lut):
    """tfhe_pbs_noalloc through the C ABI, results in fresh tensors."""
    p = eng.params
    B = a.shape[0]
    out_a = torch.full((B, n_lut, p.N), -1, dtype=torch.int32, device="cuda")
    out_b = torch.full((B, n_lut), -1, dtype=torch.int32, device="cuda")
    rc = _lib.load().tfhe_pbs_noalloc(eng.handle, _ptr(a), _ptr(b), _ptr(lut), lut.shape[0], n_lut,
                                      _ptr(out_a), _ptr(out_b), B, _stream())
    _lib.check(rc)
    return out_a, out_b


@pytest.mark.parametrize("name,batch,n_lut", [("tiny_c3", 37, 2), ("cfg1", 9, 1)])
def test_noalloc_matches_pbs_on_consecutive_calls(name, batch, n_lut):
    ps, eng = _engine(name)
    N = PARAMS[name]["N"]
    lut = device_u32(np.stack([np.zeros(N), step_body(name)])[None])
    for call in range(2):
        msgs, a, b = inputs(name, batch, seed_offset=100 + call)
        a_d, b_d = device_u32(a), device_u32(b.reshape(-1))
        want_a, want_b = eng.pbs(a_d, b_d, lut, n_lut=n_lut)
        got_a, got_b = _noalloc(eng, a_d, b_d, lut, n_lut)
        torch.cuda.synchronize()
        # same kernels on the same inputs: bit-identical, the tolerance of
        # every native-path parity test
        assert torch.equal(got_a, want_a), f"call {call}: masks differ"
        assert torch.equal(got_b, want_b), f"call {call}: bodies differ"
    eng.close()


def test_noalloc_refuses_batches_beyond_the_static_array():
    ps, eng = _engine("tiny_c3")
    n = ps.n
    too_many = (8 << 20) // 4 // (n + 1) + 1
    a = torch.zeros((too_many, ps.big), dtype=torch.int32, device="cuda")
    b = torch.zeros((too_many,), dtype=torch.int32, device="cuda")
    lut = torch.zeros((1, 2, ps.N), dtype=torch.int32, device="cuda")
    out_a = torch.empty((too_many, 1, ps.N), dtype=torch.int32, device="cuda")
    out_b = torch.empty((too_many, 1), dtype=torch.int32, device="cuda")
    rc = _lib.load().tfhe_pbs_noalloc(eng.handle, _ptr(a), _ptr(b), _ptr(lut), 1, 1, _ptr(out_a), _ptr(out_b),
                                      too_many, _stream())
    assert rc == 1
    assert b"exceeds the static scratch" in _lib.load().tfhe_last_error()
    eng.close()
