"""tfhe_pbs_noalloc: the programmable bootstrap for callers that must not
allocate device memory (an XLA custom call inside a runtime that has
preallocated the GPU, a serving loop that keeps allocation off its latency
path, code under an external memory manager).  It keeps the key-switched
intermediate in a static device array of the library instead of allocating
it, so its results must equal tfhe_pbs's, call after call, and batches that
do not fit the array must be refused with a clear error.

This file is collected last so that a run stopping at the first failure has
already run every other test; it also passes on its own in a fresh process.
One test runs the entry point as the very first bootstrap of a fresh process
(no tfhe_pbs before it) and checks that the device's free memory and the
stream-ordered pool's usage do not move across the call.
"""
import ctypes
import json
import os
import subprocess
import sys

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


# Runs in a fresh interpreter: key upload and every buffer first, then the
# no-allocation bootstrap as the process's first bootstrap of any kind.
# Modules load eagerly, so a lazily loaded kernel image cannot be mistaken
# for an allocation by the call.
_FRESH_PROCESS = r"""
import ctypes, json, sys
import numpy as np
import torch
from cuda.bindings import runtime as rt
sys.path[:0] = [TESTS, ROOT, PKG]
from pbs_cases import PARAMS, inputs, keys, step_body
from tfhe_b200 import _lib
from tfhe_b200.engine import Keys, _ptr, _stream, device_u32
from tfhe_b200.params import ParamSet

name, batch, n_lut = "tiny_c3", 37, 2
p, k = PARAMS[name], keys(name)
lg = lambda v: int(round(np.log2(v)))
ps = ParamSet(name, N=p["N"], n=p["n"], log2_beta_bs=lg(p["beta_bs"]), l_bs=p["l_bs"],
              collapse=p["collapse"], log2_beta_ks=lg(p["beta_ks"]), l_ks=p["l_ks"],
              sigma_glwe=p["sigma_glwe"], sigma_lwe=p["sigma_lwe"])
eng = Keys.create(ps, k.bsk_coeff, k.ksk[0], k.ksk[1].reshape(k.ksk[1].shape[:2]))
lib = _lib.load()
msgs, a, b = inputs(name, batch, seed_offset=300)
a_d, b_d = device_u32(a), device_u32(b.reshape(-1))
lut = device_u32(np.stack([np.zeros(p["N"]), step_body(name)])[None])
outs = [(torch.full((batch, n_lut, p["N"]), -1, dtype=torch.int32, device="cuda"),
         torch.full((batch, n_lut), -1, dtype=torch.int32, device="cuda")) for _ in range(2)]
torch.cuda.synchronize()

def pool_used_high():
    err, pool = rt.cudaDeviceGetDefaultMemPool(0)
    assert err == rt.cudaError_t.cudaSuccess
    err, v = rt.cudaMemPoolGetAttribute(pool, rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemHigh)
    assert err == rt.cudaError_t.cudaSuccess
    return int(v)

before = (torch.cuda.mem_get_info()[0], pool_used_high(), torch.cuda.memory_reserved())
rcs = []
for oa, ob in outs:
    rcs.append(lib.tfhe_pbs_noalloc(eng.handle, _ptr(a_d), _ptr(b_d), _ptr(lut), 1, n_lut,
                                    _ptr(oa), _ptr(ob), batch, _stream()))
torch.cuda.synchronize()
after = (torch.cuda.mem_get_info()[0], pool_used_high(), torch.cuda.memory_reserved())
v = ctypes.c_int32(-1)
lib.tfhe_device_status(ctypes.byref(v), 0)
want_a, want_b = eng.pbs(a_d, b_d, lut, n_lut=n_lut)
torch.cuda.synchronize()
same = all(torch.equal(oa, want_a) and torch.equal(ob, want_b) for oa, ob in outs)
print("RESULT " + json.dumps({"rcs": rcs, "before": before, "after": after, "status": v.value,
                              "same": same}))
"""


def test_noalloc_first_call_in_fresh_process_allocates_nothing():
    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    code = (f"TESTS, ROOT, PKG = {here!r}, {root!r}, {os.path.join(root, 'blind-spiking-lstm_b200')!r}\n"
            + _FRESH_PROCESS)
    env = dict(os.environ, CUDA_MODULE_LOADING="EAGER")
    proc = subprocess.run([sys.executable, "-c", code], env=env, stdout=subprocess.PIPE,
                          stderr=subprocess.STDOUT, text=True, timeout=600)
    assert proc.returncode == 0, proc.stdout[-4000:]
    line = next(ln for ln in proc.stdout.splitlines() if ln.startswith("RESULT "))
    res = json.loads(line[len("RESULT "):])
    assert res["rcs"] == [0, 0]
    free0, pool0, torch0 = res["before"]
    free1, pool1, torch1 = res["after"]
    assert free1 == free0, f"free device memory moved across the calls: {free0} -> {free1}"
    assert pool1 == pool0, f"the stream-ordered pool was used: high-water {pool0} -> {pool1}"
    assert torch1 == torch0
    assert res["status"] == 0, "a bounded wait timed out"
    # and the results are tfhe_pbs's, bit for bit, on both calls
    assert res["same"]
