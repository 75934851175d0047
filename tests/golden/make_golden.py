"""Generate the golden fixtures of the PBS path by running the REFERENCE's own
Python code (AMIAD-Research/Blind-Spiking-LSTM) in this container.

jax is not installed here, so the reference modules are imported under the
numpy-backed stand-in in ``tests/golden/jaxshim`` (jit = identity, vmap =
map-and-stack, lax.scan = loop; FFTs are numpy's).  The compiled FFI module
``cuTFHE._core`` cannot be built here either, so ``cuTFHE.multiply`` is
replaced by a stub that forwards to the reference's own JAX statement of the
kernel, ``schemas/text_jax.py:multiply_seq_monomial`` (the two share one
signature up to log2 arguments, cuTFHE/multiply.py:54-92 vs
schemas/text_jax.py:390-435).  Everything around the kernel in
``cuboot_merge`` (schemas/RLWE_jax.py:288-303: vmap, rotation by -b~ after the
blind rotation, many-LUT extraction) is the reference's code as written.

Keys and inputs come from ``oracle.tfhe_oracle.keygen`` with fixed seeds
(numpy PCG64), so only outputs are stored; the tests regenerate the keys.

Run from the repository root with REFERENCE_ROOT naming a checkout of the
reference (the output is committed and the tests never read the reference):

    REFERENCE_ROOT=<path to the reference checkout> python tests/golden/make_golden.py
    REFERENCE_ROOT=<path to the reference checkout> python tests/golden/make_golden.py cfg2
"""
from __future__ import annotations

import ast
import hashlib
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REFERENCE = os.environ.get("REFERENCE_ROOT")
if not REFERENCE or not os.path.isdir(REFERENCE):
    raise SystemExit("set REFERENCE_ROOT to a checkout of AMIAD-Research/Blind-Spiking-LSTM")

sys.path.insert(0, os.path.join(HERE, "jaxshim"))
sys.path.insert(0, REFERENCE)
sys.path.insert(0, REPO)

import jax.numpy as jnp  # noqa: E402  (the stand-in)
from schemas import polynomial_jax as PJ  # noqa: E402
from schemas import text_jax as TJ  # noqa: E402
from schemas import LWE_jax as LJ  # noqa: E402


def _install_cutfhe_stub():
    cu = types.ModuleType("cuTFHE")
    cum = types.ModuleType("cuTFHE.multiply")

    def multiply_seq_monomial(ciphertext, public_key, BSK, log_q, log_beta, l, degree,
                              collapse, all_rot_fft, n_lut):
        return TJ.multiply_seq_monomial(ciphertext, public_key, BSK, 2.0 ** log_q,
                                        2 ** log_beta, l, degree, collapse, all_rot_fft, n_lut)

    cum.multiply_seq_monomial = multiply_seq_monomial
    cu.multiply = cum
    sys.modules["cuTFHE"] = cu
    sys.modules["cuTFHE.multiply"] = cum


_install_cutfhe_stub()
from schemas import RLWE_jax as RJ  # noqa: E402
from oracle import tfhe_oracle as O  # noqa: E402
from jax import vmap  # noqa: E402


def _load_function(relpath, name, namespace):
    """Compile one top-level function of a reference file whose module
    cannot be imported (it pulls in flax), with the given globals."""
    src = open(os.path.join(REFERENCE, relpath)).read()
    tree = ast.parse(src)
    node = next(n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name == name)
    mod = ast.Module(body=[node], type_ignores=[])
    code = compile(mod, os.path.join(REFERENCE, relpath), "exec")
    exec(code, namespace)
    return namespace[name]


get_plain_LUT_ref = _load_function("nn_tfhe/utils_spike.py", "get_plain_LUT",
                                   {"jnp": jnp, "coef_rotation": PJ.coef_rotation})

Q = 2.0 ** 32

# parameter sets: tiny ones for fast CPU/GPU tests, and config 1 of the PBS
# workload (n=630, N=1024, beta 2^7 x 3, KS 2^3 x 5, collapse 3)
PARAMS = {
    "tiny_c3": dict(q=Q, N=256, n=24, beta_bs=2 ** 7, l_bs=3, collapse=3, beta_ks=2 ** 3, l_ks=5,
                    sigma_glwe=2.0 ** 7, sigma_lwe=2.0 ** 17),
    "tiny_c2": dict(q=Q, N=512, n=16, beta_bs=2 ** 15, l_bs=2, collapse=2, beta_ks=2 ** 4, l_ks=5,
                    sigma_glwe=1.0, sigma_lwe=2.0 ** 15),
    "cfg1": dict(q=Q, N=1024, n=630, beta_bs=2 ** 7, l_bs=3, collapse=3, beta_ks=2 ** 3, l_ks=5,
                 sigma_glwe=2.0 ** 7, sigma_lwe=2.0 ** 17),
    # config 2 of the PBS workload (n=742, N=2048, beta 2^15 x 2, KS 2^4 x 5,
    # collapse 2): written to its own file by `make_golden.py cfg2`
    "cfg2": dict(q=Q, N=2048, n=742, beta_bs=2 ** 15, l_bs=2, collapse=2, beta_ks=2 ** 4, l_ks=5,
                 sigma_glwe=1.0, sigma_lwe=2.0 ** 15),
}
KEY_SEED = {"tiny_c3": 11, "tiny_c2": 12, "cfg1": 13, "cfg2": 14}
INPUT_SEED = {"tiny_c3": 21, "tiny_c2": 22, "cfg1": 23, "cfg2": 24}


def special_values():
    """Torus values at and around the decomposition's rounding ties."""
    vals = [0, 1, -1, 2 ** 31, -2 ** 31, 2 ** 31 - 1, -2 ** 31 + 1, 2 ** 24, -2 ** 24,
            3 * 2 ** 24, 2 ** 24 + 2 ** 17, 2 ** 10, 2 ** 10 + 1, 2 ** 10 - 1, 2 ** 16, 2 ** 17,
            -2 ** 17, 2 ** 20, 2 ** 28 + 2 ** 27, -(2 ** 28 + 2 ** 27), 5 * 2 ** 14, 2 ** 14,
            2 ** 15 + 2 ** 14, 7 * 2 ** 12, 2 ** 12]
    return np.array(vals, dtype=np.float64)


def gen_polynomial(out):
    rng = np.random.default_rng(101)
    x = rng.integers(-2 ** 31, 2 ** 31, size=(3, 2, 256)).astype(np.float64)
    x[0, 0, : len(special_values())] = special_values()
    out["poly_x"] = x
    for beta, l in [(2 ** 7, 3), (2 ** 15, 2), (2 ** 3, 5), (2 ** 4, 5), (2 ** 13, 2)]:
        out[f"poly_dec_b{beta}_l{l}"] = np.asarray(PJ.decomposition(x, beta, l, Q))
    out["poly_cmod"] = np.asarray(PJ.centered_mod(x * 3.0 + 2 ** 31, Q))
    small = rng.integers(-64, 64, size=(4, 256)).astype(np.float64)
    out["poly_small"] = small
    out["poly_fourier"] = np.asarray(PJ.jax_fourier(small))
    out["poly_inverse"] = np.asarray(PJ.jax_inversefourier(PJ.jax_fourier(small)))
    alphas = np.array([0, 1, 5, 255, 256, 257, 511, 512, -1, -3, -256, -300, -511, 700, -700])
    out["rot_alphas"] = alphas
    out["rot_out"] = np.stack([np.asarray(PJ.coef_rotation(small[0], np.array([float(a)])))
                               for a in alphas])
    ext = []
    for a in [0, 1, 2, 3, 100, 255]:
        ea, eb = TJ.sample_extract((small[1], small[2]), a)
        ext.append(np.concatenate([np.asarray(ea), np.asarray(eb)]))
    out["extract_alphas"] = np.array([0, 1, 2, 3, 100, 255])
    out["extract_out"] = np.stack(ext)
    for c in (1, 2, 3, 4):
        out[f"binvec_{c}"] = np.asarray(TJ.all_binary_vectors(c))
    lut = np.stack([np.asarray(get_plain_LUT_ref(256, 4, i, 4.0, g))
                    for i, g in enumerate([-1.5, -0.5, 0.5, 1.5])])
    out["plain_lut_n4"] = lut


def gen_pbs(name, out, n_lut_list=(1,), batch=4, t=32, t_out=32):
    """Messages in Z_{t/2} at q/t; the step LUT's output at q/t_out."""
    p = PARAMS[name]
    N, q = p["N"], p["q"]
    keys = O.keygen(p, KEY_SEED[name])
    rng = np.random.default_rng(INPUT_SEED[name])
    msgs = rng.integers(0, t // 2, size=batch)
    a, b = O.encrypt_inputs(keys, msgs, q / t, rng)
    out[f"{name}_in_a"], out[f"{name}_in_b"], out[f"{name}_msgs"] = a, b, msgs
    ks_params = {"beta_ks": p["beta_ks"], "l_ks": p["l_ks"], "q": q}
    # KS exactly as nn_tfhe/activation.py:150
    ksk = (keys.ksk[0], keys.ksk[1])
    ca, cb = vmap(LJ.key_switch_LWE, (None, 0, None))(ksk, (a, b), ks_params)
    ca, cb = np.asarray(ca), np.asarray(cb)
    out[f"{name}_ks_a"], out[f"{name}_ks_b"] = ca, cb
    all_rot = keys.all_rot
    for n_lut in n_lut_list:
        if n_lut == 1:
            body = O.step_lut(N, t // 2, t // 4, q / t_out)
        else:
            s = 4.0
            body = sum(np.asarray(get_plain_LUT_ref(N, n_lut, i, s, g))
                       for i, g in enumerate(np.linspace(-1.5, 1.5, n_lut))) * (q / 16)
        luts = [np.zeros((batch, N)), np.broadcast_to(body, (batch, N)).copy()]
        out[f"{name}_lut{n_lut}"] = body
        # schemas/RLWE_jax.py:288-303 (kernel replaced by text_jax.multiply_seq_monomial)
        ra, rb = RJ.cuboot_merge((ca, cb), luts, keys.bsk_ordered, q, p["beta_bs"], p["l_bs"], N,
                                 p["collapse"], all_rot, n_lut)
        out[f"{name}_merge{n_lut}_a"], out[f"{name}_merge{n_lut}_b"] = np.asarray(ra), np.asarray(rb)
        # schemas/RLWE_jax.py:305-315
        acc = RJ.BR((ca, cb), luts, keys.bsk_ordered, q, p["beta_bs"], p["l_bs"], N, p["collapse"],
                    all_rot, n_lut)
        out[f"{name}_br{n_lut}"] = np.asarray(acc)
    # pure-JAX bootstrapping path (rotation before), as test_collapse.py:173
    body = O.step_lut(N, t // 2, t // 4, q / t_out)
    luts = [np.zeros((batch, N)), np.broadcast_to(body, (batch, N)).copy()]
    ba, bb = vmap(RJ.bootstrapping, in_axes=(0, 0, None, None, None, None, None, None, None))(
        (ca, cb), luts, keys.bsk_ordered, q, p["beta_bs"], p["l_bs"], N, p["collapse"], all_rot)
    out[f"{name}_boot_a"], out[f"{name}_boot_b"] = np.asarray(ba), np.asarray(bb)


def gen_all_rot(out):
    """parameters_crypto.py:86-91 at its own degree (2^11): digest only."""
    import importlib
    pc = importlib.import_module("parameters_crypto")
    arr = np.ascontiguousarray(np.asarray(pc.all_rot_possible_fourier))
    out["allrot2048_sha256"] = np.frombuffer(hashlib.sha256(arr.tobytes()).digest(), dtype=np.uint8)
    out["allrot2048_rows"] = arr[[0, 1, 2047, 2048, 4095]]


def main():
    out = {}
    gen_polynomial(out)
    gen_pbs("tiny_c3", out, n_lut_list=(1, 4), batch=6)
    gen_pbs("tiny_c2", out, n_lut_list=(1, 2), batch=6)
    gen_pbs("cfg1", out, n_lut_list=(1, 4), batch=4)
    gen_all_rot(out)
    path = os.path.join(HERE, "pbs_golden.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes,", len(out), "arrays")


def main_cfg2():
    """Config 2 (gadget 2^15, where the reference's FP64 products round):
    four ciphertexts of Z_8 (at q/16) through the reference's key switch,
    cuboot_merge and BR, the step LUT's output at q/8 (its noise, ~2^25,
    needs that margin)."""
    out = {}
    gen_pbs("cfg2", out, n_lut_list=(1,), batch=4, t=16, t_out=8)
    path = os.path.join(HERE, "pbs_cfg2_golden.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes,", len(out), "arrays")


if __name__ == "__main__":
    if sys.argv[1:] == ["cfg2"]:
        main_cfg2()
    else:
        main()
