"""The FP32 split-limb blind rotation (tfhe_fp32_*) on the GPU: with four
8-bit limbs at a 2^7 gadget it evaluates the LUT like the FP64 engine; one
CMux group against the exact integer product shows the limb count's
rounding (more limbs, smaller error); one or two ciphertexts per CTA give the
same outputs; a short run of the config-3 ablation decrypts every FP64
output."""
import numpy as np
import pytest
import torch

from oracle import tfhe_oracle as O
from pbs_cases import PARAMS, inputs, keys, ks_params, step_body

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU runs deselect -m gpu
    pytest.skip("needs a CUDA device", allow_module_level=True)

from tfhe_b200.engine import FP32Keys, centred, device_u32  # noqa: E402
from tfhe_b200.params import TINY_C3  # noqa: E402


def _ks(name, a, b):
    ka, kb = O.key_switch_LWE(keys(name).ksk, (a, b), ks_params(name))
    return device_u32(ka), device_u32(kb.reshape(-1))


def test_fp32_four_limbs_evaluates_the_lut():
    name = "tiny_c3"
    k = keys(name)
    msgs, a, b = inputs(name, 24)
    ka, kb = _ks(name, a, b)
    lut = device_u32(np.stack([np.zeros(PARAMS[name]["N"]), step_body(name)])[None])
    f = FP32Keys(TINY_C3, k.bsk_coeff, 4)
    oa, ob = f.cuboot_merge(ka, kb, lut, 1)
    out_a = centred(oa.cpu().numpy())[:, 0].astype(np.float64)
    out_b = centred(ob.cpu().numpy())[:, 0].astype(np.float64)
    dec = O.decrypt_LWE((out_a, out_b), k.sk_glwe, {"t": 32, "q": 2.0 ** 32})
    assert np.array_equal(dec, (msgs >= 8).astype(float))
    # one or two ciphertexts per CTA: the same arithmetic per ciphertext
    oa1, ob1 = f.cuboot_merge(ka, kb, lut, 1, ciphertexts_per_cta=1)
    assert torch.equal(oa1, oa) and torch.equal(ob1, ob)
    f.close()


def test_one_group_error_shrinks_with_more_limbs():
    from precision_ablation_gpu import one_group_errors
    from tfhe_b200 import client
    from tfhe_b200.params import CONFIG3
    ck = client.keygen(CONFIG3, 5)
    errs = one_group_errors(CONFIG3, ck, ("fp64", "fp32x2", "fp32x4"), samples=16)
    print(errs)
    assert errs["fp64"]["group_err_max_log2"] == 0.0            # exact at gadget 2^7 (rounding < 1/2)
    assert errs["fp32x4"]["group_err_var"] < errs["fp32x2"]["group_err_var"]


def test_short_ablation_run():
    from precision_ablation_gpu import run
    rows = {r["form"]: r for r in run(total=2048, forms=("fp64", "fp32x4"))}
    assert rows["fp64"]["failures"] == 0
    assert rows["fp32x4"]["br_pbs_per_s"] > 0
