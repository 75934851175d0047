"""Golden fixtures of the blind rotation at the reference's OWN parameter set
(parameters_crypto.py:6-32: q = 2^64 held in float64, N = 2048, n = 702,
gadget 2^13 x 2, collapse 3, sigma 2^17), recorded by running the
reference's code under the jax stand-in (see refenv.py):

  multiply_seq_monomial  schemas/text_jax.py:390-435 (the JAX statement of
                         the mul_bootstrap kernel), one CMux group and the
                         full 234-group chain
  cuboot_merge           schemas/RLWE_jax.py:288-303 (rotation by -b~ after
                         the chain, sample extraction)

Keys come from oracle.tfhe_oracle.keygen_q64 (seed 64), inputs from fixed
seeds; only outputs are stored, in tests/golden/ref64_golden.npz.  At
q = 2^64 the reference's float64 arithmetic is inexact, so these outputs
are the reference's own rounding of the chain, not exact integers.  Run from
the repository root:

    REFERENCE_ROOT=<path to the reference checkout> python tests/golden/make_ref64_golden.py
"""
from __future__ import annotations

import os
import sys
import time

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import refenv  # noqa: E402

refenv.setup()

import numpy as np  # noqa: E402

from schemas import RLWE_jax as RJ  # noqa: E402  (the reference)
from schemas import text_jax as TJ  # noqa: E402
from oracle import tfhe_oracle as O  # noqa: E402

import ref64_cases as RC  # noqa: E402


def main():
    t0 = time.time()
    case = RC.case()
    p = O.REF64
    q, N, c = p["q"], p["N"], p["collapse"]
    out = {}
    # one CMux group: the first group's key block on random accumulators
    g1 = RC.one_group_inputs(case)
    accs = []
    for i in range(g1["acc"].shape[0]):
        accs.append(np.asarray(TJ.multiply_seq_monomial(g1["acc"][i], g1["pk"][i], g1["bsk1"], q, p["beta_bs"],
                                                        p["l_bs"], N, c, case["all_rot"], 1)))
    out["group1_acc"] = np.stack(accs)
    t1 = time.time()
    # the full chain and cuboot_merge on LWEs of Z_8 messages (padding bit)
    a, b, luts = case["lwe_a"], case["lwe_b"], case["luts"]
    br = RJ.BR((a, b[:, None]), luts, case["bsk_ordered"], q, p["beta_bs"], p["l_bs"], N, c, case["all_rot"], 1)
    out["br_a"], out["br_b"] = np.asarray(br[0]), np.asarray(br[1])
    ma, mb = RJ.cuboot_merge((a, b[:, None]), luts, case["bsk_ordered"], q, p["beta_bs"], p["l_bs"], N, c,
                             case["all_rot"], 1)
    out["merge_a"], out["merge_b"] = np.asarray(ma), np.asarray(mb)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref64_golden.npz")
    np.savez_compressed(path, **out)
    print(f"one group {t1 - t0:.1f} s, chain {time.time() - t1:.1f} s; wrote {path} "
          f"{os.path.getsize(path)} bytes")


if __name__ == "__main__":
    main()
