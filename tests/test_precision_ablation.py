"""Small case of the external-product precision ablation (the full table
comes from ``python tests/precision_ablation.py``) and the packed-table LUT
used by the 4-LUT configuration."""
import numpy as np

from oracle import tfhe_oracle as O
from precision_ablation import Study, split_limbs
from tfhe_b200 import client


def test_split_limbs_recombine_exactly():
    rng = np.random.default_rng(0)
    x = rng.integers(-2 ** 31, 2 ** 31, size=1000)
    for count in (2, 3, 4):
        parts = split_limbs(x, count)
        w = -(-32 // count)
        total = sum(limb << shift for limb, shift in parts)
        assert np.array_equal(total, x)
        for limb, _ in parts[:-1]:
            assert np.all(np.abs(limb) <= 2 ** (w - 1))


def test_packed_table_lut_rotates_to_every_table():
    N, n_lut, t, t_out = 256, 4, 4, 8
    rng = np.random.default_rng(1)
    tables = rng.integers(0, 4, size=(n_lut, t))
    body = client.packed_table_lut(N, tables, t_out).view(np.int32).astype(np.float64)
    scale = 2 ** 32 // t_out
    for m in range(t):
        for jitter in (-28, 0, 28):                     # inside the half box of N/(2t) = 32 positions
            pos = m * (2 * N // (2 * t)) + jitter           # phase m q/(2t) as a position in 2N
            rot = O.coef_rotation(body, -pos)
            got = np.rint(rot[:n_lut] / scale).astype(np.int64) % t_out
            assert np.array_equal(got, tables[:, m]), (m, jitter)


def test_ablation_small_case():
    st = Study(samples=1, seed=0, groups=3)
    res = st.run()
    assert res["fp64"]["group_err_max"] == 0            # FP64 is exact at gadget 2^7
    assert res["fp32x2"]["group_err_max"] > 0
    assert res["fp32x4"]["group_err_var"] < res["fp32x2"]["group_err_var"]


def test_fp64_product_at_gadget_2_15_stays_within_a_few_units_of_exact():
    """At n=742, N=2048, gadget 2^15 x 2 the FP64 external product is not
    exact; its per-coefficient error against the exact product stays small
    (the reference's FP64 FFT carries the same bound)."""
    st = Study(samples=1, seed=1, groups=2, name="cfg2", n_lut=1, t_in=16, t_out=8, fp32=False)
    res = st.run(("fp64",))
    assert 0 < res["fp64"]["group_err_max"] <= 16
