"""Parameter sets of the PBS workloads (uint32 torus, q = 2^32).

The reference keeps its parameters as module globals
(parameters_crypto.py:6-84: q = 2^64, N = 2048, n = 702, beta_bs = 2^13,
l_bs = 2, collapse 3).  The workloads here run on a 32-bit torus:

* CONFIG1: n=630, N=1024, gadget 2^7 x 3, key switch 2^3 x 5, collapse 3,
  noise std 2^-15 (LWE) and 2^-25 (GLWE) of q; messages Z_16 + padding bit.
* CONFIG2: n=742, N=2048, gadget 2^15 x 2, key switch 2^4 x 5, collapse 2
  (742 has no factor 3); messages Z_8 + padding bit.  The noise of this set
  is not fixed by the workload; with digits up to 2^14 the bootstrapping key
  must carry at most unit noise (std 1 of 2^32) for outputs to decrypt, and
  the LWE noise is 2^-17 of q.
* CONFIG3: CONFIG1 with 4 LUTs packed per blind rotation (n_lut = 4) over
  Z_4 messages.
"""
from __future__ import annotations

from dataclasses import dataclass, replace

from ._lib import TfheParams


@dataclass(frozen=True)
class ParamSet:
    name: str
    N: int
    n: int
    log2_beta_bs: int
    l_bs: int
    collapse: int
    log2_beta_ks: int
    l_ks: int
    sigma_glwe: float     # noise std in units of q / 2^32
    sigma_lwe: float
    n_big: int = 0        # 0 -> N (inputs are LWEs under the GLWE key)
    log2_q: int = 32

    @property
    def q(self) -> float:
        return float(2 ** self.log2_q)

    @property
    def big(self) -> int:
        return self.n_big or self.N

    @property
    def G(self) -> int:
        return self.n // self.collapse

    @property
    def M(self) -> int:
        return 1 << self.collapse

    def ctypes(self) -> TfheParams:
        return TfheParams(self.N, self.n, self.big, self.log2_beta_bs, self.l_bs, self.collapse,
                          self.log2_beta_ks, self.l_ks, self.log2_q)

    def oracle_dict(self) -> dict:
        """The keys of the reference's dict_params (parameters_crypto.py)."""
        return dict(q=self.q, N=self.N, n=self.n, beta_bs=2 ** self.log2_beta_bs, l_bs=self.l_bs,
                    collapse=self.collapse, beta_ks=2 ** self.log2_beta_ks, l_ks=self.l_ks,
                    sigma_glwe=self.sigma_glwe, sigma_lwe=self.sigma_lwe)

    def bsk_bytes_fp64(self) -> int:
        """Device bytes of the FP64 Fourier bootstrapping key."""
        return self.G * 2 * (2 * self.l_bs) * self.M * (self.N // 2) * 16

    def with_(self, **kw) -> "ParamSet":
        return replace(self, **kw)


CONFIG1 = ParamSet("n630_N1024_b7x3_c3", N=1024, n=630, log2_beta_bs=7, l_bs=3, collapse=3,
                   log2_beta_ks=3, l_ks=5, sigma_glwe=2.0 ** 7, sigma_lwe=2.0 ** 17)
CONFIG2 = ParamSet("n742_N2048_b15x2_c2", N=2048, n=742, log2_beta_bs=15, l_bs=2, collapse=2,
                   log2_beta_ks=4, l_ks=5, sigma_glwe=1.0, sigma_lwe=2.0 ** 15)
CONFIG3 = CONFIG1.with_(name="n630_N1024_b7x3_c3_lut4")

# small sets for tests (same shapes as the golden fixtures)
TINY_C3 = ParamSet("n24_N256_b7x3_c3", N=256, n=24, log2_beta_bs=7, l_bs=3, collapse=3,
                   log2_beta_ks=3, l_ks=5, sigma_glwe=2.0 ** 7, sigma_lwe=2.0 ** 17)
TINY_C2 = ParamSet("n16_N512_b15x2_c2", N=512, n=16, log2_beta_bs=15, l_bs=2, collapse=2,
                   log2_beta_ks=4, l_ks=5, sigma_glwe=1.0, sigma_lwe=2.0 ** 15)

ALL = {p.name: p for p in (CONFIG1, CONFIG2, CONFIG3, TINY_C3, TINY_C2)}
