"""tfhe_b200: B200-native TFHE programmable bootstrapping (key switching,
collapsed blind rotation, many-LUT sample extraction) for the encrypted
Spike-LSTM of AMIAD-Research/Blind-Spiking-LSTM.

The compute lives in libtfhe_b200.so (sm_100a CUDA behind the C ABI of
include/tfhe_b200.h).  ``engine`` holds device-resident keys and batched
stages; ``ops`` mirrors the reference's operator surface.
"""
from ._lib import TFHEError, LIB_PATH, load, version
from .params import ParamSet, CONFIG1, CONFIG2, CONFIG3, TINY_C3, TINY_C2

__all__ = ["TFHEError", "LIB_PATH", "load", "version", "ParamSet", "CONFIG1", "CONFIG2", "CONFIG3",
           "TINY_C3", "TINY_C2"]
