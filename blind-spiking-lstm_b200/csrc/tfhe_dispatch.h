// Kernel lookup by degree: each br_inst.cu object (one per log2 N) exports
// the FP64 blind-rotation kernels and the key-FFT kernel of its degree.
#pragma once

#include "br_fp64.cuh"

namespace tfhe {

using BrKernel = void (*)(const BrArgs);
using BrConvKernel = void (*)(const BskConvArgs);

#define TFHE_DECLARE_LOGN(LG)                              \
    BrKernel br_fp64_logn_##LG(int L, bool reflayout, int kr, int kt);     \
    BrConvKernel bsk_fft_logn_##LG();

TFHE_DECLARE_LOGN(7)
TFHE_DECLARE_LOGN(8)
TFHE_DECLARE_LOGN(9)
TFHE_DECLARE_LOGN(10)
TFHE_DECLARE_LOGN(11)
TFHE_DECLARE_LOGN(12)
#undef TFHE_DECLARE_LOGN

inline BrKernel br_fp64_kernel_for(int logn, int L, bool reflayout, int kr, int kt) {
    switch (logn) {
        case 7: return br_fp64_logn_7(L, reflayout, kr, kt);
        case 8: return br_fp64_logn_8(L, reflayout, kr, kt);
        case 9: return br_fp64_logn_9(L, reflayout, kr, kt);
        case 10: return br_fp64_logn_10(L, reflayout, kr, kt);
        case 11: return br_fp64_logn_11(L, reflayout, kr, kt);
        case 12: return br_fp64_logn_12(L, reflayout, kr, kt);
        default: return nullptr;
    }
}

inline BrConvKernel bsk_fft_kernel_for(int logn) {
    switch (logn) {
        case 7: return bsk_fft_logn_7();
        case 8: return bsk_fft_logn_8();
        case 9: return bsk_fft_logn_9();
        case 10: return bsk_fft_logn_10();
        case 11: return bsk_fft_logn_11();
        case 12: return bsk_fft_logn_12();
        default: return nullptr;
    }
}

}  // namespace tfhe
