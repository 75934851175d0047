// Instantiations of the FP64 blind-rotation kernel for one degree.
// Compiled once per BR_LOGN (7 .. 12) so the degrees build in parallel.
#include "br_cluster.cuh"
#include "br_split.cuh"
#include "br_tm.cuh"
#include "tfhe_dispatch.h"

#ifndef BR_LOGN
#error "BR_LOGN must be defined (log2 of the GLWE degree)"
#endif

#define TFHE_CAT2(a, b) a##b
#define TFHE_CAT(a, b) TFHE_CAT2(a, b)

namespace tfhe {

BrKernel TFHE_CAT(br_fp64_logn_, BR_LOGN)(int L, bool reflayout, int kr, int kt, bool qtg, bool xt) {
    // the extra-thread kernels: one-CTA layout, L <= 2
    if (xt) {
        if (kr != 0 || qtg) return nullptr;
        switch (L) {
            case 1:
                if (reflayout) return kt == 2 ? br_fp64_kernel<BR_LOGN, 1, true, 0, 2, false, true>
                                              : br_fp64_kernel<BR_LOGN, 1, true, 0, 1, false, true>;
                return kt == 2 ? br_fp64_kernel<BR_LOGN, 1, false, 0, 2, false, true>
                               : br_fp64_kernel<BR_LOGN, 1, false, 0, 1, false, true>;
            case 2:
                if (reflayout) return kt == 2 ? br_fp64_kernel<BR_LOGN, 2, true, 0, 2, false, true>
                                              : br_fp64_kernel<BR_LOGN, 2, true, 0, 1, false, true>;
                return kt == 2 ? br_fp64_kernel<BR_LOGN, 2, false, 0, 2, false, true>
                               : br_fp64_kernel<BR_LOGN, 2, false, 0, 1, false, true>;
            case 3:
                if (reflayout) return kt == 2 ? br_fp64_kernel<BR_LOGN, 3, true, 0, 2, false, true>
                                              : br_fp64_kernel<BR_LOGN, 3, true, 0, 1, false, true>;
                return kt == 2 ? br_fp64_kernel<BR_LOGN, 3, false, 0, 2, false, true>
                               : br_fp64_kernel<BR_LOGN, 3, false, 0, 1, false, true>;
            default: return nullptr;
        }
    }
#define TFHE_BR_CASE(LL)                                                                         \
    case LL:                                                                                     \
        if (reflayout) return kt == 2 ? br_fp64_kernel<BR_LOGN, LL, true, 0, 2>                    \
                                      : br_fp64_kernel<BR_LOGN, LL, true, 0, 1>;                   \
        if (kr == 2) return br_fp64_kernel<BR_LOGN, LL, false, 2, 1>;                             \
        if (kr != 0) return nullptr;                                                             \
        if (qtg) return kt == 2 ? br_fp64_kernel<BR_LOGN, LL, false, 0, 2, true>                   \
                                : br_fp64_kernel<BR_LOGN, LL, false, 0, 1, true>;                  \
        return kt == 2 ? br_fp64_kernel<BR_LOGN, LL, false, 0, 2> : br_fp64_kernel<BR_LOGN, LL, false, 0, 1>;
    switch (L) {
        TFHE_BR_CASE(1)
        TFHE_BR_CASE(2)
        TFHE_BR_CASE(3)
        TFHE_BR_CASE(4)
        default: return nullptr;
    }
#undef TFHE_BR_CASE
}

BrConvKernel TFHE_CAT(bsk_fft_logn_, BR_LOGN)() { return bsk_fft_kernel<BR_LOGN>; }

BrKernel TFHE_CAT(br_split_logn_, BR_LOGN)(int L) {
    switch (L) {
        case 1: return br_split_kernel<BR_LOGN, 1, false>;
        case 2: return br_split_kernel<BR_LOGN, 2, false>;
        case 3: return br_split_kernel<BR_LOGN, 3, false>;
        default: return nullptr;
    }
}

#if BR_LOGN == 10 || BR_LOGN == 11
BrKernel TFHE_CAT(br_cluster32_logn, BR_LOGN)(int L, int S) {
    if (S == 2) {
        switch (L) {
            case 1: return br_cluster_kernel<BR_LOGN, 1, false, 2>;
            case 2: return br_cluster_kernel<BR_LOGN, 2, false, 2>;
            case 3: return br_cluster_kernel<BR_LOGN, 3, false, 2>;
            default: return nullptr;
        }
    }
    if (S == 4) {
        switch (L) {
            case 1: return br_cluster_kernel<BR_LOGN, 1, false, 4>;
            case 2: return br_cluster_kernel<BR_LOGN, 2, false, 4>;
            case 3: return br_cluster_kernel<BR_LOGN, 3, false, 4>;
            default: return nullptr;
        }
    }
    return nullptr;
}
#endif

#if BR_LOGN == 11
BrKernel br_tm32_logn11(int L) {
    switch (L) {
        case 1: return br_tm_kernel<11, 1, 3, false>;
        case 2: return br_tm_kernel<11, 2, 3, false>;
        default: return nullptr;
    }
}
#endif

}  // namespace tfhe
