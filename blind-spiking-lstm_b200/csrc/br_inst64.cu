// Instantiations of the FP64 blind-rotation kernel on the 64-bit torus
// (T64) for one degree, compiled once per BR_LOGN beside br_inst.cu.
// Shapes: the one-CTA layout with extra threads, the quarter-root-table-in-
// global layout, and the plain layout; l_bs 1 .. 3; and the cluster-pair
// kernel of small batches (br_split.cuh).
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

BrKernel TFHE_CAT(br_fp64_t64_logn_, BR_LOGN)(int L, int kt, bool qtg, bool xt) {
#define TFHE_BR64_CASE(LL)                                                                          \
    case LL:                                                                                        \
        if (xt) {                                                                                   \
            if (qtg) return nullptr;                                                                \
            return kt == 2 ? br_fp64_kernel<BR_LOGN, LL, false, 0, 2, false, true, true>              \
                           : br_fp64_kernel<BR_LOGN, LL, false, 0, 1, false, true, true>;             \
        }                                                                                           \
        if (qtg) return kt == 2 ? br_fp64_kernel<BR_LOGN, LL, false, 0, 2, true, false, true> : nullptr; \
        return kt == 2 ? br_fp64_kernel<BR_LOGN, LL, false, 0, 2, false, false, true>                 \
                       : br_fp64_kernel<BR_LOGN, LL, false, 0, 1, false, false, true>;
    switch (L) {
        TFHE_BR64_CASE(1)
        TFHE_BR64_CASE(2)
        TFHE_BR64_CASE(3)
        default: return nullptr;
    }
#undef TFHE_BR64_CASE
}

BrKernel TFHE_CAT(br_split64_logn_, BR_LOGN)(int L) {
    switch (L) {
        case 1: return br_split_kernel<BR_LOGN, 1, true>;
        case 2: return br_split_kernel<BR_LOGN, 2, true>;
        case 3: return br_split_kernel<BR_LOGN, 3, true>;
        default: return nullptr;
    }
}

#if BR_LOGN == 10 || BR_LOGN == 11
BrKernel TFHE_CAT(br_cluster64_logn, BR_LOGN)(int L, int S) {
    if (S == 2) {
        switch (L) {
            case 1: return br_cluster_kernel<BR_LOGN, 1, true, 2>;
            case 2: return br_cluster_kernel<BR_LOGN, 2, true, 2>;
            case 3: return br_cluster_kernel<BR_LOGN, 3, true, 2>;
            default: return nullptr;
        }
    }
    if (S == 4) {
        switch (L) {
            case 1: return br_cluster_kernel<BR_LOGN, 1, true, 4>;
            case 2: return br_cluster_kernel<BR_LOGN, 2, true, 4>;
            case 3: return br_cluster_kernel<BR_LOGN, 3, true, 4>;
            default: return nullptr;
        }
    }
    return nullptr;
}
#endif

#if BR_LOGN == 11
BrKernel br_tm64_logn11(int L) {
    switch (L) {
        case 1: return br_tm_kernel<11, 1, 3, true>;
        case 2: return br_tm_kernel<11, 2, 3, true>;
        default: return nullptr;
    }
}
#endif

}  // namespace tfhe
