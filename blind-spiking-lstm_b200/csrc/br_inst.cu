// Instantiations of the FP64 blind-rotation kernel for one degree.
// Compiled once per BR_LOGN (7 .. 12) so the degrees build in parallel.
#include "br_fp64.cuh"
#include "tfhe_dispatch.h"

#ifndef BR_LOGN
#error "BR_LOGN must be defined (log2 of the GLWE degree)"
#endif

#define TFHE_CAT2(a, b) a##b
#define TFHE_CAT(a, b) TFHE_CAT2(a, b)

namespace tfhe {

BrKernel TFHE_CAT(br_fp64_logn_, BR_LOGN)(int L, bool reflayout) {
    switch (L) {
        case 1: return reflayout ? br_fp64_kernel<BR_LOGN, 1, true> : br_fp64_kernel<BR_LOGN, 1, false>;
        case 2: return reflayout ? br_fp64_kernel<BR_LOGN, 2, true> : br_fp64_kernel<BR_LOGN, 2, false>;
        case 3: return reflayout ? br_fp64_kernel<BR_LOGN, 3, true> : br_fp64_kernel<BR_LOGN, 3, false>;
        case 4: return reflayout ? br_fp64_kernel<BR_LOGN, 4, true> : br_fp64_kernel<BR_LOGN, 4, false>;
        default: return nullptr;
    }
}

BrConvKernel TFHE_CAT(bsk_fft_logn_, BR_LOGN)() { return bsk_fft_kernel<BR_LOGN>; }

}  // namespace tfhe
