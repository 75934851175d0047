// Kernel lookup by degree: each br_inst.cu object (one per log2 N) exports
// the FP64 blind-rotation kernels and the key-FFT kernel of its degree.
#pragma once

#include "br_cluster.cuh"
#include "br_split.cuh"
#include "br_tm.cuh"

namespace tfhe {

using BrKernel = void (*)(const BrArgs);
using BrConvKernel = void (*)(const BskConvArgs);

#define TFHE_DECLARE_LOGN(LG)                              \
    BrKernel br_fp64_logn_##LG(int L, bool reflayout, int kr, int kt, bool qtg, bool xt);     \
    BrKernel br_fp64_t64_logn_##LG(int L, int kt, bool qtg, bool xt);                         \
    BrKernel br_split_logn_##LG(int L);                                                       \
    BrKernel br_split64_logn_##LG(int L);                                                     \
    BrConvKernel bsk_fft_logn_##LG();

TFHE_DECLARE_LOGN(7)
TFHE_DECLARE_LOGN(8)
TFHE_DECLARE_LOGN(9)
TFHE_DECLARE_LOGN(10)
TFHE_DECLARE_LOGN(11)
TFHE_DECLARE_LOGN(12)
#undef TFHE_DECLARE_LOGN

inline BrKernel br_fp64_kernel_for(int logn, int L, bool reflayout, int kr, int kt, bool qtg = false,
                                   bool xt = false) {
    switch (logn) {
        case 7: return br_fp64_logn_7(L, reflayout, kr, kt, qtg, xt);
        case 8: return br_fp64_logn_8(L, reflayout, kr, kt, qtg, xt);
        case 9: return br_fp64_logn_9(L, reflayout, kr, kt, qtg, xt);
        case 10: return br_fp64_logn_10(L, reflayout, kr, kt, qtg, xt);
        case 11: return br_fp64_logn_11(L, reflayout, kr, kt, qtg, xt);
        case 12: return br_fp64_logn_12(L, reflayout, kr, kt, qtg, xt);
        default: return nullptr;
    }
}

// the T64 kernels (q = 2^64: uint64 LWEs, int64 LUTs, uint64 outputs)
inline BrKernel br_fp64_t64_kernel_for(int logn, int L, int kt, bool qtg, bool xt) {
    switch (logn) {
        case 7: return br_fp64_t64_logn_7(L, kt, qtg, xt);
        case 8: return br_fp64_t64_logn_8(L, kt, qtg, xt);
        case 9: return br_fp64_t64_logn_9(L, kt, qtg, xt);
        case 10: return br_fp64_t64_logn_10(L, kt, qtg, xt);
        case 11: return br_fp64_t64_logn_11(L, kt, qtg, xt);
        case 12: return br_fp64_t64_logn_12(L, kt, qtg, xt);
        default: return nullptr;
    }
}

// the cluster-pair kernels of small batches (one ciphertext per two CTAs)
inline BrKernel br_split_kernel_for(int logn, int L, bool t64) {
    switch (logn) {
        case 7: return t64 ? br_split64_logn_7(L) : br_split_logn_7(L);
        case 8: return t64 ? br_split64_logn_8(L) : br_split_logn_8(L);
        case 9: return t64 ? br_split64_logn_9(L) : br_split_logn_9(L);
        case 10: return t64 ? br_split64_logn_10(L) : br_split_logn_10(L);
        case 11: return t64 ? br_split64_logn_11(L) : br_split_logn_11(L);
        case 12: return t64 ? br_split64_logn_12(L) : br_split_logn_12(L);
        default: return nullptr;
    }
}

// the kernels of one ciphertext per cluster of 2 S CTAs for small batches:
// S = 2 (four CTAs) and S = 4 (eight CTAs) at N = 1024 and 2048
BrKernel br_cluster32_logn10(int L, int S);
BrKernel br_cluster32_logn11(int L, int S);
BrKernel br_cluster64_logn10(int L, int S);
BrKernel br_cluster64_logn11(int L, int S);
inline BrKernel br_cluster_kernel_for(int logn, int L, bool t64, int S) {
    if (logn == 10) return t64 ? br_cluster64_logn10(L, S) : br_cluster32_logn10(L, S);
    if (logn == 11) return t64 ? br_cluster64_logn11(L, S) : br_cluster32_logn11(L, S);
    return nullptr;
}

// the tensor-memory kernels (three ciphertexts per CTA), N = 2048 only
BrKernel br_tm32_logn11(int L);
BrKernel br_tm64_logn11(int L);
inline BrKernel br_tm_kernel_for(int logn, int L, bool t64) {
    if (logn != 11) return nullptr;
    return t64 ? br_tm64_logn11(L) : br_tm32_logn11(L);
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

// tensor-core LWE key switch (ks_tc.cu)
struct KsTcArgs {
    const uint32_t* a_in;         // (B, n_big)
    const uint32_t* b_in;         // (B)
    const unsigned char* limbs;   // (npad, n_big * l) int8: row 4 o + t = limb t of key column o
    int n_big, n, l, log2_beta, npad;
    long long B;
    uint32_t* a_out;              // (B, n)
    uint32_t* b_out;              // (B)
    long long wait_limit;
    int* status;
    // packing epilogue (pack_T > 0): row s*T + t adds -X^t V into RLWE s of
    // pack_out (S, 2, pack_N); limb row 4 o + t with o = poly * N + coefficient
    int pack_T, pack_N;
    uint32_t* pack_out;
    // 64-bit torus words (the pointers above then address uint64 words and
    // the limb matrix has 8 rows per key column)
    bool w64;
    // the call may allocate stream-ordered scratch (the digit matrix the
    // pipelined kernel reads by TMA); false: digits computed in the kernel
    bool allow_alloc;
};
int smem_attr_once(const void* kern, size_t smem);
size_t ks_tc_smem_bytes(int l);
int ks_tc_columns();
int launch_ks_tc(const KsTcArgs& args, cudaStream_t stream);
int build_packing_limbs(const uint32_t* ksp, int n_dim, int l, int N, int8_t* limbs, cudaStream_t stream);
int build_limbs64(const unsigned long long* key, long long K, int cols, int npad, int8_t* limbs, cudaStream_t stream);

}  // namespace tfhe
