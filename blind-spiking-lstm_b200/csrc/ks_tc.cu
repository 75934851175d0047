// LWE key switching on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// key_switch_LWE (schemas/LWE_jax.py:97-117) is the integer contraction
//   a'[o] = sum_k d[k] K[k][o],   b' = b + sum_k d[k] K[k][n],   k = i*l + j
// of the gadget digits d (|d| <= 2^(log2_beta-1) <= 64, int8) of the input
// mask with the key.  Every 32-bit key word is split into four signed 8-bit
// limbs, K = sum_t limb_t 2^(8t) mod 2^32, so the contraction is four int8 x
// int8 -> int32 GEMMs; their int32 sums cannot overflow (checked by the
// launcher) and are recombined modulo 2^32 in the epilogue: bit-exact with
// the integer key switch.
//
// Tile: 128 ciphertexts x 256 limb columns (64 outputs x 4 limbs) per CTA,
// K in stages of 32 input coefficients (32*l digits).  Operands are staged
// in shared memory in the canonical K-major no-swizzle layout (8-row x
// 16-byte core matrices), two stages in flight; one thread issues
// tcgen05.mma.kind::i8 (M=128, N=256, K=32) into a TMEM accumulator and
// commits to an mbarrier per stage; the epilogue reads TMEM with tcgen05.ld.
// Every mbarrier wait is bounded: on timeout the kernel records
// TFHE_STATUS_WAIT_TIMEOUT and still releases its TMEM.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <stdint.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <set>
#include <utility>

#include "tfhe_b200.h"
#include "tfhe_dispatch.h"
#include "tfhe_internal.cuh"

namespace tfhe {

namespace {

constexpr int KTC_M = 128;          // ciphertexts per CTA (TMEM lanes)
constexpr int KTC_N = 256;          // limb columns per CTA (TMEM columns)
constexpr int KTC_COEF = 32;        // input coefficients per stage
constexpr int KTC_THREADS = 256;

__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

// shared-memory matrix descriptor: K-major, no swizzle; lbo = byte distance
// between the two 16-byte K chunks of one MMA, sbo = between 8-row groups
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    const uint32_t lo = ((saddr >> 4) & 0x3FFFu) | (((lbo >> 4) & 0x3FFFu) << 16);
    const uint32_t hi = ((sbo >> 4) & 0x3FFFu) | (1u << 14);     // descriptor version 1, layout 0
    return ((uint64_t)hi << 32) | lo;
}

// K-major descriptor of a tile written by TMA with 32-byte swizzling: rows of
// 32 bytes (one MMA's K), 8-row atoms 256 bytes apart; the leading byte
// offset is unused for swizzled K-major layouts; layout type 6 = 32B swizzle
__device__ __forceinline__ uint64_t smem_desc_sw32(uint32_t saddr) {
    const uint32_t lo = ((saddr >> 4) & 0x3FFFu) | (1u << 16);
    const uint32_t hi = ((256u >> 4) & 0x3FFFu) | (1u << 14) | (6u << 29);
    return ((uint64_t)hi << 32) | lo;
}

// instruction descriptor: D s32, A and B signed 8-bit, both K-major
constexpr uint32_t KTC_IDESC = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(KTC_N >> 3) << 17) |
                               ((uint32_t)(KTC_M >> 4) << 24);

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(tmem_d), "l"(da), "l"(db), "r"(KTC_IDESC), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&r)[8]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// gadget digit of a centred 64-bit value: rne(x / 2^sh), *rem = x - d 2^sh
// (the reference's decomposition, schemas/polynomial_jax.py:90-111, on the
// exact integer)
__device__ __forceinline__ long long rne_shift64(long long x, int sh, long long* rem) {
    long long d = x >> sh;
    const unsigned long long low = (unsigned long long)x & ((1ULL << sh) - 1ULL);
    const unsigned long long half = 1ULL << (sh - 1);
    if (low > half || (low == half && (d & 1))) {
        d += 1;
        *rem = (long long)(low - (1ULL << sh));
    } else {
        *rem = (long long)low;
    }
    return d;
}

// W64: 64-bit torus words (q = 2^64): eight 8-bit limbs per key word, digits
// from the exact integer, outputs recombined modulo 2^64
template <int L, bool PACK, bool W64>
__global__ void __launch_bounds__(KTC_THREADS, 1) ks_tc_kernel(KsTcArgs a) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ uint32_t tmem_base_slot;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    constexpr int l = L;
    constexpr int chunks = 2 * l;                        // 16-byte K chunks per row per stage
    const uint32_t a_bytes = KTC_M * chunks * 16;    // one stage of A
    const uint32_t b_bytes = KTC_N * chunks * 16;    // one stage of B
    unsigned char* bufA[2] = {smem_raw, smem_raw + a_bytes + b_bytes};
    unsigned char* bufB[2] = {smem_raw + a_bytes, smem_raw + 2 * a_bytes + b_bytes};
    const uint32_t sbo = (uint32_t)chunks * 128;     // 8 rows x 16 bytes per core matrix
    const long long row0 = (long long)blockIdx.y * KTC_M;
    const int col0 = blockIdx.x * KTC_N;             // limb column (= 4 * output)
    const int stages = a.n_big / KTC_COEF;
    const long long kstride = (long long)a.n_big * l;   // bytes per key-limb row

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_addr(&tmem_base_slot)),
                     "r"((uint32_t)KTC_N));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_fence_init();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base_slot;

    const double inv_q = ldexp(1.0, -32);
    const double beta = ldexp(1.0, a.log2_beta);
    bool ok = true;

    for (int s = 0; s < stages; ++s) {
        const int buf = s & 1;
        if (s >= 2)   // the MMAs of stage s - 2 have finished reading this buffer
            ok &= mbar_wait_bounded(&bars[buf], (uint32_t)(((s - 2) >> 1) & 1), a.wait_limit, a.status);
        // A: thread -> (row, half); 16 coefficients -> 16 l digits = l chunks
        {
            const int r = tid & (KTC_M - 1), half = tid >> 7;
            const long long row = row0 + r;
            const int i0 = s * KTC_COEF + half * 16;
            int8_t dig[16 * L];
            if (W64 && row < a.B) {
                const uint4* src = reinterpret_cast<const uint4*>(
                    reinterpret_cast<const unsigned long long*>(a.a_in) + row * a.n_big + i0);
#pragma unroll
                for (int q4 = 0; q4 < 8; ++q4) {
                    const uint4 v = src[q4];
                    const unsigned long long w[2] = {((unsigned long long)v.y << 32) | v.x,
                                                     ((unsigned long long)v.w << 32) | v.z};
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        long long x = (long long)w[e];
#pragma unroll
                        for (int j = 0; j < l; ++j) {
                            long long rem;
                            dig[(q4 * 2 + e) * l + j] = (int8_t)rne_shift64(x, 64 - (j + 1) * a.log2_beta, &rem);
                            x = rem;
                        }
                    }
                }
            } else if (row < a.B) {
                const uint4* src = reinterpret_cast<const uint4*>(a.a_in + row * a.n_big + i0);
#pragma unroll
                for (int q4 = 0; q4 < 4; ++q4) {
                    const uint4 v = src[q4];
                    const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        double x = (double)(int32_t)w[e] * inv_q;
#pragma unroll
                        for (int j = 0; j < l; ++j) {
                            const double y = x * beta;
                            const double d = rint(y);
                            x = y - d;
                            dig[(q4 * 4 + e) * l + j] = (int8_t)(int)d;
                        }
                    }
                }
            } else {
#pragma unroll
                for (int t = 0; t < 16 * l; ++t) dig[t] = 0;
            }
            unsigned char* base = bufA[buf] + (r >> 3) * sbo + (r & 7) * 16;
#pragma unroll
            for (int c = 0; c < l; ++c) {
                uint4 v;
                memcpy(&v, dig + c * 16, 16);
                *reinterpret_cast<uint4*>(base + (half * l + c) * 128) = v;
            }
        }
        // B: thread -> one limb row, 2 l chunks
        {
            const int r = tid;
            const unsigned char* src = a.limbs + (long long)(col0 + r) * kstride + (long long)s * KTC_COEF * l;
            unsigned char* base = bufB[buf] + (r >> 3) * sbo + (r & 7) * 16;
#pragma unroll
            for (int c = 0; c < chunks; ++c)
                *reinterpret_cast<uint4*>(base + c * 128) = *reinterpret_cast<const uint4*>(src + c * 16);
        }
        fence_proxy_async_smem();
        tc_fence_before();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t sa = smem_addr(bufA[buf]), sb = smem_addr(bufB[buf]);
            for (int kk = 0; kk < l; ++kk)     // K = 32 bytes = two chunks per MMA
                mma_i8(tmem, smem_desc(sa + kk * 256, 128, sbo), smem_desc(sb + kk * 256, 128, sbo),
                       (s > 0 || kk > 0) ? 1u : 0u);
            mma_commit(&bars[buf]);
        }
    }
    // every issued MMA has completed once the last stage of each buffer has
    for (int s = stages - 2; s < stages; ++s)
        if (s >= 0) ok &= mbar_wait_bounded(&bars[s & 1], (uint32_t)((s >> 1) & 1), a.wait_limit, a.status);
    tc_fence_after();

    // epilogue: warp w reads TMEM lanes 32 (w % 4) ..; warps 0-3 take limb
    // columns 0-127, warps 4-7 columns 128-255
    {
        const int r = 32 * (warp & 3) + lane;
        const long long row = row0 + r;
        const int cbase = (warp >> 2) * (KTC_N / 2);
        for (int c = cbase; c < cbase + KTC_N / 2; c += 8) {
            uint32_t v[8];
            tmem_ld8(tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)c, v);
            tmem_wait_ld();
            if (!ok || row >= a.B) continue;
            if constexpr (W64) {
                typedef unsigned long long u64;
                const int o = (col0 + c) / 8;
                u64 val = 0ULL;
#pragma unroll
                for (int t = 0; t < 8; ++t) val += (u64)(long long)(int32_t)v[t] << (8 * t);
                if constexpr (PACK) {
                    if (o >= 2 * a.pack_N) continue;
                    const long long sq = row / a.pack_T;
                    const int t = (int)(row - sq * a.pack_T);
                    const int poly = o / a.pack_N, cc = o - poly * a.pack_N;
                    int d = cc + t;
                    u64 add = 0ULL - val;                  // -X^t V: negated unless it wraps past X^N
                    if (d >= a.pack_N) {
                        d -= a.pack_N;
                        add = val;
                    }
                    atomicAdd(reinterpret_cast<u64*>(a.pack_out) + (sq * 2 + poly) * (long long)a.pack_N + d, add);
                } else {
                    if (o < a.n) reinterpret_cast<u64*>(a.a_out)[row * a.n + o] = val;
                    else if (o == a.n)
                        reinterpret_cast<u64*>(a.b_out)[row] = reinterpret_cast<const u64*>(a.b_in)[row] + val;
                }
                continue;
            }
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int o = (col0 + c) / 4 + h;
                const uint32_t val = v[4 * h] + (v[4 * h + 1] << 8) + (v[4 * h + 2] << 16) + (v[4 * h + 3] << 24);
                if constexpr (PACK) {
                    if (o >= 2 * a.pack_N) continue;
                    const long long sq = row / a.pack_T;
                    const int t = (int)(row - sq * a.pack_T);
                    const int poly = o / a.pack_N, cc = o - poly * a.pack_N;
                    int d = cc + t;
                    uint32_t add = 0u - val;               // -X^t V: negated unless it wraps past X^N
                    if (d >= a.pack_N) {
                        d -= a.pack_N;
                        add = val;
                    }
                    atomicAdd(a.pack_out + (sq * 2 + poly) * (long long)a.pack_N + d, add);
                } else {
                    if (o < a.n) a.a_out[row * a.n + o] = val;
                    else if (o == a.n) a.b_out[row] = a.b_in[row] + val;
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)KTC_N));
}

// ============================================================================
// Pipelined form: operands fed by the Tensor Memory Accelerator.
//
// The limb key tile (B) of every stage arrives by 2D TMA copies (one 32-byte
// K slice x 256 limb rows per copy with 32-byte swizzling, or one 16-byte
// chunk unswizzled; each CTA fetches its own tiles, through a tensor map over
// this GPU's memory only) into a ring of stages; the digits (A) either arrive the
// same way from a digit matrix made once per call (tc_digits_kernel) or are
// computed by 8 producer warps into the ring.  One thread issues the copies,
// one thread the MMAs; full / empty mbarriers per stage pass the ring between
// them, so loads of stage s + 1 .. s + S - 1 overlap the MMAs of stage s.
// Shared layout per stage and operand: with swizzling, [slice][row][32 B]
// (one 32-byte K slice of all rows, 8-row atoms of 256 bytes, the descriptor's
// 32-byte swizzle mode); without, and for digits the producers write,
// [chunk][row][16 B], the K-major no-swizzle canonical layout with leading
// byte offset rows * 16 and stride byte offset 128.
// ============================================================================
constexpr int KT2_THREADS = 384;               // warp 0: copies, warp 1: MMAs, warps 4-11: digits + epilogue
constexpr uint32_t KT2_SMEM_BUDGET = 200 * 1024;

__host__ __device__ constexpr uint32_t kt2_stage_bytes(int l) { return (uint32_t)(KTC_M + KTC_N) * 32u * l; }
__host__ __device__ constexpr int kt2_stages(int l) {
    return (int)(KT2_SMEM_BUDGET / kt2_stage_bytes(l)) > 4 ? 4 : (int)(KT2_SMEM_BUDGET / kt2_stage_bytes(l));
}

__device__ __forceinline__ void mbar_arrive_one(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// 2D tile copy global -> this CTA's shared memory (x: byte offset along K, a
// multiple of 16; y: row), completing its bytes on `bar`
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
            "r"(smem_addr(dst)),
        "l"(map), "r"(x), "r"(y), "r"(smem_addr(bar))
        : "memory");
}

// the gadget digits of one input word, as the one-stage kernel computes them
template <int L, bool W64>
__device__ __forceinline__ void word_digits(const void* a_in, long long idx, int log2_beta, int8_t* out) {
    if constexpr (W64) {
        long long x = (long long)reinterpret_cast<const unsigned long long*>(a_in)[idx];
#pragma unroll
        for (int j = 0; j < L; ++j) {
            long long rem;
            out[j] = (int8_t)rne_shift64(x, 64 - (j + 1) * log2_beta, &rem);
            x = rem;
        }
    } else {
        double x = (double)(int32_t)reinterpret_cast<const uint32_t*>(a_in)[idx] * ldexp(1.0, -32);
        const double beta = ldexp(1.0, log2_beta);
#pragma unroll
        for (int j = 0; j < L; ++j) {
            const double y = x * beta;
            const double d = rint(y);
            x = y - d;
            out[j] = (int8_t)(int)d;
        }
    }
}

// digit matrix (B, n_big l) int8, row-major: column i l + j = digit j of
// a_in[row][i] (the A operand of the pipelined kernel)
template <int L, bool W64>
__global__ void __launch_bounds__(256) tc_digits_kernel(const void* a_in, long long B, int n_big, int log2_beta,
                                                        int8_t* __restrict__ out) {
    const long long total = B * (long long)n_big;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        int8_t d[L];
        word_digits<L, W64>(a_in, idx, log2_beta, d);
#pragma unroll
        for (int j = 0; j < L; ++j) out[idx * L + j] = d[j];
    }
}

// 16 consecutive input words of one row -> their 16 L digits (the A staging
// of the one-stage kernel): 16-byte loads, 16-word aligned
template <int L, bool W64>
__device__ __forceinline__ void digits16(const void* a_in, long long off, int log2_beta, int8_t* dig) {
    if constexpr (W64) {
        const uint4* src = reinterpret_cast<const uint4*>(reinterpret_cast<const unsigned long long*>(a_in) + off);
#pragma unroll
        for (int q4 = 0; q4 < 8; ++q4) {
            const uint4 v = src[q4];
            const unsigned long long w[2] = {((unsigned long long)v.y << 32) | v.x, ((unsigned long long)v.w << 32) | v.z};
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                long long x = (long long)w[e];
#pragma unroll
                for (int j = 0; j < L; ++j) {
                    long long rem;
                    dig[(q4 * 2 + e) * L + j] = (int8_t)rne_shift64(x, 64 - (j + 1) * log2_beta, &rem);
                    x = rem;
                }
            }
        }
    } else {
        const uint4* src = reinterpret_cast<const uint4*>(reinterpret_cast<const uint32_t*>(a_in) + off);
        const double inv_q = ldexp(1.0, -32);
        const double beta = ldexp(1.0, log2_beta);
#pragma unroll
        for (int q4 = 0; q4 < 4; ++q4) {
            const uint4 v = src[q4];
            const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                double x = (double)(int32_t)w[e] * inv_q;
#pragma unroll
                for (int j = 0; j < L; ++j) {
                    const double y = x * beta;
                    const double d = rint(y);
                    x = y - d;
                    dig[(q4 * 4 + e) * L + j] = (int8_t)(int)d;
                }
            }
        }
    }
}

// the outputs of 8 accumulator columns c .. c + 7 of one row (the one-stage
// kernel's epilogue): limbs recombined modulo 2^32 / 2^64, then stored, or
// for packing added as -X^t V into the sequence's RLWE
template <bool PACK, bool W64>
__device__ __forceinline__ void store_cols(const KsTcArgs& a, long long row, int colabs, const uint32_t (&v)[8]) {
    if constexpr (W64) {
        typedef unsigned long long u64;
        const int o = colabs / 8;
        u64 val = 0ULL;
#pragma unroll
        for (int t = 0; t < 8; ++t) val += (u64)(long long)(int32_t)v[t] << (8 * t);
        if constexpr (PACK) {
            if (o >= 2 * a.pack_N) return;
            const long long sq = row / a.pack_T;
            const int t = (int)(row - sq * a.pack_T);
            const int poly = o / a.pack_N, cc = o - poly * a.pack_N;
            int d = cc + t;
            u64 add = 0ULL - val;
            if (d >= a.pack_N) {
                d -= a.pack_N;
                add = val;
            }
            atomicAdd(reinterpret_cast<u64*>(a.pack_out) + (sq * 2 + poly) * (long long)a.pack_N + d, add);
        } else {
            if (o < a.n) reinterpret_cast<u64*>(a.a_out)[row * a.n + o] = val;
            else if (o == a.n)
                reinterpret_cast<u64*>(a.b_out)[row] = reinterpret_cast<const u64*>(a.b_in)[row] + val;
        }
    } else {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int o = colabs / 4 + h;
            const uint32_t val = v[4 * h] + (v[4 * h + 1] << 8) + (v[4 * h + 2] << 16) + (v[4 * h + 3] << 24);
            if constexpr (PACK) {
                if (o >= 2 * a.pack_N) continue;
                const long long sq = row / a.pack_T;
                const int t = (int)(row - sq * a.pack_T);
                const int poly = o / a.pack_N, cc = o - poly * a.pack_N;
                int d = cc + t;
                uint32_t add = 0u - val;
                if (d >= a.pack_N) {
                    d -= a.pack_N;
                    add = val;
                }
                atomicAdd(a.pack_out + (sq * 2 + poly) * (long long)a.pack_N + d, add);
            } else {
                if (o < a.n) a.a_out[row * a.n + o] = val;
                else if (o == a.n) a.b_out[row] = a.b_in[row] + val;
            }
        }
    }
}

// SW: TMA copies of 32-byte K slices with 32-byte swizzling (one copy per
// MMA K step, whole 32-byte sectors) instead of 16-byte chunks
template <int L, bool PACK, bool W64, bool A_TMA, bool SW>
__global__ void __launch_bounds__(KT2_THREADS, 1)
    ks_tc2_kernel(const KsTcArgs a, const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                  int rows_fast) {
    constexpr int S = kt2_stages(L);
    constexpr int CH = 2 * L;                              // 16-byte K chunks per stage
    constexpr uint32_t A_BYTES = KTC_M * CH * 16;
    constexpr uint32_t B_BYTES = KTC_N * CH * 16;
    static_assert(S >= 2, "at least two stages in the ring");
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full[S];
    __shared__ __align__(8) uint64_t empty[S];
    __shared__ __align__(8) uint64_t done;
    __shared__ uint32_t tmem_slot;
    __shared__ int fail;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const long long row0 = (long long)(rows_fast ? blockIdx.x : blockIdx.y) * KTC_M;
    const int col0 = (int)(rows_fast ? blockIdx.y : blockIdx.x) * KTC_N;
    const int stages = a.n_big / KTC_COEF;
    volatile int* vfail = &fail;
    // a stage's copies and MMAs take microseconds: a far shorter bound than
    // the caller's keeps a faulty launch from holding the GPU for long
    const long long wlim = a.wait_limit < 200000000LL ? a.wait_limit : 200000000LL;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_slot)),
                     "r"((uint32_t)KTC_N));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (tid == 0) {
        for (int i = 0; i < S; ++i) {
            mbar_init(&full[i], A_TMA ? 1u : 1u + 256u);
            mbar_init(&empty[i], 1);
        }
        mbar_init(&done, 1);
        fail = 0;
        mbar_fence_init();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            // copies: B (and A) of stage s into slot s % S once the MMAs of
            // stage s - S have released it
            int issued = 0;
            for (int s = 0; s < stages && !*vfail; ++s) {
                const int slot = s % S;
                if (s >= S && !mbar_wait_bounded(&empty[slot], (uint32_t)(((s / S) + 1) & 1), wlim, a.status)) {
                    *vfail = 1;
                    break;
                }
                unsigned char* st = smem_raw + (size_t)slot * (A_BYTES + B_BYTES);
                mbar_arrive_expect_tx(&full[slot], B_BYTES + (A_TMA ? A_BYTES : 0u));
                const int x0 = s * KTC_COEF * L;
                if constexpr (SW) {
#pragma unroll 1
                    for (int kk = 0; kk < L; ++kk) {
                        tma_load_2d(st + A_BYTES + kk * KTC_N * 32, &tmB, x0 + kk * 32, col0, &full[slot]);
                        if constexpr (A_TMA)
                            tma_load_2d(st + kk * KTC_M * 32, &tmA, x0 + kk * 32, (int)row0, &full[slot]);
                    }
                } else {
#pragma unroll 1
                    for (int c = 0; c < CH; ++c) {
                        tma_load_2d(st + A_BYTES + c * KTC_N * 16, &tmB, x0 + c * 16, col0, &full[slot]);
                        if constexpr (A_TMA)
                            tma_load_2d(st + c * KTC_M * 16, &tmA, x0 + c * 16, (int)row0, &full[slot]);
                    }
                }
                issued = s + 1;
            }
            // this thread's copies still in flight land before the CTA ends
            for (int s = issued > S ? issued - S : 0; s < issued; ++s)
                if (!mbar_wait_bounded(&full[s % S], (uint32_t)((s / S) & 1), wlim, a.status)) *vfail = 1;
        }
    } else if (warp == 1) {
        if (lane == 0) {
            for (int s = 0; s < stages && !*vfail; ++s) {
                const int slot = s % S;
                if (!mbar_wait_bounded(&full[slot], (uint32_t)((s / S) & 1), wlim, a.status)) {
                    *vfail = 1;
                    break;
                }
                tc_fence_after();
                const uint32_t sa = smem_addr(smem_raw + (size_t)slot * (A_BYTES + B_BYTES));
                const uint32_t sb = sa + A_BYTES;
#pragma unroll
                for (int kk = 0; kk < L; ++kk) {   // K = 32 bytes = chunks 2 kk, 2 kk + 1
                    const uint64_t da = (SW && A_TMA) ? smem_desc_sw32(sa + kk * KTC_M * 32)
                                                      : smem_desc(sa + 2 * kk * KTC_M * 16, KTC_M * 16, 128);
                    const uint64_t db = SW ? smem_desc_sw32(sb + kk * KTC_N * 32)
                                           : smem_desc(sb + 2 * kk * KTC_N * 16, KTC_N * 16, 128);
                    mma_i8(tmem, da, db, (s > 0 || kk > 0) ? 1u : 0u);
                }
                mma_commit(&empty[slot]);
            }
            mma_commit(&done);              // arrives once every MMA issued above has completed
        }
    } else if (warp >= 4) {
        if constexpr (!A_TMA) {
            // digit producers: thread -> (row, half of the stage's 32 coefficients)
            const int p = tid - 128, r = p & (KTC_M - 1), half = p >> 7;
            const long long row = row0 + r;
            for (int s = 0; s < stages && !*vfail; ++s) {
                const int slot = s % S;
                if (s >= S && !mbar_wait_bounded(&empty[slot], (uint32_t)(((s / S) + 1) & 1), wlim, a.status)) {
                    *vfail = 1;
                    break;
                }
                int8_t dig[16 * L];
                if (row < a.B) {
                    digits16<L, W64>(a.a_in, row * a.n_big + s * KTC_COEF + half * 16, a.log2_beta, dig);
                } else {
#pragma unroll
                    for (int t = 0; t < 16 * L; ++t) dig[t] = 0;
                }
                unsigned char* base = smem_raw + (size_t)slot * (A_BYTES + B_BYTES) + r * 16;
#pragma unroll
                for (int c = 0; c < L; ++c) {
                    uint4 v;
                    memcpy(&v, dig + c * 16, 16);
                    *reinterpret_cast<uint4*>(base + (half * L + c) * KTC_M * 16) = v;
                }
                fence_proxy_async_smem();
                mbar_arrive_one(&full[slot]);
            }
        }
    }
    if (!mbar_wait_bounded(&done, 0, wlim, a.status)) *vfail = 1;
    tc_fence_after();
    __syncthreads();
    const bool ok = fail == 0;

    // epilogue: warp w reads TMEM lanes 32 (w % 4) ..; warps 4-7 take limb
    // columns 0-127, warps 8-11 columns 128-255
    if (warp >= 4) {
        const int wq = warp & 3;
        const long long row = row0 + 32 * wq + lane;
        const int cbase = ((warp - 4) >> 2) * (KTC_N / 2);
        for (int c = cbase; c < cbase + KTC_N / 2; c += 8) {
            uint32_t v[8];
            tmem_ld8(tmem + ((uint32_t)(32 * wq) << 16) + (uint32_t)c, v);
            tmem_wait_ld();
            if (!ok || row >= a.B) continue;
            store_cols<PACK, W64>(a, row, col0 + c, v);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)KTC_N));
}

}  // namespace

size_t ks_tc_smem_bytes(int l) { return (size_t)2 * (KTC_M + KTC_N) * 2 * l * 16; }

int ks_tc_columns() { return KTC_N; }

// the dynamic shared-memory attribute is set once per kernel and device, so
// later launches make no attribute calls (and can be captured in a graph)
static std::mutex g_tc_attr_mu;
static std::set<std::pair<int, const void*>> g_tc_attr_done;

static int tc_set_smem_once(const void* kern, size_t smem) {
    int dev = 0;
    const cudaError_t ge = cudaGetDevice(&dev);
    if (ge != cudaSuccess) return check_cuda(ge, "cudaGetDevice");
    std::lock_guard<std::mutex> lk(g_tc_attr_mu);
    if (g_tc_attr_done.count({dev, kern})) return TFHE_OK;
    const cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return check_cuda(e, "tensor-core contraction attribute");
    g_tc_attr_done.insert({dev, kern});
    return TFHE_OK;
}

template <int L, bool PACK, bool W64>
static int launch_l(const KsTcArgs& args, cudaStream_t stream) {
    const size_t smem = ks_tc_smem_bytes(L);
    const int rc = tc_set_smem_once((const void*)ks_tc_kernel<L, PACK, W64>, smem);
    if (rc != TFHE_OK) return rc;
    const dim3 grid((unsigned)(args.npad / KTC_N), (unsigned)((args.B + KTC_M - 1) / KTC_M));
    count_launch();
    ks_tc_kernel<L, PACK, W64><<<grid, KTC_THREADS, smem, stream>>>(args);
    return check_cuda(cudaGetLastError(), "tensor-core contraction launch");
}

// cuTensorMapEncodeTiled from the driver (no link against libcuda)
static PFN_cuTensorMapEncodeTiled_v12000 tma_encoder() {
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

// (rows, K) int8 matrix, row-major with K bytes per row; boxes of one 16-byte
// K chunk x box_rows rows; rows past the end read as zero
static int make_chunk_map(CUtensorMap* m, const void* base, long long K, long long rows, int box_rows, bool sw) {
    const PFN_cuTensorMapEncodeTiled_v12000 enc = tma_encoder();
    if (!enc) return fail(TFHE_ERR_INTERNAL, "tensor-core contraction: cuTensorMapEncodeTiled unavailable");
    if ((reinterpret_cast<uintptr_t>(base) & 15) || K % 16)
        return fail(TFHE_ERR_INVALID_ARGUMENT, "tensor-core contraction: operand not 16-byte aligned");
    const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)K};
    const cuuint32_t box[2] = {sw ? 32u : 16u, (cuuint32_t)box_rows};
    const cuuint32_t es[2] = {1u, 1u};
    const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void*>(base), dims, strides, box, es,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, sw ? CU_TENSOR_MAP_SWIZZLE_32B : CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? TFHE_OK : fail(TFHE_ERR_INTERNAL, "tensor-core contraction: tensor map encoding failed");
}

// TFHE_B200_TC_SW=0: 16-byte chunk copies without swizzling (for comparison)
static bool tc_swizzle() {
    static const bool on = [] {
        const char* env = getenv("TFHE_B200_TC_SW");
        return !(env && env[0] == '0');
    }();
    return on;
}

template <int L, bool PACK, bool W64>
static int launch_l2(const KsTcArgs& args, cudaStream_t stream) {
    const long long K = (long long)args.n_big * L;
    const long long rt = (args.B + KTC_M - 1) / KTC_M, ct = args.npad / KTC_N;
    // the larger operand is streamed once: tiles sharing its slice run together
    const bool rows_fast = (long long)args.npad > args.B;
    if ((rows_fast ? ct : rt) > 65535) return fail(TFHE_ERR_INVALID_ARGUMENT, "tensor-core contraction: too many tiles");
    CUtensorMap ta, tb;
    memset(&ta, 0, sizeof(ta));
    const bool sw = tc_swizzle();
    int rc = make_chunk_map(&tb, args.limbs, K, args.npad, KTC_N, sw);
    if (rc != TFHE_OK) return rc;
    int8_t* dig = nullptr;
    if (args.allow_alloc) {
        rc = check_cuda(cudaMallocAsync((void**)&dig, (size_t)(args.B * K), stream), "cudaMallocAsync(digits)");
        if (rc != TFHE_OK) return rc;
        const long long words = args.B * (long long)args.n_big;
        count_launch();
        tc_digits_kernel<L, W64><<<(unsigned)std::min<long long>((words + 255) / 256, 148LL * 16), 256, 0, stream>>>(
            args.a_in, args.B, args.n_big, args.log2_beta, dig);
        rc = check_cuda(cudaGetLastError(), "digit matrix launch");
        if (rc == TFHE_OK) rc = make_chunk_map(&ta, dig, K, args.B, KTC_M, sw);
    }
    if (rc == TFHE_OK) {
        const size_t smem = (size_t)kt2_stages(L) * kt2_stage_bytes(L);
        auto kern = dig ? (sw ? ks_tc2_kernel<L, PACK, W64, true, true> : ks_tc2_kernel<L, PACK, W64, true, false>)
                        : (sw ? ks_tc2_kernel<L, PACK, W64, false, true> : ks_tc2_kernel<L, PACK, W64, false, false>);
        rc = tc_set_smem_once((const void*)kern, smem);
        if (rc == TFHE_OK) {
            const dim3 grid = rows_fast ? dim3((unsigned)rt, (unsigned)ct) : dim3((unsigned)ct, (unsigned)rt);
            count_launch();
            kern<<<grid, KT2_THREADS, smem, stream>>>(args, ta, tb, rows_fast ? 1 : 0);
            rc = check_cuda(cudaGetLastError(), "tensor-core contraction launch");
        }
    }
    if (dig) {
        const int rc2 = check_cuda(cudaFreeAsync(dig, stream), "cudaFreeAsync(digits)");
        if (rc == TFHE_OK) rc = rc2;
    }
    return rc;
}

// TFHE_B200_TC_PIPE=0 selects the one-stage kernel (for comparison)
static bool tc_pipelined() {
    static const bool on = [] {
        const char* env = getenv("TFHE_B200_TC_PIPE");
        return !(env && env[0] == '0');
    }();
    return on;
}

template <bool PACK, bool W64>
static int launch_any(const KsTcArgs& args, cudaStream_t stream) {
    if (tc_pipelined()) {
        switch (args.l) {
            case 1: return launch_l2<1, PACK, W64>(args, stream);
            case 2: return launch_l2<2, PACK, W64>(args, stream);
            case 3: return launch_l2<3, PACK, W64>(args, stream);
            case 4: return launch_l2<4, PACK, W64>(args, stream);
            case 5: return launch_l2<5, PACK, W64>(args, stream);
            case 6: return launch_l2<6, PACK, W64>(args, stream);
            case 7: return launch_l2<7, PACK, W64>(args, stream);
            case 8: return launch_l2<8, PACK, W64>(args, stream);
            default: return fail(TFHE_ERR_INVALID_ARGUMENT, "tensor-core contraction: 1 <= l <= 8");
        }
    }
    switch (args.l) {
        case 1: return launch_l<1, PACK, W64>(args, stream);
        case 2: return launch_l<2, PACK, W64>(args, stream);
        case 3: return launch_l<3, PACK, W64>(args, stream);
        case 4: return launch_l<4, PACK, W64>(args, stream);
        case 5: return launch_l<5, PACK, W64>(args, stream);
        case 6: return launch_l<6, PACK, W64>(args, stream);
        case 7: return launch_l<7, PACK, W64>(args, stream);
        case 8: return launch_l<8, PACK, W64>(args, stream);
        default: return fail(TFHE_ERR_INVALID_ARGUMENT, "tensor-core contraction: 1 <= l <= 8");
    }
}

int launch_ks_tc(const KsTcArgs& args, cudaStream_t stream) {
    if (args.B == 0) return TFHE_OK;
    if (args.npad % KTC_N || args.n_big % KTC_COEF || (args.B + KTC_M - 1) / KTC_M > 65535)
        return fail(TFHE_ERR_INVALID_ARGUMENT, "tensor-core contraction: unsupported shape");
    const int limbs = args.w64 ? 8 : 4;
    if (args.pack_T > 0) {
        if (!args.pack_out || args.npad != limbs * 2 * args.pack_N)
            return fail(TFHE_ERR_INVALID_ARGUMENT, "tensor-core packing: bad arguments");
        return args.w64 ? launch_any<true, true>(args, stream) : launch_any<true, false>(args, stream);
    }
    return args.w64 ? launch_any<false, true>(args, stream) : launch_any<false, false>(args, stream);
}

// 8-bit limb rows of a 64-bit key matrix (K rows, cols columns, row-major):
// row 8 o + t, column k holds limb t of key[k][o] (signed, sum_t limb_t 2^(8t)
// = key[k][o] mod 2^64); rows 8 cols .. npad - 1 are zero
__global__ void limbs64_kernel(const unsigned long long* __restrict__ key, long long K, int cols, int npad,
                               int8_t* __restrict__ limbs) {
    const long long total = (long long)npad / 8 * K;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const long long o = idx / K;
        const long long k = idx - o * K;
        unsigned long long w = o < cols ? key[k * cols + o] : 0ULL;
        for (int t = 0; t < 8; ++t) {
            const int lo = (int)((w + 128ULL) & 255ULL) - 128;
            limbs[(o * 8 + t) * K + k] = (int8_t)lo;
            w = (w - (unsigned long long)(long long)lo) >> 8;
        }
    }
}

int build_limbs64(const unsigned long long* key, long long K, int cols, int npad, int8_t* limbs,
                  cudaStream_t stream) {
    const long long total = (long long)npad / 8 * K;
    const int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 32);
    count_launch();
    limbs64_kernel<<<blocks, 256, 0, stream>>>(key, K, cols, npad, limbs);
    return check_cuda(cudaGetLastError(), "64-bit limb launch");
}

// limb rows of a packing key: row 4 o + t, o = poly * N + c, column k = i l + j
// holds limb t of ksp[i][j][poly][c]
__global__ void packing_limbs_kernel(const uint32_t* __restrict__ ksp, int n_dim, int l, int N,
                                     int8_t* __restrict__ limbs) {
    const long long K = (long long)n_dim * l;
    const long long total = 2LL * N * K;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const long long o = idx / K;
        const long long k = idx - o * K;
        const int poly = (int)(o / N), c = (int)(o - (long long)poly * N);
        long long rest = ksp[(k * 2 + poly) * N + c];
        for (int t = 0; t < 4; ++t) {
            const long long lo = ((rest + 128) & 255) - 128;
            limbs[(o * 4 + t) * K + k] = (int8_t)lo;
            rest = (rest - lo) >> 8;
        }
    }
}

int build_packing_limbs(const uint32_t* ksp, int n_dim, int l, int N, int8_t* limbs, cudaStream_t stream) {
    const long long total = 2LL * N * n_dim * l;
    const int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 32);
    count_launch();
    packing_limbs_kernel<<<blocks, 256, 0, stream>>>(ksp, n_dim, l, N, limbs);
    return check_cuda(cudaGetLastError(), "packing limb launch");
}

}  // namespace tfhe
