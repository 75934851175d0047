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
#include <stdint.h>

#include <algorithm>
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

template <bool PACK, bool W64>
static int launch_any(const KsTcArgs& args, cudaStream_t stream) {
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
