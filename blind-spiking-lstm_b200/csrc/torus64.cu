// Operators on the reference's own torus, q = 2^64 (parameters_crypto.py:6:
// q = float(2**64)), for the encrypted Spike-LSTM at the reference's
// parameter set.  The reference holds these values in float64 and rounds;
// here they are uint64 words and every integer step is exact modulo 2^64:
//
//   ks64_kernel             key_switch_LWE (schemas/LWE_jax.py:97-117)
//   indices64_kernel        the rotation indices of multiply_seq_monomial
//                           (cuTFHE/multiply.py:67-79) from 64-bit masks
//   rotate_extract64_kernel rotation by -b~ and many-LUT sample extraction
//                           (schemas/RLWE_jax.py:295-303)
//   linear64_kernel         Linear.__call__ (nn_tfhe/Spike_LSTM.py:48-58)
//   lut_mul_sum64_kernel    prepare_LUT's product summed over the packed
//                           sub-LUTs (nn_tfhe/activation.py:103-106,
//                           nn_tfhe/Spike_LSTM.py:129-132)
//   trace64_kernel          pack_lwe_to_rlwe (schemas/text_jax.py:316-345)
//   pack64_kernel           packing (schemas/text_jax.py:211-239)
//   rotate_add64 / add64 / extract64   rotate_ciphertext, sums, sample_extract
//
// The blind rotation itself is the FP64 kernel of tfhe_mul_bootstrap at
// log2_q = 64 (the reference's own arithmetic at that modulus).
//
// Gadget digits follow the reference's decomposition (schemas/
// polynomial_jax.py:90-111: x = gamma / q, d = round(beta x), x = beta x - d,
// round half to even) evaluated exactly on the integer: d_j = rne(r_{j-1} /
// 2^(64 - j log2 beta)), r_j = r_{j-1} - d_j 2^(64 - j log2 beta), r_0 the
// centred value.
#include <stdint.h>

#include <algorithm>
#include <cstdlib>
#include <string>

#include "tfhe_b200.h"
#include "tfhe_dispatch.h"
#include "tfhe_internal.cuh"

namespace tfhe {
namespace t64 {

typedef unsigned long long u64;

// rne(x / 2^s) for a centred value x, s in [0, 63]; *rem = x - d 2^s
__device__ __host__ __forceinline__ long long rne_shift(long long x, int s, long long* rem) {
    if (s == 0) {
        *rem = 0;
        return x;
    }
    long long d = x >> s;
    const u64 low = (u64)x & ((1ULL << s) - 1ULL);
    const u64 half = 1ULL << (s - 1);
    if (low > half || (low == half && (d & 1))) {
        d += 1;
        *rem = (long long)(low - (1ULL << s));
    } else {
        *rem = (long long)low;
    }
    return d;
}

// ---------------------------------------------------------------- key switch
// a'[o] = sum_{i,j} d_j(a[i]) K[i l + j][o] (mod 2^64), o < n; the body
// column o = n adds to b.  Key rows (n_big l, n + 1), row-major.
constexpr int KS_TB = 64, KS_TO = 64, KS_KC = 4, KS_LMAX = 8;

__global__ void __launch_bounds__(256) ks64_kernel(const u64* __restrict__ a_in, const u64* __restrict__ b_in,
                                                   const u64* __restrict__ key, int n_big, int n, int l,
                                                   int log2_beta, u64* __restrict__ a_out, u64* __restrict__ b_out,
                                                   long long B) {
    __shared__ int dig[KS_TB][KS_KC * KS_LMAX + 1];
    __shared__ __align__(16) u64 kt[KS_KC * KS_LMAX][KS_TO];
    const int tid = threadIdx.x;
    const int ty = tid / 16, tx = tid % 16;
    const long long r0 = (long long)blockIdx.y * KS_TB;
    const int o0 = blockIdx.x * KS_TO;
    const int ld = n + 1;
    u64 acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0ULL;
    for (int i0 = 0; i0 < n_big; i0 += KS_KC) {
        for (int idx = tid; idx < KS_TB * KS_KC; idx += 256) {
            const int ct = idx / KS_KC, c = idx % KS_KC;
            const long long row = r0 + ct;
            const int i = i0 + c;
            long long x = (row < B && i < n_big) ? (long long)a_in[row * n_big + i] : 0LL;
            for (int j = 0; j < l; ++j) {
                long long rem;
                dig[ct][c * l + j] = (int)rne_shift(x, 64 - (j + 1) * log2_beta, &rem);
                x = rem;
            }
        }
        const int rows = KS_KC * l;
        for (int idx = tid; idx < rows * KS_TO; idx += 256) {
            const int r = idx / KS_TO, col = idx % KS_TO;
            const int i = i0 + r / l, j = r % l;
            const int o = o0 + col;
            kt[r][col] = (i < n_big && o <= n) ? key[((long long)i * l + j) * ld + o] : 0ULL;
        }
        __syncthreads();
        for (int r = 0; r < rows; ++r) {
#pragma unroll
            for (int cc = 0; cc < 4; ++cc) {
                const u64 d = (u64)(long long)dig[ty * 4 + cc][r];
#pragma unroll
                for (int e = 0; e < 4; ++e) acc[cc][e] += d * kt[r][tx * 4 + e];
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int cc = 0; cc < 4; ++cc) {
        const long long row = r0 + ty * 4 + cc;
        if (row >= B) continue;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int o = o0 + tx * 4 + e;
            if (o < n) a_out[row * n + o] = acc[cc][e];
            else if (o == n) b_out[row] = b_in[row] + acc[cc][e];
        }
    }
}

// ---------------------------------------------------------------- BR indices
// r[g][m] = rne(2N <a_g, p_m> / (q n_lut)) n_lut mod 2N, p_m the m-th
// binary pattern in meshgrid 'ij' order (cuTFHE/utils.py:5-8)
__global__ void indices64_kernel(const u64* __restrict__ lwe_a, int n, int collapse, int logN, int log2_nlut,
                                 int32_t* __restrict__ out, long long B) {
    const int G = n / collapse, M = 1 << collapse, N2 = 2 << logN;
    const long long total = B * G * (long long)M;
    const int s = 63 - logN + log2_nlut;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const long long k = t / ((long long)G * M);
        const int rem = (int)(t - k * G * M);
        const int g = rem / M, m = rem - g * M;
        const u64* a = lwe_a + k * n + (long long)g * collapse;
        u64 v = 0ULL;
        for (int c = 0; c < collapse; ++c)
            if ((m >> (collapse - 1 - c)) & 1) v += a[c];
        long long r;
        const long long d = rne_shift((long long)v, s, &r);
        long long idx = (d << log2_nlut) % N2;
        if (idx < 0) idx += N2;
        out[t] = (int32_t)idx;
    }
}

// ---------------------------------------------------------------- rotate / extract
// b~ = rne(2N b / (q n_lut)) n_lut; ACC <- X^(-b~) ACC; out_a[al][j] = coefficient
// al - j of the rotated mask (negacyclic), out_b[al] = rotated body[al]
__global__ void rotate_extract64_kernel(const long long* __restrict__ acc, const u64* __restrict__ b, int logN,
                                        int n_lut, int log2_nlut, u64* __restrict__ out_a, u64* __restrict__ out_b,
                                        long long B) {
    const int N = 1 << logN;
    const long long per = (long long)n_lut * N + n_lut;
    const long long total = B * per;
    const int s = 63 - logN + log2_nlut;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const long long k = t / per;
        const int r = (int)(t - k * per);
        long long rm;
        const long long bt = rne_shift((long long)b[k], s, &rm) << log2_nlut;
        const long long* a = acc + k * 2 * N;
        long long e;
        int src;
        u64* dst;
        if (r < n_lut * N) {
            const int al = r / N, j = r - al * N;
            e = (long long)al - j + bt;
            src = 0;
            dst = out_a + k * (long long)n_lut * N + r;
        } else {
            const int al = r - n_lut * N;
            e = (long long)al + bt;
            src = N;
            dst = out_b + k * n_lut + al;
        }
        e %= 2 * N;
        if (e < 0) e += 2 * N;
        const u64 v = e < N ? (u64)a[src + e] : 0ULL - (u64)a[src + e - N];
        *dst = v;
    }
}

// ---------------------------------------------------------------- linear
constexpr int LIN_JT = 4, LIN_NT = 256, CPT_MAX = 16;

__global__ void __launch_bounds__(LIN_NT) linear64_kernel(const int32_t* __restrict__ W,
                                                          const long long* __restrict__ bias, int J,
                                                          const u64* __restrict__ ct, int N, u64* __restrict__ out_a,
                                                          u64* __restrict__ out_b) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    u64* A = reinterpret_cast<u64*>(smem_raw);                   // N
    int32_t* Ws = reinterpret_cast<int32_t*>(A + N);             // LIN_JT * N
    __shared__ u64 red[LIN_JT][LIN_NT / 32];
    const int tid = threadIdx.x;
    const long long s = blockIdx.y;
    const int j0 = blockIdx.x * LIN_JT;
    const u64* a_in = ct + s * 2 * N;
    const u64* b_in = a_in + N;
    for (int i = tid; i < N; i += LIN_NT) A[i] = a_in[i];
    for (int i = tid; i < LIN_JT * N; i += LIN_NT) {
        const int jt = i / N;
        Ws[i] = (j0 + jt < J) ? W[(long long)(j0 + jt) * N + (i - jt * N)] : 0;
    }
    __syncthreads();
    u64 pb[LIN_JT];
#pragma unroll
    for (int jt = 0; jt < LIN_JT; ++jt) pb[jt] = 0ULL;
    for (int m = tid; m < N; m += LIN_NT) {
        const u64 bv = m == 0 ? b_in[0] : 0ULL - b_in[N - m];
#pragma unroll
        for (int jt = 0; jt < LIN_JT; ++jt) pb[jt] += (u64)(long long)Ws[jt * N + m] * bv;
    }
#pragma unroll
    for (int jt = 0; jt < LIN_JT; ++jt) {
        u64 v = pb[jt];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((tid & 31) == 0) red[jt][tid >> 5] = v;
    }
    u64 acc[LIN_JT][CPT_MAX];
    const int cpt = N / LIN_NT > 0 ? N / LIN_NT : 1;
#pragma unroll
    for (int jt = 0; jt < LIN_JT; ++jt)
#pragma unroll
        for (int r = 0; r < CPT_MAX; ++r) acc[jt][r] = 0ULL;
    for (int m = 0; m < N; ++m) {
        int32_t w[LIN_JT];
        bool any = false;
#pragma unroll
        for (int jt = 0; jt < LIN_JT; ++jt) {
            w[jt] = Ws[jt * N + m];
            any |= w[jt] != 0;
        }
        if (!any) continue;                           // uniform across the CTA
#pragma unroll
        for (int r = 0; r < CPT_MAX; ++r) {
            if (r >= cpt) break;
            const int c = tid + LIN_NT * r;
            if (c >= N) break;
            const int idx = c - m;
            const u64 v = idx >= 0 ? A[idx] : 0ULL - A[idx + N];
#pragma unroll
            for (int jt = 0; jt < LIN_JT; ++jt) acc[jt][r] += (u64)(long long)w[jt] * v;
        }
    }
    __syncthreads();
#pragma unroll
    for (int jt = 0; jt < LIN_JT; ++jt) {
        const int j = j0 + jt;
        if (j >= J) break;
        u64* dst = out_a + (s * J + j) * (long long)N;
#pragma unroll
        for (int r = 0; r < CPT_MAX; ++r) {
            if (r >= cpt) break;
            const int c = tid + LIN_NT * r;
            if (c >= N) break;
            if (c == 0) dst[0] = acc[jt][r];
            else dst[N - c] = 0ULL - acc[jt][r];
        }
        if (tid == 0) {
            u64 v = (u64)bias[j];
            for (int w = 0; w < LIN_NT / 32; ++w) v += red[jt][w];
            out_b[s * J + j] = v;
        }
    }
}

// ---------------------------------------------------------------- LUT x RLWE
constexpr int LM_NT = 256;

__global__ void __launch_bounds__(LM_NT) lut_mul_sum64_kernel(const long long* __restrict__ P, int G, int Kp,
                                                              const u64* __restrict__ ct, int N,
                                                              u64* __restrict__ out) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    u64* A = reinterpret_cast<u64*>(smem_raw);              // N
    u64* Bp = A + N;                                         // N
    long long* Ps = reinterpret_cast<long long*>(Bp + N);    // N
    const int tid = threadIdx.x;
    const int k = blockIdx.x;
    const long long s = blockIdx.y;
    const int cpt = N / LM_NT > 0 ? N / LM_NT : 1;
    u64 acc_a[CPT_MAX], acc_b[CPT_MAX];
#pragma unroll
    for (int r = 0; r < CPT_MAX; ++r) acc_a[r] = acc_b[r] = 0ULL;
    for (int g = 0; g < G; ++g) {
        const u64* src = ct + ((s * G + g) * (long long)Kp + k) * 2 * N;
        const long long* lut = P + ((long long)g * Kp + k) * N;
        for (int i = tid; i < N; i += LM_NT) {
            A[i] = src[i];
            Bp[i] = src[N + i];
            Ps[i] = lut[i];
        }
        __syncthreads();
        for (int m = 0; m < N; ++m) {
            const long long w = Ps[m];
            if (w == 0) continue;                     // uniform across the CTA
#pragma unroll
            for (int r = 0; r < CPT_MAX; ++r) {
                if (r >= cpt) break;
                const int c = tid + LM_NT * r;
                if (c >= N) break;
                const int idx = c - m;
                const u64 va = idx >= 0 ? A[idx] : 0ULL - A[idx + N];
                const u64 vb = idx >= 0 ? Bp[idx] : 0ULL - Bp[idx + N];
                acc_a[r] += (u64)w * va;
                acc_b[r] += (u64)w * vb;
            }
        }
        __syncthreads();
    }
    u64* dst = out + (s * Kp + k) * 2 * (long long)N;
#pragma unroll
    for (int r = 0; r < CPT_MAX; ++r) {
        if (r >= cpt) break;
        const int c = tid + LM_NT * r;
        if (c >= N) break;
        dst[c] = acc_a[r];
        dst[N + c] = acc_b[r];
    }
}

// ---------------------------------------------------------------- FFT helpers
template <int LOGH, int s>
__device__ __forceinline__ void fwd(double2* polys, int npoly, const double2* tw, int tid, int nt) {
    if constexpr (s < Plan<LOGH>::NS) {
        stage_all<LOGH, s, false>(polys, npoly, tw, tid, nt);
        __syncthreads();
        fwd<LOGH, s + 1>(polys, npoly, tw, tid, nt);
    }
}

template <int LOGH, int s>
__device__ __forceinline__ void inv(double2* polys, int npoly, const double2* tw, int tid, int nt) {
    if constexpr (s >= 0) {
        stage_all<LOGH, s, true>(polys, npoly, tw, tid, nt);
        __syncthreads();
        inv<LOGH, s - 1>(polys, npoly, tw, tid, nt);
    }
}

constexpr int LIMBS = 4;     // 16-bit signed limbs of a 64-bit key word

// signed 16-bit limb t of a 64-bit word: w = sum_t limb_t 2^(16 t) mod 2^64
__device__ __forceinline__ int limb16(u64 w, int t) {
    int lo = 0;
    for (int i = 0; i <= t; ++i) {
        lo = (int)((w + 0x8000ULL) & 0xFFFFULL) - 0x8000;
        w = (w - (u64)(long long)lo) >> 16;
    }
    return lo;
}

// 64-bit key polynomials (npoly, N) -> the folded Fourier transform of each of
// their four 16-bit limbs: dst (npoly, LIMBS, H), position order
template <int LOGN>
__global__ void __launch_bounds__(256) limb_fft64_kernel(const u64* __restrict__ src, const double2* qt,
                                                         const double2* tw, double2* __restrict__ dst) {
    constexpr int N = 1 << LOGN;
    constexpr int H = N / 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* buf = reinterpret_cast<double2*>(smem_raw);
    const long long pi = blockIdx.x;
    const int t = blockIdx.y;
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int i = tid; i < H; i += nt) {
        const double lo = (double)limb16(src[pi * N + i], t);
        const double hi = (double)limb16(src[pi * N + i + H], t);
        const double2 w = qt[i];
        buf[swz(i)] = make_double2(fma(w.x, lo, w.y * hi), fma(w.y, lo, -w.x * hi));
    }
    __syncthreads();
    fwd<LOGN - 1, 0>(buf, 1, tw, tid, nt);
    for (int p = tid; p < H; p += nt) dst[(pi * LIMBS + t) * H + p] = buf[swz(p)];
}

// ---------------------------------------------------------------- LUT x RLWE by FFT
// The same sums with small LUTs (the step LUTs of the layer hold 0 / +-1):
// each ciphertext word is split into four signed 16-bit limbs, each limb
// polynomial multiplied by the LUT in the folded FP64 Fourier domain and the
// G products summed there; a limb's result is below G N 2^15 2^8 = 2^36 for
// |LUT| <= 2^8, so it rounds to the exact integer, and the limbs recombine
// exactly modulo 2^64.  A CTA whose LUTs exceed 2^8 takes the direct sums of
// lut_mul_sum64_kernel instead (block-uniform), so the result is exact for
// any LUT.  One CTA per (group slot k, sequence s), the two output
// polynomials in turn; shared memory: 9 H complex values.
constexpr int LF_NT = 512;
constexpr long long LF_MAX_LUT = 256;

template <int LOGN>
__global__ void __launch_bounds__(LF_NT) lut_fft64_kernel(const long long* __restrict__ P, int G, int Kp,
                                                          const u64* __restrict__ ct, const double2* qt,
                                                          const double2* tw, u64* __restrict__ out) {
    constexpr int N = 1 << LOGN;
    constexpr int H = N / 2;
    constexpr int LOGH = LOGN - 1;
    constexpr int SL = H >= LF_NT ? H / LF_NT : 1;
    constexpr double inv_h = 1.0 / H;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* work = reinterpret_cast<double2*>(smem_raw);    // 5 H: LUT, 4 limbs
    double2* acc = work + 5 * H;                              // 4 H: limb products summed over g
    __shared__ int big;
    const int tid = threadIdx.x, nt = blockDim.x;
    const int k = blockIdx.x;
    const long long s = blockIdx.y;

    if (tid == 0) big = 0;
    __syncthreads();
    for (int g = 0; g < G; ++g) {
        const long long* lut = P + ((long long)g * Kp + k) * N;
        for (int i = tid; i < N; i += nt)
            if (lut[i] > LF_MAX_LUT || lut[i] < -LF_MAX_LUT) big = 1;
    }
    __syncthreads();
    if (big) {
        // direct negacyclic sums (lut_mul_sum64_kernel's operations)
        u64* A = reinterpret_cast<u64*>(smem_raw);
        u64* Bp = A + N;
        long long* Ps = reinterpret_cast<long long*>(Bp + N);
        constexpr int CPT = N / LF_NT > 0 ? N / LF_NT : 1;
        u64 acc_a[CPT], acc_b[CPT];
#pragma unroll
        for (int r = 0; r < CPT; ++r) acc_a[r] = acc_b[r] = 0ULL;
        for (int g = 0; g < G; ++g) {
            const u64* src = ct + ((s * G + g) * (long long)Kp + k) * 2 * N;
            const long long* lut = P + ((long long)g * Kp + k) * N;
            for (int i = tid; i < N; i += nt) {
                A[i] = src[i];
                Bp[i] = src[N + i];
                Ps[i] = lut[i];
            }
            __syncthreads();
            for (int m = 0; m < N; ++m) {
                const long long w = Ps[m];
                if (w == 0) continue;
#pragma unroll
                for (int r = 0; r < CPT; ++r) {
                    const int c = tid + LF_NT * r;
                    if (c >= N) break;
                    const int idx = c - m;
                    const u64 va = idx >= 0 ? A[idx] : 0ULL - A[idx + N];
                    const u64 vb = idx >= 0 ? Bp[idx] : 0ULL - Bp[idx + N];
                    acc_a[r] += (u64)w * va;
                    acc_b[r] += (u64)w * vb;
                }
            }
            __syncthreads();
        }
        u64* dst = out + (s * Kp + k) * 2 * (long long)N;
#pragma unroll
        for (int r = 0; r < CPT; ++r) {
            const int c = tid + LF_NT * r;
            if (c >= N) break;
            dst[c] = acc_a[r];
            dst[N + c] = acc_b[r];
        }
        return;
    }

    for (int pass = 0; pass < 2; ++pass) {
        for (int g = 0; g < G; ++g) {
            const u64* src = ct + ((s * G + g) * (long long)Kp + k) * 2 * N + pass * N;
            const long long* lut = P + ((long long)g * Kp + k) * N;
            // fold + twist of the LUT and of the four limbs of the polynomial
            for (int i = tid; i < H; i += nt) {
                const double2 w = qt[i];
                {
                    const double lo = (double)lut[i], hi = (double)lut[i + H];
                    work[swz(i)] = make_double2(fma(w.x, lo, w.y * hi), fma(w.y, lo, -w.x * hi));
                }
                const u64 xl = src[i], xh = src[i + H];
#pragma unroll
                for (int t = 0; t < LIMBS; ++t) {
                    const double lo = (double)limb16(xl, t), hi = (double)limb16(xh, t);
                    work[(size_t)(1 + t) * H + swz(i)] = make_double2(fma(w.x, lo, w.y * hi), fma(w.y, lo, -w.x * hi));
                }
            }
            __syncthreads();
            fwd<LOGH, 0>(work, 5, tw, tid, nt);
            for (int p = tid; p < H; p += nt) {
                const double2 f = work[swz(p)];
#pragma unroll
                for (int t = 0; t < LIMBS; ++t) {
                    const double2 v = c_mul(f, work[(size_t)(1 + t) * H + swz(p)]);
                    double2& a = acc[(size_t)t * H + swz(p)];
                    if (g == 0) a = v;
                    else a = make_double2(a.x + v.x, a.y + v.y);
                }
            }
            __syncthreads();
        }
        inv<LOGH, Plan<LOGH>::NS - 1>(acc, LIMBS, tw, tid, nt);
        u64* dst = out + (s * Kp + k) * 2 * (long long)N + pass * N;
#pragma unroll
        for (int sl = 0; sl < SL; ++sl) {
            const int i = tid + sl * nt;
            if (i >= H) continue;
            const double2 w = c_conj(qt[i]);
            u64 lo = 0ULL, hi = 0ULL;
#pragma unroll
            for (int t = 0; t < LIMBS; ++t) {
                const double2 u = c_mul(w, acc[(size_t)t * H + swz(i)]);
                lo += (u64)(long long)rint(u.x * inv_h) << (16 * t);
                hi += (u64)(long long)rint(-u.y * inv_h) << (16 * t);
            }
            dst[i] = lo;
            dst[i + H] = hi;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- trace
struct Trace64Args {
    const u64* lwe_a;          // (R, N)
    const u64* lwe_b;          // (R)
    const double2* key;        // [step][level][2][LIMBS][H], position order
    const double2* qt;
    const double2* tw;
    int log2_beta, l, steps;
    u64* out;                  // (R, 2, N)
};

// pack_lwe_to_rlwe on Z/2^64 for one LWE per CTA:
//   lwe <- rne(lwe / N) (modulus_switch to q/N, text_jax.py:173-187)
//   rlwe = trivial_embedding(lwe) (A[0] = a[0], A[i] = -a[N-i], B[0] = b)
//   for step i, k = 2^(log2 N - i) + 1:
//     (A', B') = automorphism X -> X^k of (A, B)
//     (A_ks, B_ks) = sum_j dec_j(A') * galois_key[i][j], exact: each 16-bit
//                    key limb's FP64 product is an integer below 2^40
//     rlwe += (A_ks, B' + B_ks)
constexpr int TRACE_NT = 512;     // one LWE per CTA (the CTA's shared memory holds its whole trace)

template <int LOGN>
__global__ void __launch_bounds__(TRACE_NT) trace64_kernel(const Trace64Args args) {
    constexpr int N = 1 << LOGN;
    constexpr int H = N / 2;
    constexpr int LOGH = LOGN - 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* dig = reinterpret_cast<double2*>(smem_raw);        // l * H
    double2* res = dig + (size_t)args.l * H;                     // 2 * H
    u64* accA = reinterpret_cast<u64*>(res + 2 * H);             // N
    u64* accB = accA + N;                                        // N
    u64* permA = accB + N;                                       // N
    u64* permB = permA + N;                                      // N
    const int tid = threadIdx.x, nt = blockDim.x;
    const long long r = blockIdx.x;
    constexpr double inv_h = 1.0 / H;

    const u64* a = args.lwe_a + r * N;
    for (int i = tid; i < N; i += nt) {
        long long rm;
        const u64 ms = (u64)rne_shift((long long)a[i == 0 ? 0 : N - i], LOGN, &rm);
        accA[i] = i == 0 ? ms : 0ULL - ms;
        accB[i] = i == 0 ? (u64)rne_shift((long long)args.lwe_b[r], LOGN, &rm) : 0ULL;
    }
    __syncthreads();

    for (int st = 0; st < args.steps; ++st) {
        const int k = (1 << (args.steps - st)) + 1;
        for (int j = tid; j < N; j += nt) {
            const int dst = (int)(((long long)j * k) % (2 * N));
            const int t = dst % N;
            permA[t] = dst >= N ? 0ULL - accA[j] : accA[j];
            permB[t] = dst >= N ? 0ULL - accB[j] : accB[j];
        }
        __syncthreads();
        // gadget digits of A', fold + twist
        for (int i = tid; i < H; i += nt) {
            long long xl = (long long)permA[i], xh = (long long)permA[i + H];
            const double2 w = args.qt[i];
            for (int lvl = 0; lvl < args.l; ++lvl) {
                const int sh = 64 - (lvl + 1) * args.log2_beta;
                long long rl, rh;
                const double dl = (double)rne_shift(xl, sh, &rl);
                const double dh = (double)rne_shift(xh, sh, &rh);
                xl = rl;
                xh = rh;
                dig[(size_t)lvl * H + swz(i)] = make_double2(fma(w.x, dl, w.y * dh), fma(w.y, dl, -w.x * dh));
            }
        }
        __syncthreads();
        fwd<LOGH, 0>(dig, args.l, args.tw, tid, nt);
        const double2* key = args.key + (size_t)st * args.l * 2 * LIMBS * H;
        u64 ksA[CPT_MAX], ksB[CPT_MAX];        // coefficient c = i and i + H of thread i
        for (int limb = 0; limb < LIMBS; ++limb) {
            for (int p = tid; p < H; p += nt) {
                double2 o0 = make_double2(0.0, 0.0), o1 = make_double2(0.0, 0.0);
                for (int lvl = 0; lvl < args.l; ++lvl) {
                    const double2 d = dig[(size_t)lvl * H + swz(p)];
                    c_mac(o0, d, key[(((size_t)lvl * 2 + 0) * LIMBS + limb) * H + p]);
                    c_mac(o1, d, key[(((size_t)lvl * 2 + 1) * LIMBS + limb) * H + p]);
                }
                res[swz(p)] = o0;
                res[H + swz(p)] = o1;
            }
            __syncthreads();
            inv<LOGH, Plan<LOGH>::NS - 1>(res, 2, args.tw, tid, nt);
            int slot = 0;
            for (int i = tid; i < H; i += nt, ++slot) {
                const double2 w = c_conj(args.qt[i]);
                const double2 ua = c_mul(w, res[swz(i)]);
                const double2 ub = c_mul(w, res[H + swz(i)]);
                const int sh = 16 * limb;
                const u64 a0 = (u64)(long long)rint(ua.x * inv_h) << sh;
                const u64 a1 = (u64)(long long)rint(-ua.y * inv_h) << sh;
                const u64 b0 = (u64)(long long)rint(ub.x * inv_h) << sh;
                const u64 b1 = (u64)(long long)rint(-ub.y * inv_h) << sh;
                if (limb == 0) {
                    ksA[2 * slot] = a0;
                    ksA[2 * slot + 1] = a1;
                    ksB[2 * slot] = b0;
                    ksB[2 * slot + 1] = b1;
                } else {
                    ksA[2 * slot] += a0;
                    ksA[2 * slot + 1] += a1;
                    ksB[2 * slot] += b0;
                    ksB[2 * slot + 1] += b1;
                }
            }
            __syncthreads();
        }
        int slot = 0;
        for (int i = tid; i < H; i += nt, ++slot) {
            accA[i] += ksA[2 * slot];
            accA[i + H] += ksA[2 * slot + 1];
            accB[i] += permB[i] + ksB[2 * slot];
            accB[i + H] += permB[i + H] + ksB[2 * slot + 1];
        }
        __syncthreads();
    }
    u64* dst = args.out + r * 2 * N;
    for (int i = tid; i < N; i += nt) {
        dst[i] = accA[i];
        dst[N + i] = accB[i];
    }
}

// The same trace with the four limbs' products transformed back together:
// the pointwise stage writes all 2 x LIMBS output spectra, one inverse pass
// runs over the eight polynomials (every thread busy, a quarter of the
// barriers), and the accumulators live in the registers of the threads that
// own their coefficients (thread i: coefficients i and i + H of its slots),
// the permuted copies passing through the spectra's space.  Every value is
// computed by trace64_kernel's operations in the same order, so the outputs
// are identical.  Shared memory: (l + 2 LIMBS) H complex values.
template <int LOGN>
__global__ void __launch_bounds__(TRACE_NT) trace64_fused_kernel(const Trace64Args args) {
    constexpr int N = 1 << LOGN;
    constexpr int H = N / 2;
    constexpr int LOGH = LOGN - 1;
    constexpr int SL = H >= TRACE_NT ? H / TRACE_NT : 1;     // coefficient slots per thread
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* dig = reinterpret_cast<double2*>(smem_raw);        // l * H
    double2* res = dig + (size_t)args.l * H;                     // 2 LIMBS * H
    u64* permA = reinterpret_cast<u64*>(res);                    // N (in res, before the products)
    u64* permB = permA + N;                                      // N
    const int tid = threadIdx.x, nt = blockDim.x;
    const long long r = blockIdx.x;
    constexpr double inv_h = 1.0 / H;

    u64 accA[SL][2], accB[SL][2];
    const u64* a = args.lwe_a + r * N;
#pragma unroll
    for (int sl = 0; sl < SL; ++sl) {
        const int i = tid + sl * nt;
#pragma unroll
        for (int hf = 0; hf < 2; ++hf) {
            accA[sl][hf] = accB[sl][hf] = 0ULL;
            if (i >= H) continue;
            const int c = i + hf * H;
            long long rm;
            const u64 ms = (u64)rne_shift((long long)a[c == 0 ? 0 : N - c], LOGN, &rm);
            accA[sl][hf] = c == 0 ? ms : 0ULL - ms;
            accB[sl][hf] = c == 0 ? (u64)rne_shift((long long)args.lwe_b[r], LOGN, &rm) : 0ULL;
        }
    }

    for (int st = 0; st < args.steps; ++st) {
        const int k = (1 << (args.steps - st)) + 1;
        // automorphism X -> X^k of the owned coefficients, into shared memory
#pragma unroll
        for (int sl = 0; sl < SL; ++sl) {
            const int i = tid + sl * nt;
            if (i >= H) continue;
#pragma unroll
            for (int hf = 0; hf < 2; ++hf) {
                const int j = i + hf * H;
                const int dst = (int)(((long long)j * k) % (2 * N));
                const int t = dst % N;
                permA[t] = dst >= N ? 0ULL - accA[sl][hf] : accA[sl][hf];
                permB[t] = dst >= N ? 0ULL - accB[sl][hf] : accB[sl][hf];
            }
        }
        __syncthreads();
        // gadget digits of A', fold + twist; B' of the owned coefficients kept
        u64 pB[SL][2];
#pragma unroll
        for (int sl = 0; sl < SL; ++sl) {
            const int i = tid + sl * nt;
            pB[sl][0] = pB[sl][1] = 0ULL;
            if (i >= H) continue;
            pB[sl][0] = permB[i];
            pB[sl][1] = permB[i + H];
            long long xl = (long long)permA[i], xh = (long long)permA[i + H];
            const double2 w = args.qt[i];
            for (int lvl = 0; lvl < args.l; ++lvl) {
                const int sh = 64 - (lvl + 1) * args.log2_beta;
                long long rl, rh;
                const double dl = (double)rne_shift(xl, sh, &rl);
                const double dh = (double)rne_shift(xh, sh, &rh);
                xl = rl;
                xh = rh;
                dig[(size_t)lvl * H + swz(i)] = make_double2(fma(w.x, dl, w.y * dh), fma(w.y, dl, -w.x * dh));
            }
        }
        __syncthreads();
        fwd<LOGH, 0>(dig, args.l, args.tw, tid, nt);
        const double2* key = args.key + (size_t)st * args.l * 2 * LIMBS * H;
        for (int p = tid; p < H; p += nt) {
            for (int limb = 0; limb < LIMBS; ++limb) {
                double2 o0 = make_double2(0.0, 0.0), o1 = make_double2(0.0, 0.0);
                for (int lvl = 0; lvl < args.l; ++lvl) {
                    const double2 d = dig[(size_t)lvl * H + swz(p)];
                    c_mac(o0, d, key[(((size_t)lvl * 2 + 0) * LIMBS + limb) * H + p]);
                    c_mac(o1, d, key[(((size_t)lvl * 2 + 1) * LIMBS + limb) * H + p]);
                }
                res[(size_t)(2 * limb) * H + swz(p)] = o0;
                res[(size_t)(2 * limb + 1) * H + swz(p)] = o1;
            }
        }
        __syncthreads();
        inv<LOGH, Plan<LOGH>::NS - 1>(res, 2 * LIMBS, args.tw, tid, nt);
#pragma unroll
        for (int sl = 0; sl < SL; ++sl) {
            const int i = tid + sl * nt;
            if (i >= H) continue;
            const double2 w = c_conj(args.qt[i]);
            u64 ka0 = 0ULL, ka1 = 0ULL, kb0 = 0ULL, kb1 = 0ULL;
#pragma unroll
            for (int limb = 0; limb < LIMBS; ++limb) {
                const double2 ua = c_mul(w, res[(size_t)(2 * limb) * H + swz(i)]);
                const double2 ub = c_mul(w, res[(size_t)(2 * limb + 1) * H + swz(i)]);
                const int sh = 16 * limb;
                ka0 += (u64)(long long)rint(ua.x * inv_h) << sh;
                ka1 += (u64)(long long)rint(-ua.y * inv_h) << sh;
                kb0 += (u64)(long long)rint(ub.x * inv_h) << sh;
                kb1 += (u64)(long long)rint(-ub.y * inv_h) << sh;
            }
            accA[sl][0] += ka0;
            accA[sl][1] += ka1;
            accB[sl][0] += pB[sl][0] + kb0;
            accB[sl][1] += pB[sl][1] + kb1;
        }
        __syncthreads();
    }
    u64* dst = args.out + r * 2 * N;
#pragma unroll
    for (int sl = 0; sl < SL; ++sl) {
        const int i = tid + sl * nt;
        if (i >= H) continue;
        dst[i] = accA[sl][0];
        dst[i + H] = accA[sl][1];
        dst[N + i] = accB[sl][0];
        dst[N + i + H] = accB[sl][1];
    }
}

// ---------------------------------------------------------------- packing
constexpr int PK_TB = 64, PK_TO = 64, PK_KC = 4, PK_LMAX = 8;

__global__ void __launch_bounds__(256) pack64_kernel(const u64* __restrict__ lwe_a, int n_dim, int T, long long S,
                                                     const u64* __restrict__ ksp, int N, int l, int log2_beta,
                                                     u64* __restrict__ out) {
    __shared__ int dig[PK_TB][PK_KC * PK_LMAX + 1];
    __shared__ __align__(16) u64 kt[PK_KC * PK_LMAX][PK_TO];
    const int tid = threadIdx.x;
    const int ty = tid / 16, tx = tid % 16;
    const long long r0 = (long long)blockIdx.y * PK_TB;
    const int o0 = blockIdx.x * PK_TO;
    const long long rows_total = S * T;
    const int cols = 2 * N;
    u64 acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0ULL;
    for (int i0 = 0; i0 < n_dim; i0 += PK_KC) {
        for (int idx = tid; idx < PK_TB * PK_KC; idx += 256) {
            const int rr = idx / PK_KC, c = idx % PK_KC;
            const long long row = r0 + rr;
            const int i = i0 + c;
            long long x = (row < rows_total && i < n_dim) ? (long long)lwe_a[row * n_dim + i] : 0LL;
            for (int j = 0; j < l; ++j) {
                long long rem;
                dig[rr][c * l + j] = (int)rne_shift(x, 64 - (j + 1) * log2_beta, &rem);
                x = rem;
            }
        }
        const int krows = PK_KC * l;
        for (int idx = tid; idx < krows * PK_TO; idx += 256) {
            const int kr = idx / PK_TO, col = idx % PK_TO;
            const int i = i0 + kr / l, j = kr % l;
            const int o = o0 + col;
            kt[kr][col] = (i < n_dim && o < cols) ? ksp[((long long)i * l + j) * cols + o] : 0ULL;
        }
        __syncthreads();
        for (int kr = 0; kr < krows; ++kr) {
#pragma unroll
            for (int cc = 0; cc < 4; ++cc) {
                const u64 d = (u64)(long long)dig[ty * 4 + cc][kr];
#pragma unroll
                for (int e = 0; e < 4; ++e) acc[cc][e] += d * kt[kr][tx * 4 + e];
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int cc = 0; cc < 4; ++cc) {
        const long long row = r0 + ty * 4 + cc;
        if (row >= rows_total) continue;
        const long long s = row / T;
        const int t = (int)(row - s * T);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int o = o0 + tx * 4 + e;
            if (o >= cols) continue;
            const int poly = o / N, c = o - poly * N;
            int d = c + t;
            u64 v = 0ULL - acc[cc][e];              // -X^t V: negated unless it wraps past X^N
            if (d >= N) {
                d -= N;
                v = acc[cc][e];
            }
            atomicAdd(out + (s * 2 + poly) * (long long)N + d, v);
        }
    }
}

__global__ void pack_init64_kernel(const u64* __restrict__ lwe_b, int T, long long S, int N, u64* __restrict__ out) {
    const long long total = S * 2 * (long long)N;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long s = i / (2 * N);
        const int rem = (int)(i - s * 2 * N);
        const int poly = rem / N, c = rem - poly * N;
        out[i] = (poly == 1 && c < T) ? lwe_b[s * T + c] : 0ULL;
    }
}

// ---------------------------------------------------------------- small ops
__global__ void rotate_add64_kernel(const u64* __restrict__ x, int rot, const u64* __restrict__ y, long long S,
                                    int N, u64* __restrict__ out) {
    const long long total = S * 2 * (long long)N;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long row = i / N;
        const int c = (int)(i - row * N);
        int src = c - rot;                         // rot in [0, 2N)
        int wraps = 0;
        if (src < 0) {
            src += N;
            ++wraps;
        }
        if (src < 0) {
            src += N;
            ++wraps;
        }
        u64 v = x[row * N + src];
        if (wraps & 1) v = 0ULL - v;
        out[i] = v + (y ? y[i] : 0ULL);
    }
}

__global__ void add64_kernel(const u64* __restrict__ x, const u64* __restrict__ y, long long n,
                             u64* __restrict__ out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = x[i] + y[i];
}

// LWEs of coefficients 0 .. count-1 of RLWEs (S, 2, N)
__global__ void extract64_kernel(const u64* __restrict__ acc, int N, int count, u64* __restrict__ out_a,
                                 u64* __restrict__ out_b, long long S) {
    const long long total = S * count * (long long)N;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const long long k = t / ((long long)count * N);
        const int rem = (int)(t - k * count * (long long)N);
        const int al = rem / N, j = rem % N;
        const u64* a = acc + k * 2 * N;
        const int e = al - j;
        out_a[t] = e >= 0 ? a[e] : 0ULL - a[e + N];
        if (j == 0) out_b[k * count + al] = a[N + al];
    }
}

int grid_for(long long total) {
    return (int)std::max<long long>(1, std::min<long long>((total + 255) / 256, 148LL * 16));
}

int log2_exact(long long v) {
    int r = 0;
    while ((1LL << r) < v) ++r;
    return (1LL << r) == v ? r : -1;
}

bool valid_degree(int N) { return N >= 128 && N <= 4096 && log2_exact(N) > 0; }

int max_smem() {
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    return v;
}

size_t trace_smem(int N, int l) {
    return (size_t)(l + 2) * (N / 2) * sizeof(double2) + 4 * (size_t)N * sizeof(u64);
}

size_t trace_fused_smem(int N, int l) { return (size_t)(l + 2 * LIMBS) * (N / 2) * sizeof(double2); }

// the fused-limb kernel where its spectra fit in shared memory
// (TFHE_B200_TRACE_FUSED=0: the limb-by-limb kernel, for comparison)
static bool trace_fused_enabled() {
    static const bool on = [] {
        const char* env = getenv("TFHE_B200_TRACE_FUSED");
        return !(env && env[0] == '0');
    }();
    return on;
}

template <int LOGN>
int launch_trace(const Trace64Args& a, long long R, cudaStream_t stream) {
    int dev = 0, optin = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
        optin = 0;
    const size_t fsmem = trace_fused_smem(1 << LOGN, a.l);
    const bool fused = trace_fused_enabled() && fsmem <= (size_t)optin;
    const size_t smem = fused ? fsmem : trace_smem(1 << LOGN, a.l);
    const void* kern = fused ? (const void*)trace64_fused_kernel<LOGN> : (const void*)trace64_kernel<LOGN>;
    TFHE_TRY(smem_attr_once(kern, smem));
    count_launch();
    if (fused) trace64_fused_kernel<LOGN><<<(unsigned)R, TRACE_NT, smem, stream>>>(a);
    else trace64_kernel<LOGN><<<(unsigned)R, TRACE_NT, smem, stream>>>(a);
    return check_cuda(cudaGetLastError(), "trace (2^64) launch");
}

template <int LOGN>
int launch_limb_fft(const u64* src, long long npoly, const FftPlan* pl, double2* dst, cudaStream_t stream) {
    const size_t smem = (size_t)(1 << (LOGN - 1)) * sizeof(double2);
    count_launch();
    limb_fft64_kernel<LOGN><<<dim3((unsigned)npoly, LIMBS), 256, smem, stream>>>(src, pl->qt, pl->tw, dst);
    return check_cuda(cudaGetLastError(), "limb FFT launch");
}

#define T64_DISPATCH(LOGN_VAL, CALL)                                                              \
    switch (LOGN_VAL) {                                                                           \
        case 7: return CALL(7);                                                                   \
        case 8: return CALL(8);                                                                   \
        case 9: return CALL(9);                                                                   \
        case 10: return CALL(10);                                                                 \
        case 11: return CALL(11);                                                                 \
        case 12: return CALL(12);                                                                 \
        default: return fail(TFHE_ERR_INVALID_ARGUMENT, "degree must be a power of two in [128, 4096]"); \
    }

}  // namespace t64
}  // namespace tfhe

using namespace tfhe;
using namespace tfhe::t64;

struct tfhe64_galois_keys {
    int N = 0, log2_beta = 0, l = 0, steps = 0, device = 0;
    double2* key = nullptr;     // [steps][l][2][LIMBS][H]
};

extern "C" {

int tfhe64_keyswitch(const uint64_t* ksk, int32_t n_big, int32_t n, int32_t l_ks, int32_t log2_beta_ks,
                     const uint64_t* a_in, const uint64_t* b_in, uint64_t* a_out, uint64_t* b_out, int64_t batch,
                     void* stream) {
    if (n_big <= 0 || n <= 0) return fail(TFHE_ERR_INVALID_ARGUMENT, "keyswitch64: dimensions must be positive");
    if (l_ks < 1 || l_ks > KS_LMAX || log2_beta_ks < 1 || log2_beta_ks > 16 || log2_beta_ks * l_ks > 64)
        return fail(TFHE_ERR_INVALID_ARGUMENT, "keyswitch64: need 1 <= l <= 8, log2 beta <= 16, l log2 beta <= 64");
    if (batch < 0) return fail(TFHE_ERR_INVALID_ARGUMENT, "keyswitch64: negative batch");
    if (batch == 0) return TFHE_OK;
    if (!ksk || !a_in || !b_in || !a_out || !b_out) return fail(TFHE_ERR_INVALID_ARGUMENT, "keyswitch64: NULL buffer");
    if ((batch + KS_TB - 1) / KS_TB > 65535) return fail(TFHE_ERR_INVALID_ARGUMENT, "keyswitch64: batch too large");
    const dim3 grid((n + 1 + KS_TO - 1) / KS_TO, (unsigned)((batch + KS_TB - 1) / KS_TB));
    count_launch();
    ks64_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(
        reinterpret_cast<const u64*>(a_in), reinterpret_cast<const u64*>(b_in), reinterpret_cast<const u64*>(ksk),
        n_big, n, l_ks, log2_beta_ks, reinterpret_cast<u64*>(a_out), reinterpret_cast<u64*>(b_out), batch);
    return check_cuda(cudaGetLastError(), "keyswitch64 launch");
}

int tfhe64_rotation_indices(const uint64_t* lwe_a, int32_t n, int32_t collapse, int32_t N, int32_t n_lut,
                            int32_t* indices, int64_t batch, void* stream) {
    if (!valid_degree(N)) return fail(TFHE_ERR_INVALID_ARGUMENT, "indices64: N must be a power of two in [128, 4096]");
    if (collapse < 1 || collapse > 4 || n <= 0 || n % collapse)
        return fail(TFHE_ERR_INVALID_ARGUMENT, "indices64: n must be a positive multiple of collapse (1..4)");
    const int ln = log2_exact(n_lut);
    if (ln < 0 || n_lut > N) return fail(TFHE_ERR_INVALID_ARGUMENT, "indices64: n_lut must be a power of two <= N");
    if (batch < 0) return fail(TFHE_ERR_INVALID_ARGUMENT, "indices64: negative batch");
    if (batch == 0) return TFHE_OK;
    if (!lwe_a || !indices) return fail(TFHE_ERR_INVALID_ARGUMENT, "indices64: NULL buffer");
    const long long total = batch * (n / collapse) * (1LL << collapse);
    count_launch();
    indices64_kernel<<<grid_for(total), 256, 0, (cudaStream_t)stream>>>(reinterpret_cast<const u64*>(lwe_a), n,
                                                                        collapse, log2_exact(N), ln, indices, batch);
    return check_cuda(cudaGetLastError(), "indices64 launch");
}

int tfhe64_rotate_extract(const int64_t* acc, const uint64_t* b, int32_t N, int32_t n_lut, uint64_t* out_a,
                          uint64_t* out_b, int64_t batch, void* stream) {
    if (!valid_degree(N)) return fail(TFHE_ERR_INVALID_ARGUMENT, "rotate/extract64: N must be a power of two");
    const int ln = log2_exact(n_lut);
    if (ln < 0 || n_lut > N) return fail(TFHE_ERR_INVALID_ARGUMENT, "rotate/extract64: n_lut must be a power of two <= N");
    if (batch < 0) return fail(TFHE_ERR_INVALID_ARGUMENT, "rotate/extract64: negative batch");
    if (batch == 0) return TFHE_OK;
    if (!acc || !b || !out_a || !out_b) return fail(TFHE_ERR_INVALID_ARGUMENT, "rotate/extract64: NULL buffer");
    const long long total = batch * ((long long)n_lut * N + n_lut);
    count_launch();
    rotate_extract64_kernel<<<grid_for(total), 256, 0, (cudaStream_t)stream>>>(
        reinterpret_cast<const long long*>(acc), reinterpret_cast<const u64*>(b), log2_exact(N), n_lut, ln,
        reinterpret_cast<u64*>(out_a), reinterpret_cast<u64*>(out_b), batch);
    return check_cuda(cudaGetLastError(), "rotate/extract64 launch");
}

int tfhe64_linear_extract(const int32_t* weights, const int64_t* bias, int32_t J, const uint64_t* rlwe, int64_t S,
                          int32_t N, uint64_t* out_a, uint64_t* out_b, void* stream) {
    if (!valid_degree(N)) return fail(TFHE_ERR_INVALID_ARGUMENT, "linear64: N must be a power of two in [128, 4096]");
    if (J < 0 || S < 0) return fail(TFHE_ERR_INVALID_ARGUMENT, "linear64: negative size");
    if (J == 0 || S == 0) return TFHE_OK;
    if (!weights || !bias || !rlwe || !out_a || !out_b) return fail(TFHE_ERR_INVALID_ARGUMENT, "linear64: null pointer");
    if (S > 65535) return fail(TFHE_ERR_INVALID_ARGUMENT, "linear64: at most 65535 ciphertexts per call");
    const size_t smem = (size_t)N * sizeof(u64) + (size_t)LIN_JT * N * sizeof(int32_t);
    TFHE_TRY(smem_attr_once((const void*)linear64_kernel, smem));
    const dim3 grid((J + LIN_JT - 1) / LIN_JT, (unsigned)S);
    count_launch();
    linear64_kernel<<<grid, LIN_NT, smem, (cudaStream_t)stream>>>(
        weights, reinterpret_cast<const long long*>(bias), J, reinterpret_cast<const u64*>(rlwe), N,
        reinterpret_cast<u64*>(out_a), reinterpret_cast<u64*>(out_b));
    return check_cuda(cudaGetLastError(), "linear64 launch");
}

// LUT products in the Fourier domain (TFHE_B200_LUT_FFT=0: the direct sums)
static bool lut_fft_enabled() {
    static const bool on = [] {
        const char* env = getenv("TFHE_B200_LUT_FFT");
        return !(env && env[0] == '0');
    }();
    return on;
}

int tfhe64_lut_mul_sum(const int64_t* luts, int32_t groups, int32_t per_group, const uint64_t* rlwe, int64_t S,
                       int32_t N, uint64_t* out, void* stream) {
    if (!valid_degree(N)) return fail(TFHE_ERR_INVALID_ARGUMENT, "lut product64: N must be a power of two");
    if (groups < 1 || per_group < 0 || S < 0) return fail(TFHE_ERR_INVALID_ARGUMENT, "lut product64: bad sizes");
    if (per_group == 0 || S == 0) return TFHE_OK;
    if (!luts || !rlwe || !out) return fail(TFHE_ERR_INVALID_ARGUMENT, "lut product64: null pointer");
    if (S > 65535) return fail(TFHE_ERR_INVALID_ARGUMENT, "lut product64: at most 65535 sequences per call");
    if (lut_fft_enabled() && N <= 2048) {
        const FftPlan* pl = get_plan(N);
        if (!pl) return TFHE_ERR_INTERNAL;
        const size_t fsmem = (size_t)9 * (N / 2) * sizeof(double2);
        const int logn = log2_exact(N);
        const void* kern = logn == 7   ? (const void*)lut_fft64_kernel<7>
                           : logn == 8  ? (const void*)lut_fft64_kernel<8>
                           : logn == 9  ? (const void*)lut_fft64_kernel<9>
                           : logn == 10 ? (const void*)lut_fft64_kernel<10>
                                        : (const void*)lut_fft64_kernel<11>;
        TFHE_TRY(smem_attr_once(kern, fsmem));
        const dim3 grid((unsigned)per_group, (unsigned)S);
        const long long* P = reinterpret_cast<const long long*>(luts);
        const u64* ct = reinterpret_cast<const u64*>(rlwe);
        u64* o = reinterpret_cast<u64*>(out);
        cudaStream_t st = (cudaStream_t)stream;
        count_launch();
        switch (logn) {
            case 7: lut_fft64_kernel<7><<<grid, LF_NT, fsmem, st>>>(P, groups, per_group, ct, pl->qt, pl->tw, o); break;
            case 8: lut_fft64_kernel<8><<<grid, LF_NT, fsmem, st>>>(P, groups, per_group, ct, pl->qt, pl->tw, o); break;
            case 9: lut_fft64_kernel<9><<<grid, LF_NT, fsmem, st>>>(P, groups, per_group, ct, pl->qt, pl->tw, o); break;
            case 10: lut_fft64_kernel<10><<<grid, LF_NT, fsmem, st>>>(P, groups, per_group, ct, pl->qt, pl->tw, o); break;
            default: lut_fft64_kernel<11><<<grid, LF_NT, fsmem, st>>>(P, groups, per_group, ct, pl->qt, pl->tw, o); break;
        }
        return check_cuda(cudaGetLastError(), "lut product64 (FFT) launch");
    }
    const size_t smem = 3 * (size_t)N * sizeof(u64);
    TFHE_TRY(smem_attr_once((const void*)lut_mul_sum64_kernel, smem));
    const dim3 grid((unsigned)per_group, (unsigned)S);
    count_launch();
    lut_mul_sum64_kernel<<<grid, LM_NT, smem, (cudaStream_t)stream>>>(
        reinterpret_cast<const long long*>(luts), groups, per_group, reinterpret_cast<const u64*>(rlwe), N,
        reinterpret_cast<u64*>(out));
    return check_cuda(cudaGetLastError(), "lut product64 launch");
}

int tfhe64_galois_keys_create(int32_t N, int32_t log2_beta, int32_t l, const uint64_t* keys, void* stream,
                              tfhe64_galois_keys** out) {
    if (!out) return fail(TFHE_ERR_INVALID_ARGUMENT, "galois keys64: null output");
    *out = nullptr;
    if (!valid_degree(N)) return fail(TFHE_ERR_INVALID_ARGUMENT, "galois keys64: N must be a power of two");
    // exactness: |digit| <= 2^(log2_beta - 1), |limb| <= 2^15, N l terms < 2^50
    if (l < 1 || l > 8 || log2_beta < 1 || log2_beta > 16 || log2_beta * l > 64 ||
        (long long)N * l * (1LL << (log2_beta - 1)) * (1LL << 15) >= (1LL << 50))
        return fail(TFHE_ERR_INVALID_ARGUMENT, "galois keys64: need 1 <= l <= 8, l log2 beta <= 64, exact products");
    if (!keys) return fail(TFHE_ERR_INVALID_ARGUMENT, "galois keys64: null key pointer");
    if (trace_smem(N, l) > (size_t)max_smem())
        return fail(TFHE_ERR_INVALID_ARGUMENT, "galois keys64: l levels at this degree exceed shared memory");
    const FftPlan* pl = get_plan(N);
    if (!pl) return TFHE_ERR_INTERNAL;
    auto* gk = new tfhe64_galois_keys();
    gk->N = N;
    gk->log2_beta = log2_beta;
    gk->l = l;
    gk->steps = log2_exact(N);
    cudaGetDevice(&gk->device);
    const long long npoly = (long long)gk->steps * l * 2;
    cudaStream_t st = (cudaStream_t)stream;
    int rc = check_cuda(cudaMalloc(&gk->key, (size_t)npoly * LIMBS * (N / 2) * sizeof(double2)),
                        "cudaMalloc(galois key64)");
    if (rc == TFHE_OK) {
        const u64* src = reinterpret_cast<const u64*>(keys);
#define T64_LIMB_FFT(LG) launch_limb_fft<LG>(src, npoly, pl, gk->key, st)
        rc = [&]() -> int { T64_DISPATCH(log2_exact(N), T64_LIMB_FFT) }();
#undef T64_LIMB_FFT
    }
    if (rc == TFHE_OK) rc = check_cuda(cudaStreamSynchronize(st), "galois key64 upload");
    if (rc != TFHE_OK) {
        cudaFree(gk->key);
        delete gk;
        return rc;
    }
    *out = gk;
    return TFHE_OK;
}

int tfhe64_galois_keys_destroy(tfhe64_galois_keys* gk) {
    if (!gk) return TFHE_OK;
    cudaFree(gk->key);
    delete gk;
    return TFHE_OK;
}

int tfhe64_pack_lwe_to_rlwe(const tfhe64_galois_keys* gk, const uint64_t* lwe_a, const uint64_t* lwe_b, int64_t R,
                            uint64_t* out, void* stream) {
    if (!gk) return fail(TFHE_ERR_INVALID_ARGUMENT, "pack_lwe_to_rlwe64: null keys");
    if (R < 0) return fail(TFHE_ERR_INVALID_ARGUMENT, "pack_lwe_to_rlwe64: negative count");
    if (R == 0) return TFHE_OK;
    if (!lwe_a || !lwe_b || !out) return fail(TFHE_ERR_INVALID_ARGUMENT, "pack_lwe_to_rlwe64: null pointer");
    if (R > 2147483647LL) return fail(TFHE_ERR_INVALID_ARGUMENT, "pack_lwe_to_rlwe64: too many ciphertexts");
    const FftPlan* pl = get_plan(gk->N);
    if (!pl) return TFHE_ERR_INTERNAL;
    Trace64Args a{reinterpret_cast<const u64*>(lwe_a), reinterpret_cast<const u64*>(lwe_b), gk->key, pl->qt, pl->tw,
                  gk->log2_beta, gk->l, gk->steps, reinterpret_cast<u64*>(out)};
    cudaStream_t st = (cudaStream_t)stream;
#define T64_TRACE(LG) launch_trace<LG>(a, R, st)
    T64_DISPATCH(log2_exact(gk->N), T64_TRACE)
#undef T64_TRACE
}

int tfhe64_pack_lwes(const uint64_t* ksp, int32_t n_dim, int32_t N, int32_t log2_beta, int32_t l,
                     const uint64_t* lwe_a, const uint64_t* lwe_b, int32_t T, int64_t S, uint64_t* out, void* stream) {
    if (!valid_degree(N)) return fail(TFHE_ERR_INVALID_ARGUMENT, "packing64: N must be a power of two in [128, 4096]");
    if (l < 1 || l > PK_LMAX || log2_beta < 1 || log2_beta > 16 || log2_beta * l > 64)
        return fail(TFHE_ERR_INVALID_ARGUMENT, "packing64: need 1 <= l <= 8, log2 beta <= 16, l log2 beta <= 64");
    if (n_dim < 1 || T < 0 || T > N || S < 0) return fail(TFHE_ERR_INVALID_ARGUMENT, "packing64: bad sizes (T <= N)");
    if (S == 0) return TFHE_OK;
    if (!ksp || !out || (T > 0 && (!lwe_a || !lwe_b))) return fail(TFHE_ERR_INVALID_ARGUMENT, "packing64: null pointer");
    const long long total = S * 2 * (long long)N;
    count_launch();
    pack_init64_kernel<<<grid_for(total), 256, 0, (cudaStream_t)stream>>>(reinterpret_cast<const u64*>(lwe_b), T, S,
                                                                          N, reinterpret_cast<u64*>(out));
    const int rc = check_cuda(cudaGetLastError(), "packing64 init launch");
    if (rc != TFHE_OK) return rc;
    if (T == 0) return TFHE_OK;
    const long long rows = S * T;
    if ((rows + PK_TB - 1) / PK_TB > 65535) return fail(TFHE_ERR_INVALID_ARGUMENT, "packing64: too many LWEs per call");
    const dim3 grid((2 * N + PK_TO - 1) / PK_TO, (unsigned)((rows + PK_TB - 1) / PK_TB));
    count_launch();
    pack64_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(reinterpret_cast<const u64*>(lwe_a), n_dim, T, S,
                                                          reinterpret_cast<const u64*>(ksp), N, l, log2_beta,
                                                          reinterpret_cast<u64*>(out));
    return check_cuda(cudaGetLastError(), "packing64 launch");
}

int64_t tfhe64_tc_limb_rows(int32_t cols) {
    if (cols < 1) return 0;
    const long long rows = 8LL * cols;
    const int tile = ks_tc_columns();
    return (rows + tile - 1) / tile * tile;
}

int tfhe64_tc_limbs(const uint64_t* key, int64_t K, int32_t cols, int8_t* limbs, void* stream) {
    if (!key || !limbs) return fail(TFHE_ERR_INVALID_ARGUMENT, "limbs64: null pointer");
    if (K < 1 || cols < 1) return fail(TFHE_ERR_INVALID_ARGUMENT, "limbs64: bad sizes");
    return build_limbs64(reinterpret_cast<const u64*>(key), K, cols, (int)tfhe64_tc_limb_rows(cols), limbs,
                         (cudaStream_t)stream);
}

// the int32 sums of the tensor-core contraction cannot overflow: digits
// |d| <= 2^(log2_beta - 1) <= 64, limbs |v| <= 128, K terms
static bool tc_contraction_fits(long long K, int log2_beta) {
    return log2_beta >= 1 && log2_beta <= 7 && K * (1LL << (log2_beta - 1)) * 128 < (1LL << 31);
}

int tfhe64_keyswitch_tc(const int8_t* limbs, int32_t n_big, int32_t n, int32_t l_ks, int32_t log2_beta_ks,
                        const uint64_t* a_in, const uint64_t* b_in, uint64_t* a_out, uint64_t* b_out, int64_t batch,
                        void* stream) {
    if (n_big <= 0 || n <= 0 || n_big % 32) return fail(TFHE_ERR_INVALID_ARGUMENT, "keyswitch64 (tc): n_big % 32");
    if (l_ks < 1 || l_ks > 8 || !tc_contraction_fits((long long)n_big * l_ks, log2_beta_ks))
        return fail(TFHE_ERR_INVALID_ARGUMENT, "keyswitch64 (tc): digits must fit 8 bits without int32 overflow");
    if (batch < 0) return fail(TFHE_ERR_INVALID_ARGUMENT, "keyswitch64 (tc): negative batch");
    if (batch == 0) return TFHE_OK;
    if (!limbs || !a_in || !b_in || !a_out || !b_out) return fail(TFHE_ERR_INVALID_ARGUMENT, "keyswitch64 (tc): NULL");
    if (reinterpret_cast<uintptr_t>(a_in) & 15) return fail(TFHE_ERR_INVALID_ARGUMENT, "keyswitch64 (tc): a_in alignment");
    KsTcArgs args{reinterpret_cast<const uint32_t*>(a_in), reinterpret_cast<const uint32_t*>(b_in),
                  reinterpret_cast<const unsigned char*>(limbs), n_big, n, l_ks, log2_beta_ks,
                  (int)tfhe64_tc_limb_rows(n + 1), batch, reinterpret_cast<uint32_t*>(a_out),
                  reinterpret_cast<uint32_t*>(b_out), WAIT_LIMIT_CYCLES, device_status_word(), 0, 0, nullptr, true,
                  true};
    if (!args.status) return fail(TFHE_ERR_INTERNAL, "device status word unavailable");
    return launch_ks_tc(args, (cudaStream_t)stream);
}

int tfhe64_pack_lwes_tc(const int8_t* limbs, int32_t n_dim, int32_t N, int32_t log2_beta, int32_t l,
                        const uint64_t* lwe_a, const uint64_t* lwe_b, int32_t T, int64_t S, uint64_t* out,
                        void* stream) {
    if (!valid_degree(N)) return fail(TFHE_ERR_INVALID_ARGUMENT, "packing64 (tc): N must be a power of two");
    if (l < 1 || l > 8 || n_dim < 32 || n_dim % 32 || !tc_contraction_fits((long long)n_dim * l, log2_beta))
        return fail(TFHE_ERR_INVALID_ARGUMENT, "packing64 (tc): n_dim % 32, digits in 8 bits, no int32 overflow");
    if (T < 0 || T > N || S < 0) return fail(TFHE_ERR_INVALID_ARGUMENT, "packing64 (tc): bad sizes (T <= N)");
    if (S == 0) return TFHE_OK;
    if (!limbs || !out || (T > 0 && (!lwe_a || !lwe_b))) return fail(TFHE_ERR_INVALID_ARGUMENT, "packing64 (tc): NULL");
    if (T > 0 && (reinterpret_cast<uintptr_t>(lwe_a) & 15))
        return fail(TFHE_ERR_INVALID_ARGUMENT, "packing64 (tc): lwe_a alignment");
    const long long total = S * 2 * (long long)N;
    count_launch();
    pack_init64_kernel<<<grid_for(total), 256, 0, (cudaStream_t)stream>>>(reinterpret_cast<const u64*>(lwe_b), T, S,
                                                                          N, reinterpret_cast<u64*>(out));
    const int rc = check_cuda(cudaGetLastError(), "packing64 (tc) init launch");
    if (rc != TFHE_OK || T == 0) return rc;
    KsTcArgs args{reinterpret_cast<const uint32_t*>(lwe_a), nullptr, reinterpret_cast<const unsigned char*>(limbs),
                  n_dim, 0, l, log2_beta, (int)tfhe64_tc_limb_rows(2 * N), S * T, nullptr, nullptr,
                  WAIT_LIMIT_CYCLES, device_status_word(), T, N, reinterpret_cast<uint32_t*>(out), true, true};
    if (!args.status) return fail(TFHE_ERR_INTERNAL, "device status word unavailable");
    return launch_ks_tc(args, (cudaStream_t)stream);
}

int tfhe64_rlwe_rotate_add(const uint64_t* x, int32_t rot, const uint64_t* y, int64_t S, int32_t N, uint64_t* out,
                           void* stream) {
    if (!valid_degree(N)) return fail(TFHE_ERR_INVALID_ARGUMENT, "rotate/add64: N must be a power of two");
    if (S < 0) return fail(TFHE_ERR_INVALID_ARGUMENT, "rotate/add64: negative count");
    if (S == 0) return TFHE_OK;
    if (!x || !out) return fail(TFHE_ERR_INVALID_ARGUMENT, "rotate/add64: null pointer");
    if (x == out && rot % (2 * N) != 0)
        return fail(TFHE_ERR_INVALID_ARGUMENT, "rotate/add64: out may not alias x when rotating");
    const int r = ((rot % (2 * N)) + 2 * N) % (2 * N);
    count_launch();
    rotate_add64_kernel<<<grid_for(S * 2 * (long long)N), 256, 0, (cudaStream_t)stream>>>(
        reinterpret_cast<const u64*>(x), r, reinterpret_cast<const u64*>(y), S, N, reinterpret_cast<u64*>(out));
    return check_cuda(cudaGetLastError(), "rotate/add64 launch");
}

int tfhe64_add(const uint64_t* x, const uint64_t* y, int64_t n, uint64_t* out, void* stream) {
    if (n < 0) return fail(TFHE_ERR_INVALID_ARGUMENT, "add64: negative count");
    if (n == 0) return TFHE_OK;
    if (!x || !y || !out) return fail(TFHE_ERR_INVALID_ARGUMENT, "add64: null pointer");
    count_launch();
    add64_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(reinterpret_cast<const u64*>(x),
                                                               reinterpret_cast<const u64*>(y), n,
                                                               reinterpret_cast<u64*>(out));
    return check_cuda(cudaGetLastError(), "add64 launch");
}

int tfhe64_sample_extract(const uint64_t* rlwe, int32_t N, int32_t count, uint64_t* out_a, uint64_t* out_b,
                          int64_t S, void* stream) {
    if (!valid_degree(N)) return fail(TFHE_ERR_INVALID_ARGUMENT, "extract64: N must be a power of two");
    if (count < 1 || count > N) return fail(TFHE_ERR_INVALID_ARGUMENT, "extract64: count must be in [1, N]");
    if (S < 0) return fail(TFHE_ERR_INVALID_ARGUMENT, "extract64: negative count");
    if (S == 0) return TFHE_OK;
    if (!rlwe || !out_a || !out_b) return fail(TFHE_ERR_INVALID_ARGUMENT, "extract64: null pointer");
    count_launch();
    extract64_kernel<<<grid_for(S * count * (long long)N), 256, 0, (cudaStream_t)stream>>>(
        reinterpret_cast<const u64*>(rlwe), N, count, reinterpret_cast<u64*>(out_a), reinterpret_cast<u64*>(out_b), S);
    return check_cuda(cudaGetLastError(), "extract64 launch");
}

}  // extern "C"
