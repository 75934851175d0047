// Operators of one encrypted Spike-LSTM timestep around the programmable
// bootstrap (nn_tfhe/Spike_LSTM.py:15-62, 103-184):
//
//   linear_extract_kernel   Linear.__call__: plaintext weight polynomial x
//                           RLWE, sample_extract at 0, + bias
//   lut_mul_sum_kernel      prepare_LUT's multiply_plaintext_ciphertext and
//                           the sum over the packed sub-LUTs
//   trace_pack_kernel       pack_lwe_to_rlwe: modulus switch to q/N, trivial
//                           embedding, log2 N automorphism + key switch steps
//   pack_ks_kernel          packing: LWE list -> RLWE with the packing key
//   rlwe_rotate_add_kernel  rotate_ciphertext / sum_ciphertext_ciphertext
//
// Torus values are uint32 (q = 2^32).  Every product of an integer
// plaintext with a ciphertext is computed exactly modulo 2^32 (the
// reference rounds FP64 FFT products that are exact at these sizes and
// reduces them modulo q).  The trace keeps its running sum unreduced in
// float64, as the reference does, because the next step's decomposition
// depends on the unreduced value.
#include <algorithm>
#include <string>

#include "tfhe_b200.h"
#include "tfhe_dispatch.h"
#include "tfhe_internal.cuh"

namespace tfhe {

// ---------------------------------------------------------------- linear
// P_A = W_j(X) A_s(X) mod X^N + 1; the LWE of coefficient 0 is
// a'[0] = P_A[0], a'[i] = -P_A[N - i] (schemas/text_jax.py:191-208) and
// b' = P_B[0] + bias_j (Spike_LSTM.py:48-58).
constexpr int LIN_JT = 4;      // outputs per CTA
constexpr int LIN_NT = 256;

__global__ void __launch_bounds__(LIN_NT) linear_extract_kernel(const int32_t* __restrict__ W,
                                                                const int32_t* __restrict__ bias, int J,
                                                                const uint32_t* __restrict__ ct, int N,
                                                                uint32_t* __restrict__ out_a,
                                                                uint32_t* __restrict__ out_b) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint32_t* A = reinterpret_cast<uint32_t*>(smem_raw);            // N
    int32_t* Ws = reinterpret_cast<int32_t*>(A + N);                // LIN_JT * N
    __shared__ uint32_t red[LIN_JT][LIN_NT / 32];
    const int tid = threadIdx.x;
    const long long s = blockIdx.y;
    const int j0 = blockIdx.x * LIN_JT;
    const uint32_t* a_in = ct + s * 2 * N;
    const uint32_t* b_in = a_in + N;
    for (int i = tid; i < N; i += LIN_NT) A[i] = a_in[i];
    for (int i = tid; i < LIN_JT * N; i += LIN_NT) {
        const int jt = i / N;
        Ws[i] = (j0 + jt < J) ? W[(long long)(j0 + jt) * N + (i - jt * N)] : 0;
    }
    __syncthreads();

    // b' = sum_m W[m] B[-m]: B[0] for m = 0, -B[N - m] otherwise
    uint32_t pb[LIN_JT];
#pragma unroll
    for (int jt = 0; jt < LIN_JT; ++jt) pb[jt] = 0u;
    for (int m = tid; m < N; m += LIN_NT) {
        const uint32_t bv = m == 0 ? b_in[0] : 0u - b_in[N - m];
#pragma unroll
        for (int jt = 0; jt < LIN_JT; ++jt) pb[jt] += (uint32_t)Ws[jt * N + m] * bv;
    }
#pragma unroll
    for (int jt = 0; jt < LIN_JT; ++jt) {
        uint32_t v = pb[jt];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((tid & 31) == 0) red[jt][tid >> 5] = v;
    }

    // every thread owns coefficients c = tid + LIN_NT * r of P_A
    constexpr int CPT_MAX = 16;                      // N <= 4096
    uint32_t acc[LIN_JT][CPT_MAX];
    const int cpt = N / LIN_NT > 0 ? N / LIN_NT : 1;
#pragma unroll
    for (int jt = 0; jt < LIN_JT; ++jt)
#pragma unroll
        for (int r = 0; r < CPT_MAX; ++r) acc[jt][r] = 0u;
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
            const uint32_t v = idx >= 0 ? A[idx] : 0u - A[idx + N];
#pragma unroll
            for (int jt = 0; jt < LIN_JT; ++jt) acc[jt][r] += (uint32_t)w[jt] * v;
        }
    }
    __syncthreads();
#pragma unroll
    for (int jt = 0; jt < LIN_JT; ++jt) {
        const int j = j0 + jt;
        if (j >= J) break;
        uint32_t* dst = out_a + (s * J + j) * (long long)N;
#pragma unroll
        for (int r = 0; r < CPT_MAX; ++r) {
            if (r >= cpt) break;
            const int c = tid + LIN_NT * r;
            if (c >= N) break;
            if (c == 0) dst[0] = acc[jt][r];
            else dst[N - c] = 0u - acc[jt][r];
        }
        if (tid == 0) {
            uint32_t v = (uint32_t)bias[j];
            for (int w = 0; w < LIN_NT / 32; ++w) v += red[jt][w];
            out_b[s * J + j] = v;
        }
    }
}

// ---------------------------------------------------------------- LUT x RLWE
// out[s][k] = sum_{g < G} P[g][k](X) * ct[s][g][k] (both polynomials),
// the products of prepare_LUT (nn_tfhe/activation.py:103-106) summed over
// the packed sub-LUTs (Spike_LSTM.py:129-132, 160-163).
constexpr int LM_NT = 256;

__global__ void __launch_bounds__(LM_NT) lut_mul_sum_kernel(const int32_t* __restrict__ P, int G, int Kp,
                                                            const uint32_t* __restrict__ ct, int N,
                                                            uint32_t* __restrict__ out) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint32_t* A = reinterpret_cast<uint32_t*>(smem_raw);   // N
    uint32_t* B = A + N;                                    // N
    int32_t* Ps = reinterpret_cast<int32_t*>(B + N);        // N
    const int tid = threadIdx.x;
    const int k = blockIdx.x;
    const long long s = blockIdx.y;
    constexpr int CPT_MAX = 16;
    const int cpt = N / LM_NT > 0 ? N / LM_NT : 1;
    uint32_t acc_a[CPT_MAX], acc_b[CPT_MAX];
#pragma unroll
    for (int r = 0; r < CPT_MAX; ++r) acc_a[r] = acc_b[r] = 0u;
    for (int g = 0; g < G; ++g) {
        const uint32_t* src = ct + ((s * G + g) * (long long)Kp + k) * 2 * N;
        const int32_t* lut = P + ((long long)g * Kp + k) * N;
        for (int i = tid; i < N; i += LM_NT) {
            A[i] = src[i];
            B[i] = src[N + i];
            Ps[i] = lut[i];
        }
        __syncthreads();
        for (int m = 0; m < N; ++m) {
            const int32_t w = Ps[m];
            if (w == 0) continue;                     // uniform across the CTA
#pragma unroll
            for (int r = 0; r < CPT_MAX; ++r) {
                if (r >= cpt) break;
                const int c = tid + LM_NT * r;
                if (c >= N) break;
                const int idx = c - m;
                const uint32_t va = idx >= 0 ? A[idx] : 0u - A[idx + N];
                const uint32_t vb = idx >= 0 ? B[idx] : 0u - B[idx + N];
                acc_a[r] += (uint32_t)w * va;
                acc_b[r] += (uint32_t)w * vb;
            }
        }
        __syncthreads();
    }
    uint32_t* dst = out + (s * Kp + k) * 2 * (long long)N;
#pragma unroll
    for (int r = 0; r < CPT_MAX; ++r) {
        if (r >= cpt) break;
        const int c = tid + LM_NT * r;
        if (c >= N) break;
        dst[c] = acc_a[r];
        dst[N + c] = acc_b[r];
    }
}

// ---------------------------------------------------------------- trace
struct TraceArgs {
    const uint32_t* lwe_a;     // (R, N)
    const uint32_t* lwe_b;     // (R)
    const double2* key;        // [step][level][2][H] position order
    const double2* qt;
    const double2* tw;
    int log2_beta, l, steps;
    uint32_t* out;             // (R, 2, N)
};

template <int LOGH, int s>
__device__ __forceinline__ void forward_all(double2* polys, int npoly, const double2* tw, int tid, int nt) {
    if constexpr (s < Plan<LOGH>::NS) {
        stage_all<LOGH, s, false>(polys, npoly, tw, tid, nt);
        __syncthreads();
        forward_all<LOGH, s + 1>(polys, npoly, tw, tid, nt);
    }
}

template <int LOGH, int s>
__device__ __forceinline__ void inverse_all(double2* polys, int npoly, const double2* tw, int tid, int nt) {
    if constexpr (s >= 0) {
        stage_all<LOGH, s, true>(polys, npoly, tw, tid, nt);
        __syncthreads();
        inverse_all<LOGH, s - 1>(polys, npoly, tw, tid, nt);
    }
}

__device__ __forceinline__ double cmod_q32(double x) {
    const double q = 4294967296.0;
    return x - q * rint(x * (1.0 / q));
}

// pack_lwe_to_rlwe (schemas/text_jax.py:316-345) for one LWE per CTA:
//   lwe <- round(lwe / N) (modulus_switch to q/N, text_jax.py:173-187)
//   rlwe = trivial_embedding(lwe) (A[0] = a[0], A[i] = -a[N-i], B[0] = b)
//   for step i: k = 2^(log2 N - i) + 1,
//     (A', B') = automorphism X -> X^k of (A, B),
//     (A_ks, B_ks) = sum_j dec_j(A')(X) * galois_key[i][j]  (FP64, rounded)
//     rlwe += (cmod(A_ks), cmod(B' + B_ks))   (no reduction of the sum)
// The output is reduced modulo 2^32.
template <int LOGN>
__global__ void __launch_bounds__(256) trace_pack_kernel(const TraceArgs args) {
    constexpr int N = 1 << LOGN;
    constexpr int H = N / 2;
    constexpr int LOGH = LOGN - 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* dig = reinterpret_cast<double2*>(smem_raw);        // l * H
    double2* res = dig + (size_t)args.l * H;                     // 2 * H
    double* accA = reinterpret_cast<double*>(res + 2 * H);       // N
    double* accB = accA + N;                                     // N
    double* permA = accB + N;                                    // N
    double* permB = permA + N;                                   // N
    const int tid = threadIdx.x, nt = blockDim.x;
    const long long r = blockIdx.x;
    const double q = 4294967296.0, inv_q = 1.0 / q;
    const double beta = ldexp(1.0, args.log2_beta);
    constexpr double inv_h = 1.0 / H;
    constexpr double inv_n = 1.0 / N;

    const uint32_t* a = args.lwe_a + r * N;
    for (int i = tid; i < N; i += nt) {
        const double ms = rint((double)(int32_t)a[i == 0 ? 0 : N - i] * inv_n);
        accA[i] = i == 0 ? ms : -ms;
        accB[i] = i == 0 ? rint((double)(int32_t)args.lwe_b[r] * inv_n) : 0.0;
    }
    __syncthreads();

    for (int st = 0; st < args.steps; ++st) {
        const int k = (1 << (args.steps - st)) + 1;
        for (int j = tid; j < N; j += nt) {
            const int dst = (int)(((long long)j * k) % (2 * N));
            const int t = dst % N;
            const double sg = dst >= N ? -1.0 : 1.0;
            permA[t] = sg * accA[j];
            permB[t] = sg * accB[j];
        }
        __syncthreads();
        // gadget digits of A' (polynomial_jax.py:90-111), fold + twist
        for (int i = tid; i < H; i += nt) {
            double xl = permA[i] * inv_q, xh = permA[i + H] * inv_q;
            const double2 w = args.qt[i];
            for (int lvl = 0; lvl < args.l; ++lvl) {
                const double yl = xl * beta, yh = xh * beta;
                const double dl = rint(yl), dh = rint(yh);
                xl = yl - dl;
                xh = yh - dh;
                dig[(size_t)lvl * H + swz(i)] = make_double2(fma(w.x, dl, w.y * dh), fma(w.y, dl, -w.x * dh));
            }
        }
        __syncthreads();
        forward_all<LOGH, 0>(dig, args.l, args.tw, tid, nt);
        const double2* key = args.key + (size_t)st * args.l * 2 * H;
        for (int p = tid; p < H; p += nt) {
            double2 o0 = make_double2(0.0, 0.0), o1 = make_double2(0.0, 0.0);
            for (int lvl = 0; lvl < args.l; ++lvl) {
                const double2 d = dig[(size_t)lvl * H + swz(p)];
                c_mac(o0, d, key[((size_t)lvl * 2 + 0) * H + p]);
                c_mac(o1, d, key[((size_t)lvl * 2 + 1) * H + p]);
            }
            res[swz(p)] = o0;
            res[H + swz(p)] = o1;
        }
        __syncthreads();
        inverse_all<LOGH, Plan<LOGH>::NS - 1>(res, 2, args.tw, tid, nt);
        for (int i = tid; i < H; i += nt) {
            const double2 w = c_conj(args.qt[i]);
            const double2 ua = c_mul(w, res[swz(i)]);
            const double2 ub = c_mul(w, res[H + swz(i)]);
            accA[i] += cmod_q32(rint(ua.x * inv_h));
            accA[i + H] += cmod_q32(rint(-ua.y * inv_h));
            accB[i] += cmod_q32(permB[i] + rint(ub.x * inv_h));
            accB[i + H] += cmod_q32(permB[i + H] + rint(-ub.y * inv_h));
        }
        __syncthreads();
    }
    uint32_t* dst = args.out + r * 2 * N;
    for (int i = tid; i < N; i += nt) {
        dst[i] = (uint32_t)(long long)accA[i];
        dst[N + i] = (uint32_t)(long long)accB[i];
    }
}

// integer polynomials (npoly, N) -> folded Fourier (npoly, H), position order
template <int LOGN>
__global__ void __launch_bounds__(256) poly_fft_kernel(const uint32_t* __restrict__ src, long long npoly,
                                                       const double2* qt, const double2* tw,
                                                       double2* __restrict__ dst) {
    constexpr int N = 1 << LOGN;
    constexpr int H = N / 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* buf = reinterpret_cast<double2*>(smem_raw);
    const long long pi = blockIdx.x;
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int i = tid; i < H; i += nt) {
        const double lo = (double)(int32_t)src[pi * N + i];
        const double hi = (double)(int32_t)src[pi * N + i + H];
        const double2 w = qt[i];
        buf[swz(i)] = make_double2(fma(w.x, lo, w.y * hi), fma(w.y, lo, -w.x * hi));
    }
    __syncthreads();
    forward_all<LOGN - 1, 0>(buf, 1, tw, tid, nt);
    for (int p = tid; p < H; p += nt) dst[pi * H + p] = buf[swz(p)];
}

// ---------------------------------------------------------------- packing
// packing (schemas/text_jax.py:211-239): for the LWEs (a_t, b_t), t < T,
//   V_t = sum_{i,j} dec_j(a_t[i]) KSP[i][j]   (KSP[i][j] = (pk, b) of the
//   GLEV row of lwe_sk[i], get_packing_KSK, schemas/RLWE_jax.py:205-215)
//   result = (-sum_t X^t V_t^pk, packed_b - sum_t X^t V_t^b), packed_b[t] = b_t
// as a u32 contraction (rows = LWEs, columns = the 2N words of V) whose
// epilogue adds -X^t V_t into the packed RLWE with atomics (integer
// additions modulo 2^32 commute, so the result is deterministic).
constexpr int PK_TB = 64, PK_TO = 64, PK_KC = 16, PK_LMAX = 4;

__global__ void __launch_bounds__(256) pack_ks_kernel(const uint32_t* __restrict__ lwe_a, int n_dim, int T,
                                                      long long S, const uint32_t* __restrict__ ksp, int N,
                                                      int l, int log2_beta, uint32_t* __restrict__ out) {
    __shared__ int dig[PK_TB][PK_KC * PK_LMAX + 1];
    __shared__ __align__(16) uint32_t kt[PK_KC * PK_LMAX][PK_TO];
    const int tid = threadIdx.x;
    const int ty = tid / 16, tx = tid % 16;
    const long long r0 = (long long)blockIdx.y * PK_TB;
    const int o0 = blockIdx.x * PK_TO;
    const long long rows_total = S * T;
    const double inv_q = ldexp(1.0, -32);
    const double beta = ldexp(1.0, log2_beta);
    const int cols = 2 * N;
    uint32_t acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0u;
    for (int i0 = 0; i0 < n_dim; i0 += PK_KC) {
        for (int idx = tid; idx < PK_TB * PK_KC; idx += 256) {
            const int rr = idx / PK_KC, c = idx % PK_KC;
            const long long row = r0 + rr;
            const int i = i0 + c;
            const uint32_t v = (row < rows_total && i < n_dim) ? lwe_a[row * n_dim + i] : 0u;
            double x = (double)(int32_t)v * inv_q;
            for (int j = 0; j < l; ++j) {
                const double y = x * beta;
                const double d = rint(y);
                x = y - d;
                dig[rr][c * l + j] = (int)d;
            }
        }
        const int krows = PK_KC * l;
        for (int idx = tid; idx < krows * PK_TO; idx += 256) {
            const int kr = idx / PK_TO, col = idx % PK_TO;
            const int i = i0 + kr / l, j = kr % l;
            const int o = o0 + col;
            kt[kr][col] = (i < n_dim && o < cols) ? ksp[((long long)i * l + j) * cols + o] : 0u;
        }
        __syncthreads();
        for (int kr = 0; kr < krows; ++kr) {
            const uint4 kv = *reinterpret_cast<const uint4*>(&kt[kr][tx * 4]);
#pragma unroll
            for (int cc = 0; cc < 4; ++cc) {
                const uint32_t d = (uint32_t)dig[ty * 4 + cc][kr];
                acc[cc][0] += d * kv.x;
                acc[cc][1] += d * kv.y;
                acc[cc][2] += d * kv.z;
                acc[cc][3] += d * kv.w;
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
            uint32_t v = 0u - acc[cc][e];
            if (d >= N) {
                d -= N;
                v = acc[cc][e];
            }
            atomicAdd(out + (s * 2 + poly) * (long long)N + d, v);
        }
    }
}

__global__ void pack_init_kernel(const uint32_t* __restrict__ lwe_b, int T, long long S, int N,
                                 uint32_t* __restrict__ out) {
    const long long total = S * 2 * (long long)N;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long s = i / (2 * N);
        const int rem = (int)(i - s * 2 * N);
        const int poly = rem / N, c = rem - poly * N;
        out[i] = (poly == 1 && c < T) ? lwe_b[s * T + c] : 0u;
    }
}

// ---------------------------------------------------------------- small ops
// out[s] = X^rot * x[s] + y[s] (y may be null): rotate_ciphertext
// (schemas/text_jax.py:348-362) and sum_ciphertext_ciphertext (:24-41)
__global__ void rlwe_rotate_add_kernel(const uint32_t* __restrict__ x, int rot, const uint32_t* __restrict__ y,
                                       long long S, int N, uint32_t* __restrict__ out) {
    const long long total = S * 2 * (long long)N;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long row = i / N;
        const int c = (int)(i - row * N);
        int src = c - rot;                         // rot in [0, 2N): src in (-2N, N)
        int wraps = 0;
        if (src < 0) {
            src += N;
            ++wraps;
        }
        if (src < 0) {
            src += N;
            ++wraps;
        }
        uint32_t v = x[row * N + src];
        if (wraps & 1) v = 0u - v;
        out[i] = v + (y ? y[i] : 0u);
    }
}

__global__ void u32_add_kernel(const uint32_t* __restrict__ x, const uint32_t* __restrict__ y, long long n,
                               uint32_t* __restrict__ out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = x[i] + y[i];
}

static int grid_for(long long total) {
    return (int)std::max<long long>(1, std::min<long long>((total + 255) / 256, 148LL * 16));
}

}  // namespace tfhe

// ================================================================ C ABI
using namespace tfhe;

struct tfhe_packing_key {
    int n_dim = 0, N = 0, log2_beta = 0, l = 0, device = 0;
    uint32_t* ksp = nullptr;        // (n_dim, l, 2, N)
    int8_t* limbs = nullptr;        // (8 N, n_dim l) int8 limbs for the tensor cores, or null
};

struct tfhe_galois_keys {
    int N = 0, log2_beta = 0, l = 0, steps = 0, device = 0;
    double2* key = nullptr;     // [steps][l][2][H]
};

namespace {

int log2_exact(long long v) {
    int r = 0;
    while ((1LL << r) < v) ++r;
    return (1LL << r) == v ? r : -1;
}

bool valid_degree(int N) { return N >= 128 && N <= 4096 && log2_exact(N) > 0; }

size_t trace_smem(int N, int l) {
    const size_t H = N / 2;
    return (size_t)(l + 2) * H * sizeof(double2) + 4 * (size_t)N * sizeof(double);
}

int max_smem() {
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    return v;
}

template <int LOGN>
int launch_trace(const TraceArgs& a, long long R, size_t smem, cudaStream_t stream) {
    auto kern = trace_pack_kernel<LOGN>;
    TFHE_TRY(smem_attr_once((const void*)kern, smem));
    count_launch();
    kern<<<(unsigned)R, 256, smem, stream>>>(a);
    return check_cuda(cudaGetLastError(), "trace kernel launch");
}

template <int LOGN>
int launch_poly_fft(const uint32_t* src, long long npoly, const FftPlan* pl, double2* dst, cudaStream_t stream) {
    const size_t smem = (size_t)(1 << (LOGN - 1)) * sizeof(double2);
    count_launch();
    poly_fft_kernel<LOGN><<<(unsigned)npoly, 256, smem, stream>>>(src, npoly, pl->qt, pl->tw, dst);
    return check_cuda(cudaGetLastError(), "polynomial FFT launch");
}

int dispatch_trace(int N, const TraceArgs& a, long long R, size_t smem, cudaStream_t stream) {
    switch (log2_exact(N)) {
        case 7: return launch_trace<7>(a, R, smem, stream);
        case 8: return launch_trace<8>(a, R, smem, stream);
        case 9: return launch_trace<9>(a, R, smem, stream);
        case 10: return launch_trace<10>(a, R, smem, stream);
        case 11: return launch_trace<11>(a, R, smem, stream);
        case 12: return launch_trace<12>(a, R, smem, stream);
        default: return fail(TFHE_ERR_INVALID_ARGUMENT, "degree must be a power of two in [128, 4096]");
    }
}

int dispatch_poly_fft(int N, const uint32_t* src, long long npoly, const FftPlan* pl, double2* dst,
                      cudaStream_t stream) {
    switch (log2_exact(N)) {
        case 7: return launch_poly_fft<7>(src, npoly, pl, dst, stream);
        case 8: return launch_poly_fft<8>(src, npoly, pl, dst, stream);
        case 9: return launch_poly_fft<9>(src, npoly, pl, dst, stream);
        case 10: return launch_poly_fft<10>(src, npoly, pl, dst, stream);
        case 11: return launch_poly_fft<11>(src, npoly, pl, dst, stream);
        case 12: return launch_poly_fft<12>(src, npoly, pl, dst, stream);
        default: return fail(TFHE_ERR_INVALID_ARGUMENT, "degree must be a power of two in [128, 4096]");
    }
}

}  // namespace

extern "C" {

int tfhe_linear_extract(const int32_t* weights, const int32_t* bias, int32_t J, const uint32_t* rlwe, int64_t S,
                        int32_t N, uint32_t* out_a, uint32_t* out_b, void* stream) {
    if (!valid_degree(N)) return fail(TFHE_ERR_INVALID_ARGUMENT, "linear: N must be a power of two in [128, 4096]");
    if (J < 0 || S < 0) return fail(TFHE_ERR_INVALID_ARGUMENT, "linear: negative size");
    if (J == 0 || S == 0) return TFHE_OK;
    if (!weights || !bias || !rlwe || !out_a || !out_b)
        return fail(TFHE_ERR_INVALID_ARGUMENT, "linear: null pointer");
    if (S > 65535) return fail(TFHE_ERR_INVALID_ARGUMENT, "linear: at most 65535 ciphertexts per call");
    const size_t smem = (size_t)N * sizeof(uint32_t) + (size_t)LIN_JT * N * sizeof(int32_t);
    TFHE_TRY(smem_attr_once((const void*)linear_extract_kernel, smem));
    const dim3 grid((J + LIN_JT - 1) / LIN_JT, (unsigned)S);
    count_launch();
    linear_extract_kernel<<<grid, LIN_NT, smem, (cudaStream_t)stream>>>(weights, bias, J, rlwe, N, out_a, out_b);
    return check_cuda(cudaGetLastError(), "linear kernel launch");
}

int tfhe_lut_mul_sum(const int32_t* luts, int32_t groups, int32_t per_group, const uint32_t* rlwe, int64_t S,
                     int32_t N, uint32_t* out, void* stream) {
    if (!valid_degree(N)) return fail(TFHE_ERR_INVALID_ARGUMENT, "lut product: N must be a power of two in [128, 4096]");
    if (groups < 1 || per_group < 0 || S < 0) return fail(TFHE_ERR_INVALID_ARGUMENT, "lut product: bad sizes");
    if (per_group == 0 || S == 0) return TFHE_OK;
    if (!luts || !rlwe || !out) return fail(TFHE_ERR_INVALID_ARGUMENT, "lut product: null pointer");
    if (S > 65535) return fail(TFHE_ERR_INVALID_ARGUMENT, "lut product: at most 65535 sequences per call");
    const size_t smem = 3 * (size_t)N * sizeof(uint32_t);
    TFHE_TRY(smem_attr_once((const void*)lut_mul_sum_kernel, smem));
    const dim3 grid((unsigned)per_group, (unsigned)S);
    count_launch();
    lut_mul_sum_kernel<<<grid, LM_NT, smem, (cudaStream_t)stream>>>(luts, groups, per_group, rlwe, N, out);
    return check_cuda(cudaGetLastError(), "lut product launch");
}

int tfhe_galois_keys_create(int32_t N, int32_t log2_beta, int32_t l, const uint32_t* keys, void* stream,
                            tfhe_galois_keys** out) {
    // keys: device u32 (log2 N steps, l, 2, N): step i is the key switching
    // key from the automorphism X -> X^(2^(log2 N - i) + 1) of the secret
    // back to the secret (get_galois_key, schemas/RLWE_jax.py:218-226)
    if (!out) return fail(TFHE_ERR_INVALID_ARGUMENT, "galois keys: null output");
    *out = nullptr;
    if (!valid_degree(N)) return fail(TFHE_ERR_INVALID_ARGUMENT, "galois keys: N must be a power of two in [128, 4096]");
    if (l < 1 || l > 16 || log2_beta < 1 || log2_beta * l > 32)
        return fail(TFHE_ERR_INVALID_ARGUMENT, "galois keys: need 1 <= l <= 16 and l * log2_beta <= 32");
    if (!keys) return fail(TFHE_ERR_INVALID_ARGUMENT, "galois keys: null key pointer");
    if (trace_smem(N, l) > (size_t)max_smem())
        return fail(TFHE_ERR_INVALID_ARGUMENT, "galois keys: l levels at this degree exceed shared memory");
    const FftPlan* pl = get_plan(N);
    if (!pl) return TFHE_ERR_INTERNAL;
    auto* gk = new tfhe_galois_keys();
    gk->N = N;
    gk->log2_beta = log2_beta;
    gk->l = l;
    gk->steps = log2_exact(N);
    cudaGetDevice(&gk->device);
    const long long npoly = (long long)gk->steps * l * 2;
    int rc = check_cuda(cudaMalloc(&gk->key, (size_t)npoly * (N / 2) * sizeof(double2)), "cudaMalloc(galois key)");
    if (rc == TFHE_OK) rc = dispatch_poly_fft(N, keys, npoly, pl, gk->key, (cudaStream_t)stream);
    if (rc == TFHE_OK) rc = check_cuda(cudaStreamSynchronize((cudaStream_t)stream), "galois key upload");
    if (rc != TFHE_OK) {
        cudaFree(gk->key);
        delete gk;
        return rc;
    }
    *out = gk;
    return TFHE_OK;
}

int tfhe_galois_keys_destroy(tfhe_galois_keys* gk) {
    if (!gk) return TFHE_OK;
    cudaFree(gk->key);
    delete gk;
    return TFHE_OK;
}

int tfhe_pack_lwe_to_rlwe(const tfhe_galois_keys* gk, const uint32_t* lwe_a, const uint32_t* lwe_b, int64_t R,
                          uint32_t* out, void* stream) {
    if (!gk) return fail(TFHE_ERR_INVALID_ARGUMENT, "pack_lwe_to_rlwe: null keys");
    if (R < 0) return fail(TFHE_ERR_INVALID_ARGUMENT, "pack_lwe_to_rlwe: negative count");
    if (R == 0) return TFHE_OK;
    if (!lwe_a || !lwe_b || !out) return fail(TFHE_ERR_INVALID_ARGUMENT, "pack_lwe_to_rlwe: null pointer");
    if (R > 2147483647LL) return fail(TFHE_ERR_INVALID_ARGUMENT, "pack_lwe_to_rlwe: too many ciphertexts");
    const FftPlan* pl = get_plan(gk->N);
    if (!pl) return TFHE_ERR_INTERNAL;
    TraceArgs a{lwe_a, lwe_b, gk->key, pl->qt, pl->tw, gk->log2_beta, gk->l, gk->steps, out};
    return dispatch_trace(gk->N, a, R, trace_smem(gk->N, gk->l), (cudaStream_t)stream);
}

int tfhe_pack_lwes(const uint32_t* ksp, int32_t n_dim, int32_t N, int32_t log2_beta, int32_t l,
                   const uint32_t* lwe_a, const uint32_t* lwe_b, int32_t T, int64_t S, uint32_t* out, void* stream) {
    if (!valid_degree(N)) return fail(TFHE_ERR_INVALID_ARGUMENT, "packing: N must be a power of two in [128, 4096]");
    if (l < 1 || l > PK_LMAX || log2_beta < 1 || log2_beta * l > 32)
        return fail(TFHE_ERR_INVALID_ARGUMENT, "packing: need 1 <= l <= 4 and l * log2_beta <= 32");
    if (n_dim < 1 || T < 0 || T > N || S < 0) return fail(TFHE_ERR_INVALID_ARGUMENT, "packing: bad sizes (T <= N)");
    if (S == 0) return TFHE_OK;
    if (!ksp || !out || (T > 0 && (!lwe_a || !lwe_b))) return fail(TFHE_ERR_INVALID_ARGUMENT, "packing: null pointer");
    const long long total = S * 2 * (long long)N;
    count_launch();
    pack_init_kernel<<<grid_for(total), 256, 0, (cudaStream_t)stream>>>(lwe_b, T, S, N, out);
    const int rc = check_cuda(cudaGetLastError(), "packing init launch");
    if (rc != TFHE_OK) return rc;
    if (T == 0) return TFHE_OK;
    const long long rows = S * T;
    if ((rows + PK_TB - 1) / PK_TB > 65535) return fail(TFHE_ERR_INVALID_ARGUMENT, "packing: too many LWEs per call");
    const dim3 grid((2 * N + PK_TO - 1) / PK_TO, (unsigned)((rows + PK_TB - 1) / PK_TB));
    count_launch();
    pack_ks_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(lwe_a, n_dim, T, S, ksp, N, l, log2_beta, out);
    return check_cuda(cudaGetLastError(), "packing launch");
}

int tfhe_packing_key_create(const uint32_t* ksp, int32_t n_dim, int32_t N, int32_t log2_beta, int32_t l,
                            void* stream, tfhe_packing_key** out) {
    if (!out) return fail(TFHE_ERR_INVALID_ARGUMENT, "packing key: null output");
    *out = nullptr;
    if (!valid_degree(N)) return fail(TFHE_ERR_INVALID_ARGUMENT, "packing key: N must be a power of two in [128, 4096]");
    if (l < 1 || l > PK_LMAX || log2_beta < 1 || log2_beta * l > 32 || n_dim < 1)
        return fail(TFHE_ERR_INVALID_ARGUMENT, "packing key: need n_dim >= 1, 1 <= l <= 4, l * log2_beta <= 32");
    if (!ksp) return fail(TFHE_ERR_INVALID_ARGUMENT, "packing key: null key");
    cudaStream_t st = (cudaStream_t)stream;
    auto* k = new tfhe_packing_key();
    k->n_dim = n_dim;
    k->N = N;
    k->log2_beta = log2_beta;
    k->l = l;
    cudaGetDevice(&k->device);
    const size_t words = (size_t)n_dim * l * 2 * N;
    int rc = check_cuda(cudaMalloc(&k->ksp, words * sizeof(uint32_t)), "cudaMalloc(packing key)");
    if (rc == TFHE_OK)
        rc = check_cuda(cudaMemcpyAsync(k->ksp, ksp, words * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st),
                        "packing key copy");
    // int8 limbs where the digits fit int8 and the int32 sums cannot overflow
    const long long K = (long long)n_dim * l;
    const bool tc = log2_beta <= 7 && n_dim % 32 == 0 && K * (1LL << (log2_beta - 1)) * 128 < (1LL << 31) &&
                    (8 * N) % ks_tc_columns() == 0;
    if (rc == TFHE_OK && tc) {
        rc = check_cuda(cudaMalloc(&k->limbs, (size_t)8 * N * K), "cudaMalloc(packing limbs)");
        if (rc == TFHE_OK) rc = build_packing_limbs(k->ksp, n_dim, l, N, k->limbs, st);
    }
    if (rc == TFHE_OK) rc = check_cuda(cudaStreamSynchronize(st), "packing key upload");
    if (rc != TFHE_OK) {
        cudaFree(k->ksp);
        cudaFree(k->limbs);
        delete k;
        return rc;
    }
    *out = k;
    return TFHE_OK;
}

int tfhe_packing_key_destroy(tfhe_packing_key* key) {
    if (!key) return TFHE_OK;
    cudaFree(key->ksp);
    cudaFree(key->limbs);
    delete key;
    return TFHE_OK;
}

int tfhe_packing_key_uses_tensor_cores(const tfhe_packing_key* key) { return key && key->limbs ? 1 : 0; }

int tfhe_pack_lwes_with_key(const tfhe_packing_key* key, const uint32_t* lwe_a, const uint32_t* lwe_b, int32_t T,
                            int64_t S, uint32_t* out, int32_t tensor_cores, void* stream) {
    if (!key) return fail(TFHE_ERR_INVALID_ARGUMENT, "packing: null key");
    if (tensor_cores < -1 || tensor_cores > 1) return fail(TFHE_ERR_INVALID_ARGUMENT, "packing: tensor_cores in {-1, 0, 1}");
    const int N = key->N;
    const bool tc = key->limbs && tensor_cores != 0 && T > 0 && (reinterpret_cast<uintptr_t>(lwe_a) & 15) == 0;
    if (!tc) return tfhe_pack_lwes(key->ksp, key->n_dim, N, key->log2_beta, key->l, lwe_a, lwe_b, T, S, out, stream);
    if (T > N || S < 0) return fail(TFHE_ERR_INVALID_ARGUMENT, "packing: bad sizes (T <= N)");
    if (S == 0) return TFHE_OK;
    if (!lwe_a || !lwe_b || !out) return fail(TFHE_ERR_INVALID_ARGUMENT, "packing: null pointer");
    const long long total = S * 2 * (long long)N;
    count_launch();
    pack_init_kernel<<<grid_for(total), 256, 0, (cudaStream_t)stream>>>(lwe_b, T, S, N, out);
    const int rc = check_cuda(cudaGetLastError(), "packing init launch");
    if (rc != TFHE_OK) return rc;
    KsTcArgs a{lwe_a, nullptr, reinterpret_cast<const unsigned char*>(key->limbs), key->n_dim, 0, key->l,
               key->log2_beta, 8 * N, S * T, nullptr, nullptr, WAIT_LIMIT_CYCLES, device_status_word(), T, N, out,
               false, true};
    return launch_ks_tc(a, (cudaStream_t)stream);
}

int tfhe_rlwe_rotate_add(const uint32_t* x, int32_t rot, const uint32_t* y, int64_t S, int32_t N, uint32_t* out,
                         void* stream) {
    if (!valid_degree(N)) return fail(TFHE_ERR_INVALID_ARGUMENT, "rotate/add: N must be a power of two in [128, 4096]");
    if (S < 0) return fail(TFHE_ERR_INVALID_ARGUMENT, "rotate/add: negative count");
    if (S == 0) return TFHE_OK;
    if (!x || !out) return fail(TFHE_ERR_INVALID_ARGUMENT, "rotate/add: null pointer");
    if (x == out && rot % (2 * N) != 0)
        return fail(TFHE_ERR_INVALID_ARGUMENT, "rotate/add: out may not alias x when rotating");
    const int r = ((rot % (2 * N)) + 2 * N) % (2 * N);
    count_launch();
    rlwe_rotate_add_kernel<<<grid_for(S * 2 * (long long)N), 256, 0, (cudaStream_t)stream>>>(x, r, y, S, N, out);
    return check_cuda(cudaGetLastError(), "rotate/add launch");
}

int tfhe_u32_add(const uint32_t* x, const uint32_t* y, int64_t n, uint32_t* out, void* stream) {
    if (n < 0) return fail(TFHE_ERR_INVALID_ARGUMENT, "add: negative count");
    if (n == 0) return TFHE_OK;
    if (!x || !y || !out) return fail(TFHE_ERR_INVALID_ARGUMENT, "add: null pointer");
    count_launch();
    u32_add_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(x, y, n, out);
    return check_cuda(cudaGetLastError(), "add launch");
}

}  // extern "C"
