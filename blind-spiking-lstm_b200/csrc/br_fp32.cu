// The FP32 split-limb form of the blind rotation (the precision ablation of
// the external product): the collapsed CMux chain of multiply_seq_monomial
// (schemas/text_jax.py:390-435, cuTFHE/multiply.py:54-92) with every FFT in
// FP32 and the bootstrapping key split into P signed limbs,
//   K = sum_t limb_t 2^(s_t),   s_t = t * ceil(32 / P)  (limb widths 16.16,
//   11.11.10, 8.8.8.8),
// so that each limb's product with the gadget digits is an FP32 FFT product
// that rounds to an integer; the limb results are recombined exactly,
//   ACC' = sum_t round(y_t) 2^(s_t)  mod 2^32.
// Where |y_t| or the FFT's rounding exceed FP32's 24-bit mantissa the rounded
// limb result is off by some units, shifted by 2^(s_t): that error is what the
// ablation measures against the FP64 engine and the exact integer product.
//
// Layout: one CTA holds K ciphertexts, 256 threads.  The H = N/2-point
// negacyclic folding (z_i = psi^i (p_i - i p_{i+H}), psi = e^(-i pi / N),
// evaluation at psi^(4j+1)) of the FP64 kernel, with a radix-2 DIF forward
// transform (natural -> bit-reversed order) and DIT inverse (bit-reversed ->
// natural), all in shared memory.  Keys are stored as FP32 spectra times 1/H
// in bit-reversed position order: [G][2 out][2 in][L][M][P][H] float2.
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "tfhe_b200.h"
#include "tfhe_dispatch.h"
#include "tfhe_internal.cuh"

namespace tfhe {
namespace f32 {

constexpr int NT = 256;

struct Tables {
    float2* root = nullptr;   // 2N: e^(-i pi k / N)
    float2* tw = nullptr;     // H/2: e^(-2 pi i k / H)
};

struct Args {
    const float2* bsk;        // [G][2][2][L][M][P][H]
    const float2* root;
    const float2* tw;
    int G, M, collapse, P;
    long long B;
    const uint32_t* lwe_a;    // (B, n)
    const uint32_t* lwe_b;    // (B)
    const uint32_t* lut;      // (B|1, 2, N)
    long long lut_stride;
    int n_lut, lwe_n;
    int log2_beta;
    uint32_t* out_a;          // (B, n_lut, N)
    uint32_t* out_b;          // (B, n_lut)
    uint32_t* acc_out;        // (B, 2, N): the accumulator after the chain, unrotated (or null)
};

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {     // a * conj(b)
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ void cmac(float2& acc, float2 a, float2 b) {
    acc.x = fmaf(a.x, b.x, fmaf(-a.y, b.y, acc.x));
    acc.y = fmaf(a.x, b.y, fmaf(a.y, b.x, acc.y));
}

// forward DIF over npoly contiguous H-point polynomials: natural -> bit-reversed
template <int LOGH>
__device__ __forceinline__ void fft_fwd(float2* x, int npoly, const float2* tw) {
    constexpr int H = 1 << LOGH;
    for (int s = 0; s < LOGH; ++s) {
        const int lspan = LOGH - 1 - s, span = 1 << lspan;
        for (int idx = threadIdx.x; idx < npoly * (H / 2); idx += NT) {
            const int poly = idx >> (LOGH - 1), b = idx & (H / 2 - 1);
            const int pos = b & (span - 1);
            const int i0 = ((b >> lspan) << (lspan + 1)) + pos, i1 = i0 + span;
            float2* y = x + (size_t)poly * H;
            const float2 u = y[i0], v = y[i1];
            y[i0] = make_float2(u.x + v.x, u.y + v.y);
            y[i1] = cmul(make_float2(u.x - v.x, u.y - v.y), tw[pos << s]);
        }
        __syncthreads();
    }
}

// inverse DIT: bit-reversed -> natural, unnormalised (times H)
template <int LOGH>
__device__ __forceinline__ void fft_inv(float2* x, int npoly, const float2* tw) {
    constexpr int H = 1 << LOGH;
    for (int s = LOGH - 1; s >= 0; --s) {
        const int lspan = LOGH - 1 - s, span = 1 << lspan;
        for (int idx = threadIdx.x; idx < npoly * (H / 2); idx += NT) {
            const int poly = idx >> (LOGH - 1), b = idx & (H / 2 - 1);
            const int pos = b & (span - 1);
            const int i0 = ((b >> lspan) << (lspan + 1)) + pos, i1 = i0 + span;
            float2* y = x + (size_t)poly * H;
            const float2 u = y[i0], v = cmulc(y[i1], tw[pos << s]);
            y[i0] = make_float2(u.x + v.x, u.y + v.y);
            y[i1] = make_float2(u.x - v.x, u.y - v.y);
        }
        __syncthreads();
    }
}

__device__ __forceinline__ int limb_shift(int t, int P) { return t * ((32 + P - 1) / P); }

// signed limb t of a centred 32-bit word (limb widths ceil(32/P), the last
// limb takes the rest): sum_t limb_t 2^(s_t) == v exactly
__device__ __forceinline__ int limb_of(int v, int t, int P) {
    long long r = v;
    const int w = (32 + P - 1) / P;
    int lo = 0;
    for (int i = 0; i <= t; ++i) {
        if (i == P - 1) return (int)r;
        const long long half = 1LL << (w - 1), mod = 1LL << w;
        lo = (int)(((r + half) & (mod - 1)) - half);
        r = (r - lo) >> w;
    }
    return lo;
}

// key spectra: bsk_coeff (2 side, 2 mask/body, G*M, L, N) uint32 ->
// [G][2 out][2 in][L][M][P][H] FP32 spectra times 1/H, bit-reversed order
template <int LOGN>
__global__ void __launch_bounds__(NT) key_fft32_kernel(const uint32_t* __restrict__ bsk, int G, int M, int L, int P,
                                                       const float2* root, const float2* tw,
                                                       float2* __restrict__ dst) {
    constexpr int N = 1 << LOGN, H = N / 2;
    __shared__ float2 buf[H];
    __shared__ float2 tws[H / 2];
    // blockIdx.x enumerates (g, out, in, l, m, t)
    long long id = blockIdx.x;
    const int t = (int)(id % P); id /= P;
    const int m = (int)(id % M); id /= M;
    const int l = (int)(id % L); id /= L;
    const int in = (int)(id % 2); id /= 2;
    const int out = (int)(id % 2); id /= 2;
    const int g = (int)id;
    for (int i = threadIdx.x; i < H / 2; i += NT) tws[i] = tw[i];
    const uint32_t* src = bsk + ((((size_t)in * 2 + out) * G * M + (size_t)g * M + m) * L + l) * N;
    const float inv_h = 1.0f / H;
    for (int i = threadIdx.x; i < H; i += NT) {
        const float lo = (float)limb_of((int)src[i], t, P) * inv_h;
        const float hi = (float)limb_of((int)src[i + H], t, P) * inv_h;
        buf[i] = cmul(root[i], make_float2(lo, -hi));
    }
    __syncthreads();
    fft_fwd<LOGN - 1>(buf, 1, tws);
    float2* d = dst + (size_t)blockIdx.x * H;
    for (int i = threadIdx.x; i < H; i += NT) d[i] = buf[i];
}

template <int LOGN, int L, int K>
__global__ void __launch_bounds__(NT) br_fp32_kernel(const Args a) {
    constexpr int N = 1 << LOGN, H = N / 2, LOGH = LOGN - 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* spec = reinterpret_cast<float2*>(smem_raw);            // [K][2L][H]
    float2* outs = spec + (size_t)K * 2 * L * H;                    // [K][2][H]
    float2* roots = outs + (size_t)K * 2 * H;                       // [2N]
    float2* tws = roots + 2 * N;                                     // [H/2]
    uint32_t* acc = reinterpret_cast<uint32_t*>(tws + H / 2);       // [K][2][N]
    int* rot = reinterpret_cast<int*>(acc + (size_t)K * 2 * N);     // [K][M]
    const int tid = threadIdx.x;
    const int M = a.M, P = a.P;
    for (int i = tid; i < 2 * N; i += NT) roots[i] = a.root[i];
    for (int i = tid; i < H / 2; i += NT) tws[i] = a.tw[i];
    const long long ct0 = (long long)blockIdx.x * K;
    for (int i = tid; i < K * 2 * N; i += NT) {
        const int k = i / (2 * N);
        const long long ct = min(ct0 + k, a.B - 1);
        acc[i] = a.lut[ct * a.lut_stride + (i - k * 2 * N)];
    }
    const double q = 4294967296.0;
    const double beta = ldexp(1.0, a.log2_beta);
    __syncthreads();

    for (int g = 0; g < a.G; ++g) {
        for (int t = tid; t < K * M; t += NT) {
            const int k = t / M, m = t - k * M;
            const long long ct = min(ct0 + k, a.B - 1);
            double v = 0.0;
            const uint32_t* la = a.lwe_a + ct * a.lwe_n + (long long)g * a.collapse;
            for (int c = 0; c < a.collapse; ++c)
                if ((m >> (a.collapse - 1 - c)) & 1) v += (double)(int32_t)la[c];
            const int ri = (int)(rint((2.0 * N * v) / (q * a.n_lut)) * a.n_lut) % (2 * N);
            rot[t] = ri < 0 ? ri + 2 * N : ri;
        }
        // gadget digits (float64 steps of polynomial_jax.py:90-111), folded
        for (int i = tid; i < K * 2 * H; i += NT) {
            const int k = i / (2 * H), rem = i - k * 2 * H, c = rem / H, j = rem - c * H;
            double xl = (double)(int32_t)acc[(k * 2 + c) * N + j] / q;
            double xh = (double)(int32_t)acc[(k * 2 + c) * N + j + H] / q;
            const float2 w = roots[j];
            for (int lv = 0; lv < L; ++lv) {
                const double yl = xl * beta, yh = xh * beta;
                const double dl = rint(yl), dh = rint(yh);
                xl = yl - dl;
                xh = yh - dh;
                spec[((size_t)k * 2 * L + c * L + lv) * H + j] = cmul(w, make_float2((float)dl, (float)-dh));
            }
        }
        __syncthreads();
        fft_fwd<LOGH>(spec, K * 2 * L, tws);
        for (int i = tid; i < K * 2 * N; i += NT) acc[i] = 0u;
        const float2* kg = a.bsk + (size_t)g * 2 * 2 * L * M * P * H;
        for (int t = 0; t < P; ++t) {
            for (int p = tid; p < H; p += NT) {
                const int f = (int)(__brev((unsigned)p) >> (32 - LOGH));
                const int ex = 4 * f + 1;
                float2 Y[K][2];
#pragma unroll
                for (int k = 0; k < K; ++k) Y[k][0] = Y[k][1] = make_float2(0.f, 0.f);
                for (int c = 0; c < 2; ++c) {
                    for (int lv = 0; lv < L; ++lv) {
                        float2 d[K];
#pragma unroll
                        for (int k = 0; k < K; ++k) d[k] = spec[((size_t)k * 2 * L + c * L + lv) * H + p];
#pragma unroll
                        for (int o = 0; o < 2; ++o) {
                            float2 S[K];
#pragma unroll
                            for (int k = 0; k < K; ++k) S[k] = make_float2(0.f, 0.f);
                            const float2* kp = kg + ((((size_t)o * 2 + c) * L + lv) * M * P + t) * H + p;
                            for (int m = 0; m < M; ++m) {
                                const float2 key = kp[(size_t)m * P * H];
#pragma unroll
                                for (int k = 0; k < K; ++k) {
                                    const float2 r = roots[(rot[k * M + m] * ex) & (2 * N - 1)];
                                    cmac(S[k], key, r);
                                }
                            }
#pragma unroll
                            for (int k = 0; k < K; ++k) cmac(Y[k][o], d[k], S[k]);
                        }
                    }
                }
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    outs[((size_t)k * 2 + 0) * H + p] = Y[k][0];
                    outs[((size_t)k * 2 + 1) * H + p] = Y[k][1];
                }
            }
            __syncthreads();
            fft_inv<LOGH>(outs, K * 2, tws);
            const int sh = limb_shift(t, P);
            for (int i = tid; i < K * 2 * H; i += NT) {
                const int k = i / (2 * H), rem = i - k * 2 * H, o = rem / H, j = rem - o * H;
                const float2 u = cmulc(outs[((size_t)k * 2 + o) * H + j], roots[j]);
                const long long lo = __float2ll_rn(u.x), hi = __float2ll_rn(-u.y);
                acc[(k * 2 + o) * N + j] += (uint32_t)((unsigned long long)lo << sh);
                acc[(k * 2 + o) * N + j + H] += (uint32_t)((unsigned long long)hi << sh);
            }
            __syncthreads();
        }
    }
    if (a.acc_out) {
        for (int i = tid; i < K * 2 * N; i += NT) {
            const int k = i / (2 * N);
            if (ct0 + k < a.B) a.acc_out[(ct0 + k) * 2 * N + (i - k * 2 * N)] = acc[i];
        }
        return;
    }
    // rotation by -b~ then many-LUT extraction (schemas/RLWE_jax.py:295-303)
    for (int i = tid; i < K * a.n_lut * (N + 1); i += NT) {
        const int k = i / (a.n_lut * (N + 1)), rem = i - k * a.n_lut * (N + 1);
        const long long ct = ct0 + k;
        if (ct >= a.B) continue;
        const double bb = (double)(int32_t)a.lwe_b[ct];
        const int bt = (int)(rint((2.0 * N * bb) / (q * a.n_lut)) * a.n_lut);
        const int al = rem / (N + 1), j = rem - al * (N + 1);
        const uint32_t* ac = acc + (size_t)k * 2 * N;
        int e, src;
        if (j < N) {
            e = al - j + bt;
            src = 0;
        } else {
            e = al + bt;
            src = N;
        }
        e %= 2 * N;
        if (e < 0) e += 2 * N;
        const uint32_t v = e < N ? ac[src + e] : 0u - ac[src + e - N];
        if (j < N) a.out_a[(ct * a.n_lut + al) * (long long)N + j] = v;
        else a.out_b[ct * a.n_lut + al] = v;
    }
}

static std::mutex g_mu;
static std::map<std::pair<int, int>, Tables> g_tables;   // (device, N)

static int tables_for(int N, Tables* out) {
    int dev = 0;
    const cudaError_t ge = cudaGetDevice(&dev);
    if (ge != cudaSuccess) return check_cuda(ge, "cudaGetDevice");
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_tables.find({dev, N});
    if (it != g_tables.end()) {
        *out = it->second;
        return TFHE_OK;
    }
    const int H = N / 2;
    std::vector<float2> root(2 * N), tw(H / 2);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int k = 0; k < 2 * N; ++k) {
        const long double ang = pi * (long double)k / (long double)N;
        root[k] = make_float2((float)cosl(ang), (float)-sinl(ang));
    }
    for (int k = 0; k < H / 2; ++k) {
        const long double ang = 2.0L * pi * (long double)k / (long double)H;
        tw[k] = make_float2((float)cosl(ang), (float)-sinl(ang));
    }
    Tables t;
    int rc = check_cuda(cudaMalloc(&t.root, root.size() * sizeof(float2)), "cudaMalloc(fp32 roots)");
    if (rc == TFHE_OK) rc = check_cuda(cudaMalloc(&t.tw, tw.size() * sizeof(float2)), "cudaMalloc(fp32 twiddles)");
    if (rc == TFHE_OK)
        rc = check_cuda(cudaMemcpy(t.root, root.data(), root.size() * sizeof(float2), cudaMemcpyHostToDevice),
                        "fp32 roots upload");
    if (rc == TFHE_OK)
        rc = check_cuda(cudaMemcpy(t.tw, tw.data(), tw.size() * sizeof(float2), cudaMemcpyHostToDevice),
                        "fp32 twiddles upload");
    if (rc != TFHE_OK) {
        cudaFree(t.root);
        cudaFree(t.tw);
        return rc;
    }
    g_tables[{dev, N}] = t;
    *out = t;
    return TFHE_OK;
}

static size_t smem_bytes(int N, int L, int K, int M) {
    const int H = N / 2;
    return (size_t)K * 2 * L * H * 8 + (size_t)K * 2 * H * 8 + (size_t)2 * N * 8 + (size_t)(H / 2) * 8 +
           (size_t)K * 2 * N * 4 + (size_t)K * M * 4;
}

template <int LOGN, int L, int K>
static int launch_br(const Args& a, cudaStream_t stream) {
    const size_t smem = smem_bytes(1 << LOGN, L, K, a.M);
    TFHE_TRY(smem_attr_once((const void*)br_fp32_kernel<LOGN, L, K>, smem));
    const long long grid = (a.B + K - 1) / K;
    count_launch();
    br_fp32_kernel<LOGN, L, K><<<(unsigned)grid, NT, smem, stream>>>(a);
    return check_cuda(cudaGetLastError(), "fp32 blind rotation launch");
}

template <int LOGN>
static int launch_key_fft(const uint32_t* bsk, int G, int M, int L, int P, const Tables& t, float2* dst,
                          cudaStream_t stream) {
    const long long blocks = (long long)G * 2 * 2 * L * M * P;
    count_launch();
    key_fft32_kernel<LOGN><<<(unsigned)blocks, NT, 0, stream>>>(bsk, G, M, L, P, t.root, t.tw, dst);
    return check_cuda(cudaGetLastError(), "fp32 key FFT launch");
}

}  // namespace f32
}  // namespace tfhe

using namespace tfhe;

struct tfhe_fp32_keys {
    tfhe_params p;
    int G = 0, M = 0, limbs = 0, device = 0;
    float2* bsk = nullptr;
    f32::Tables tables;
};

extern "C" {

int tfhe_fp32_keys_create(const tfhe_params* p, const uint32_t* bsk_coeff, int32_t limbs, void* stream,
                          tfhe_fp32_keys** out) {
    if (!out) return fail(TFHE_ERR_INVALID_ARGUMENT, "fp32 keys: null output");
    *out = nullptr;
    if (!p || !bsk_coeff) return fail(TFHE_ERR_INVALID_ARGUMENT, "fp32 keys: null argument");
    if (p->log2_q != 32) return fail(TFHE_ERR_INVALID_ARGUMENT, "fp32 keys: log2_q must be 32");
    if (p->N != 256 && p->N != 1024 && p->N != 2048)
        return fail(TFHE_ERR_INVALID_ARGUMENT, "fp32 keys: N in {256, 1024, 2048}");
    if (p->l_bs < 1 || p->l_bs > 3 || p->collapse < 1 || p->collapse > 3 || p->n % p->collapse)
        return fail(TFHE_ERR_INVALID_ARGUMENT, "fp32 keys: l_bs <= 3, collapse <= 3 dividing n");
    if (limbs < 2 || limbs > 4) return fail(TFHE_ERR_INVALID_ARGUMENT, "fp32 keys: 2 to 4 limbs");
    auto* k = new tfhe_fp32_keys();
    k->p = *p;
    k->M = 1 << p->collapse;
    k->G = p->n / p->collapse;
    k->limbs = limbs;
    cudaGetDevice(&k->device);
    cudaStream_t st = (cudaStream_t)stream;
    const size_t words = (size_t)2 * 2 * k->G * k->M * p->l_bs * p->N;
    uint32_t* dev_coeff = nullptr;
    int rc = f32::tables_for(p->N, &k->tables);
    if (rc == TFHE_OK) rc = check_cuda(cudaMalloc(&dev_coeff, words * 4), "cudaMalloc(fp32 key staging)");
    if (rc == TFHE_OK)
        rc = check_cuda(cudaMalloc(&k->bsk, (size_t)k->G * 2 * 2 * p->l_bs * k->M * limbs * (p->N / 2) * 8),
                        "cudaMalloc(fp32 key)");
    if (rc == TFHE_OK)
        rc = check_cuda(cudaMemcpyAsync(dev_coeff, bsk_coeff, words * 4, cudaMemcpyHostToDevice, st),
                        "fp32 key upload");
    if (rc == TFHE_OK) {
        switch (p->N) {
            case 256: rc = f32::launch_key_fft<8>(dev_coeff, k->G, k->M, p->l_bs, limbs, k->tables, k->bsk, st); break;
            case 1024: rc = f32::launch_key_fft<10>(dev_coeff, k->G, k->M, p->l_bs, limbs, k->tables, k->bsk, st); break;
            default: rc = f32::launch_key_fft<11>(dev_coeff, k->G, k->M, p->l_bs, limbs, k->tables, k->bsk, st); break;
        }
    }
    if (rc == TFHE_OK) rc = check_cuda(cudaStreamSynchronize(st), "fp32 key build");
    cudaFree(dev_coeff);
    if (rc != TFHE_OK) {
        cudaFree(k->bsk);
        delete k;
        return rc;
    }
    *out = k;
    return TFHE_OK;
}

void tfhe_fp32_keys_destroy(tfhe_fp32_keys* k) {
    if (!k) return;
    cudaFree(k->bsk);
    delete k;
}

int tfhe_fp32_cuboot_merge(const tfhe_fp32_keys* k, const uint32_t* lwe_a, const uint32_t* lwe_b,
                           const uint32_t* lut, int64_t lut_count, int32_t n_lut, uint32_t* out_a, uint32_t* out_b,
                           uint32_t* acc_out, int64_t batch, int32_t ciphertexts_per_cta, void* stream) {
    if (!k) return fail(TFHE_ERR_INVALID_ARGUMENT, "fp32 blind rotation: null keys");
    if (batch < 0) return fail(TFHE_ERR_INVALID_ARGUMENT, "fp32 blind rotation: negative batch");
    if (batch == 0) return TFHE_OK;
    if (!lwe_a || !lwe_b || !lut || (!acc_out && (!out_a || !out_b)))
        return fail(TFHE_ERR_INVALID_ARGUMENT, "fp32 blind rotation: NULL buffer");
    if (lut_count != 1 && lut_count != batch)
        return fail(TFHE_ERR_INVALID_ARGUMENT, "fp32 blind rotation: lut_count must be 1 or batch");
    const int N = k->p.N;
    if (n_lut < 1 || n_lut > N || (n_lut & (n_lut - 1)))
        return fail(TFHE_ERR_INVALID_ARGUMENT, "fp32 blind rotation: n_lut a power of two <= N");
    const int K = ciphertexts_per_cta <= 0 ? 2 : ciphertexts_per_cta;
    if (K != 1 && K != 2) return fail(TFHE_ERR_INVALID_ARGUMENT, "fp32 blind rotation: 1 or 2 ciphertexts per CTA");
    if ((batch + K - 1) / K > 2147483647LL) return fail(TFHE_ERR_INVALID_ARGUMENT, "fp32 blind rotation: batch");
    f32::Args a{k->bsk, k->tables.root, k->tables.tw, k->G, k->M, k->p.collapse, k->limbs, batch, lwe_a, lwe_b,
                lut, lut_count == 1 ? 0 : 2LL * N, n_lut, k->p.n, k->p.log2_beta_bs, out_a, out_b, acc_out};
    cudaStream_t st = (cudaStream_t)stream;
    const int L = k->p.l_bs;
#define F32_CASE(LG, LL)                                                              \
    if (N == (1 << LG) && L == LL)                                                    \
        return K == 1 ? f32::launch_br<LG, LL, 1>(a, st) : f32::launch_br<LG, LL, 2>(a, st);
    F32_CASE(8, 1) F32_CASE(8, 2) F32_CASE(8, 3)
    F32_CASE(10, 1) F32_CASE(10, 2) F32_CASE(10, 3)
    F32_CASE(11, 1) F32_CASE(11, 2)
#undef F32_CASE
    return fail(TFHE_ERR_INVALID_ARGUMENT, "fp32 blind rotation: unsupported N / l_bs");
}

}  // extern "C"
