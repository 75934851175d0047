// Batched blind rotation (collapsed CMux chain) in FP64, K ciphertexts per CTA.
//
// Semantics follow the reference's JAX statement of the kernel
// (schemas/text_jax.py:390-435, cuTFHE/multiply.py:54-92): for each group g
//   dec   = decomposition(ACC)                    (polynomial_jax.py:90-111)
//   ACC'  = cmod_q(round(iFFT( sum_bc DEC_F[bc] * sum_m ROT[r_gm] BSK[g,a,bc,m] )))
// with the group's rotation indices r = round(2N <a_g,p> / (q n_lut)) n_lut
// mod 2N (multiply.py:70-79).  Decomposition, rounding and the centred
// reduction are the reference's float64 operations, so every stage but the
// FFT rounding is bit-identical; with |FFT error| < 1/2 the products are too.
//
// Work mapping (2 K H/8 butterfly owners; XT kernels run 512 threads):
//  * each owner thread has one radix-8 butterfly (k, a, n1) of the first
//    forward / last inverse superstage and keeps ACC[k][a][n1 + (H/8) n2] and
//    ACC[k][a][n1 + (H/8) n2 + H] (n2 < 8) in registers across groups;
//  * middle superstages run over all polynomials in shared memory;
//  * the pointwise stage gives each thread one slot p for KT ciphertexts, so
//    every key word a thread loads serves KT ciphertexts.
#pragma once

#include "tfhe_internal.cuh"

namespace tfhe {

// ciphertexts sharing one thread's key loads in the pointwise stage; the
// CTA's ciphertext count K is always a multiple of it (launcher)
constexpr int br_kt(int logn, int L) { return (L <= 3 && logn <= 11) ? 2 : 1; }

// whether small-K launches of the one-CTA layout get extra threads (the XT
// kernels, instantiated for L <= 3; larger L launch exactly the owners)
constexpr bool br_extra_threads(int L) { return L <= 3; }

struct BrArgs {
    const double2* bsk;       // native [G][2][P/2][M][H][2]; reference layout (G,2,L,2,M,H)
    const double2* all_rot;   // reference layout only: (2N, H)
    const double2* qt;
    const double2* qr;        // qt in rotation order (rot_slot): the QTG layout's only root table
    const double2* tw;
    const uint16_t* freq;
    int G, M, collapse, K;
    long long B;
    int log2_beta, log2_q;
    // native inputs (u32 torus)
    const uint32_t* lwe_a;    // (B, lwe_n) key-switched masks
    const uint32_t* lwe_b;    // (B)
    const uint32_t* lut;      // (B|1, 2, N)
    long long lut_stride;     // 0 or 2N
    int n_lut, lwe_n;
    // reference-layout inputs (mul_bootstrap drop-in)
    const int64_t* ct_init;   // (B|1, 2, N)
    long long ct_stride;      // 0 or 2N
    const int32_t* indices;   // (B, G, M)
    // outputs
    uint32_t* acc_out;        // (B, 2, N): ACC rotated by -b~ (BR)
    uint32_t* out_a;          // (B, n_lut, N): extracted masks
    uint32_t* out_b;          // (B, n_lut)
    int64_t* out_i64;         // (B, 2, N): reference-layout result
    // key ring (KR > 0): stages of the shared-memory ring, wait bound
    int ring_stages;
    int prefetch;             // L1 prefetch of the next pattern's key words: 1 on, 0 off, -1 by path
    int l2_prefetch;          // 1: bring the next group's key block into L2 during each group
    // the 64-bit torus (T64 kernels, q = 2^64): the roles of lwe_a, lwe_b,
    // lut, acc_out, out_a, out_b on uint64 words
    const unsigned long long* lwe_a64;
    const unsigned long long* lwe_b64;
    const long long* lut64;
    unsigned long long* acc_out64;
    unsigned long long* out_a64;
    unsigned long long* out_b64;
    long long wait_limit;     // clock cycles per mbarrier wait
    int* status;              // device status word (tfhe_device_status)
};

// the key words of digits 2j and 2j+1 of one slot: one 32-byte load (the
// native key layout keeps them adjacent; p 32-byte aligned)
__device__ __forceinline__ void ldg_pair(const double2* p, double2& x, double2& y) {
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(x.x), "=d"(x.y), "=d"(y.x), "=d"(y.y) : "l"(p));
}

// exp(-i pi n / 16), n = 1..7
__device__ __forceinline__ double2 root32(int n) {
    constexpr double C[8] = {1.0, 0.98078528040323044913, 0.92387953251128675613, 0.83146961230254523708,
                             0.70710678118654752440, 0.55557023301960222474, 0.38268343236508977173,
                             0.19509032201612826785};
    return make_double2(C[n], -C[8 - n]);
}

// The twist factors zeta^(n1 + (N/16) n2) = zeta^n1 exp(-i pi n2 / 16) and
// the first superstage's twiddles W_H^(n1 k2) = (W_H^n1)^k2 (n2, k2 = 0..7)
// of the butterfly a thread owns, from two table reads and 13 products
// instead of 15 reads (a few ulp from the table values).  Where the root
// table is in global memory (QTG) the reads are the costlier side: n=630
// N=1024 went from 166.7 to 156.4 ms per 16384 ciphertexts; with the table in
// shared memory (n=742 N=2048) the 52 extra FP64 instructions cost more
// (280.7 -> 285.4 ms), so that layout keeps the reads.
template <int LOGN>
__device__ __forceinline__ void owned_factors(const double2* qr, const double2* tw, int n1, double2 (&wt)[8],
                                              double2 (&w0)[8]) {
    const double2 z = qr[rot_slot<LOGN>(n1)];
    wt[0] = z;
#pragma unroll
    for (int n2 = 1; n2 < 8; ++n2) wt[n2] = c_mul(z, root32(n2));
    const double2 u = tw[n1];
    w0[0] = make_double2(1.0, 0.0);
    w0[1] = u;
    w0[2] = c_mul(u, u);
    w0[3] = c_mul(w0[2], u);
    w0[4] = c_mul(w0[2], w0[2]);
    w0[5] = c_mul(w0[4], u);
    w0[6] = c_mul(w0[4], w0[2]);
    w0[7] = c_mul(w0[4], w0[3]);
}

// coefficient of X^e (any integer e) of a negacyclic polynomial in smem
template <int LOGN>
__device__ __forceinline__ uint32_t ncoef(const uint32_t* p, int e) {
    constexpr int N = 1 << LOGN;
    e &= (2 * N - 1);
    const uint32_t v = p[e & (N - 1)];
    return (e < N) ? v : (0u - v);
}

template <int LOGN>
__device__ __forceinline__ unsigned long long ncoef64(const unsigned long long* p, int e) {
    constexpr int N = 1 << LOGN;
    e &= (2 * N - 1);
    const unsigned long long v = p[e & (N - 1)];
    return (e < N) ? v : (0ULL - v);
}

// inverse superstages s = S0 .. 1 (descending) over the 2K output polys
template <int LOGH, int s>
__device__ __forceinline__ void inverse_middle(double2* dec, int K, int P, const double2* tw, int tid, int nt) {
    if constexpr (s >= 1) {
        using PL = Plan<LOGH>;
        constexpr int R = PL::radix(s);
        constexpr int S = PL::span(s);
        constexpr int PER = PL::H / R;
        const double2* tws = tw + PL::tw_offset(s);
        const int total = 2 * K * PER;
        for (int t = tid; t < total; t += nt) {
            const int poly = t / PER;
            double2* base = dec + (size_t)(poly >> 1) * P * PL::H + (poly & 1) * PL::H;
            dit_stage<R, S>(base, tws, t % PER);
        }
        __syncthreads();
        inverse_middle<LOGH, s - 1>(dec, K, P, tw, tid, nt);
    }
}

template <int LOGH, int s>
__device__ __forceinline__ void forward_middle(double2* dec, int npoly, const double2* tw, int tid, int nt) {
    using PL = Plan<LOGH>;
    if constexpr (s < PL::NS) {
        stage_all<LOGH, s, false>(dec, npoly, tw, tid, nt);
        __syncthreads();
        forward_middle<LOGH, s + 1>(dec, npoly, tw, tid, nt);
    }
}

// KR = 0: key words read from global memory by every thread (any K).
// KR > 0: K == KR ciphertexts per CTA and the key streamed through a
// shared-memory ring by 1D bulk copies; the device key layout is then
// [G][4/KR parts][2 out][M][P][NT slots] so each (group, part, out, pattern)
// chunk of P * NT words is contiguous (NT = KR H / 4 = threads per CTA).
// QTG: the quarter root table is read from global memory (L1-cached) instead
// of shared memory, so two CTAs of half the ciphertexts fit on one SM.
// XT: the CTA may have more threads than the 2 K N/16 butterfly owners.
// T64: the native path on the 64-bit torus (uint64 LWEs and outputs, int64
// LUTs, q = 2^64 in the float64 chain as the reference's own arithmetic).
template <int LOGN, int L, bool REFLAYOUT, int KR, int KTP, bool QTG = false, bool XT = false, bool T64 = false>
__global__ void __launch_bounds__(KR > 0 ? KR * (1 << LOGN) / 8 : 512, 1) br_fp64_kernel(const BrArgs args) {
    constexpr int N = 1 << LOGN;
    constexpr int H = N / 2;
    constexpr int LOGH = LOGN - 1;
    constexpr int P = 2 * L;
    constexpr int Q8 = H / 8;
    constexpr int KT = KTP;                // ciphertexts per thread in the pointwise stage
    using PL = Plan<LOGH>;

    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int K = args.K;
    const int M = args.M;
    double2* dec = reinterpret_cast<double2*>(smem_raw);           // K * P * H
    double2* qt_s = dec + (size_t)K * P * H;                        // N / 2 (unless QTG)
    const double2* qt = QTG ? args.qt : qt_s;
    // root r of the quarter table: the shared copy is stored swizzled (qsw),
    // which keeps the X^r lookups of the pointwise stage free of bank
    // conflicts (n=742 N=2048: 280.3 -> 277.9 ms per 16384 ciphertexts,
    // together with the level-fused prologue)
    auto qtab = [&](int r) { return QTG ? qt[r] : qt[qsw<LOGN>(r)]; };
    double2* tw = QTG ? qt_s : qt_s + N / 2;                        // PL::TW
    uint16_t* freq = reinterpret_cast<uint16_t*>(tw + PL::TW);      // H
    int* rot = reinterpret_cast<int*>(freq + H);                    // K * M
    int* bexp = rot + K * M;                                        // K
    // key ring: 128-byte aligned stages, then one mbarrier per stage
    const size_t ring_off = ((reinterpret_cast<uintptr_t>(bexp + K) - reinterpret_cast<uintptr_t>(smem_raw)) + 127) & ~size_t(127);
    double2* ring = reinterpret_cast<double2*>(smem_raw + ring_off);
    uint64_t* bars = reinterpret_cast<uint64_t*>(ring + (size_t)(KR > 0 ? args.ring_stages : 0) * P * (KR * H / 4));

    const int tid = threadIdx.x;
    const int nt = blockDim.x;
    // persistent CTAs: this CTA takes ciphertext sets blockIdx.x, +gridDim.x, ...
    // so every SM walks the key in lockstep for the whole launch
    const long long nsets = (args.B + K - 1) / K;
    const long long my_sets = blockIdx.x < nsets ? (nsets - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;

    if constexpr (!QTG)
        for (int i = tid; i < N / 2; i += nt) qt_s[qsw<LOGN>(i)] = args.qt[i];
    for (int i = tid; i < PL::TW; i += nt) tw[i] = args.tw[i];
    for (int i = tid; i < H; i += nt) freq[i] = args.freq[i];

    // key ring: chunk q of the launch = key words [q * P * NT, (q+1) * P * NT)
    constexpr int RNT = KR * H / 4;                 // threads (= slots per part) in ring mode
    constexpr int NPART = KR > 0 ? 4 / KR : 1;
    const int ring_nc = NPART * 2 * M;              // chunks per group
    const long long ring_set = (long long)args.G * ring_nc;   // chunks per ciphertext set
    const long long ring_total = my_sets * ring_set;          // chunks this CTA consumes
    const uint32_t ring_bytes = (uint32_t)(P * RNT * sizeof(double2));
    if constexpr (KR > 0) {
        if (tid == 0) {
            for (int st = 0; st < args.ring_stages; ++st) mbar_init(&bars[st], 1);
            mbar_fence_init();
        }
        __syncthreads();
        if (tid == 0) {
            for (int st = 0; st < args.ring_stages && st < ring_total; ++st) {
                mbar_arrive_expect_tx(&bars[st], ring_bytes);
                bulk_load(ring + (size_t)st * P * RNT, args.bsk + (size_t)(st % ring_set) * P * RNT, ring_bytes,
                          &bars[st]);
            }
        }
    }

    // the butterfly this thread owns in the first / last superstage
    // a CTA may have more threads than owned butterflies (2 K N/16): the
    // others shadow an owner's butterfly in the register-resident
    // superstages without storing anything, and share the shared-memory
    // superstages and the pointwise stage
    const bool owner = !XT || tid < 2 * K * Q8;
    const int otid = owner ? tid : tid % (2 * K * Q8);
    const int ok = otid / (2 * Q8);
    const int oa = (otid / Q8) & 1;
    const int on1 = otid % Q8;

    const double q = ldexp(1.0, args.log2_q);
    const double inv_q = ldexp(1.0, -args.log2_q);
    const double beta = ldexp(1.0, args.log2_beta);
    // q^-1 beta: the first level's beta acc / q in one (exact) product
    const double inv_qb = ldexp(1.0, args.log2_beta - args.log2_q);
    constexpr double inv_h = 1.0 / H;

    for (long long iter = 0; iter < my_sets; ++iter) {
    const long long ct0 = (blockIdx.x + iter * gridDim.x) * K;
    const long long oct = min(ct0 + ok, args.B - 1);

    double acc_lo[8], acc_hi[8];
    if constexpr (REFLAYOUT) {
        const int64_t* src = args.ct_init + oct * args.ct_stride + oa * N;
#pragma unroll
        for (int n2 = 0; n2 < 8; ++n2) {
            acc_lo[n2] = (double)src[on1 + Q8 * n2];
            acc_hi[n2] = (double)src[on1 + Q8 * n2 + H];
        }
    } else if constexpr (T64) {
        const long long* src = args.lut64 + oct * args.lut_stride + oa * N;
#pragma unroll
        for (int n2 = 0; n2 < 8; ++n2) {
            acc_lo[n2] = (double)src[on1 + Q8 * n2];
            acc_hi[n2] = (double)src[on1 + Q8 * n2 + H];
        }
    } else {
        const uint32_t* src = args.lut + oct * args.lut_stride + oa * N;
#pragma unroll
        for (int n2 = 0; n2 < 8; ++n2) {
            acc_lo[n2] = (double)(int32_t)src[on1 + Q8 * n2];
            acc_hi[n2] = (double)(int32_t)src[on1 + Q8 * n2 + H];
        }
    }
    __syncthreads();

    for (int g = 0; g < args.G; ++g) {
        if constexpr (KR == 0 && !REFLAYOUT) {
            // the next group's key block (all CTAs together: each its share)
            // into L2 while this group runs
            if (tid == 0 && g + 1 < args.G && args.l2_prefetch) {
                const size_t block = (size_t)2 * P * M * H * sizeof(double2);
                const size_t share = ((block / gridDim.x) + 255) & ~(size_t)255;
                const size_t off = (size_t)blockIdx.x * share;
                if (off < block) {
                    const size_t len = min(share, block - off);
                    const char* base = reinterpret_cast<const char*>(args.bsk + (size_t)(g + 1) * 2 * P * M * H);
                    prefetch_l2_bulk(base + off, (uint32_t)len);
                }
            }
        }
        // rotation index of every (ciphertext, pattern) of this group
        for (int t = tid; t < K * M; t += nt) {
            const int k = t / M;
            const int m = t - k * M;
            const long long ct = min(ct0 + k, args.B - 1);
            int r;
            if constexpr (REFLAYOUT) {
                r = args.indices[(ct * args.G + g) * M + m];
            } else if constexpr (T64) {
                // rne(2N <a_g, p_m> / (q n_lut)) n_lut mod 2N on the exact group sum
                unsigned long long v = 0ULL;
                const unsigned long long* a = args.lwe_a64 + ct * args.lwe_n + (long long)g * args.collapse;
                for (int c = 0; c < args.collapse; ++c)
                    if ((m >> (args.collapse - 1 - c)) & 1) v += a[c];
                const int ln = __ffs(args.n_lut) - 1;
                const long long d = rne_div_pow2((long long)v, 63 - LOGN + ln);
                r = (int)((d << ln) & (2 * N - 1));
            } else {
                // <a_g, pattern m>, patterns in meshgrid 'ij' order
                double v = 0.0;
                const uint32_t* a = args.lwe_a + ct * args.lwe_n + (long long)g * args.collapse;
                for (int c = 0; c < args.collapse; ++c)
                    if ((m >> (args.collapse - 1 - c)) & 1) v += (double)(int32_t)a[c];
                const double idx = rint((2.0 * N * v) / (q * args.n_lut)) * args.n_lut;
                int ri = (int)idx % (2 * N);
                r = ri < 0 ? ri + 2 * N : ri;
            }
            rot[t] = r;
        }

        // prologue: gadget digits of the owned coefficients (float64 steps of
        // polynomial_jax.py:98-111), fold + twist, first DIF superstage
        {
            double2* pk = dec + (size_t)ok * P * H + oa * H;
            double2 w0[8];
            [[maybe_unused]] double2 wt[8];
            if constexpr (QTG) {
                owned_factors<LOGN>(args.qr, tw, on1, wt, w0);
            } else {
                w0[0] = make_double2(1.0, 0.0);
#pragma unroll
                for (int k2 = 1; k2 < 8; ++k2) w0[k2] = tw[(k2 - 1) * Q8 + on1];
            }
            if constexpr (!QTG && L <= 2) {
                // all L digits of a coefficient pair at once, so its twist
                // factor is read once per group rather than once per level
                // (the same operations on every value as the level loop below)
                double2 v[L][8];
#pragma unroll
                for (int n2 = 0; n2 < 8; ++n2) {
                    double xlo = 0.0, xhi = 0.0;
                    const double2 w = qtab(on1 + Q8 * n2);   // zeta^i
#pragma unroll
                    for (int lvl = 0; lvl < L; ++lvl) {
                        const double ylo = lvl == 0 ? acc_lo[n2] * inv_qb : xlo * beta;
                        const double dlo = rint(ylo);
                        xlo = ylo - dlo;
                        const double yhi = lvl == 0 ? acc_hi[n2] * inv_qb : xhi * beta;
                        const double dhi = rint(yhi);
                        xhi = yhi - dhi;
                        v[lvl][n2] = make_double2(fma(w.x, dlo, w.y * dhi), fma(w.y, dlo, -w.x * dhi));
                    }
                }
#pragma unroll
                for (int lvl = 0; lvl < L; ++lvl) {
                    dft8<false>(v[lvl]);
#pragma unroll
                    for (int k2 = 1; k2 < 8; ++k2) v[lvl][k2] = c_mul(v[lvl][k2], w0[k2]);
                    double2* poly = pk + lvl * 2 * H;
#pragma unroll
                    for (int k2 = 0; k2 < 8; ++k2)
                        if (owner) poly[swz(on1 + Q8 * k2)] = v[lvl][k2];
                }
            } else {
                double x_lo[8], x_hi[8];
#pragma unroll
                for (int lvl = 0; lvl < L; ++lvl) {
                    double2 v[8];
#pragma unroll
                    for (int n2 = 0; n2 < 8; ++n2) {
                        const double ylo = lvl == 0 ? acc_lo[n2] * inv_qb : x_lo[n2] * beta;
                        const double dlo = rint(ylo);
                        x_lo[n2] = ylo - dlo;
                        const double yhi = lvl == 0 ? acc_hi[n2] * inv_qb : x_hi[n2] * beta;
                        const double dhi = rint(yhi);
                        x_hi[n2] = yhi - dhi;
                        const double2 w = QTG ? wt[n2] : qtab(on1 + Q8 * n2);   // zeta^i
                        v[n2] = make_double2(fma(w.x, dlo, w.y * dhi), fma(w.y, dlo, -w.x * dhi));
                    }
                    dft8<false>(v);
#pragma unroll
                    for (int k2 = 1; k2 < 8; ++k2) v[k2] = c_mul(v[k2], w0[k2]);
                    double2* poly = pk + lvl * 2 * H;
#pragma unroll
                    for (int k2 = 0; k2 < 8; ++k2)
                        if (owner) poly[swz(on1 + Q8 * k2)] = v[k2];
                }
            }
        }
        __syncthreads();
        forward_middle<LOGH, 1>(dec, K * P, tw, tid, nt);

        if constexpr (KR > 0) {
            // pointwise with the key streamed through the ring: chunk
            // (part, out a, pattern m) holds the P key words of every slot of
            // the part; thread tid owns slot part * NT + tid for all KR
            // ciphertexts, so every staged key word is read once.
            double2 d[KR][P];
            double2 o0[KR], o1[KR];
            int e = 0;
            for (int c = 0; c < ring_nc; ++c) {
                const long long qi = iter * ring_set + (long long)g * ring_nc + c;
                const int st = (int)(qi % args.ring_stages);
                const uint32_t par = (uint32_t)((qi / args.ring_stages) & 1);
                const int part = c / (2 * M);
                const int a = (c / M) & 1;
                const int m = c % M;
                const int p = part * RNT + tid;
                if (a == 0 && m == 0) {
#pragma unroll
                    for (int kt = 0; kt < KR; ++kt) {
#pragma unroll
                        for (int bc = 0; bc < P; ++bc) d[kt][bc] = dec[(size_t)kt * P * H + bc * H + swz(p)];
                        o0[kt] = o1[kt] = make_double2(0.0, 0.0);
                    }
                    e = 4 * freq[p] + 1;
                }
                mbar_wait_bounded(&bars[st], par, args.wait_limit, args.status);
                const double2* chunk = ring + (size_t)st * P * RNT;
                double2 t[KR];
#pragma unroll
                for (int kt = 0; kt < KR; ++kt) t[kt] = make_double2(0.0, 0.0);
#pragma unroll
                for (int bc = 0; bc < P; ++bc) {
                    const double2 kv = chunk[bc * RNT + tid];
#pragma unroll
                    for (int kt = 0; kt < KR; ++kt) c_mac(t[kt], kv, d[kt][bc]);
                }
#pragma unroll
                for (int kt = 0; kt < KR; ++kt) {
                    const double2 w = root2n<LOGN, !QTG>(qt, rot[kt * M + m] * e);
                    if (a == 0) c_mac(o0[kt], w, t[kt]);
                    else c_mac(o1[kt], w, t[kt]);
                }
                if (a == 1 && m == M - 1) {
#pragma unroll
                    for (int kt = 0; kt < KR; ++kt) {
                        dec[(size_t)kt * P * H + swz(p)] = o0[kt];
                        dec[(size_t)kt * P * H + H + swz(p)] = o1[kt];
                    }
                }
                __syncthreads();                      // stage st fully read
                if (tid == 0 && qi + args.ring_stages < ring_total) {
                    const long long qn = qi + args.ring_stages;
                    fence_proxy_async_smem();
                    mbar_arrive_expect_tx(&bars[st], ring_bytes);
                    bulk_load(ring + (size_t)st * P * RNT, args.bsk + (size_t)(qn % ring_set) * P * RNT, ring_bytes,
                              &bars[st]);
                }
            }
        } else {
            // pointwise: out[a] = sum_m X^{r_m} * sum_bc BSK[g,a,bc,m] * DEC[bc].
            // One thread per (slot, group of KT ciphertexts): every key word is
            // loaded once into registers and used for KT ciphertexts.
            {
                const size_t gbase = (size_t)g * 2 * P * M * H;
                const int KG = K / KT;
                for (int t = tid; t < KG * H; t += nt) {
                    const int kg = t % KG;
                    const int p = t / KG;
                    double2 d[KT][P];
    #pragma unroll
                    for (int kt = 0; kt < KT; ++kt)
    #pragma unroll
                        for (int bc = 0; bc < P; ++bc) d[kt][bc] = dec[(size_t)(kg * KT + kt) * P * H + bc * H + swz(p)];
                    const int j = freq[p];
                    const int e = 4 * j + 1;                       // evaluation point zeta^e
                    // reference layout index of the same point (or its conjugate)
                    const bool cj = REFLAYOUT && (e >= N);
                    const int jr = REFLAYOUT ? (cj ? (N - 1 - 2 * j) : 2 * j) : p;
                    double2 o0[KT], o1[KT];
    #pragma unroll
                    for (int kt = 0; kt < KT; ++kt) o0[kt] = o1[kt] = make_double2(0.0, 0.0);
                    const double2* kb = args.bsk + gbase + jr;          // reference layout
                    const double2* kb2 = args.bsk + gbase + 2 * (size_t)p; // native: pairs of digits
#pragma unroll 1
                    for (int m = 0; m < M; ++m) {
                        if (args.prefetch > 0 || (args.prefetch < 0 && 2 * P * KT > 16)) {
                            // next pattern of this slot, or the first pattern of
                            // this thread's next slot: into L1 while this one computes
                            const double2* nb = REFLAYOUT ? kb + (size_t)(m + 1) * H : kb2 + (size_t)(m + 1) * H * 2;
                            if (m + 1 == M) {
                                const int tn = t + nt;
                                const int pn = tn / KG;
                                nb = (tn < KG * H) ? args.bsk + gbase + 2 * (size_t)pn : nullptr;
                                if (REFLAYOUT) nb = nullptr;
                            }
                            if (nb) {
                                if constexpr (REFLAYOUT) {
#pragma unroll
                                    for (int bc = 0; bc < 2 * P; ++bc) prefetch_l1(nb + (size_t)bc * M * H);
                                } else {
#pragma unroll
                                    for (int j = 0; j < P; ++j) prefetch_l1(nb + (size_t)j * M * H * 2);
                                }
                            }
                        }
                        double2 w[KT];
#pragma unroll
                        for (int kt = 0; kt < KT; ++kt) {
                            const int r = rot[(kg * KT + kt) * M + m];
                            if constexpr (REFLAYOUT) {
                                w[kt] = __ldg(args.all_rot + (size_t)r * H + jr);
                                if (cj) w[kt] = c_conj(w[kt]);
                            } else {
                                w[kt] = QTG ? root2n_rot<LOGN>(args.qr, r * e) : root2n<LOGN, true>(qt, r * e);
                            }
                        }
                        if constexpr (2 * P * KT <= 16) {
                            // both outputs' key words of this pattern in flight before use
                            double2 k0[P], k1[P];
                            if constexpr (REFLAYOUT) {
#pragma unroll
                                for (int bc = 0; bc < P; ++bc) {
                                    k0[bc] = __ldg(kb + ((size_t)bc * M + m) * H);
                                    k1[bc] = __ldg(kb + ((size_t)(P + bc) * M + m) * H);
                                }
                            } else {
#pragma unroll
                                for (int j = 0; j < P / 2; ++j) {
                                    ldg_pair(kb2 + ((size_t)j * M + m) * H * 2, k0[2 * j], k0[2 * j + 1]);
                                    ldg_pair(kb2 + ((size_t)(P / 2 + j) * M + m) * H * 2, k1[2 * j], k1[2 * j + 1]);
                                }
                            }
                            double2 t0[KT], t1[KT];
#pragma unroll
                            for (int kt = 0; kt < KT; ++kt) t0[kt] = t1[kt] = make_double2(0.0, 0.0);
#pragma unroll
                            for (int bc = 0; bc < P; ++bc) {
                                if (cj) { k0[bc] = c_conj(k0[bc]); k1[bc] = c_conj(k1[bc]); }
#pragma unroll
                                for (int kt = 0; kt < KT; ++kt) {
                                    c_mac(t0[kt], k0[bc], d[kt][bc]);
                                    c_mac(t1[kt], k1[bc], d[kt][bc]);
                                }
                            }
#pragma unroll
                            for (int kt = 0; kt < KT; ++kt) {
                                c_mac(o0[kt], w[kt], t0[kt]);
                                c_mac(o1[kt], w[kt], t1[kt]);
                            }
                        } else {
                            // one output at a time: P key words in flight
#pragma unroll
                            for (int a = 0; a < 2; ++a) {
                                double2 kv[P];
                                if constexpr (REFLAYOUT) {
#pragma unroll
                                    for (int bc = 0; bc < P; ++bc) kv[bc] = __ldg(kb + ((size_t)(a * P + bc) * M + m) * H);
                                } else {
#pragma unroll
                                    for (int j = 0; j < P / 2; ++j)
                                        ldg_pair(kb2 + ((size_t)(a * (P / 2) + j) * M + m) * H * 2, kv[2 * j], kv[2 * j + 1]);
                                }
                                double2 t[KT];
#pragma unroll
                                for (int kt = 0; kt < KT; ++kt) t[kt] = make_double2(0.0, 0.0);
#pragma unroll
                                for (int bc = 0; bc < P; ++bc) {
                                    if (cj) kv[bc] = c_conj(kv[bc]);
#pragma unroll
                                    for (int kt = 0; kt < KT; ++kt) c_mac(t[kt], kv[bc], d[kt][bc]);
                                }
#pragma unroll
                                for (int kt = 0; kt < KT; ++kt) {
                                    if (a == 0) c_mac(o0[kt], w[kt], t[kt]);
                                    else c_mac(o1[kt], w[kt], t[kt]);
                                }
                            }
                        }
                    }
    #pragma unroll
                    for (int kt = 0; kt < KT; ++kt) {
                        double2* pk = dec + (size_t)(kg * KT + kt) * P * H;
                        pk[swz(p)] = o0[kt];
                        pk[H + swz(p)] = o1[kt];
                    }
                }
            }
        }
        __syncthreads();
        inverse_middle<LOGH, PL::NS - 1>(dec, K, P, tw, tid, nt);

        // last DIT superstage, untwist, round, centred reduction
        {
            double2* poly = dec + (size_t)ok * P * H + oa * H;
            double2 v[8];
#pragma unroll
            for (int k2 = 0; k2 < 8; ++k2) v[k2] = poly[swz(on1 + Q8 * k2)];
            [[maybe_unused]] double2 wt[8];
            if constexpr (QTG) {
                double2 w0[8];
                owned_factors<LOGN>(args.qr, tw, on1, wt, w0);
#pragma unroll
                for (int k2 = 1; k2 < 8; ++k2) v[k2] = c_mul(v[k2], c_conj(w0[k2]));
            } else {
                twiddle<8, Q8, true>(v, tw, on1);
            }
            dft8<true>(v);
#pragma unroll
            for (int n2 = 0; n2 < 8; ++n2) {
                const double2 u = c_mul(c_conj(QTG ? wt[n2] : qtab(on1 + Q8 * n2)), v[n2]);
                // the native key is stored times 1/H (bsk_fft_kernel), which
                // already applied the inverse transform's 1/H, exactly
                double rlo, rhi;
                if constexpr (REFLAYOUT) {
                    rlo = rint(u.x * inv_h);
                    rhi = rint(-u.y * inv_h);
                } else {
                    rlo = rint(u.x);
                    rhi = rint(-u.y);
                }
                acc_lo[n2] = rlo - q * rint(rlo * inv_q);
                acc_hi[n2] = rhi - q * rint(rhi * inv_q);
            }
        }
        __syncthreads();
    }

    // ---------------------------------------------------------------- epilogue
    if constexpr (REFLAYOUT) {
        if (owner && ct0 + ok < args.B) {
            int64_t* dst = args.out_i64 + (ct0 + ok) * 2 * N + oa * N;
#pragma unroll
            for (int n2 = 0; n2 < 8; ++n2) {
                dst[on1 + Q8 * n2] = __double2ll_rn(acc_lo[n2]);
                dst[on1 + Q8 * n2 + H] = __double2ll_rn(acc_hi[n2]);
            }
        }
    } else if constexpr (T64) {
        // ACC to shared memory as uint64 words, then rotate by -b~ and
        // extract, exactly as below on the 64-bit torus
        typedef unsigned long long u64;
        u64* acc = reinterpret_cast<u64*>(smem_raw);                 // [K][2][N]
        if (owner) {
            u64* dst = acc + (size_t)ok * 2 * N + oa * N;
#pragma unroll
            for (int n2 = 0; n2 < 8; ++n2) {
                dst[on1 + Q8 * n2] = (u64)__double2ll_rn(acc_lo[n2]);
                dst[on1 + Q8 * n2 + H] = (u64)__double2ll_rn(acc_hi[n2]);
            }
        }
        for (int k = tid; k < K; k += nt) {
            const long long ct = min(ct0 + k, args.B - 1);
            const int ln = __ffs(args.n_lut) - 1;
            bexp[k] = (int)((rne_div_pow2((long long)args.lwe_b64[ct], 63 - LOGN + ln) << ln) & (2 * N - 1));
        }
        __syncthreads();
        const int kv = (int)min((long long)K, args.B - ct0);
        if (args.acc_out64) {
            for (int t = tid; t < kv * 2 * N; t += nt) {
                const int k = t / (2 * N);
                const int rem = t - k * 2 * N;
                const int a = rem / N;
                const int i = rem - a * N;
                args.acc_out64[(ct0 + k) * 2 * N + rem] = ncoef64<LOGN>(acc + (size_t)k * 2 * N + a * N, i + bexp[k]);
            }
        }
        if (args.out_a64) {
            const int nl = args.n_lut;
            for (int t = tid; t < kv * nl * N; t += nt) {
                const int k = t / (nl * N);
                const int rem = t - k * nl * N;
                const int al = rem / N;
                const int j = rem - al * N;
                args.out_a64[(ct0 + k) * nl * N + rem] = ncoef64<LOGN>(acc + (size_t)k * 2 * N, al - j + bexp[k]);
            }
            for (int t = tid; t < kv * nl; t += nt) {
                const int k = t / nl;
                const int al = t - k * nl;
                args.out_b64[(ct0 + k) * nl + al] = ncoef64<LOGN>(acc + (size_t)k * 2 * N + N, al + bexp[k]);
            }
        }
    } else {
        // ACC to shared memory as u32, then rotate by -b~ (RLWE_jax.py:295-297)
        // and, for the PBS, extract n_lut LWEs (RLWE_jax.py:301-303)
        uint32_t* acc = reinterpret_cast<uint32_t*>(smem_raw);       // [K][2][N]
        if (owner) {
            uint32_t* dst = acc + (size_t)ok * 2 * N + oa * N;
#pragma unroll
            for (int n2 = 0; n2 < 8; ++n2) {
                dst[on1 + Q8 * n2] = (uint32_t)(long long)acc_lo[n2];
                dst[on1 + Q8 * n2 + H] = (uint32_t)(long long)acc_hi[n2];
            }
        }
        for (int k = tid; k < K; k += nt) {
            const long long ct = min(ct0 + k, args.B - 1);
            const double b = (double)(int32_t)args.lwe_b[ct];
            bexp[k] = (int)(rint((2.0 * N * b) / (q * args.n_lut)) * args.n_lut);
        }
        __syncthreads();
        const int kv = (int)min((long long)K, args.B - ct0);
        if (args.acc_out) {
            for (int t = tid; t < kv * 2 * N; t += nt) {
                const int k = t / (2 * N);
                const int rem = t - k * 2 * N;
                const int a = rem / N;
                const int i = rem - a * N;
                args.acc_out[(ct0 + k) * 2 * N + rem] = ncoef<LOGN>(acc + (size_t)k * 2 * N + a * N, i + bexp[k]);
            }
        }
        if (args.out_a) {
            const int nl = args.n_lut;
            for (int t = tid; t < kv * nl * N; t += nt) {
                const int k = t / (nl * N);
                const int rem = t - k * nl * N;
                const int al = rem / N;
                const int j = rem - al * N;
                args.out_a[(ct0 + k) * nl * N + rem] = ncoef<LOGN>(acc + (size_t)k * 2 * N, al - j + bexp[k]);
            }
            for (int t = tid; t < kv * nl; t += nt) {
                const int k = t / nl;
                const int al = t - k * nl;
                args.out_b[(ct0 + k) * nl + al] = ncoef<LOGN>(acc + (size_t)k * 2 * N + N, al + bexp[k]);
            }
        }
    }
    __syncthreads();               // shared memory is reused by the next set
    }
}

// ----------------------------------------------------------------------------
// Forward FFT of the coefficient-domain bootstrapping key into the device
// layout [G][2 out][P/2][M][H][2] (position order; the two digits bc = 2j,
// 2j+1 of a slot adjacent), P = 2L, bc = level * 2 + in.
// Source: uint32 (2 in = left/right, 2 out = mask/body, G*M, L, N), the
// layout of get_boostrapping_key_collapse (schemas/RLWE_jax.py:162-197).
// The reference transforms the same integers with jax_fourier and permutes
// (nn_tfhe/activation.py:49-53, cuTFHE/multiply.py:81-86).
// ----------------------------------------------------------------------------
struct BskConvArgs {
    const uint32_t* src;
    const unsigned long long* src64;   // the 64-bit torus's key (then src is unused)
    double2* dst;
    const double2* qt;
    const double2* tw;
    int G, M, L;
    long long npoly;   // 2 * 2 * G * M * L
    int ring_nt;       // 0: [G][2][P/2][M][H][2]; > 0: [G][H/ring_nt][2][M][P][ring_nt]
};

template <int LOGN>
__global__ void __launch_bounds__(256) bsk_fft_kernel(const BskConvArgs a) {
    constexpr int N = 1 << LOGN;
    constexpr int H = N / 2;
    constexpr int LOGH = LOGN - 1;
    constexpr int PPC = (2048 / H) > 0 ? (2048 / H) : 1;   // polys per CTA (<= 32 KB)
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* buf = reinterpret_cast<double2*>(smem_raw);
    const int tid = threadIdx.x, nt = blockDim.x;
    const long long p0 = (long long)blockIdx.x * PPC;
    const int P = 2 * a.L;
    const long long GM = (long long)a.G * a.M;

    for (int idx = tid; idx < PPC * H; idx += nt) {
        const int lp = idx / H, i = idx % H;
        const long long pi = min(p0 + lp, a.npoly - 1);
        double lo, hi;
        if (a.src64) {
            const unsigned long long* s64 = a.src64 + pi * N;
            lo = (double)(long long)s64[i];
            hi = (double)(long long)s64[i + H];
        } else {
            const uint32_t* s = a.src + pi * N;
            lo = (double)(int32_t)s[i];
            hi = (double)(int32_t)s[i + H];
        }
        const double2 w = a.qt[i];
        buf[lp * H + swz(i)] = make_double2(fma(w.x, lo, w.y * hi), fma(w.y, lo, -w.x * hi));
    }
    __syncthreads();
    forward_middle<LOGH, 0>(buf, PPC, a.tw, tid, nt);
    for (int idx = tid; idx < PPC * H; idx += nt) {
        const int lp = idx / H, p = idx % H;
        const long long pi = p0 + lp;
        if (pi >= a.npoly) continue;
        const int lvl = (int)(pi % a.L);
        const long long gm = (pi / a.L) % GM;
        const int out = (int)((pi / (a.L * GM)) % 2);
        const int in = (int)(pi / (2 * a.L * GM));
        const long long g = gm / a.M;
        const int m = (int)(gm % a.M);
        const int bc = lvl * 2 + in;
        size_t di;
        if (a.ring_nt > 0) {
            const int parts = H / a.ring_nt;
            di = ((((size_t)g * parts + p / a.ring_nt) * 2 + out) * a.M + m) * P + bc;
            di = di * a.ring_nt + p % a.ring_nt;
        } else {
            di = ((((size_t)(g * 2 + out) * (P / 2) + bc / 2) * a.M + m) * H + p) * 2 + (bc & 1);
        }
        // times 1/H: a power of two, so every product and sum of the blind
        // rotation comes out exactly 1/H times the unscaled one, and the
        // inverse transform's 1/H needs no multiply of its own
        const double2 v = buf[lp * H + swz(p)];
        a.dst[di] = make_double2(v.x * (1.0 / H), v.y * (1.0 / H));
    }
}

}  // namespace tfhe
