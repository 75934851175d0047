// Large-batch blind rotation with the accumulators in tensor memory.
//
// br_fp64_kernel keeps every ciphertext's accumulator in the registers of
// the threads that own its radix-8 butterflies, so 512 threads hold at most
// K = 2 ciphertexts at N = 2048, and each key word loaded in the pointwise
// stage serves two ciphertexts.  Here the accumulators live in tensor memory
// (TMEM, 256 KB per SM) between groups: a thread owns several butterflies in
// turn, loading its accumulator words with tcgen05.ld before the prologue and
// storing them with tcgen05.st after the last superstage, so K = 3
// ciphertexts fit one CTA of 512 threads (shared memory: 3 x 4 digit spectra
// of N/2 points, 192 KB, plus the tables), and every key word serves three.
// TMEM is private per thread here: thread t of warp w uses lane
// 32 (w % 4) + t % 32, columns (slot * 4 + w / 4) * 32 .. + 31 for its slot-th
// butterfly, 32 words = the 16 float64 accumulator values.
//
// Every value is computed by br_fp64_kernel's operations in the same order
// (the level-fused prologue, the FFT stages, the pointwise contraction of
// each ciphertext in digit order per pattern, the rounding), so the outputs
// are bit-identical to it.  Native layout only (uint32 or the 64-bit torus),
// l_bs <= 2, the root table in shared memory.
#pragma once

#include "br_fp64.cuh"

namespace tfhe {

constexpr int BR_TM_THREADS = 512;
constexpr uint32_t BR_TM_COLS = 256;          // TMEM columns allocated per CTA

__device__ __forceinline__ void tm_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}

__device__ __forceinline__ void tm_st16(uint32_t taddr, const uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16};" ::"r"(taddr),
        "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]), "r"(r[9]),
        "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
        : "memory");
}

__device__ __forceinline__ void tm_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tm_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// 8 float64 values <-> 16 words
__device__ __forceinline__ void pack8(const double (&v)[8], uint32_t (&w)[16]) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const unsigned long long b = (unsigned long long)__double_as_longlong(v[i]);
        w[2 * i] = (uint32_t)b;
        w[2 * i + 1] = (uint32_t)(b >> 32);
    }
}

__device__ __forceinline__ void unpack8(const uint32_t (&w)[16], double (&v)[8]) {
#pragma unroll
    for (int i = 0; i < 8; ++i)
        v[i] = __longlong_as_double((long long)(((unsigned long long)w[2 * i + 1] << 32) | w[2 * i]));
}

// shared memory of br_tm_kernel: K x P digit spectra, the tables, rotation
// indices and b~ (the accumulator words of the epilogue reuse the spectra)
inline size_t br_tm_smem(int N, int L, int K, int M, size_t table_bytes) {
    const int H = N / 2;
    return (size_t)K * 2 * L * H * sizeof(double2) + table_bytes + (size_t)(K * M + K) * sizeof(int) + 16;
}

template <int LOGN, int L, int K, bool T64>
__global__ void __launch_bounds__(BR_TM_THREADS, 1) br_tm_kernel(const BrArgs args) {
    constexpr int N = 1 << LOGN;
    constexpr int H = N / 2;
    constexpr int LOGH = LOGN - 1;
    constexpr int P = 2 * L;
    constexpr int Q8 = H / 8;
    constexpr int OWN = 2 * K * Q8;                                   // radix-8 butterflies per set
    constexpr int SLOTS = (OWN + BR_TM_THREADS - 1) / BR_TM_THREADS;  // butterflies per thread
    using PL = Plan<LOGH>;
    static_assert(L <= 2, "the level-fused prologue (l_bs <= 2)");
    static_assert(SLOTS * 4 * 32 <= (int)BR_TM_COLS, "TMEM columns per lane");
    static_assert(OWN % 32 == 0, "whole warps per butterfly slot");

    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ uint32_t tmem_slot;
    const int M = args.M;
    double2* dec = reinterpret_cast<double2*>(smem_raw);           // K * P * H
    double2* qt_s = dec + (size_t)K * P * H;                        // N / 2, swizzled
    double2* tw = qt_s + N / 2;                                     // PL::TW
    uint16_t* freq = reinterpret_cast<uint16_t*>(tw + PL::TW);      // H
    int* rot = reinterpret_cast<int*>(freq + H);                    // K * M
    int* bexp = rot + K * M;                                        // K
    auto qtab = [&](int r) { return qt_s[qsw<LOGN>(r)]; };

    const int tid = threadIdx.x, nt = blockDim.x, warp = tid >> 5;
    const long long nsets = (args.B + K - 1) / K;
    const long long my_sets = blockIdx.x < nsets ? (nsets - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;

    for (int i = tid; i < N / 2; i += nt) qt_s[qsw<LOGN>(i)] = args.qt[i];
    for (int i = tid; i < PL::TW; i += nt) tw[i] = args.tw[i];
    for (int i = tid; i < H; i += nt) freq[i] = args.freq[i];
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_slot)),
                     "r"(BR_TM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot + ((uint32_t)(32 * (warp & 3)) << 16);
    auto tcol = [&](int slot) { return (uint32_t)((slot * 4 + (warp >> 2)) * 32); };

    const double q = ldexp(1.0, args.log2_q);
    const double inv_q = ldexp(1.0, -args.log2_q);
    const double beta = ldexp(1.0, args.log2_beta);
    const double inv_qb = ldexp(1.0, args.log2_beta - args.log2_q);

    for (long long iter = 0; iter < my_sets; ++iter) {
        const long long ct0 = (blockIdx.x + iter * gridDim.x) * K;
        // ACC of every owned butterfly from the LUT, into TMEM
#pragma unroll
        for (int sl = 0; sl < SLOTS; ++sl) {
            const int ob = tid + sl * nt;
            if (ob >= OWN) continue;                                // warp-uniform
            const int ok = ob / (2 * Q8), oa = (ob / Q8) & 1, on1 = ob % Q8;
            const long long oct = min(ct0 + ok, args.B - 1);
            double lo[8], hi[8];
            if constexpr (T64) {
                const long long* src = args.lut64 + oct * args.lut_stride + oa * N;
#pragma unroll
                for (int n2 = 0; n2 < 8; ++n2) {
                    lo[n2] = (double)src[on1 + Q8 * n2];
                    hi[n2] = (double)src[on1 + Q8 * n2 + H];
                }
            } else {
                const uint32_t* src = args.lut + oct * args.lut_stride + oa * N;
#pragma unroll
                for (int n2 = 0; n2 < 8; ++n2) {
                    lo[n2] = (double)(int32_t)src[on1 + Q8 * n2];
                    hi[n2] = (double)(int32_t)src[on1 + Q8 * n2 + H];
                }
            }
            uint32_t w[16];
            pack8(lo, w);
            tm_st16(tmem + tcol(sl), w);
            pack8(hi, w);
            tm_st16(tmem + tcol(sl) + 16, w);
        }
        tm_wait_st();
        __syncthreads();

        for (int g = 0; g < args.G; ++g) {
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
            // rotation indices of this group (br_fp64_kernel's formulas)
            for (int t = tid; t < K * M; t += nt) {
                const int k = t / M;
                const int m = t - k * M;
                const long long ct = min(ct0 + k, args.B - 1);
                int r;
                if constexpr (T64) {
                    unsigned long long v = 0ULL;
                    const unsigned long long* a = args.lwe_a64 + ct * args.lwe_n + (long long)g * args.collapse;
                    for (int c = 0; c < args.collapse; ++c)
                        if ((m >> (args.collapse - 1 - c)) & 1) v += a[c];
                    const int ln = __ffs(args.n_lut) - 1;
                    const long long d = rne_div_pow2((long long)v, 63 - LOGN + ln);
                    r = (int)((d << ln) & (2 * N - 1));
                } else {
                    double v = 0.0;
                    const uint32_t* a = args.lwe_a + ct * args.lwe_n + (long long)g * args.collapse;
                    for (int c = 0; c < args.collapse; ++c)
                        if ((m >> (args.collapse - 1 - c)) & 1) v += (double)(int32_t)a[c];
                    const double idx = rint((2.0 * N * v) / (q * args.n_lut)) * args.n_lut;
                    const int ri = (int)idx % (2 * N);
                    r = ri < 0 ? ri + 2 * N : ri;
                }
                rot[t] = r;
            }

            // prologue: every owned butterfly's digits (level-fused), fold +
            // twist, first DIF superstage
#pragma unroll
            for (int sl = 0; sl < SLOTS; ++sl) {
                const int ob = tid + sl * nt;
                if (ob >= OWN) continue;
                const int ok = ob / (2 * Q8), oa = (ob / Q8) & 1, on1 = ob % Q8;
                double acc_lo[8], acc_hi[8];
                {
                    uint32_t w[16];
                    tm_ld16(tmem + tcol(sl), w);
                    tm_wait_ld();
                    unpack8(w, acc_lo);
                    tm_ld16(tmem + tcol(sl) + 16, w);
                    tm_wait_ld();
                    unpack8(w, acc_hi);
                }
                double2* pk = dec + (size_t)ok * P * H + oa * H;
                double2 w0[8];
                w0[0] = make_double2(1.0, 0.0);
#pragma unroll
                for (int k2 = 1; k2 < 8; ++k2) w0[k2] = tw[(k2 - 1) * Q8 + on1];
                double2 v[L][8];
#pragma unroll
                for (int n2 = 0; n2 < 8; ++n2) {
                    double xlo = 0.0, xhi = 0.0;
                    const double2 w = qtab(on1 + Q8 * n2);
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
                    for (int k2 = 0; k2 < 8; ++k2) poly[swz(on1 + Q8 * k2)] = v[lvl][k2];
                }
            }
            __syncthreads();
            forward_middle<LOGH, 1>(dec, K * P, tw, tid, nt);

            // pointwise: one thread per slot for all K ciphertexts; every key
            // word loaded serves K of them
            {
                const size_t gbase = (size_t)g * 2 * P * M * H;
                for (int p = tid; p < H; p += nt) {
                    double2 d[K][P];
#pragma unroll
                    for (int kt = 0; kt < K; ++kt)
#pragma unroll
                        for (int bc = 0; bc < P; ++bc) d[kt][bc] = dec[(size_t)kt * P * H + bc * H + swz(p)];
                    const int j = freq[p];
                    const int e = 4 * j + 1;
                    double2 o0[K], o1[K];
#pragma unroll
                    for (int kt = 0; kt < K; ++kt) o0[kt] = o1[kt] = make_double2(0.0, 0.0);
                    const double2* kb2 = args.bsk + gbase + 2 * (size_t)p;
#pragma unroll 1
                    for (int m = 0; m < M; ++m) {
                        // both outputs' key words of this pattern in flight, then
                        // each ciphertext in turn (its own digit order, as the
                        // one-CTA kernel contracts it)
                        double2 k0[P], k1[P];
#pragma unroll
                        for (int jj = 0; jj < P / 2; ++jj) {
                            ldg_pair(kb2 + ((size_t)jj * M + m) * H * 2, k0[2 * jj], k0[2 * jj + 1]);
                            ldg_pair(kb2 + ((size_t)(P / 2 + jj) * M + m) * H * 2, k1[2 * jj], k1[2 * jj + 1]);
                        }
#pragma unroll
                        for (int kt = 0; kt < K; ++kt) {
                            const double2 w = root2n<LOGN, true>(qt_s, rot[kt * M + m] * e);
                            double2 t0 = make_double2(0.0, 0.0), t1 = make_double2(0.0, 0.0);
#pragma unroll
                            for (int bc = 0; bc < P; ++bc) {
                                c_mac(t0, k0[bc], d[kt][bc]);
                                c_mac(t1, k1[bc], d[kt][bc]);
                            }
                            c_mac(o0[kt], w, t0);
                            c_mac(o1[kt], w, t1);
                        }
                    }
#pragma unroll
                    for (int kt = 0; kt < K; ++kt) {
                        double2* pk = dec + (size_t)kt * P * H;
                        pk[swz(p)] = o0[kt];
                        pk[H + swz(p)] = o1[kt];
                    }
                }
            }
            __syncthreads();
            inverse_middle<LOGH, PL::NS - 1>(dec, K, P, tw, tid, nt);

            // last DIT superstage, untwist, round, centred reduction; ACC to TMEM
#pragma unroll
            for (int sl = 0; sl < SLOTS; ++sl) {
                const int ob = tid + sl * nt;
                if (ob >= OWN) continue;
                const int ok = ob / (2 * Q8), oa = (ob / Q8) & 1, on1 = ob % Q8;
                double2* poly = dec + (size_t)ok * P * H + oa * H;
                double2 v[8];
#pragma unroll
                for (int k2 = 0; k2 < 8; ++k2) v[k2] = poly[swz(on1 + Q8 * k2)];
                twiddle<8, Q8, true>(v, tw, on1);
                dft8<true>(v);
                double acc_lo[8], acc_hi[8];
#pragma unroll
                for (int n2 = 0; n2 < 8; ++n2) {
                    const double2 u = c_mul(c_conj(qtab(on1 + Q8 * n2)), v[n2]);
                    const double rlo = rint(u.x);
                    const double rhi = rint(-u.y);
                    acc_lo[n2] = rlo - q * rint(rlo * inv_q);
                    acc_hi[n2] = rhi - q * rint(rhi * inv_q);
                }
                uint32_t w[16];
                pack8(acc_lo, w);
                tm_st16(tmem + tcol(sl), w);
                pack8(acc_hi, w);
                tm_st16(tmem + tcol(sl) + 16, w);
            }
            tm_wait_st();
            __syncthreads();
        }

        // epilogue: ACC words to shared memory, rotation by -b~, extraction
        // (br_fp64_kernel's epilogue)
        if constexpr (T64) {
            typedef unsigned long long u64;
            u64* acc = reinterpret_cast<u64*>(smem_raw);                     // [K][2][N]
#pragma unroll
            for (int sl = 0; sl < SLOTS; ++sl) {
                const int ob = tid + sl * nt;
                if (ob >= OWN) continue;
                const int ok = ob / (2 * Q8), oa = (ob / Q8) & 1, on1 = ob % Q8;
                double lo[8], hi[8];
                uint32_t w[16];
                tm_ld16(tmem + tcol(sl), w);
                tm_wait_ld();
                unpack8(w, lo);
                tm_ld16(tmem + tcol(sl) + 16, w);
                tm_wait_ld();
                unpack8(w, hi);
                u64* dst = acc + (size_t)ok * 2 * N + oa * N;
#pragma unroll
                for (int n2 = 0; n2 < 8; ++n2) {
                    dst[on1 + Q8 * n2] = (u64)__double2ll_rn(lo[n2]);
                    dst[on1 + Q8 * n2 + H] = (u64)__double2ll_rn(hi[n2]);
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
                    const int jx = rem - al * N;
                    args.out_a64[(ct0 + k) * nl * N + rem] = ncoef64<LOGN>(acc + (size_t)k * 2 * N, al - jx + bexp[k]);
                }
                for (int t = tid; t < kv * nl; t += nt) {
                    const int k = t / nl;
                    const int al = t - k * nl;
                    args.out_b64[(ct0 + k) * nl + al] = ncoef64<LOGN>(acc + (size_t)k * 2 * N + N, al + bexp[k]);
                }
            }
        } else {
            uint32_t* acc = reinterpret_cast<uint32_t*>(smem_raw);           // [K][2][N]
#pragma unroll
            for (int sl = 0; sl < SLOTS; ++sl) {
                const int ob = tid + sl * nt;
                if (ob >= OWN) continue;
                const int ok = ob / (2 * Q8), oa = (ob / Q8) & 1, on1 = ob % Q8;
                double lo[8], hi[8];
                uint32_t w[16];
                tm_ld16(tmem + tcol(sl), w);
                tm_wait_ld();
                unpack8(w, lo);
                tm_ld16(tmem + tcol(sl) + 16, w);
                tm_wait_ld();
                unpack8(w, hi);
                uint32_t* dst = acc + (size_t)ok * 2 * N + oa * N;
#pragma unroll
                for (int n2 = 0; n2 < 8; ++n2) {
                    dst[on1 + Q8 * n2] = (uint32_t)(long long)lo[n2];
                    dst[on1 + Q8 * n2 + H] = (uint32_t)(long long)hi[n2];
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
                    const int jx = rem - al * N;
                    args.out_a[(ct0 + k) * nl * N + rem] = ncoef<LOGN>(acc + (size_t)k * 2 * N, al - jx + bexp[k]);
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
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_slot), "r"(BR_TM_COLS));
}

}  // namespace tfhe
