// Small-batch blind rotation: one ciphertext per cluster of two CTAs.
//
// The latency of one ciphertext is its walk over all G groups; a single CTA
// walks it on one SM.  Here CTA r (r = 0, 1: its rank in the cluster) owns
// ACC polynomial r (the mask for r = 0, the body for r = 1):
//   * the prologue takes the L gadget digits of its own polynomial only
//     (digits bc = 2 lvl + r) and transforms them: L forward FFTs, not 2L;
//   * after one cluster barrier, the pointwise stage of CTA r computes output
//     r over all P = 2L digits, reading the peer's L digit spectra from its
//     shared memory (distributed shared memory, no copy) and only the key
//     words of output r (half the key);
//   * one inverse FFT gives the next ACC polynomial r, which is again the
//     polynomial this CTA decomposes in the next group.
// So each SM does half the work of the one-CTA kernel, and the pair exchanges
// nothing but the digit spectra read in place.  Every value is computed by
// the same operations in the same order as br_fp64_kernel's native and T64
// paths (the digits, the FFT stages, the key contraction in digit order per
// pattern, the rounding), so the outputs are bit-identical to them.
//
// Digit spectra are double-buffered by group parity: CTA r rewrites buffer
// s & 1 in step s + 2 only after passing the barrier of step s + 1, which the
// peer reaches after its pointwise reads of step s.  A last cluster barrier
// keeps each CTA's shared memory alive until the peer has finished with it.
// The barriers are hardware cluster barriers reached the same number of
// times by every thread of both CTAs (the loop bounds depend only on the
// cluster index), so they always complete.
#pragma once

#include "br_fp64.cuh"

namespace tfhe {

constexpr int BR_SPLIT_THREADS = 512;

__device__ __forceinline__ uint32_t cluster_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

__device__ __forceinline__ uint32_t cluster_index_x() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(r));
    return r;
}

__device__ __forceinline__ uint32_t cluster_count_x() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%nclusterid.x;" : "=r"(r));
    return r;
}

// all threads of both CTAs; release / acquire orders the shared-memory
// writes before it with the peer's reads after it
__device__ __forceinline__ void cluster_barrier() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// address of the same shared-memory location in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t peer_smem(const void* p, uint32_t rank) {
    uint32_t out;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(out) : "r"(smem_addr(p)), "r"(rank));
    return out;
}

__device__ __forceinline__ double2 ld_peer(uint32_t addr) {
    double2 v;
    asm volatile("ld.shared::cluster.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"(addr) : "memory");
    return v;
}

// inverse superstages s = S0 .. 1 of one polynomial (inverse_middle's
// operations on a single output)
template <int LOGH, int s>
__device__ __forceinline__ void inverse_middle_one(double2* poly, const double2* tw, int tid, int nt) {
    if constexpr (s >= 1) {
        using PL = Plan<LOGH>;
        constexpr int R = PL::radix(s);
        constexpr int S = PL::span(s);
        constexpr int PER = PL::H / R;
        const double2* tws = tw + PL::tw_offset(s);
        for (int t = tid; t < PER; t += nt) dit_stage<R, S>(poly, tws, t);
        __syncthreads();
        inverse_middle_one<LOGH, s - 1>(poly, tw, tid, nt);
    }
}

// shared memory of br_split_kernel: digit spectra [2][L][H], the output
// polynomial [H], the tables, the rotation indices of every group and b~
inline size_t br_split_smem(int N, int L, int G, int M, size_t table_bytes) {
    const int H = N / 2;
    return (size_t)(2 * L + 1) * H * sizeof(double2) + table_bytes + ((size_t)G * M + 1) * sizeof(int) + 16;
}

template <int LOGN, int L, bool T64>
__global__ void __launch_bounds__(BR_SPLIT_THREADS, 1) br_split_kernel(const BrArgs args) {
    constexpr int N = 1 << LOGN;
    constexpr int H = N / 2;
    constexpr int LOGH = LOGN - 1;
    constexpr int P = 2 * L;
    constexpr int Q8 = H / 8;
    using PL = Plan<LOGH>;
    static_assert(Q8 <= BR_SPLIT_THREADS, "one radix-8 butterfly owner per thread at most");

    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int M = args.M;
    double2* spec = reinterpret_cast<double2*>(smem_raw);   // [2 parity][L][H]
    double2* outp = spec + 2 * L * H;                        // [H]
    double2* qt_s = outp + H;                                // N / 2, swizzled
    double2* tw = qt_s + N / 2;                              // PL::TW
    uint16_t* freq = reinterpret_cast<uint16_t*>(tw + PL::TW);
    int* rot_all = reinterpret_cast<int*>(freq + H);         // G * M
    int* bexp = rot_all + (size_t)args.G * M;                // 1
    auto qtab = [&](int r) { return qt_s[qsw<LOGN>(r)]; };

    const int tid = threadIdx.x;
    const int nt = blockDim.x;
    const int r = (int)cluster_rank();
    const long long cl = cluster_index_x();
    const long long ncl = cluster_count_x();
    const long long mine = cl < args.B ? (args.B - cl + ncl - 1) / ncl : 0;

    for (int i = tid; i < N / 2; i += nt) qt_s[qsw<LOGN>(i)] = args.qt[i];
    for (int i = tid; i < PL::TW; i += nt) tw[i] = args.tw[i];
    for (int i = tid; i < H; i += nt) freq[i] = args.freq[i];
    const uint32_t peer_spec = peer_smem(spec, (uint32_t)(r ^ 1));
    cluster_barrier();                                       // the peer has started

    const bool owner = tid < Q8;
    const int on1 = tid;
    const double q = ldexp(1.0, args.log2_q);
    const double inv_q = ldexp(1.0, -args.log2_q);
    const double beta = ldexp(1.0, args.log2_beta);
    const double inv_qb = ldexp(1.0, args.log2_beta - args.log2_q);

    int step = 0;
    for (long long it = 0; it < mine; ++it) {
        const long long ct = cl + it * ncl;
        double acc_lo[8], acc_hi[8];
        if (owner) {
            if constexpr (T64) {
                const long long* src = args.lut64 + ct * args.lut_stride + r * N;
#pragma unroll
                for (int n2 = 0; n2 < 8; ++n2) {
                    acc_lo[n2] = (double)src[on1 + Q8 * n2];
                    acc_hi[n2] = (double)src[on1 + Q8 * n2 + H];
                }
            } else {
                const uint32_t* src = args.lut + ct * args.lut_stride + r * N;
#pragma unroll
                for (int n2 = 0; n2 < 8; ++n2) {
                    acc_lo[n2] = (double)(int32_t)src[on1 + Q8 * n2];
                    acc_hi[n2] = (double)(int32_t)src[on1 + Q8 * n2 + H];
                }
            }
        } else {
#pragma unroll
            for (int n2 = 0; n2 < 8; ++n2) acc_lo[n2] = acc_hi[n2] = 0.0;
        }
        // rotation indices of every group of this ciphertext, up front (the
        // formulas of br_fp64_kernel), so no group waits on a global load;
        // read after the first group's barriers
        for (int t = tid; t < args.G * M; t += nt) {
            const int g = t / M, m = t - g * M;
            int rr;
            if constexpr (T64) {
                unsigned long long v = 0ULL;
                const unsigned long long* a = args.lwe_a64 + ct * args.lwe_n + (long long)g * args.collapse;
                for (int c = 0; c < args.collapse; ++c)
                    if ((m >> (args.collapse - 1 - c)) & 1) v += a[c];
                const int ln = __ffs(args.n_lut) - 1;
                const long long d = rne_div_pow2((long long)v, 63 - LOGN + ln);
                rr = (int)((d << ln) & (2 * N - 1));
            } else {
                double v = 0.0;
                const uint32_t* a = args.lwe_a + ct * args.lwe_n + (long long)g * args.collapse;
                for (int c = 0; c < args.collapse; ++c)
                    if ((m >> (args.collapse - 1 - c)) & 1) v += (double)(int32_t)a[c];
                const double idx = rint((2.0 * N * v) / (q * args.n_lut)) * args.n_lut;
                const int ri = (int)idx % (2 * N);
                rr = ri < 0 ? ri + 2 * N : ri;
            }
            rot_all[t] = rr;
        }

        for (int g = 0; g < args.G; ++g, ++step) {
            double2* mine_spec = spec + (size_t)(step & 1) * L * H;
            const uint32_t peer_base = peer_spec + (uint32_t)((step & 1) * L * H * sizeof(double2));
            // the next group's key words of output r into L2 (each cluster its
            // share), as the one-CTA kernel does for its whole block
            if (tid == 0 && g + 1 < args.G && args.l2_prefetch) {
                const size_t half = (size_t)P * M * H * sizeof(double2);      // output r's block
                const size_t share = ((half / (size_t)ncl) + 255) & ~(size_t)255;
                const size_t off = (size_t)cl * share;
                if (off < half) {
                    const size_t len = min(share, half - off);
                    const char* base = reinterpret_cast<const char*>(args.bsk + (size_t)(g + 1) * 2 * P * M * H +
                                                                     (size_t)r * P * M * H);
                    prefetch_l2_bulk(base + off, (uint32_t)len);
                }
            }
            const int* rot = rot_all + (size_t)g * M;

            // prologue: the digits of this CTA's polynomial, fold + twist,
            // first DIF superstage
            if (owner) {
                double2 w0[8];
                w0[0] = make_double2(1.0, 0.0);
#pragma unroll
                for (int k2 = 1; k2 < 8; ++k2) w0[k2] = tw[(k2 - 1) * Q8 + on1];
                if constexpr (L <= 2) {
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
                        double2* poly = mine_spec + lvl * H;
#pragma unroll
                        for (int k2 = 0; k2 < 8; ++k2) poly[swz(on1 + Q8 * k2)] = v[lvl][k2];
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
                            const double2 w = qtab(on1 + Q8 * n2);
                            v[n2] = make_double2(fma(w.x, dlo, w.y * dhi), fma(w.y, dlo, -w.x * dhi));
                        }
                        dft8<false>(v);
#pragma unroll
                        for (int k2 = 1; k2 < 8; ++k2) v[k2] = c_mul(v[k2], w0[k2]);
                        double2* poly = mine_spec + lvl * H;
#pragma unroll
                        for (int k2 = 0; k2 < 8; ++k2) poly[swz(on1 + Q8 * k2)] = v[k2];
                    }
                }
            }
            __syncthreads();
            forward_middle<LOGH, 1>(mine_spec, L, tw, tid, nt);
            cluster_barrier();                               // both CTAs' digit spectra are complete

            // pointwise: output r = sum_m X^{r_m} * sum_bc BSK[g, r, bc, m] * DEC[bc]
            {
                const size_t gbase = (size_t)g * 2 * P * M * H;
                for (int p = tid; p < H; p += nt) {
                    double2 d[P];
#pragma unroll
                    for (int lvl = 0; lvl < L; ++lvl) {
                        const double2 own = mine_spec[lvl * H + swz(p)];
                        const double2 other =
                            ld_peer(peer_base + (uint32_t)((lvl * H + swz(p)) * sizeof(double2)));
                        d[2 * lvl + r] = own;
                        d[2 * lvl + (r ^ 1)] = other;
                    }
                    const int j = freq[p];
                    const int e = 4 * j + 1;
                    double2 o = make_double2(0.0, 0.0);
                    const double2* kb2 = args.bsk + gbase + 2 * (size_t)p + (size_t)r * (P / 2) * M * H * 2;
                    // one ciphertext per SM leaves little to hide a key load's
                    // latency behind: the key words of MC patterns are all in
                    // flight before the first of them is contracted (the
                    // contraction keeps the pattern order: same operations,
                    // same order as the one-CTA kernel)
                    constexpr int MC = (8 / P) >= 4 ? 4 : ((8 / P) >= 2 ? 2 : 1);
#pragma unroll 1
                    for (int m0 = 0; m0 < M; m0 += MC) {
                        double2 k[MC][P];
#pragma unroll
                        for (int mc = 0; mc < MC; ++mc)
                            if (m0 + mc < M) {
#pragma unroll
                                for (int jj = 0; jj < P / 2; ++jj)
                                    ldg_pair(kb2 + ((size_t)jj * M + m0 + mc) * H * 2, k[mc][2 * jj],
                                             k[mc][2 * jj + 1]);
                            }
#pragma unroll
                        for (int mc = 0; mc < MC; ++mc)
                            if (m0 + mc < M) {
                                double2 t = make_double2(0.0, 0.0);
#pragma unroll
                                for (int bc = 0; bc < P; ++bc) c_mac(t, k[mc][bc], d[bc]);
                                const double2 w = root2n<LOGN, true>(qt_s, rot[m0 + mc] * e);
                                c_mac(o, w, t);
                            }
                    }
                    outp[swz(p)] = o;
                }
            }
            __syncthreads();
            inverse_middle_one<LOGH, PL::NS - 1>(outp, tw, tid, nt);

            // last DIT superstage, untwist, round, centred reduction
            if (owner) {
                double2 v[8];
#pragma unroll
                for (int k2 = 0; k2 < 8; ++k2) v[k2] = outp[swz(on1 + Q8 * k2)];
                twiddle<8, Q8, true>(v, tw, on1);
                dft8<true>(v);
#pragma unroll
                for (int n2 = 0; n2 < 8; ++n2) {
                    const double2 u = c_mul(c_conj(qtab(on1 + Q8 * n2)), v[n2]);
                    const double rlo = rint(u.x);
                    const double rhi = rint(-u.y);
                    acc_lo[n2] = rlo - q * rint(rlo * inv_q);
                    acc_hi[n2] = rhi - q * rint(rhi * inv_q);
                }
            } else {
                // written on every path, so the accumulator is dead (no
                // registers held) between the prologue and this point
#pragma unroll
                for (int n2 = 0; n2 < 8; ++n2) acc_lo[n2] = acc_hi[n2] = 0.0;
            }
            __syncthreads();
        }

        // epilogue: polynomial r rotated by -b~; CTA 0 extracts the masks,
        // CTA 1 the bodies
        if constexpr (T64) {
            typedef unsigned long long u64;
            u64* acc = reinterpret_cast<u64*>(outp);          // N words
            if (owner) {
#pragma unroll
                for (int n2 = 0; n2 < 8; ++n2) {
                    acc[on1 + Q8 * n2] = (u64)__double2ll_rn(acc_lo[n2]);
                    acc[on1 + Q8 * n2 + H] = (u64)__double2ll_rn(acc_hi[n2]);
                }
            }
            if (tid == 0) {
                const int ln = __ffs(args.n_lut) - 1;
                bexp[0] = (int)((rne_div_pow2((long long)args.lwe_b64[ct], 63 - LOGN + ln) << ln) & (2 * N - 1));
            }
            __syncthreads();
            const int bx = bexp[0];
            if (args.acc_out64)
                for (int i = tid; i < N; i += nt) args.acc_out64[ct * 2 * N + r * N + i] = ncoef64<LOGN>(acc, i + bx);
            const int nl = args.n_lut;
            if (args.out_a64 && r == 0)
                for (int t = tid; t < nl * N; t += nt) {
                    const int al = t / N;
                    const int jx = t - al * N;
                    args.out_a64[ct * nl * N + t] = ncoef64<LOGN>(acc, al - jx + bx);
                }
            if (args.out_b64 && r == 1)
                for (int al = tid; al < nl; al += nt) args.out_b64[ct * nl + al] = ncoef64<LOGN>(acc, al + bx);
        } else {
            uint32_t* acc = reinterpret_cast<uint32_t*>(outp);
            if (owner) {
#pragma unroll
                for (int n2 = 0; n2 < 8; ++n2) {
                    acc[on1 + Q8 * n2] = (uint32_t)(long long)acc_lo[n2];
                    acc[on1 + Q8 * n2 + H] = (uint32_t)(long long)acc_hi[n2];
                }
            }
            if (tid == 0) {
                const double b = (double)(int32_t)args.lwe_b[ct];
                bexp[0] = (int)(rint((2.0 * N * b) / (q * args.n_lut)) * args.n_lut);
            }
            __syncthreads();
            const int bx = bexp[0];
            if (args.acc_out)
                for (int i = tid; i < N; i += nt) args.acc_out[ct * 2 * N + r * N + i] = ncoef<LOGN>(acc, i + bx);
            const int nl = args.n_lut;
            if (args.out_a && r == 0)
                for (int t = tid; t < nl * N; t += nt) {
                    const int al = t / N;
                    const int jx = t - al * N;
                    args.out_a[ct * nl * N + t] = ncoef<LOGN>(acc, al - jx + bx);
                }
            if (args.out_b && r == 1)
                for (int al = tid; al < nl; al += nt) args.out_b[ct * nl + al] = ncoef<LOGN>(acc, al + bx);
        }
        __syncthreads();                                     // outp is reused by the next ciphertext
    }
    cluster_barrier();                                       // the peer no longer reads this CTA's spectra
}

}  // namespace tfhe
