// Small-batch blind rotation: one ciphertext per cluster of 2 S CTAs
// (S = 2: four CTAs, S = 4: eight).
//
// At batch 1 the cluster-pair kernel (br_split.cuh) spends about half of each
// group in the pointwise stage (n=742 N=2048: 8.8k of 16.6k cycles; n=630
// N=1024 with eight patterns: 12.0k of 18.9k), pulling output r's half of the
// group's key into one SM.  Here CTA (r, h) (cluster rank r + 2 h, h < S) owns
// ACC polynomial r and part h of the S parts of the spectrum's positions:
//   * the prologue transforms the gadget digits of polynomial r at the levels
//     lvl with lvl % S == h (one forward FFT at most where l_bs <= S);
//   * after a cluster barrier, the pointwise stage computes output r at the
//     positions of part h, from the cluster's digit spectra (distributed
//     shared memory) and the key words of those positions only: 1 / (2 S) of
//     the group's key per SM;
//   * the inverse superstages but the last stay inside a part (their
//     butterfly groups span at most H/8 positions, a part at least H/4);
//     after a second cluster barrier the S CTAs of polynomial r each run the
//     last superstage over all parts (8/S of its 8 points per part), so each
//     holds the whole next ACC polynomial r for its next prologue.
// Where a part holds fewer positions than the CTA has threads, TPS = 2 or 4
// adjacent lanes share a position, lane u contracting the u-th M/TPS
// patterns, and each lane continues the sum of the lanes before it after a
// shuffle, so the sum over patterns keeps its order.  Every value is computed by the
// same operations in the same order as br_fp64_kernel (digits, FFT stages,
// the key contraction in digit order per pattern, the twist products in
// pattern order, the rounding), so the outputs are bit-identical to it.
//
// Shared memory is single-buffered.  CTA (r, h) rewrites its digit spectra in
// group g + 1 only after the second barrier of group g, which every CTA
// reaches after its pointwise reads of group g; it rewrites its output part in
// group g + 1 only after the first barrier of group g + 1, which the other CTAs
// of polynomial r reach after their last-superstage reads of group g.  A
// barrier after each ciphertext's last group keeps the output parts alive for
// those reads before the epilogue reuses them, and a last one keeps each CTA's
// shared memory until no peer reads it.  Every thread of the cluster reaches
// the same barriers the same number of times (loop bounds depend only on the
// cluster index).
#pragma once

#include "br_split.cuh"

namespace tfhe {

constexpr int BR_CLUSTER_THREADS = 512;
constexpr int BR_CLUSTER_MAX_M = 8;   // patterns (collapse <= 3)

// shared memory of br_cluster_kernel: the own digit levels [ceil(L/S)][H],
// the output polynomial [H] (part h used), the tables, the rotation indices
// of every group and b~
inline size_t br_cluster_smem(int N, int L, int G, int M, size_t table_bytes, int S) {
    const int H = N / 2;
    const int LH = (L + S - 1) / S;
    return (size_t)(LH + 1) * H * sizeof(double2) + table_bytes + ((size_t)G * M + 1) * sizeof(int) + 16;
}

// inverse superstages s = S0 .. 1 over the butterflies of part h of the
// NP parts of one polynomial (their groups of R * span <= H / 8 positions lie
// inside a part of H / NP >= H / 4)
template <int LOGH, int s, int NP>
__device__ __forceinline__ void inverse_middle_part(double2* poly, int h, const double2* tw, int tid, int nt) {
    if constexpr (s >= 1) {
        using PL = Plan<LOGH>;
        constexpr int R = PL::radix(s);
        constexpr int SP = PL::span(s);
        constexpr int PERP = PL::H / R / NP;
        static_assert(PERP % SP == 0, "whole butterfly groups per part");
        const double2* tws = tw + PL::tw_offset(s);
        for (int t = tid; t < PERP; t += nt) dit_stage<R, SP>(poly, tws, h * PERP + t);
        __syncthreads();
        inverse_middle_part<LOGH, s - 1, NP>(poly, h, tw, tid, nt);
    }
}

template <int LOGN, int L, bool T64, int S>
__global__ void __launch_bounds__(BR_CLUSTER_THREADS, 1) br_cluster_kernel(const BrArgs args) {
    constexpr int N = 1 << LOGN;
    constexpr int H = N / 2;
    constexpr int LOGH = LOGN - 1;
    constexpr int P = 2 * L;
    constexpr int Q8 = H / 8;
    constexpr int LH = (L + S - 1) / S;                  // own digit levels at most
    constexpr int PART = H / S;                          // positions per part
    constexpr int PPP = 8 / S;                           // last-superstage points per part
    constexpr int TPS = BR_CLUSTER_THREADS / PART;       // lanes per position in the pointwise stage
    using PL = Plan<LOGH>;
    static_assert(S == 2 || S == 4, "clusters of four or eight CTAs");
    static_assert(TPS == 1 || TPS == 2 || TPS == 4, "one, two or four lanes per position");
    static_assert(Q8 * PPP == PART, "the last superstage reads 8/S points of each part");

    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int M = args.M;
    double2* spec = reinterpret_cast<double2*>(smem_raw);   // [LH][H]: levels h, h + S, ...
    double2* outp = spec + LH * H;                           // [H]
    double2* qt_s = outp + H;                                // N / 2, swizzled
    double2* tw = qt_s + N / 2;                              // PL::TW
    uint16_t* freq = reinterpret_cast<uint16_t*>(tw + PL::TW);
    int* rot_all = reinterpret_cast<int*>(freq + H);         // G * M
    int* bexp = rot_all + (size_t)args.G * M;                // 1
    auto qtab = [&](int x) { return qt_s[qsw<LOGN>(x)]; };

    const int tid = threadIdx.x;
    const int nt = blockDim.x;
    const int rank = (int)cluster_rank();
    const int r = rank & 1;                                  // ACC polynomial / output
    const int h = rank >> 1;                                 // part of the positions, levels mod S
    const long long cl = cluster_index_x();
    const long long ncl = cluster_count_x();
    const long long mine = cl < args.B ? (args.B - cl + ncl - 1) / ncl : 0;
    const int cl32 = (int)cl, ncl32 = (int)ncl;              // at most the SM count

    for (int i = tid; i < N / 2; i += nt) qt_s[qsw<LOGN>(i)] = args.qt[i];
    for (int i = tid; i < PL::TW; i += nt) tw[i] = args.tw[i];
    for (int i = tid; i < H; i += nt) freq[i] = args.freq[i];
    uint32_t spec_of[2 * S];                                 // digit spectra of each rank
#pragma unroll
    for (int k = 0; k < 2 * S; ++k) spec_of[k] = peer_smem(spec, (uint32_t)k);
    uint32_t out_of[S];                                      // output parts of polynomial r
#pragma unroll
    for (int k = 0; k < S; ++k) out_of[k] = peer_smem(outp, (uint32_t)(r + 2 * k));
    cluster_barrier();                                       // every CTA of the cluster has started

    const bool owner = tid < Q8;
    const int on1 = tid;
    const int nown = h < L ? (L - 1 - h) / S + 1 : 0;        // own digit levels
    const double q = ldexp(1.0, args.log2_q);
    const double inv_q = ldexp(1.0, -args.log2_q);
    const double beta = ldexp(1.0, args.log2_beta);
    const double inv_qb = ldexp(1.0, args.log2_beta - args.log2_q);

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
        // rotation indices of every group (br_fp64_kernel's formulas), up
        // front; read after the first group's barriers
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

        for (int g = 0; g < args.G; ++g) {
            // the next group's key words of (output r, part h) into L2: one
            // region (digit pair, pattern) per cluster in turn
            if (g + 1 < args.G && args.l2_prefetch) {
                const int regions = (P / 2) * M;
                for (int i = tid; i < regions; i += nt)
                    if (i % ncl32 == cl32) {
                        const double2* base = args.bsk + (size_t)(g + 1) * 2 * P * M * H +
                                              (size_t)r * (P / 2) * M * H * 2 + (size_t)i * H * 2 +
                                              (size_t)h * PART * 2;
                        prefetch_l2_bulk(base, (uint32_t)(PART * 2 * sizeof(double2)));
                    }
            }
            const int* rot = rot_all + (size_t)g * M;

            // prologue: the digit levels lvl = h, h + S, ... of polynomial r,
            // fold + twist, first DIF superstage
            if (owner) {
                double2 w0[8];
                w0[0] = make_double2(1.0, 0.0);
#pragma unroll
                for (int k2 = 1; k2 < 8; ++k2) w0[k2] = tw[(k2 - 1) * Q8 + on1];
                if constexpr (LH == 1) {
                    // l_bs <= S: one own level at most (lvl = h), its digits
                    // from the chain run up to it (the chain's operations, so
                    // the same digits); one straight-line body keeps the
                    // registers low
                    if (nown > 0) {
                        double2 v[8];
#pragma unroll
                        for (int n2 = 0; n2 < 8; ++n2) {
                            double ylo = acc_lo[n2] * inv_qb;
                            double dlo = rint(ylo);
                            double yhi = acc_hi[n2] * inv_qb;
                            double dhi = rint(yhi);
#pragma unroll
                            for (int l2 = 1; l2 < L; ++l2)
                                if (l2 <= h) {
                                    ylo = (ylo - dlo) * beta;
                                    dlo = rint(ylo);
                                    yhi = (yhi - dhi) * beta;
                                    dhi = rint(yhi);
                                }
                            const double2 w = qtab(on1 + Q8 * n2);
                            v[n2] = make_double2(fma(w.x, dlo, w.y * dhi), fma(w.y, dlo, -w.x * dhi));
                        }
                        dft8<false>(v);
#pragma unroll
                        for (int k2 = 1; k2 < 8; ++k2) v[k2] = c_mul(v[k2], w0[k2]);
#pragma unroll
                        for (int k2 = 0; k2 < 8; ++k2) spec[swz(on1 + Q8 * k2)] = v[k2];
                    }
                } else {
                    // l_bs > S: every level's digits and transform (the chain
                    // runs through all of them), stored for the own levels
                    // only, so every part runs one instruction stream
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
                        double2* poly = spec + (lvl / S) * H;
                        const bool own_level = (lvl % S) == h;
#pragma unroll
                        for (int k2 = 0; k2 < 8; ++k2)
                            if (own_level) poly[swz(on1 + Q8 * k2)] = v[k2];
                    }
                }
            }
            __syncthreads();
            forward_middle<LOGH, 1>(spec, nown, tw, tid, nt);
            cluster_barrier();                               // all digit spectra are complete

            // pointwise: output r at the positions of part h,
            // out = sum_m X^{r_m} * sum_bc BSK[g, r, bc, m] * DEC[bc]
            {
                const size_t gbase = (size_t)g * 2 * P * M * H;
                const int p = h * PART + tid / TPS;
                double2 d[P];
#pragma unroll
                for (int lvl = 0; lvl < L; ++lvl)
#pragma unroll
                    for (int in = 0; in < 2; ++in) {
                        const int src = in + 2 * (lvl % S);          // rank holding digit (lvl, in)
                        const int e_off = (lvl / S) * H + swz(p);
                        d[2 * lvl + in] = src == rank ? spec[e_off]
                                                      : ld_peer(spec_of[src] + (uint32_t)(e_off * sizeof(double2)));
                    }
                const int j = freq[p];
                const int e = 4 * j + 1;
                const double2* kb2 = args.bsk + gbase + 2 * (size_t)p + (size_t)r * (P / 2) * M * H * 2;
                double2 o = make_double2(0.0, 0.0);
                if constexpr (TPS == 1) {
                    // br_split_kernel's contraction: the key words of MC
                    // patterns in flight together
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
                } else {
                    // lane u of the position contracts patterns
                    // [u M/TPS, (u+1) M/TPS) (M a multiple of TPS); lane 0
                    // also applies its twists, the other lanes keep their
                    // sums until the total of the lanes before them arrives
                    const int u = tid % TPS;
                    const int mlen = M / TPS;
                    const int mbeg = u * mlen;
                    double2 tt[BR_CLUSTER_MAX_M / 2];
#pragma unroll
                    for (int i = 0; i < BR_CLUSTER_MAX_M / 2; ++i) {
                        tt[i] = make_double2(0.0, 0.0);
                        if (i < mlen) {
                            const int m = mbeg + i;
                            double2 k[P];
#pragma unroll
                            for (int jj = 0; jj < P / 2; ++jj)
                                ldg_pair(kb2 + ((size_t)jj * M + m) * H * 2, k[2 * jj], k[2 * jj + 1]);
                            double2 t = make_double2(0.0, 0.0);
#pragma unroll
                            for (int bc = 0; bc < P; ++bc) c_mac(t, k[bc], d[bc]);
                            if (u == 0) {
                                const double2 w = root2n<LOGN, true>(qt_s, rot[m] * e);
                                c_mac(o, w, t);
                            } else {
                                tt[i] = t;
                            }
                        }
                    }
#pragma unroll
                    for (int lane = 1; lane < TPS; ++lane) {
                        // lane `lane` continues the sum of lanes 0 .. lane - 1
                        double2 prev;
                        prev.x = __shfl_up_sync(0xffffffffu, o.x, 1);
                        prev.y = __shfl_up_sync(0xffffffffu, o.y, 1);
                        if (u == lane) {
                            o = prev;
#pragma unroll
                            for (int i = 0; i < BR_CLUSTER_MAX_M / 2; ++i)
                                if (i < mlen) {
                                    const double2 w = root2n<LOGN, true>(qt_s, rot[mbeg + i] * e);
                                    c_mac(o, w, tt[i]);
                                }
                        }
                    }
                    if (u == TPS - 1) outp[swz(p)] = o;
                }
            }
            __syncthreads();
            inverse_middle_part<LOGH, PL::NS - 1, S>(outp, h, tw, tid, nt);
            cluster_barrier();                               // every part of output r is transformed

            // last DIT superstage over all parts, untwist, round, centred
            // reduction: the whole next ACC polynomial r
            if (owner) {
                double2 v[8];
#pragma unroll
                for (int k2 = 0; k2 < 8; ++k2) {
                    const int e_off = swz(on1 + Q8 * k2);
                    v[k2] = k2 / PPP == h ? outp[e_off] : ld_peer(out_of[k2 / PPP] + (uint32_t)(e_off * sizeof(double2)));
                }
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
        }
        cluster_barrier();                                   // the peers have read this CTA's output part

        // epilogue: polynomial r rotated by -b~; the CTAs of polynomial 0
        // extract the masks, those of polynomial 1 the bodies, each part h
        // of the words
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
                for (int i = h * (N / S) + tid; i < (h + 1) * (N / S); i += nt)
                    args.acc_out64[ct * 2 * N + r * N + i] = ncoef64<LOGN>(acc, i + bx);
            const int nl = args.n_lut;
            if (args.out_a64 && r == 0)
                for (int t = h * nl * (N / S) + tid; t < (h + 1) * nl * (N / S); t += nt) {
                    const int al = t / N;
                    const int jx = t - al * N;
                    args.out_a64[ct * nl * N + t] = ncoef64<LOGN>(acc, al - jx + bx);
                }
            if (args.out_b64 && r == 1 && h == 0)
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
                for (int i = h * (N / S) + tid; i < (h + 1) * (N / S); i += nt)
                    args.acc_out[ct * 2 * N + r * N + i] = ncoef<LOGN>(acc, i + bx);
            const int nl = args.n_lut;
            if (args.out_a && r == 0)
                for (int t = h * nl * (N / S) + tid; t < (h + 1) * nl * (N / S); t += nt) {
                    const int al = t / N;
                    const int jx = t - al * N;
                    args.out_a[ct * nl * N + t] = ncoef<LOGN>(acc, al - jx + bx);
                }
            if (args.out_b && r == 1 && h == 0)
                for (int al = tid; al < nl; al += nt) args.out_b[ct * nl + al] = ncoef<LOGN>(acc, al + bx);
        }
        __syncthreads();                                     // outp is reused by the next ciphertext
    }
    cluster_barrier();                                       // no peer reads this CTA's shared memory any more
}

}  // namespace tfhe
