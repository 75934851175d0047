// Internal declarations of the B200 TFHE programmable-bootstrapping engine.
//
// Polynomials of Z_q[X]/(X^N+1) are carried in the "folded" negacyclic
// Fourier domain: a real polynomial p of degree N is evaluated at the N/2
// points zeta^(4j+1), zeta = exp(-i*pi/N), j in [0, N/2), through one
// H = N/2 point complex FFT of z_k = zeta^k (p_k - i p_{k+H}).  Those points
// hold one root of every conjugate pair, so pointwise products in this
// domain are negacyclic products.  The FFT is decimation-in-frequency
// (forward) / decimation-in-time (inverse) without reordering: Fourier
// values live in "position" order p, with frequency j = freq[p]
// (mixed-radix digit reversal), and every key stored on the device uses
// the same order so the pointwise stage never permutes.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <mutex>
#include <string>

// return a non-OK status from the enclosing function
#define TFHE_TRY(expr)                          \
    do {                                        \
        const int _rc = (expr);                 \
        if (_rc != TFHE_OK) return _rc;         \
    } while (0)

namespace tfhe {

// ----------------------------------------------------------------------------
// status handling shared by the C entry points
// ----------------------------------------------------------------------------
void set_error(const std::string& msg);
// the per-device word kernels set on a bounded-wait timeout (tfhe_device_status)
int* device_status_word();
// counts one kernel launch by this library (tfhe_launch_count)
void count_launch();
// bound of every mbarrier wait, in clock cycles (about 2 s)
constexpr long long WAIT_LIMIT_CYCLES = 4000000000LL;
int fail(int code, const std::string& msg);
int check_cuda(cudaError_t e, const char* what);

// ----------------------------------------------------------------------------
// complex helpers (double2 as re, im)
// ----------------------------------------------------------------------------
__device__ __forceinline__ double2 c_add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 c_sub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 c_mul(double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 c_conj(double2 a) { return make_double2(a.x, -a.y); }
// acc += a * b
__device__ __forceinline__ void c_mac(double2& acc, double2 a, double2 b) {
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(a.y, b.x, acc.y);
}
// multiply by -i, +i
__device__ __forceinline__ double2 c_mul_mi(double2 a) { return make_double2(a.y, -a.x); }
__device__ __forceinline__ double2 c_mul_pi(double2 a) { return make_double2(-a.y, a.x); }

// ----------------------------------------------------------------------------
// radix plan of an H = 2^h point transform: the first superstage is radix 8
// (the register-resident stage of the blind rotation), the others radix 8
// or 16, as few superstages as possible:
//   H = 64: 8.8   128: 8.16   256: 8.8.4   512: 8.8.8   1024: 8.8.16   2048: 8.16.16
// ----------------------------------------------------------------------------
constexpr int plan_stages(int logh) { return logh <= 7 ? 2 : 3; }
constexpr int plan_radix(int logh, int s) {
    return logh == 6 ? 8
         : logh == 7 ? (s == 0 ? 8 : 16)
         : logh == 8 ? (s < 2 ? 8 : 4)
         : logh == 9 ? 8
         : logh == 10 ? (s < 2 ? 8 : 16)
         : (s == 0 ? 8 : 16);                       // logh == 11
}

template <int LOGH>
struct Plan {
    static_assert(LOGH >= 6 && LOGH <= 11, "transform size H = 64 .. 2048");
    static constexpr int H = 1 << LOGH;
    static constexpr int NS = plan_stages(LOGH);    // superstages
    static constexpr int radix(int s) { return plan_radix(LOGH, s); }
    // span of superstage s (elements between the inputs of one butterfly)
    static constexpr int span(int s) {
        int prod = 1;
        for (int i = 0; i <= s; ++i) prod *= radix(i);
        return H / prod;
    }
    // offset of superstage s's twiddle table (R-1 rows of span entries)
    static constexpr int tw_offset(int s) {
        int off = 0;
        for (int i = 0; i < s; ++i) off += (radix(i) - 1) * span(i);
        return off;
    }
    static constexpr int TW = tw_offset(NS);        // total per-stage twiddles
};

// XOR swizzle of 16-byte elements inside 128-byte rows (row r = e >> 3,
// column e & 7 XOR (r ^ r >> 1) & 7): the warp accesses of every superstage
// (strides 1, 2, 4, 8 and 16 elements, spans 8..128) and of the pointwise
// stage take the minimum of 4 wavefronts per 32 16-byte requests.
__device__ __forceinline__ int swz(int e) { return e ^ (((e >> 3) ^ (e >> 4)) & 7); }

// slot of root r in the swizzled shared-memory quarter table: the low three
// bits (16-byte bank group) are XORed with bits 3.. and bits log2 N - 3..,
// so both a warp's run of consecutive roots and the X^r lookups of one
// pointwise pass (roots N/8 apart) fall in distinct bank groups
template <int LOGN>
__device__ __forceinline__ int qsw(int r) {
    return r ^ (((r >> 3) ^ (r >> (LOGN - 3))) & 7);
}

// exp(-i pi idx / N) for any idx, from the quarter table qt[r] =
// exp(-i pi r / N), r in [0, N/2) (stored at qsw(r) when SW)
template <int LOGN, bool SW = false>
__device__ __forceinline__ double2 root2n(const double2* qt, int idx) {
    constexpr int N = 1 << LOGN;
    idx &= (2 * N - 1);
    const int quad = idx >> (LOGN - 1);
    const int r = idx & (N / 2 - 1);
    const double2 w = qt[SW ? qsw<LOGN>(r) : r];
    // multiply by (-i)^quad with selects (lanes take different quadrants)
    const bool odd = quad & 1, neg = quad & 2;
    const double x = odd ? w.y : w.x;
    const double y = odd ? -w.x : w.y;
    return neg ? make_double2(-x, -y) : make_double2(x, y);
}

// Slot of root r in the rotation-order copy of the quarter table.  The X^r
// factors one warp needs in the pointwise stage have table indices that
// differ by multiples of N/8 (the slots' evaluation points differ in the last
// superstage's digit), so r, r + N/8, r + N/4 and r + 3N/8 are stored side by
// side: a warp's lookups then touch about two or three 128-byte lines instead
// of five or six.
template <int LOGN>
__device__ __forceinline__ int rot_slot(int r) {
    constexpr int E = (1 << LOGN) / 8;
    return ((r & (E - 1)) << 2) | (r >> (LOGN - 3));
}

// root2n from the rotation-order table
template <int LOGN>
__device__ __forceinline__ double2 root2n_rot(const double2* qr, int idx) {
    constexpr int N = 1 << LOGN;
    idx &= (2 * N - 1);
    const int quad = idx >> (LOGN - 1);
    const double2 w = qr[rot_slot<LOGN>(idx & (N / 2 - 1))];
    const bool odd = quad & 1, neg = quad & 2;
    const double x = odd ? w.y : w.x;
    const double y = odd ? -w.x : w.y;
    return neg ? make_double2(-x, -y) : make_double2(x, y);
}

// ----------------------------------------------------------------------------
// small DFTs in registers, natural order in and out
// ----------------------------------------------------------------------------
template <bool INV>
__device__ __forceinline__ void dft2(double2& a, double2& b) {
    const double2 t = a;
    a = c_add(t, b);
    b = c_sub(t, b);
}

template <bool INV>
__device__ __forceinline__ void dft4(double2 (&v)[4]) {
    double2 a0 = c_add(v[0], v[2]), a2 = c_sub(v[0], v[2]);
    double2 a1 = c_add(v[1], v[3]), a3 = c_sub(v[1], v[3]);
    a3 = INV ? c_mul_pi(a3) : c_mul_mi(a3);
    v[0] = c_add(a0, a1);
    v[2] = c_sub(a0, a1);
    v[1] = c_add(a2, a3);
    v[3] = c_sub(a2, a3);
}

template <bool INV>
__device__ __forceinline__ void dft8(double2 (&v)[8]) {
    constexpr double R2 = 0.70710678118654752440084436210485;
    // span-4 butterflies with exp(-+2 pi i n / 8)
    double2 a[8];
#pragma unroll
    for (int n = 0; n < 4; ++n) {
        a[n] = c_add(v[n], v[n + 4]);
        a[n + 4] = c_sub(v[n], v[n + 4]);
    }
    if (!INV) {
        a[5] = make_double2(R2 * (a[5].x + a[5].y), R2 * (a[5].y - a[5].x));
        a[6] = c_mul_mi(a[6]);
        a[7] = make_double2(R2 * (a[7].y - a[7].x), -R2 * (a[7].x + a[7].y));
    } else {
        a[5] = make_double2(R2 * (a[5].x - a[5].y), R2 * (a[5].x + a[5].y));
        a[6] = c_mul_pi(a[6]);
        a[7] = make_double2(-R2 * (a[7].x + a[7].y), R2 * (a[7].x - a[7].y));
    }
    // span-2 butterflies on each half with exp(-+2 pi i n / 4)
    double2 b[8];
#pragma unroll
    for (int h = 0; h < 8; h += 4) {
        b[h + 0] = c_add(a[h + 0], a[h + 2]);
        b[h + 2] = c_sub(a[h + 0], a[h + 2]);
        b[h + 1] = c_add(a[h + 1], a[h + 3]);
        b[h + 3] = c_sub(a[h + 1], a[h + 3]);
        b[h + 3] = INV ? c_mul_pi(b[h + 3]) : c_mul_mi(b[h + 3]);
    }
    // span-1 butterflies; results land bit-reversed: X[k] = c[bitrev3(k)]
    double2 c[8];
#pragma unroll
    for (int h = 0; h < 8; h += 2) {
        c[h] = c_add(b[h], b[h + 1]);
        c[h + 1] = c_sub(b[h], b[h + 1]);
    }
    v[0] = c[0]; v[1] = c[4]; v[2] = c[2]; v[3] = c[6];
    v[4] = c[1]; v[5] = c[5]; v[6] = c[3]; v[7] = c[7];
}

// exp(-+ i pi m / 8), m = 0..7
__device__ __forceinline__ double2 w16(int m, bool inv) {
    constexpr double C[8] = {1.0, 0.92387953251128675613, 0.70710678118654752440, 0.38268343236508977173,
                             0.0, -0.38268343236508977173, -0.70710678118654752440, -0.92387953251128675613};
    constexpr double S[8] = {0.0, 0.38268343236508977173, 0.70710678118654752440, 0.92387953251128675613,
                             1.0, 0.92387953251128675613, 0.70710678118654752440, 0.38268343236508977173};
    return make_double2(C[m], inv ? S[m] : -S[m]);
}

// 16-point DFT: four radix-2 DIF stages with constant twiddles, then the
// bit-reversal permutation
template <bool INV>
__device__ __forceinline__ void dft16(double2 (&v)[16]) {
#pragma unroll
    for (int half = 8; half >= 1; half >>= 1) {
#pragma unroll
        for (int blk = 0; blk < 16; blk += 2 * half) {
#pragma unroll
            for (int j = 0; j < half; ++j) {
                const double2 a = v[blk + j], b = v[blk + j + half];
                v[blk + j] = c_add(a, b);
                const double2 d = c_sub(a, b);
                const int m = j * (8 / half);                 // angle pi * m / 8
                if (m == 0) v[blk + j + half] = d;
                else if (m == 4) v[blk + j + half] = INV ? c_mul_pi(d) : c_mul_mi(d);
                else v[blk + j + half] = c_mul(d, w16(m, INV));
            }
        }
    }
    double2 t[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) t[k] = v[((k & 1) << 3) | ((k & 2) << 1) | ((k & 4) >> 1) | ((k & 8) >> 3)];
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = t[k];
}

template <int R, bool INV>
__device__ __forceinline__ void dft(double2 (&v)[R]) {
    if constexpr (R == 16) dft16<INV>(v);
    else if constexpr (R == 8) dft8<INV>(v);
    else if constexpr (R == 4) dft4<INV>(v);
    else dft2<INV>(v[0], v[1]);
}

// ----------------------------------------------------------------------------
// superstages on one swizzled polynomial in shared memory
//
// forward (DIF) superstage at radix R, span S, butterfly b in [0, H/R):
//   n1 = b % S, base = (b / S) R S + n1, inputs x[base + S n2],
//   y = DFT_R(x), y[k2] *= W_{RS}^{n1 k2}, output y[k2] -> base + S k2.
// inverse (DIT) superstage undoes it with conjugate twiddles (times R).
// tw: per-stage table, row k2-1 of length S holds W_{RS}^{n1 k2}.
// ----------------------------------------------------------------------------
template <int R, int S, bool INV>
__device__ __forceinline__ void twiddle(double2 (&v)[R], const double2* tw, int n1) {
    if constexpr (S > 1) {
#pragma unroll
        for (int k2 = 1; k2 < R; ++k2) {
            const double2 w = tw[(k2 - 1) * S + n1];
            v[k2] = c_mul(v[k2], INV ? c_conj(w) : w);
        }
    }
}

template <int R, int S>
__device__ __forceinline__ void dif_stage(double2* poly, const double2* tw, int b) {
    const int n1 = b % S;
    const int base = (b / S) * R * S + n1;
    double2 v[R];
#pragma unroll
    for (int n2 = 0; n2 < R; ++n2) v[n2] = poly[swz(base + S * n2)];
    dft<R, false>(v);
    twiddle<R, S, false>(v, tw, n1);
#pragma unroll
    for (int k2 = 0; k2 < R; ++k2) poly[swz(base + S * k2)] = v[k2];
}

template <int R, int S>
__device__ __forceinline__ void dit_stage(double2* poly, const double2* tw, int b) {
    const int n1 = b % S;
    const int base = (b / S) * R * S + n1;
    double2 v[R];
#pragma unroll
    for (int k2 = 0; k2 < R; ++k2) v[k2] = poly[swz(base + S * k2)];
    twiddle<R, S, true>(v, tw, n1);
    dft<R, true>(v);
#pragma unroll
    for (int n2 = 0; n2 < R; ++n2) poly[swz(base + S * n2)] = v[n2];
}

// superstage s over `npoly` consecutive polynomials, spread over the CTA
// one butterfly with its twiddles already in registers
template <int R, int S, bool INV>
__device__ __forceinline__ void stage_bfly(double2* poly, const double2 (&w)[R], int b) {
    const int n1 = b % S;
    const int base = (b / S) * R * S + n1;
    double2 v[R];
    if (!INV) {
#pragma unroll
        for (int n2 = 0; n2 < R; ++n2) v[n2] = poly[swz(base + S * n2)];
        dft<R, false>(v);
#pragma unroll
        for (int k2 = 1; k2 < R; ++k2) v[k2] = c_mul(v[k2], w[k2]);
#pragma unroll
        for (int k2 = 0; k2 < R; ++k2) poly[swz(base + S * k2)] = v[k2];
    } else {
#pragma unroll
        for (int k2 = 0; k2 < R; ++k2) v[k2] = poly[swz(base + S * k2)];
#pragma unroll
        for (int k2 = 1; k2 < R; ++k2) v[k2] = c_mul(v[k2], c_conj(w[k2]));
        dft<R, true>(v);
#pragma unroll
        for (int n2 = 0; n2 < R; ++n2) poly[swz(base + S * n2)] = v[n2];
    }
}

template <int LOGH, int s, bool INV>
__device__ __forceinline__ void stage_all(double2* polys, int npoly, const double2* tw_all, int tid, int nt) {
    using P = Plan<LOGH>;
    constexpr int R = P::radix(s);
    constexpr int S = P::span(s);
    constexpr int PER = P::H / R;
    const double2* tw = tw_all + P::tw_offset(s);
    const int total = npoly * PER;
    if (S > 1 && R <= 8 && nt % PER == 0) {
        // every task of this thread is the same butterfly of another
        // polynomial: load its twiddles once
        const int b = tid % PER;
        double2 w[R];
        w[0] = make_double2(1.0, 0.0);
#pragma unroll
        for (int k2 = 1; k2 < R; ++k2) w[k2] = tw[(k2 - 1) * S + b % S];
        for (int t = tid; t < total; t += nt) stage_bfly<R, S, INV>(polys + (t / PER) * P::H, w, b);
        return;
    }
    for (int t = tid; t < total; t += nt) {
        double2* poly = polys + (t / PER) * P::H;
        if (INV) dit_stage<R, S>(poly, tw, t % PER);
        else dif_stage<R, S>(poly, tw, t % PER);
    }
}

// rne(x / 2^s) of a centred 64-bit value, 1 <= s <= 63 (the reference's
// round half to even, on the exact integer)
__device__ __forceinline__ long long rne_div_pow2(long long x, int s) {
    long long d = x >> s;
    const unsigned long long low = (unsigned long long)x & ((1ULL << s) - 1ULL);
    const unsigned long long half = 1ULL << (s - 1);
    if (low > half || (low == half && (d & 1))) d += 1;
    return d;
}

// ----------------------------------------------------------------------------
// asynchronous 1D bulk copies into this CTA's own shared memory, and mbarriers
// ----------------------------------------------------------------------------
// device status word values (tfhe_device_status)
constexpr int TFHE_STATUS_WAIT_TIMEOUT = 1;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void prefetch_l1(const void* p) {
    asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

// hint: bring [p, p + bytes) into L2 (p 16-byte aligned, bytes a multiple of
// 16); nothing waits for it
__device__ __forceinline__ void prefetch_l2_bulk(const void* p, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// make barrier initialisation visible to the async (TMA) proxy
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// order this thread's earlier generic-proxy shared-memory accesses before
// later async-proxy writes to the same buffer
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// global -> shared bulk copy completing `bytes` of transaction on `bar`;
// dst, src 16-byte aligned, bytes a multiple of 16
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// wait for phase `parity` of `bar` for at most `limit` clock cycles; on
// timeout record TFHE_STATUS_WAIT_TIMEOUT in *status and return false (the
// caller carries on, so every thread still reaches every barrier)
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, long long limit, int* status) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > limit) {
            if (status) atomicExch(status, TFHE_STATUS_WAIT_TIMEOUT);
            return false;
        }
    }
    return true;
}

// ----------------------------------------------------------------------------
// device-resident FFT plan for one degree (built once per device and N)
// ----------------------------------------------------------------------------
struct FftPlan {
    int N = 0;
    double2* qt = nullptr;     // N/2: exp(-i pi r / N)
    double2* qr = nullptr;     // the same N/2 roots in rotation order (rot_slot)
    double2* tw = nullptr;     // Plan<LOGH>::TW per-stage twiddles
    uint16_t* freq = nullptr;  // H: frequency of each position
    int tw_count = 0;
};

// returns nullptr (and sets the error) when the table cannot be built
const FftPlan* get_plan(int N);

// host helpers used by the launchers
int plan_tw_count(int logh);
size_t br_table_bytes(int N);

}  // namespace tfhe
