// C entry points, FFT plans, key upload, key switching and sample extraction
// of the B200 TFHE PBS engine.  See include/tfhe_b200.h for the contract.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <initializer_list>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <tuple>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/tfhe_b200.h"
#include "tfhe_dispatch.h"
#include "tfhe_internal.cuh"

struct tfhe_keys {
    tfhe_params p;
    int device = -1;
    int G = 0, M = 0;
    double2* bsk = nullptr;     // [G][2][L][M][N/2][2] FP64 Fourier, position order
    uint32_t* ksk = nullptr;    // [n_big * l_ks][ldk]: columns 0..n-1 mask, n body
    int ldk = 0;
    const tfhe::FftPlan* plan = nullptr;
    int64_t bytes = 0;
    int ring_kr = 0;            // > 0: key in the ring layout for K == ring_kr per CTA
    tfhe_tuning tune = {0, -1, -1, -1, -1};   // launch shapes (0 / -1: automatic)
    unsigned char* ksk_limbs = nullptr;  // int8 limbs of the key-switching key for the tensor cores
    int ks_npad = 0;                     // limb rows (4 (n+1) rounded up to the CTA tile)
};

namespace tfhe {

// ---------------------------------------------------------------- errors
static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

int check_cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return TFHE_OK;
    const std::string msg = std::string(what) + ": " + cudaGetErrorString(e);
    if (e == cudaErrorMemoryAllocation) return fail(TFHE_ERR_OUT_OF_MEMORY, msg);
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return fail(TFHE_ERR_NO_DEVICE, msg);
    return fail(TFHE_ERR_INTERNAL, msg);
}


// ---------------------------------------------------------------- FFT plans
static int ilog2(long long v) {
    int r = -1;
    while (v) { v >>= 1; ++r; }
    return r;
}

static bool is_pow2(long long v) { return v > 0 && (v & (v - 1)) == 0; }

// radix sequence of an H = 2^logh point transform (same as Plan<LOGH>)
static std::vector<int> radices(int logh) {
    std::vector<int> r;
    for (int st = 0; st < plan_stages(logh); ++st) r.push_back(plan_radix(logh, st));
    return r;
}

int plan_tw_count(int logh) {
    const std::vector<int> r = radices(logh);
    const int H = 1 << logh;
    int prod = 1, total = 0;
    for (int R : r) {
        prod *= R;
        total += (R - 1) * (H / prod);
    }
    return total;
}

// exp(-i pi k / N) with the angle reduced in long double
static double2 root(long long k, int N) {
    k %= 2LL * N;
    if (k < 0) k += 2LL * N;
    const long double pi = 3.141592653589793238462643383279502884L;
    const long double ang = pi * (long double)k / (long double)N;
    return make_double2((double)cosl(ang), (double)(-sinl(ang)));
}

static void build_tables(int N, std::vector<double2>& qt, std::vector<double2>& tw, std::vector<uint16_t>& freq) {
    const int H = N / 2;
    const int logh = ilog2(H);
    qt.resize(N / 2);
    for (int r = 0; r < N / 2; ++r) qt[r] = root(r, N);
    const std::vector<int> rs = radices(logh);
    tw.clear();
    int prod = 1;
    for (int R : rs) {
        prod *= R;
        const int S = H / prod;
        for (int k2 = 1; k2 < R; ++k2)
            for (int n1 = 0; n1 < S; ++n1)
                tw.push_back(root((long long)(2 * N / (R * S)) * n1 * k2, N));
    }
    // frequency of position p: p = S1 * k2 + pos_{S1}(k1) for k = R1 k1 + k2
    freq.resize(H);
    for (int p = 0; p < H; ++p) {
        int rem = p, size = H, mult = 1, k = 0;
        for (int R : rs) {
            const int S = size / R;
            const int k2 = rem / S;
            k += mult * k2;
            mult *= R;
            rem %= S;
            size = S;
        }
        freq[p] = (uint16_t)k;
    }
}

static std::mutex g_plan_mu;
static std::map<std::pair<int, int>, FftPlan*> g_plans;   // (device, N)

// The status word kernels write on a bounded-wait timeout: one static word
// per device, so no entry point ever allocates device memory for it.  Its
// device address is looked up once per device (the host-side name is not a
// device address) and cached.
static __device__ int g_device_status_word;
static std::map<int, int*> g_status;                      // device -> address of the word

int* device_status_word() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    std::lock_guard<std::mutex> lk(g_plan_mu);
    auto it = g_status.find(dev);
    if (it != g_status.end()) return it->second;
    int* w = nullptr;
    if (cudaGetSymbolAddress((void**)&w, g_device_status_word) != cudaSuccess) return nullptr;
    g_status[dev] = w;
    return w;
}

const FftPlan* get_plan(int N) {
    int dev = 0;
    if (check_cuda(cudaGetDevice(&dev), "cudaGetDevice") != TFHE_OK) return nullptr;
    std::lock_guard<std::mutex> lk(g_plan_mu);
    auto it = g_plans.find({dev, N});
    if (it != g_plans.end()) return it->second;
    std::vector<double2> qt, tw;
    std::vector<uint16_t> freq;
    build_tables(N, qt, tw, freq);
    FftPlan* pl = new FftPlan();
    pl->N = N;
    pl->tw_count = (int)tw.size();
    // rotation-order copy: root r at ((r mod N/8) << 2) | (r div N/8), as rot_slot
    std::vector<double2> qr(qt.size());
    for (int r = 0; r < N / 2; ++r) qr[((r % (N / 8)) << 2) | (r / (N / 8))] = qt[r];
    bool ok = cudaMalloc(&pl->qt, qt.size() * sizeof(double2)) == cudaSuccess &&
              cudaMalloc(&pl->qr, qr.size() * sizeof(double2)) == cudaSuccess &&
              cudaMalloc(&pl->tw, tw.size() * sizeof(double2)) == cudaSuccess &&
              cudaMalloc(&pl->freq, freq.size() * sizeof(uint16_t)) == cudaSuccess &&
              cudaMemcpy(pl->qt, qt.data(), qt.size() * sizeof(double2), cudaMemcpyHostToDevice) == cudaSuccess &&
              cudaMemcpy(pl->qr, qr.data(), qr.size() * sizeof(double2), cudaMemcpyHostToDevice) == cudaSuccess &&
              cudaMemcpy(pl->tw, tw.data(), tw.size() * sizeof(double2), cudaMemcpyHostToDevice) == cudaSuccess &&
              cudaMemcpy(pl->freq, freq.data(), freq.size() * sizeof(uint16_t), cudaMemcpyHostToDevice) == cudaSuccess;
    if (!ok) {
        set_error("FFT plan upload failed: " + std::string(cudaGetErrorString(cudaGetLastError())));
        cudaFree(pl->qt);
        cudaFree(pl->qr);
        cudaFree(pl->tw);
        cudaFree(pl->freq);
        delete pl;
        return nullptr;
    }
    g_plans[{dev, N}] = pl;
    return pl;
}

size_t br_table_bytes(int N) {
    const int H = N / 2;
    return (size_t)(N / 2) * sizeof(double2) + (size_t)plan_tw_count(ilog2(H)) * sizeof(double2) +
           (size_t)H * sizeof(uint16_t);
}

static int sm_count() {
    static int cached[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return 148;
    if (!cached[dev]) {
        int v = 0;
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
        cached[dev] = v;
    }
    return cached[dev];
}

static int max_smem_optin() {
    static int cached[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return 48 * 1024;
    if (!cached[dev]) {
        int v = 0;
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess || v <= 0)
            v = 48 * 1024;
        cached[dev] = v;
    }
    return cached[dev];
}

// ---------------------------------------------------------------- BR launch
struct BrShape {
    int K = 0, nt = 0;
    size_t smem = 0;
    int kr = 0, stages = 0;   // key ring (kr > 0)
    int kt = 1;               // ciphertexts per thread in the pointwise stage
    bool qtg = false;         // quarter root table in global memory (two CTAs per SM)
    bool xt = false;          // more threads than butterfly owners (XT kernels)
};

static int max_smem_per_sm() {
    static int cached[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return 0;          // unknown: never place two CTAs per SM
    if (!cached[dev]) {
        int v = 0;
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess || v <= 0)
            v = 0;
        cached[dev] = v > 0 ? v : -1;
    }
    return cached[dev] > 0 ? cached[dev] : 0;
}


// a mbarrier wait gives up after this many cycles (about 2 s)

// ciphertexts per CTA: as many as 512 threads and shared memory allow, or
// TFHE_B200_K (tuning: K = 1 lets two CTAs share an SM)
static int k_override() {
    static const int v = [] {
        const char* env = getenv("TFHE_B200_K");
        return env ? atoi(env) : 0;
    }();
    return v;
}

static BrShape br_shape(int N, int L, int M, long long B, int k_request = 0, bool allow_qtg = false) {
    const int H = N / 2, Q8 = H / 8;
    const size_t per_ct = (size_t)2 * L * H * sizeof(double2);
    const size_t limit = (size_t)max_smem_optin();
    BrShape s;
    int K = std::max(1, 512 / (2 * Q8));
    const int kreq = k_request > 0 ? k_request : k_override();
    if (kreq > 0) {
        K = std::min(K, kreq);
    } else {
        // a batch smaller than one full wave: spread it over every SM, since
        // a CTA's time grows with its ciphertext count while idle SMs add nothing
        const long long sms = std::max(1, sm_count());
        const long long per_sm = (B + sms - 1) / sms;
        if (per_sm < K) K = (int)std::max<long long>(1, per_sm);
    }
    K = (int)std::min<long long>(K, std::max<long long>(B, 1));
    const int KT = (K % 2 == 0 && br_kt(ilog2(N), L) == 2) ? 2 : 1;
    while (K >= KT) {
        const size_t smem = per_ct * K + br_table_bytes(N) + (size_t)(K * M + K) * sizeof(int) + 16;
        if (smem <= limit) {
            s.K = K;
            // 2 K N/16 threads own the butterflies of the register-resident
            // superstages; where the kernel allows extra threads they make it
            // 512 whatever K is, all of them sharing the shared-memory
            // superstages and the pointwise stage, so a batch under one wave
            // (small K) still runs 16 warps per SM
            s.nt = br_extra_threads(L) ? std::max(K * 2 * Q8, 512) : K * 2 * Q8;
            s.xt = s.nt > K * 2 * Q8;
            s.smem = smem;
            s.kt = (K % KT == 0) ? KT : 1;
            // two CTAs per SM where they fit once the quarter root table is
            // read from global memory (automatic shapes halve K for it): their
            // phases drift apart, so one CTA's FFT overlaps the other's key
            // loads (n=630 N=1024: 181.2 -> 166.8 ms per 16384 ciphertexts)
            // (only for batches beyond one CTA per SM: below that the one-CTA
            // layout of 512 threads is the faster of the two)
            if (allow_qtg && s.kt == 2 && B > (long long)K * std::max(1, sm_count())) {
                const int K2 = (kreq <= 0 && K % 4 == 0) ? K / 2 : K;
                const size_t smem2 = per_ct * K2 + br_table_bytes(N) - (size_t)(N / 2) * sizeof(double2) +
                                     (size_t)(K2 * M + K2) * sizeof(int) + 16;
                if (2 * (smem2 + 1024) <= (size_t)max_smem_per_sm()) {
                    s.K = K2;
                    s.nt = K2 * 2 * Q8;
                    s.xt = false;
                    s.smem = smem2;
                    s.kt = 2;
                    s.qtg = true;
                }
            }
            return s;
        }
        K -= KT;
    }
    return s;
}

// Key-ring shape: K = KR = 2 ciphertexts per CTA, NT = KR H / 4 threads,
// chunks of 2L * NT key words, as many stages (2..4) as shared memory holds.
// Opt-in with TFHE_B200_KEY_RING=1 when the keys are created: on B200 the
// per-thread loads of the plain kernel are merged across SMs at L2 (all CTAs
// walk the key in lockstep) while bulk copies are not, so the plain kernel
// is faster for the workloads measured here.
static BrShape ring_shape(int N, int L, int M) {
    BrShape s;
    const char* env = getenv("TFHE_B200_KEY_RING");
    if (!env || env[0] != '1') return s;
    const int H = N / 2, KR = 2, P = 2 * L;
    const int nt = KR * H / 4;
    if (nt < 64 || nt > 512 || KR * P > 12) return s;
    const size_t chunk = (size_t)P * nt * sizeof(double2);
    size_t base = (size_t)KR * P * H * sizeof(double2) + br_table_bytes(N) + (size_t)(KR * M + KR) * sizeof(int);
    base = (base + 127) & ~(size_t)127;
    const size_t limit = (size_t)max_smem_optin();
    if (base + 2 * (chunk + 8) > limit) return s;
    const int stages = (int)std::min<size_t>(4, (limit - base) / (chunk + 8));
    s.K = KR;
    s.nt = nt;
    s.kr = KR;
    s.stages = stages;
    s.smem = base + stages * chunk + stages * 8;
    return s;
}

// kernel attributes set once per kernel (also keeps launches capturable in a
// CUDA graph after the first, uncaptured launch) and occupancy per shape
static std::mutex g_attr_mu;
static std::map<std::pair<int, const void*>, int> g_attr_smem;
static std::map<std::tuple<int, const void*, int, size_t>, int> g_occupancy;

// the dynamic shared-memory attribute of a kernel, raised once per device
// and size (later launches make no attribute call, and can be captured)
int smem_attr_once(const void* kern, size_t smem) {
    int dev = 0;
    TFHE_TRY(check_cuda(cudaGetDevice(&dev), "cudaGetDevice"));
    std::lock_guard<std::mutex> lk(g_attr_mu);
    int& have = g_attr_smem[{dev, kern}];
    if (have < (int)smem) {
        TFHE_TRY(check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                            "cudaFuncSetAttribute(dynamic shared memory)"));
        have = (int)smem;
    }
    return TFHE_OK;
}

static int prepare_kernel(const void* kern, int nt, size_t smem, int* per_sm) {
    int dev = 0;
    TFHE_TRY(check_cuda(cudaGetDevice(&dev), "cudaGetDevice"));
    std::lock_guard<std::mutex> lk(g_attr_mu);
    int& have = g_attr_smem[{dev, kern}];
    if (have < (int)smem) {
        TFHE_TRY(check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                            "cudaFuncSetAttribute(blind rotation)"));
        have = (int)smem;
    }
    auto key = std::make_tuple(dev, kern, nt, smem);
    auto it = g_occupancy.find(key);
    if (it == g_occupancy.end()) {
        int v = 1;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, kern, nt, smem) != cudaSuccess || v < 1) v = 1;
        it = g_occupancy.emplace(key, v).first;
    }
    *per_sm = it->second;
    return TFHE_OK;
}

// One ciphertext per cluster of two CTAs (br_split.cuh) for batches that fit
// in one wave of clusters.  TFHE_B200_SPLIT=0 turns it off; an explicitly
// requested shape (tuning, TFHE_B200_K) never takes it.
static bool split_enabled() {
    static const bool on = [] {
        const char* env = getenv("TFHE_B200_SPLIT");
        return !(env && env[0] == '0');
    }();
    return on;
}

// one ciphertext per cluster of `csize` CTAs: grid csize * B
static int launch_cluster(BrKernel kern, int nt, size_t smem, int csize, const BrArgs& args, int N,
                          cudaStream_t stream, const tfhe_tuning* tune, const char* what) {
    int per_sm = 1;
    TFHE_TRY(prepare_kernel((const void*)kern, nt, smem, &per_sm));
    BrArgs a = args;
    const FftPlan* pl = get_plan(N);
    if (!pl) return TFHE_ERR_INTERNAL;
    a.qt = pl->qt;
    a.qr = pl->qr;
    a.tw = pl->tw;
    a.freq = pl->freq;
    a.K = 1;
    a.l2_prefetch = (tune && tune->l2_prefetch == 0) ? 0 : 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(csize * args.B), 1, 1);
    cfg.blockDim = dim3(nt, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = csize;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    count_launch();
    return check_cuda(cudaLaunchKernelEx(&cfg, kern, a), what);
}

static int launch_split(const BrArgs& args, int N, int L, cudaStream_t stream, const tfhe_tuning* tune) {
    const bool t64 = args.lwe_a64 != nullptr;
    BrKernel kern = br_split_kernel_for(ilog2(N), L, t64);
    if (!kern) return fail(TFHE_ERR_INVALID_ARGUMENT, "unsupported degree / levels");
    return launch_cluster(kern, BR_SPLIT_THREADS, br_split_smem(N, L, args.G, args.M, br_table_bytes(N)), 2, args, N,
                          stream, tune, "blind rotation launch (cluster pair)");
}

// one ciphertext per cluster of 2 S CTAs (br_cluster.cuh)
static int launch_cluster_s(const BrArgs& args, int N, int L, int S, cudaStream_t stream, const tfhe_tuning* tune) {
    const bool t64 = args.lwe_a64 != nullptr;
    BrKernel kern = br_cluster_kernel_for(ilog2(N), L, t64, S);
    if (!kern) return fail(TFHE_ERR_INVALID_ARGUMENT, "unsupported degree / levels");
    return launch_cluster(kern, BR_CLUSTER_THREADS, br_cluster_smem(N, L, args.G, args.M, br_table_bytes(N), S),
                          2 * S, args, N, stream, tune,
                          S == 4 ? "blind rotation launch (cluster of eight)" : "blind rotation launch (cluster of four)");
}

// clusters of `csize` CTAs of this kernel that can be resident at once (a
// GPC whose free SMs are not a multiple of the cluster size leaves some out),
// cached per device, kernel and shape
static long long resident_clusters(BrKernel kern, int nt, size_t smem, int csize) {
    if (!kern) return 0;
    if (smem > (size_t)max_smem_optin()) return 0;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    static std::mutex mu;
    static std::map<std::tuple<int, const void*, size_t>, long long> cache;
    std::lock_guard<std::mutex> lk(mu);
    auto key = std::make_tuple(dev, (const void*)kern, smem);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    long long n = 0;
    if (cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) == cudaSuccess) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)(csize * std::max(1, sm_count())), 1, 1);
        cfg.blockDim = dim3(nt, 1, 1);
        cfg.dynamicSmemBytes = smem;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = csize;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int c = 0;
        if (cudaOccupancyMaxActiveClusters(&c, (const void*)kern, &cfg) == cudaSuccess) n = c;
    }
    cudaGetLastError();   // a refused query only disables the cluster form
    cache.emplace(key, n);
    return n;
}

static long long split_resident_clusters(int N, int L, int G, int M, bool t64) {
    return resident_clusters(br_split_kernel_for(ilog2(N), L, t64), BR_SPLIT_THREADS,
                             br_split_smem(N, L, G, M, br_table_bytes(N)), 2);
}

// One ciphertext per cluster of 2 S CTAs (br_cluster.cuh): eight CTAs (S = 4)
// or four (S = 2) at N = 1024 and 2048, for batches that fit one wave of
// such clusters (eight at N = 1024 needs at least four patterns); each SM then pulls 1 / (2 S) of a group's key in the
// pointwise stage.  TFHE_B200_QUAD=0 turns both off (the pair then takes those
// batches), TFHE_B200_OCTET=0 only the clusters of eight.
static bool quad_enabled() {
    static const bool on = [] {
        const char* env = getenv("TFHE_B200_QUAD");
        return !(env && env[0] == '0');
    }();
    return on;
}

static bool octet_enabled() {
    static const bool on = [] {
        const char* env = getenv("TFHE_B200_OCTET");
        return !(env && env[0] == '0');
    }();
    return on;
}

// CTAs per polynomial (S = 4 or 2) of the widest cluster form that takes this
// batch, 0 for none
static int cluster_form(int N, int L, int G, int M, long long B, bool reflayout, int kr, const tfhe_tuning* tune,
                        bool t64) {
    const bool requested = (tune && tune->ciphertexts_per_cta > 0) || k_override() > 0;
    if (kr != 0 || reflayout || requested || L > 3 || M > BR_CLUSTER_MAX_M || M < 2 || !quad_enabled() ||
        !split_enabled() || B < 1)
        return 0;
    for (int S : {4, 2}) {
        if (S == 4 && !octet_enabled()) continue;
        if (2 * S * B > sm_count()) continue;
        // lanes per position in the pointwise stage: each takes M / lanes patterns
        const int lanes = BR_CLUSTER_THREADS / (N / 2 / S);
        if (lanes > 1 && M % lanes != 0) continue;
        BrKernel kern = br_cluster_kernel_for(ilog2(N), L, t64, S);
        if (!kern) continue;
        if (B <= resident_clusters(kern, BR_CLUSTER_THREADS, br_cluster_smem(N, L, G, M, br_table_bytes(N), S),
                                   2 * S))
            return S;
    }
    return 0;
}

static bool split_applies(int N, int L, int G, int M, long long B, bool reflayout, int kr,
                          const tfhe_tuning* tune, bool t64) {
    const bool requested = (tune && tune->ciphertexts_per_cta > 0) || k_override() > 0;
    if (kr != 0 || reflayout || requested || L > 3 || !split_enabled() || B < 1 || 2 * B > sm_count()) return false;
    return B <= split_resident_clusters(N, L, G, M, t64);
}

// the arguments of ciphertexts full .. B - 1 of a launch
static BrArgs args_after(const BrArgs& args, long long full, int N) {
    BrArgs tail = args;
    tail.B = args.B - full;
    if (tail.lwe_a) tail.lwe_a += full * args.lwe_n;
    if (tail.lwe_b) tail.lwe_b += full;
    if (tail.lut) tail.lut += full * args.lut_stride;
    if (tail.ct_init) tail.ct_init += full * args.ct_stride;
    if (tail.indices) tail.indices += full * (long long)args.G * args.M;
    if (tail.acc_out) tail.acc_out += full * 2 * N;
    if (tail.out_a) tail.out_a += full * args.n_lut * N;
    if (tail.out_b) tail.out_b += full * args.n_lut;
    if (tail.out_i64) tail.out_i64 += full * 2 * N;
    if (tail.lwe_a64) tail.lwe_a64 += full * args.lwe_n;
    if (tail.lwe_b64) tail.lwe_b64 += full;
    if (tail.lut64) tail.lut64 += full * args.lut_stride;
    if (tail.acc_out64) tail.acc_out64 += full * 2 * N;
    if (tail.out_a64) tail.out_a64 += full * args.n_lut * N;
    if (tail.out_b64) tail.out_b64 += full * args.n_lut;
    return tail;
}

// Three ciphertexts per CTA with the accumulators in tensor memory
// (br_tm.cuh) at N = 2048, l_bs <= 2: requested with ciphertexts_per_cta = 3,
// or automatic when TFHE_B200_TM=1; whole rounds of 3 x SMs ciphertexts go to
// it, the rest to the launch shapes below.
static bool tm_default() {
    static const bool on = [] {
        const char* env = getenv("TFHE_B200_TM");
        return env && env[0] == '1';
    }();
    return on;
}

static int launch_tm(const BrArgs& args, int N, int L, cudaStream_t stream, const tfhe_tuning* tune,
                     long long full) {
    const bool t64 = args.lwe_a64 != nullptr;
    BrKernel kern = br_tm_kernel_for(ilog2(N), L, t64);
    if (!kern) return fail(TFHE_ERR_INVALID_ARGUMENT, "unsupported degree / levels");
    const size_t smem = br_tm_smem(N, L, 3, args.M, br_table_bytes(N));
    int per_sm = 1;
    TFHE_TRY(prepare_kernel((const void*)kern, BR_TM_THREADS, smem, &per_sm));
    BrArgs a = args;
    const FftPlan* pl = get_plan(N);
    if (!pl) return TFHE_ERR_INTERNAL;
    a.qt = pl->qt;
    a.qr = pl->qr;
    a.tw = pl->tw;
    a.freq = pl->freq;
    a.K = 3;
    a.B = full;
    a.l2_prefetch = (tune && tune->l2_prefetch == 0) ? 0 : 1;
    count_launch();
    kern<<<(unsigned)sm_count(), BR_TM_THREADS, smem, stream>>>(a);
    return check_cuda(cudaGetLastError(), "blind rotation launch (tensor memory)");
}

static int launch_br(BrArgs args, int N, int L, bool reflayout, int kr, cudaStream_t stream,
                     int* status = nullptr, const tfhe_tuning* tune = nullptr) {
    const int logn = ilog2(N);
    const bool requested = (tune && tune->ciphertexts_per_cta > 0) || k_override() > 0;
    if (const int S = cluster_form(N, L, args.G, args.M, args.B, reflayout, kr, tune, args.lwe_a64 != nullptr))
        return launch_cluster_s(args, N, L, S, stream, tune);
    if (split_applies(N, L, args.G, args.M, args.B, reflayout, kr, tune, args.lwe_a64 != nullptr))
        return launch_split(args, N, L, stream, tune);
    if (!reflayout && kr == 0 && N == 2048 && L <= 2 &&
        ((tune && tune->ciphertexts_per_cta == 3) || (!requested && tm_default())) &&
        br_tm_smem(N, L, 3, args.M, br_table_bytes(N)) <= (size_t)max_smem_optin()) {
        const long long round = 3LL * sm_count();
        const long long full = (args.B / round) * round;
        if (full > 0) {
            TFHE_TRY(launch_tm(args, N, L, stream, tune, full));
            if (full == args.B) return TFHE_OK;
            tfhe_tuning rest_tune = tune ? *tune : tfhe_tuning{0, -1, -1, -1, -1};
            if (rest_tune.ciphertexts_per_cta == 3) rest_tune.ciphertexts_per_cta = 0;
            return launch_br(args_after(args, full, N), N, L, reflayout, kr, stream, status, &rest_tune);
        }
    }
    const BrShape sh = kr > 0 ? ring_shape(N, L, args.M)
                              : br_shape(N, L, args.M, args.B, tune ? tune->ciphertexts_per_cta : 0, !reflayout);
    if (kr > 0 && sh.kr != kr) return fail(TFHE_ERR_INVALID_ARGUMENT, "key ring layout not available for these keys");
    const bool t64 = args.lwe_a64 != nullptr;
    BrKernel kern = t64 ? (kr == 0 ? br_fp64_t64_kernel_for(logn, L, sh.kt, sh.qtg, sh.xt) : nullptr)
                        : br_fp64_kernel_for(logn, L, reflayout, kr, sh.kt, sh.qtg, sh.xt);
    if (!kern) return fail(TFHE_ERR_INVALID_ARGUMENT, "unsupported degree / levels");
    if (sh.K < 1)
        return fail(TFHE_ERR_INVALID_ARGUMENT,
                    "degree " + std::to_string(N) + " with l=" + std::to_string(L) +
                        " does not fit in shared memory");
    const FftPlan* pl = get_plan(N);
    if (!pl) return TFHE_ERR_INTERNAL;
    args.qt = pl->qt;
    args.qr = pl->qr;
    args.tw = pl->tw;
    args.freq = pl->freq;
    args.K = sh.K;
    args.ring_stages = sh.stages;
    args.wait_limit = WAIT_LIMIT_CYCLES;
    // L1 prefetch of the next pattern's key words: off by default.  With the
    // next group's key block prefetched into L2 it costs time at every
    // parameter set measured (n=630 N=1024: 181.2 ms off vs 207.8 ms on per
    // 16384 ciphertexts); TFHE_B200_PREFETCH=1 or the keys' tuning turns it on
    static const int prefetch_env = [] {
        const char* env = getenv("TFHE_B200_PREFETCH");
        return env ? (env[0] == '1' ? 1 : 0) : 0;
    }();
    args.prefetch = (tune && tune->prefetch >= 0) ? tune->prefetch : prefetch_env;
    args.l2_prefetch = (tune && tune->l2_prefetch == 0) ? 0 : 1;
    args.status = status ? status : device_status_word();
    if (!args.status) return fail(TFHE_ERR_INTERNAL, "device status word unavailable");
    int per_sm = 1;
    TFHE_TRY(prepare_kernel((const void*)kern, sh.nt, sh.smem, &per_sm));
    // persistent CTAs: as many as fit on the SMs, looping over ciphertext
    // sets, so all SMs walk the key in lockstep; TFHE_B200_PERSISTENT=0 (or
    // the keys' tuning) launches one CTA per set instead
    const long long sets = (args.B + sh.K - 1) / sh.K;
    static const bool persistent_env = [] {
        const char* env = getenv("TFHE_B200_PERSISTENT");
        return !(env && env[0] == '0');
    }();
    const bool persistent = (tune && tune->persistent >= 0) ? tune->persistent != 0 : persistent_env;
    const long long grid = persistent ? std::min<long long>(sets, (long long)sm_count() * per_sm) : sets;
    // A last round of at most one ciphertext per SM runs as its own launch of
    // the small-batch shape (one ciphertext per CTA, 512 threads): that is
    // faster than a partly filled round of K ciphertexts per CTA (n=742
    // N=2048: 3.9 against 4.95 ms).  Not for explicitly requested shapes.
    if (persistent && kr == 0 && sh.K > 1 && !requested && sets > grid) {
        const long long full = (sets / grid) * grid * sh.K;      // ciphertexts in whole rounds
        const long long rest = args.B - full;
        if (rest > 0 && rest <= sm_count()) {
            BrArgs head = args;
            head.B = full;
            count_launch();
            kern<<<(unsigned)grid, sh.nt, sh.smem, stream>>>(head);
            TFHE_TRY(check_cuda(cudaGetLastError(), "blind rotation launch"));
            return launch_br(args_after(args, full, N), N, L, reflayout, 0, stream, status, tune);
        }
    }
    count_launch();
    kern<<<(unsigned)grid, sh.nt, sh.smem, stream>>>(args);
    return check_cuda(cudaGetLastError(), "blind rotation launch");
}

// ---------------------------------------------------------------- key switch
// out[k][o] = sum_{i,j} d_j(a[k][i]) KSK[i*l + j][o] (mod 2^32); o = n is the
// body column (added to b).  Digits are the float64 steps of
// decomposition (schemas/polynomial_jax.py:98-111) at base 2^log2_beta_ks.
constexpr int KS_TB = 64, KS_TO = 64, KS_KC = 8, KS_LMAX = 8;

// Key rows are addressed by strides so the device layout and the
// reference layout (mask (l, n_big, n), body (l, n_big)) share the kernel:
// mask(i, j, o) = ka[i*si + j*sj + o], body(i, j) = kb[i*bi + j*bj].
struct KsKey {
    const uint32_t* ka;
    const uint32_t* kb;
    long long si, sj, bi, bj;
};

__global__ void __launch_bounds__(256) ks_kernel(const uint32_t* __restrict__ a_in,
                                                 const uint32_t* __restrict__ b_in, const KsKey key,
                                                 int n_big, int n, int l, int log2_beta,
                                                 uint32_t* __restrict__ a_out, uint32_t* __restrict__ b_out,
                                                 long long B) {
    __shared__ int dig[KS_TB][KS_KC * KS_LMAX + 1];
    __shared__ __align__(16) uint32_t kt[KS_KC * KS_LMAX][KS_TO];
    const int tid = threadIdx.x;
    const int ty = tid / 16, tx = tid % 16;
    const long long r0 = (long long)blockIdx.y * KS_TB;
    const int o0 = blockIdx.x * KS_TO;
    const double inv_q = ldexp(1.0, -32);
    const double beta = ldexp(1.0, log2_beta);
    uint32_t acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0u;

    for (int i0 = 0; i0 < n_big; i0 += KS_KC) {
        for (int idx = tid; idx < KS_TB * KS_KC; idx += 256) {
            const int ct = idx / KS_KC, c = idx % KS_KC;
            const long long row = r0 + ct;
            const int i = i0 + c;
            const uint32_t v = (row < B && i < n_big) ? a_in[row * n_big + i] : 0u;
            double x = (double)(int32_t)v * inv_q;
            for (int j = 0; j < l; ++j) {
                const double y = x * beta;
                const double d = rint(y);
                x = y - d;
                dig[ct][c * l + j] = (int)d;
            }
        }
        const int rows = KS_KC * l;
        for (int idx = tid; idx < rows * KS_TO; idx += 256) {
            const int r = idx / KS_TO, col = idx % KS_TO;
            const int i = i0 + r / l, j = r % l;
            const int o = o0 + col;
            uint32_t v = 0u;
            if (i < n_big) {
                if (o < n) v = key.ka[i * key.si + j * key.sj + o];
                else if (o == n) v = key.kb[i * key.bi + j * key.bj];
            }
            kt[r][col] = v;
        }
        __syncthreads();
        for (int r = 0; r < rows; ++r) {
            const uint4 kv = *reinterpret_cast<const uint4*>(&kt[r][tx * 4]);
#pragma unroll
            for (int cc = 0; cc < 4; ++cc) {
                const uint32_t d = (uint32_t)dig[ty * 4 + cc][r];
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
        if (row >= B) continue;
#pragma unroll
        for (int oo = 0; oo < 4; ++oo) {
            const int o = o0 + tx * 4 + oo;
            if (o < n) a_out[row * n + o] = acc[cc][oo];
            else if (o == n) b_out[row] = b_in[row] + acc[cc][oo];
        }
    }
}

static int launch_ks_key(const KsKey& key, int n_big, int n, int l, int log2_beta, const uint32_t* a_in,
                         const uint32_t* b_in, uint32_t* a_out, uint32_t* b_out, long long B, cudaStream_t stream) {
    if (B == 0) return TFHE_OK;
    const dim3 grid((n + 1 + KS_TO - 1) / KS_TO, (unsigned)((B + KS_TB - 1) / KS_TB));
    count_launch();
    ks_kernel<<<grid, 256, 0, stream>>>(a_in, b_in, key, n_big, n, l, log2_beta, a_out, b_out, B);
    return check_cuda(cudaGetLastError(), "key switch launch");
}

static int launch_ks(const tfhe_keys* k, const uint32_t* a_in, const uint32_t* b_in, uint32_t* a_out,
                     uint32_t* b_out, long long B, cudaStream_t stream) {
    // the tensor-core kernel reads the input rows with 16-byte loads
    if (k->ksk_limbs && k->tune.ks_tensor_cores != 0 && (reinterpret_cast<uintptr_t>(a_in) & 15) == 0) {
        int* status = device_status_word();
        if (!status) return fail(TFHE_ERR_INTERNAL, "device status word unavailable");
        KsTcArgs args{a_in, b_in, k->ksk_limbs, k->p.n_big, k->p.n, k->p.l_ks, k->p.log2_beta_ks, k->ks_npad, B,
                      a_out, b_out, WAIT_LIMIT_CYCLES, status, 0, 0, nullptr};
        return launch_ks_tc(args, stream);
    }
    const long long ldk = k->ldk, l = k->p.l_ks;
    const KsKey key{k->ksk, k->ksk + k->p.n, l * ldk, ldk, l * ldk, ldk};
    return launch_ks_key(key, k->p.n_big, k->p.n, k->p.l_ks, k->p.log2_beta_ks, a_in, b_in, a_out, b_out, B,
                         stream);
}

// ---------------------------------------------------------------- extraction
// out_a[k][al][j] = coefficient of X^(al - j) of the mask (negacyclic),
// out_b[k][al] = body[al]  (schemas/text_jax.py:191-208)
__global__ void extract_kernel(const uint32_t* __restrict__ acc, int N, int n_lut, uint32_t* __restrict__ out_a,
                               uint32_t* __restrict__ out_b, long long B) {
    const long long total = B * n_lut * (long long)N;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const long long k = t / ((long long)n_lut * N);
        const int rem = (int)(t - k * n_lut * (long long)N);
        const int al = rem / N, j = rem % N;
        const uint32_t* a = acc + k * 2 * N;
        const int e = al - j;
        out_a[t] = e >= 0 ? a[e] : (0u - a[e + N]);
        if (j == 0) out_b[k * n_lut + al] = a[N + al];
    }
}

// rotation by -b~ then many-LUT extraction on int64 values of the reference
// (schemas/RLWE_jax.py:295-303), keeping its +-q/2 representatives
__global__ void rotate_extract_i64_kernel(const int64_t* __restrict__ acc, const double* __restrict__ b, int N,
                                          int n_lut, double q, int64_t* __restrict__ out_acc,
                                          int64_t* __restrict__ out_a, int64_t* __restrict__ out_b, long long B) {
    const long long per = 2LL * N + (long long)n_lut * N + n_lut;
    const long long total = B * per;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const long long k = t / per;
        const int r = (int)(t - k * per);
        const int bt = (int)(rint((2.0 * N * b[k]) / (q * n_lut)) * n_lut);
        const int64_t* a = acc + k * 2 * N;
        int e, src;
        int64_t* dst;
        if (r < 2 * N) {                        // rotated ACC
            if (!out_acc) continue;
            const int comp = r / N;
            e = (r % N) + bt;
            src = comp * N;
            dst = out_acc + k * 2 * N + r;
        } else if (r < 2 * N + n_lut * N) {     // extracted masks
            if (!out_a) continue;
            const int rr = r - 2 * N;
            const int al = rr / N, j = rr % N;
            e = al - j + bt;
            src = 0;
            dst = out_a + k * (long long)n_lut * N + rr;
        } else {                                // extracted bodies
            if (!out_b) continue;
            const int al = r - 2 * N - n_lut * N;
            e = al + bt;
            src = N;
            dst = out_b + k * n_lut + al;
        }
        e %= 2 * N;
        if (e < 0) e += 2 * N;
        *dst = e < N ? a[src + e] : -a[src + e - N];
    }
}

// FP64 FMA throughput probe: 8 independent chains per thread
__global__ void fp64_fma_probe_kernel(int iters, double* out) {
    double a[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = 1.0 + 1e-9 * (threadIdx.x + i);
    const double m = 0.999999999, c = 1e-12;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < 8; ++i) a[i] = fma(a[i], m, c);
    }
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += a[i];
    if (s == 12345.678) out[0] = s;   // keeps the chains live
}

// waits on a barrier that nothing arrives on: the bounded wait must give
// up after `limit` cycles and record the timeout in *status
__global__ void wait_timeout_probe_kernel(long long limit, int* status, int* result) {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        mbar_fence_init();
    }
    __syncthreads();
    const bool ok = mbar_wait_bounded(&bar, 0, limit, status);
    if (threadIdx.x == 0) *result = ok ? 1 : 0;
}

// ---------------------------------------------------------------- validation
static int validate_params(const tfhe_params* p) {
    if (!p) return fail(TFHE_ERR_INVALID_ARGUMENT, "params is NULL");
    if (!is_pow2(p->N) || p->N < 128 || p->N > 4096) return fail(TFHE_ERR_INVALID_ARGUMENT, "unsupported degree N");
    if (p->l_bs < 1 || p->l_bs > 4) return fail(TFHE_ERR_INVALID_ARGUMENT, "unsupported l_bs (1..4)");
    if (p->collapse < 1 || p->collapse > 4) return fail(TFHE_ERR_INVALID_ARGUMENT, "unsupported collapse (1..4)");
    if (p->n <= 0 || p->n % p->collapse) return fail(TFHE_ERR_INVALID_ARGUMENT, "n must be a positive multiple of collapse");
    if (p->n_big <= 0) return fail(TFHE_ERR_INVALID_ARGUMENT, "n_big must be positive");
    if (p->log2_q != 32 && p->log2_q != 64)
        return fail(TFHE_ERR_INVALID_ARGUMENT, "native entry points need log2_q == 32 (tfhe_*) or 64 (tfhe64_*)");
    if (p->log2_beta_bs < 1 || p->log2_beta_bs * p->l_bs > p->log2_q)
        return fail(TFHE_ERR_INVALID_ARGUMENT, "log2_beta_bs * l_bs must be in [1, log2_q]");
    if (p->l_ks < 1 || p->l_ks > KS_LMAX || p->log2_beta_ks < 1 || p->log2_beta_ks * p->l_ks > p->log2_q)
        return fail(TFHE_ERR_INVALID_ARGUMENT, "unsupported key-switch base / levels");
    if (p->log2_q == 64 && p->l_bs > 3)
        return fail(TFHE_ERR_INVALID_ARGUMENT, "the 64-bit blind rotation supports l_bs 1..3");
    if (br_shape(p->N, p->l_bs, 1 << p->collapse, 1).K < 1)
        return fail(TFHE_ERR_INVALID_ARGUMENT, "degree / levels do not fit in shared memory");
    return TFHE_OK;
}

// log2_q: the torus the calling entry point works on (32: tfhe_*, 64: tfhe64_*)
static int check_keys(const tfhe_keys* k, int log2_q = 32) {
    if (!k) return fail(TFHE_ERR_INVALID_ARGUMENT, "keys is NULL");
    if (k->p.log2_q != log2_q)
        return fail(TFHE_ERR_INVALID_ARGUMENT, log2_q == 32 ? "keys are for q = 2^64: use the tfhe64_* entry points"
                                                            : "keys are for q = 2^32: use the tfhe_* entry points");
    int dev = -1;
    TFHE_TRY(check_cuda(cudaGetDevice(&dev), "cudaGetDevice"));
    if (dev != k->device)
        return fail(TFHE_ERR_INVALID_ARGUMENT, "keys live on device " + std::to_string(k->device) +
                                                   " but device " + std::to_string(dev) + " is current");
    return TFHE_OK;
}

static int upload_ksk(tfhe_keys* k, const uint32_t* ksk_a, const uint32_t* ksk_b, cudaStream_t stream) {
    const tfhe_params& p = k->p;
    k->ldk = (p.n + 1 + 3) / 4 * 4;
    const size_t rows = (size_t)p.n_big * p.l_ks;
    std::vector<uint32_t> host(rows * k->ldk, 0u);
    for (int j = 0; j < p.l_ks; ++j)
        for (int i = 0; i < p.n_big; ++i) {
            uint32_t* dst = host.data() + ((size_t)i * p.l_ks + j) * k->ldk;
            std::memcpy(dst, ksk_a + ((size_t)j * p.n_big + i) * p.n, (size_t)p.n * sizeof(uint32_t));
            dst[p.n] = ksk_b[(size_t)j * p.n_big + i];
        }
    const size_t bytes = host.size() * sizeof(uint32_t);
    TFHE_TRY(check_cuda(cudaMalloc(&k->ksk, bytes), "cudaMalloc(ksk)"));
    k->bytes += (int64_t)bytes;
    TFHE_TRY(check_cuda(cudaMemcpyAsync(k->ksk, host.data(), bytes, cudaMemcpyHostToDevice, stream), "ksk upload"));
    // int8 limbs for the tensor-core key switch, where its int32 sums cannot
    // overflow: n_big * l * 2^(log2_beta - 1) * 128 < 2^31, digits within int8
    const long long ktot = (long long)p.n_big * p.l_ks;
    const bool tc_ok = p.n_big % 32 == 0 && p.l_ks <= 8 && p.log2_beta_ks <= 7 &&
                       ktot * (1LL << (p.log2_beta_ks - 1)) * 128 < (1LL << 31);
    if (tc_ok) {
        const int cols = ks_tc_columns();
        k->ks_npad = (4 * (p.n + 1) + cols - 1) / cols * cols;
        std::vector<int8_t> lim((size_t)k->ks_npad * ktot, 0);
        for (long long kk = 0; kk < ktot; ++kk)
            for (int o = 0; o <= p.n; ++o) {
                long long rest = host[(size_t)kk * k->ldk + o];
                for (int t = 0; t < 4; ++t) {
                    const long long lo = ((rest + 128) & 255) - 128;
                    lim[((size_t)o * 4 + t) * ktot + kk] = (int8_t)lo;
                    rest = (rest - lo) >> 8;
                }
            }
        TFHE_TRY(check_cuda(cudaMalloc(&k->ksk_limbs, lim.size()), "cudaMalloc(ksk limbs)"));
        k->bytes += (int64_t)lim.size();
        TFHE_TRY(check_cuda(cudaMemcpyAsync(k->ksk_limbs, lim.data(), lim.size(), cudaMemcpyHostToDevice, stream),
                            "ksk limb upload"));
        // the host vector must outlive the copy
        return check_cuda(cudaStreamSynchronize(stream), "ksk upload sync");
    }
    return check_cuda(cudaStreamSynchronize(stream), "ksk upload sync");
}

static int keys_common(const tfhe_params* params, tfhe_keys** out, tfhe_keys** made, int log2_q = 32) {
    if (!out) return fail(TFHE_ERR_INVALID_ARGUMENT, "keys_out is NULL");
    *out = nullptr;
    TFHE_TRY(validate_params(params));
    if (params->log2_q != log2_q)
        return fail(TFHE_ERR_INVALID_ARGUMENT, log2_q == 32 ? "tfhe_keys_create* need log2_q == 32"
                                                            : "tfhe64_keys_create needs log2_q == 64");
    tfhe_keys* k = new tfhe_keys();
    k->p = *params;
    k->G = params->n / params->collapse;
    k->M = 1 << params->collapse;
    if (check_cuda(cudaGetDevice(&k->device), "cudaGetDevice") != TFHE_OK) {
        delete k;
        return TFHE_ERR_NO_DEVICE;
    }
    k->plan = get_plan(params->N);
    if (!k->plan) {
        delete k;
        return TFHE_ERR_INTERNAL;
    }
    // the key ring layout has no 64-bit kernels
    k->ring_kr = params->log2_q == 32 ? ring_shape(params->N, params->l_bs, k->M).kr : 0;
    *made = k;
    return TFHE_OK;
}

static void keys_free(tfhe_keys* k) {
    if (!k) return;
    cudaFree(k->bsk);
    cudaFree(k->ksk);
    cudaFree(k->ksk_limbs);
    delete k;
}

static std::atomic<long long> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
static long long launch_count() { return g_launches.load(std::memory_order_relaxed); }

// The bootstrapping key (2 in, 2 out, G M, L, N) words of elem bytes (4: the
// 32-bit torus, 8: the 64-bit one) -> the FP64 Fourier layout the blind
// rotation reads, converted on the device.
static int upload_bsk(tfhe_keys* k, const void* bsk_coeff, size_t elem, cudaStream_t stream) {
    const tfhe_params& p = k->p;
    const int N = p.N, H = N / 2, L = p.l_bs;
    const long long npoly = 4LL * k->G * k->M * L;
    const size_t src_bytes = (size_t)npoly * N * elem;
    const size_t dst_bytes = (size_t)npoly * H * sizeof(double2);
    void* d_src = nullptr;
    int rc = check_cuda(cudaMalloc(&d_src, src_bytes), "cudaMalloc(bsk staging)");
    if (rc == TFHE_OK) rc = check_cuda(cudaMalloc(&k->bsk, dst_bytes), "cudaMalloc(bsk)");
    if (rc == TFHE_OK) {
        k->bytes += (int64_t)dst_bytes;
        rc = check_cuda(cudaMemcpyAsync(d_src, bsk_coeff, src_bytes, cudaMemcpyHostToDevice, stream), "bsk upload");
    }
    if (rc == TFHE_OK) {
        BskConvArgs ca{elem == 4 ? static_cast<const uint32_t*>(d_src) : nullptr,
                       elem == 8 ? static_cast<const unsigned long long*>(d_src) : nullptr,
                       k->bsk, k->plan->qt, k->plan->tw, k->G, k->M, L, npoly,
                       k->ring_kr > 0 ? k->ring_kr * H / 4 : 0};
        const int ppc = std::max(1, 2048 / H);
        const size_t smem = (size_t)ppc * H * sizeof(double2);
        BrConvKernel kern = bsk_fft_kernel_for(ilog2(N));
        rc = check_cuda(cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                        "cudaFuncSetAttribute(bsk fft)");
        if (rc == TFHE_OK) {
            count_launch();
            kern<<<(unsigned)((npoly + ppc - 1) / ppc), 256, smem, stream>>>(ca);
            rc = check_cuda(cudaGetLastError(), "bsk fft launch");
        }
        if (rc == TFHE_OK) rc = check_cuda(cudaStreamSynchronize(stream), "bsk fft");
    }
    cudaFree(d_src);
    return rc;
}


}  // namespace tfhe

using namespace tfhe;

// ============================================================================
// C ABI
// ============================================================================
extern "C" {

const char* tfhe_version(void) { return "tfhe_b200 1 (sm_100a, FP64 batched blind rotation)"; }

const char* tfhe_last_error(void) { return g_last_error.c_str(); }

int tfhe_mul_bootstrap(void* stream, const int64_t* ct_init, int64_t ct_elems, const void* bsk,
                       const int64_t* bsk_dims, const void* all_rot_fft, int64_t all_rot_rows,
                       const int32_t* indices, int64_t log2_beta, int64_t log2_q, int64_t l, int64_t degree,
                       int64_t* out, int64_t batch) {
    switch (degree) {
        case 128: case 256: case 512: case 1024: case 2048: case 4096: break;
        default: return fail(TFHE_ERR_INVALID_ARGUMENT, "Unsupported degree");
    }
    if (l < 1 || l > 4) return fail(TFHE_ERR_INVALID_ARGUMENT, "Unsupported l");
    if (!bsk_dims) return fail(TFHE_ERR_INVALID_ARGUMENT, "bsk_dims is NULL");
    const int64_t G = bsk_dims[0], A = bsk_dims[1], Lb = bsk_dims[2], C = bsk_dims[3], M = bsk_dims[4],
                  D = bsk_dims[5];
    if (A != 2 || C != 2 || Lb != l || D != degree / 2 || M < 1 || M > 16 || !is_pow2(M) || G < 1)
        return fail(TFHE_ERR_INVALID_ARGUMENT, "bsk must be (G, 2, l, 2, M, degree/2) with M a power of two <= 16");
    if (all_rot_rows != 2 * degree) return fail(TFHE_ERR_INVALID_ARGUMENT, "all_rot_fft must have 2*degree rows");
    if (log2_q < 2 || log2_q > 64 || log2_beta < 1 || log2_beta > 62)
        return fail(TFHE_ERR_INVALID_ARGUMENT, "unsupported log2_q / log2_beta");
    if (batch < 0) return fail(TFHE_ERR_INVALID_ARGUMENT, "negative batch");
    if (ct_elems != 2 * degree && ct_elems != 2 * degree * batch)
        return fail(TFHE_ERR_INVALID_ARGUMENT, "ct_init must hold 2N or batch*2N elements");
    if (batch == 0) return TFHE_OK;
    if (!ct_init || !bsk || !all_rot_fft || !indices || !out)
        return fail(TFHE_ERR_INVALID_ARGUMENT, "NULL buffer");
    BrArgs a{};
    a.bsk = static_cast<const double2*>(bsk);
    a.all_rot = static_cast<const double2*>(all_rot_fft);
    a.G = (int)G;
    a.M = (int)M;
    a.collapse = ilog2(M);
    a.B = batch;
    a.log2_beta = (int)log2_beta;
    a.log2_q = (int)log2_q;
    a.ct_init = ct_init;
    a.ct_stride = (ct_elems > 2 * degree) ? 2 * degree : 0;
    a.indices = indices;
    a.out_i64 = out;
    a.n_lut = 1;
    return launch_br(a, (int)degree, (int)l, true, 0, static_cast<cudaStream_t>(stream));
}

int tfhe_keys_create(const tfhe_params* params, const uint32_t* bsk_coeff, const uint32_t* ksk_a,
                     const uint32_t* ksk_b, void* stream_v, tfhe_keys** keys_out) {
    tfhe_keys* k = nullptr;
    TFHE_TRY(keys_common(params, keys_out, &k));
    if (!bsk_coeff || !ksk_a || !ksk_b) {
        keys_free(k);
        return fail(TFHE_ERR_INVALID_ARGUMENT, "NULL key buffer");
    }
    cudaStream_t stream = static_cast<cudaStream_t>(stream_v);
    int rc = upload_bsk(k, bsk_coeff, sizeof(uint32_t), stream);
    if (rc == TFHE_OK) rc = upload_ksk(k, ksk_a, ksk_b, stream);
    if (rc != TFHE_OK) {
        keys_free(k);
        return rc;
    }
    *keys_out = k;
    return TFHE_OK;
}

int tfhe_keys_create_fourier(const tfhe_params* params, const double* bsk_ordered, const uint32_t* ksk_a,
                             const uint32_t* ksk_b, void* stream_v, tfhe_keys** keys_out) {
    tfhe_keys* k = nullptr;
    TFHE_TRY(keys_common(params, keys_out, &k));
    if (!bsk_ordered || !ksk_a || !ksk_b) {
        keys_free(k);
        return fail(TFHE_ERR_INVALID_ARGUMENT, "NULL key buffer");
    }
    cudaStream_t stream = static_cast<cudaStream_t>(stream_v);
    const tfhe_params& p = *params;
    const int N = p.N, H = N / 2, L = p.l_bs, P = 2 * L, G = k->G, M = k->M;
    std::vector<double2> qt, tw;
    std::vector<uint16_t> freq;
    build_tables(N, qt, tw, freq);
    // bsk_ordered (2 out, 2 in, L, G*M, H) at zeta^(2j+1) -> [G][2][P/2][M][H][2]
    // at zeta^(4 freq[p] + 1) (the point or the conjugate of its partner)
    const size_t total = (size_t)G * 2 * P * M * H;
    std::vector<double2> host(total);
    const double2* src = reinterpret_cast<const double2*>(bsk_ordered);
    for (int g = 0; g < G; ++g)
        for (int a = 0; a < 2; ++a)
            for (int lvl = 0; lvl < L; ++lvl)
                for (int c = 0; c < 2; ++c)
                    for (int m = 0; m < M; ++m) {
                        const double2* row = src + ((((size_t)a * 2 + c) * L + lvl) * ((size_t)G * M) + (size_t)g * M + m) * H;
                        const int rnt = k->ring_kr > 0 ? k->ring_kr * H / 4 : 0;
                        const int bc = lvl * 2 + c;
                        for (int pp = 0; pp < H; ++pp) {
                            const int j = freq[pp];
                            const int e = 4 * j + 1;
                            size_t di;
                            if (rnt > 0) {
                                di = ((((size_t)g * (H / rnt) + pp / rnt) * 2 + a) * M + m) * P + bc;
                                di = di * rnt + pp % rnt;
                            } else {
                                di = (((((size_t)g * 2 + a) * (P / 2) + bc / 2) * M + m) * H + pp) * 2 + (bc & 1);
                            }
                            // times 1/H, as bsk_fft_kernel stores the native key
                            const double2 w = e < N ? row[2 * j] : make_double2(row[N - 1 - 2 * j].x, -row[N - 1 - 2 * j].y);
                            host[di] = make_double2(w.x / H, w.y / H);
                        }
                    }
    int rc = check_cuda(cudaMalloc(&k->bsk, total * sizeof(double2)), "cudaMalloc(bsk)");
    if (rc == TFHE_OK) {
        k->bytes += (int64_t)(total * sizeof(double2));
        rc = check_cuda(cudaMemcpyAsync(k->bsk, host.data(), total * sizeof(double2), cudaMemcpyHostToDevice, stream),
                        "bsk upload");
    }
    if (rc == TFHE_OK) rc = check_cuda(cudaStreamSynchronize(stream), "bsk upload sync");
    if (rc == TFHE_OK) rc = upload_ksk(k, ksk_a, ksk_b, stream);
    if (rc != TFHE_OK) {
        keys_free(k);
        return rc;
    }
    *keys_out = k;
    return TFHE_OK;
}

void tfhe_keys_destroy(tfhe_keys* keys) { keys_free(keys); }

int64_t tfhe_keys_device_bytes(const tfhe_keys* keys) { return keys ? keys->bytes : 0; }

// ---------------------------------------------------------------- the 64-bit torus
int tfhe64_keys_create(const tfhe_params* params, const uint64_t* bsk_coeff, void* stream, tfhe_keys** keys_out) {
    tfhe_keys* k = nullptr;
    TFHE_TRY(keys_common(params, keys_out, &k, 64));
    if (!bsk_coeff) {
        keys_free(k);
        return fail(TFHE_ERR_INVALID_ARGUMENT, "NULL key buffer");
    }
    const int rc = upload_bsk(k, bsk_coeff, sizeof(uint64_t), static_cast<cudaStream_t>(stream));
    if (rc != TFHE_OK) {
        keys_free(k);
        return rc;
    }
    *keys_out = k;
    return TFHE_OK;
}

static int br_native64(const tfhe_keys* keys, const uint64_t* lwe_a, const uint64_t* lwe_b, const int64_t* lut,
                       int64_t lut_count, int32_t n_lut, uint64_t* acc_out, uint64_t* out_a, uint64_t* out_b,
                       int64_t batch, cudaStream_t stream) {
    TFHE_TRY(check_keys(keys, 64));
    const tfhe_params& p = keys->p;
    if (batch < 0) return fail(TFHE_ERR_INVALID_ARGUMENT, "negative batch");
    if (n_lut < 1 || n_lut > p.N || (n_lut & (n_lut - 1)))
        return fail(TFHE_ERR_INVALID_ARGUMENT, "n_lut must be a power of two in [1, N]");
    if (lut_count != 1 && lut_count != batch) return fail(TFHE_ERR_INVALID_ARGUMENT, "lut_count must be 1 or batch");
    if (batch == 0) return TFHE_OK;
    if (!lwe_a || !lwe_b || !lut || !(acc_out || (out_a && out_b)))
        return fail(TFHE_ERR_INVALID_ARGUMENT, "NULL buffer");
    BrArgs a{};
    a.bsk = keys->bsk;
    a.G = keys->G;
    a.M = keys->M;
    a.collapse = p.collapse;
    a.B = batch;
    a.log2_beta = p.log2_beta_bs;
    a.log2_q = 64;
    a.lwe_a64 = reinterpret_cast<const unsigned long long*>(lwe_a);
    a.lwe_b64 = reinterpret_cast<const unsigned long long*>(lwe_b);
    a.lut64 = reinterpret_cast<const long long*>(lut);
    a.lut_stride = lut_count == 1 ? 0 : 2LL * p.N;
    a.n_lut = n_lut;
    a.lwe_n = p.n;
    a.acc_out64 = reinterpret_cast<unsigned long long*>(acc_out);
    a.out_a64 = reinterpret_cast<unsigned long long*>(out_a);
    a.out_b64 = reinterpret_cast<unsigned long long*>(out_b);
    return launch_br(a, p.N, p.l_bs, false, 0, stream, nullptr, &keys->tune);
}

int tfhe64_blind_rotate(const tfhe_keys* keys, const uint64_t* lwe_a, const uint64_t* lwe_b, const int64_t* lut,
                        int64_t lut_count, int32_t n_lut, uint64_t* acc_out, int64_t batch, void* stream) {
    if (!acc_out && batch > 0) return fail(TFHE_ERR_INVALID_ARGUMENT, "NULL buffer");
    return br_native64(keys, lwe_a, lwe_b, lut, lut_count, n_lut, acc_out, nullptr, nullptr, batch,
                       static_cast<cudaStream_t>(stream));
}

int tfhe64_cuboot_merge(const tfhe_keys* keys, const uint64_t* lwe_a, const uint64_t* lwe_b, const int64_t* lut,
                        int64_t lut_count, int32_t n_lut, uint64_t* out_a, uint64_t* out_b, int64_t batch,
                        void* stream) {
    if ((!out_a || !out_b) && batch > 0) return fail(TFHE_ERR_INVALID_ARGUMENT, "NULL buffer");
    return br_native64(keys, lwe_a, lwe_b, lut, lut_count, n_lut, nullptr, out_a, out_b, batch,
                       static_cast<cudaStream_t>(stream));
}

int tfhe_keyswitch(const tfhe_keys* keys, const uint32_t* a_in, const uint32_t* b_in, uint32_t* a_out,
                   uint32_t* b_out, int64_t batch, void* stream) {
    TFHE_TRY(check_keys(keys));
    if (batch < 0) return fail(TFHE_ERR_INVALID_ARGUMENT, "negative batch");
    if (batch > 0 && (!a_in || !b_in || !a_out || !b_out)) return fail(TFHE_ERR_INVALID_ARGUMENT, "NULL buffer");
    return launch_ks(keys, a_in, b_in, a_out, b_out, batch, static_cast<cudaStream_t>(stream));
}

static int br_native(const tfhe_keys* keys, const uint32_t* lwe_a, const uint32_t* lwe_b, const uint32_t* lut,
                     int64_t lut_count, int32_t n_lut, uint32_t* acc_out, uint32_t* out_a, uint32_t* out_b,
                     int64_t batch, cudaStream_t stream, int* status = nullptr) {
    const tfhe_params& p = keys->p;
    if (n_lut < 1 || n_lut > p.N) return fail(TFHE_ERR_INVALID_ARGUMENT, "n_lut must be in [1, N]");
    if (lut_count != 1 && lut_count != batch) return fail(TFHE_ERR_INVALID_ARGUMENT, "lut_count must be 1 or batch");
    BrArgs a{};
    a.bsk = keys->bsk;
    a.G = keys->G;
    a.M = keys->M;
    a.collapse = p.collapse;
    a.B = batch;
    a.log2_beta = p.log2_beta_bs;
    a.log2_q = 32;
    a.lwe_a = lwe_a;
    a.lwe_b = lwe_b;
    a.lut = lut;
    a.lut_stride = lut_count == 1 ? 0 : 2LL * p.N;
    a.n_lut = n_lut;
    a.lwe_n = p.n;
    a.acc_out = acc_out;
    a.out_a = out_a;
    a.out_b = out_b;
    return launch_br(a, p.N, p.l_bs, false, keys->ring_kr, stream, status, &keys->tune);
}

int tfhe_blind_rotate(const tfhe_keys* keys, const uint32_t* lwe_a, const uint32_t* lwe_b, const uint32_t* lut,
                      int64_t lut_count, int32_t n_lut, uint32_t* acc_out, int64_t batch, void* stream) {
    TFHE_TRY(check_keys(keys));
    if (batch < 0) return fail(TFHE_ERR_INVALID_ARGUMENT, "negative batch");
    if (batch == 0) return TFHE_OK;
    if (!lwe_a || !lwe_b || !lut || !acc_out) return fail(TFHE_ERR_INVALID_ARGUMENT, "NULL buffer");
    return br_native(keys, lwe_a, lwe_b, lut, lut_count, n_lut, acc_out, nullptr, nullptr, batch,
                     static_cast<cudaStream_t>(stream));
}

int tfhe_sample_extract(const uint32_t* acc, int32_t N, int32_t n_lut, uint32_t* out_a, uint32_t* out_b,
                        int64_t batch, void* stream) {
    if (!is_pow2(N) || N < 2) return fail(TFHE_ERR_INVALID_ARGUMENT, "N must be a power of two");
    if (n_lut < 1 || n_lut > N) return fail(TFHE_ERR_INVALID_ARGUMENT, "n_lut must be in [1, N]");
    if (batch < 0) return fail(TFHE_ERR_INVALID_ARGUMENT, "negative batch");
    if (batch == 0) return TFHE_OK;
    if (!acc || !out_a || !out_b) return fail(TFHE_ERR_INVALID_ARGUMENT, "NULL buffer");
    const long long total = batch * (long long)n_lut * N;
    const int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 32);
    count_launch();
    extract_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(acc, N, n_lut, out_a, out_b, batch);
    return check_cuda(cudaGetLastError(), "sample extract launch");
}

int tfhe_cuboot_merge(const tfhe_keys* keys, const uint32_t* lwe_a, const uint32_t* lwe_b, const uint32_t* lut,
                      int64_t lut_count, int32_t n_lut, uint32_t* out_a, uint32_t* out_b, int64_t batch,
                      void* stream) {
    TFHE_TRY(check_keys(keys));
    if (batch < 0) return fail(TFHE_ERR_INVALID_ARGUMENT, "negative batch");
    if (batch == 0) return TFHE_OK;
    if (!lwe_a || !lwe_b || !lut || !out_a || !out_b) return fail(TFHE_ERR_INVALID_ARGUMENT, "NULL buffer");
    return br_native(keys, lwe_a, lwe_b, lut, lut_count, n_lut, nullptr, out_a, out_b, batch,
                     static_cast<cudaStream_t>(stream));
}

int tfhe_pbs(const tfhe_keys* keys, const uint32_t* a_in, const uint32_t* b_in, const uint32_t* lut,
             int64_t lut_count, int32_t n_lut, uint32_t* out_a, uint32_t* out_b, int64_t batch, void* stream_v) {
    TFHE_TRY(check_keys(keys));
    if (batch < 0) return fail(TFHE_ERR_INVALID_ARGUMENT, "negative batch");
    if (batch == 0) return TFHE_OK;
    if (!a_in || !b_in || !lut || !out_a || !out_b) return fail(TFHE_ERR_INVALID_ARGUMENT, "NULL buffer");
    cudaStream_t stream = static_cast<cudaStream_t>(stream_v);
    const size_t n = (size_t)keys->p.n;
    uint32_t* ks = nullptr;
    TFHE_TRY(check_cuda(cudaMallocAsync(&ks, (size_t)batch * (n + 1) * sizeof(uint32_t), stream),
                        "cudaMallocAsync(key-switch output)"));
    uint32_t* ks_b = ks + (size_t)batch * n;
    int rc = launch_ks(keys, a_in, b_in, ks, ks_b, batch, stream);
    if (rc == TFHE_OK)
        rc = br_native(keys, ks, ks_b, lut, lut_count, n_lut, nullptr, out_a, out_b, batch, stream);
    const int rc2 = check_cuda(cudaFreeAsync(ks, stream), "cudaFreeAsync(key-switch output)");
    return rc != TFHE_OK ? rc : rc2;
}

// tfhe_pbs from host buffers: the batch is cut into chunks; chunk i's
// host -> device copy runs on its own stream while chunk i-1 computes on the
// caller's stream and chunk i-2's outputs return on a third stream.  Two
// device slots alternate; events order every reuse of a slot after the
// work that last read it.
int tfhe_pbs_host(const tfhe_keys* keys, const uint32_t* a_host, const uint32_t* b_host, const uint32_t* lut_host,
                  int64_t lut_count, int32_t n_lut, uint32_t* out_a_host, uint32_t* out_b_host, int64_t batch,
                  int64_t chunk, void* stream_v) {
    TFHE_TRY(check_keys(keys));
    if (batch < 0 || chunk < 0) return fail(TFHE_ERR_INVALID_ARGUMENT, "negative batch or chunk");
    if (batch == 0) return TFHE_OK;
    if (!a_host || !b_host || !lut_host || !out_a_host || !out_b_host)
        return fail(TFHE_ERR_INVALID_ARGUMENT, "NULL buffer");
    if (lut_count != 1 && lut_count != batch) return fail(TFHE_ERR_INVALID_ARGUMENT, "lut_count must be 1 or batch");
    if (n_lut < 1 || n_lut > keys->p.N) return fail(TFHE_ERR_INVALID_ARGUMENT, "n_lut out of range");
    cudaStream_t stream = static_cast<cudaStream_t>(stream_v);
    const tfhe_params& p = keys->p;
    // automatic chunks: about an eighth of the batch, a whole number of
    // blind-rotation waves (SMs x ciphertexts per CTA) so no chunk ends on a
    // partly idle wave
    long long C = chunk;
    if (C == 0) {
        const BrShape sh = br_shape(p.N, p.l_bs, keys->M, std::max<long long>(batch, 1 << 20),
                                    keys->tune.ciphertexts_per_cta, true);
        const long long wave = (long long)std::max(1, sm_count()) * std::max(1, sh.K) * (sh.qtg ? 2 : 1);
        C = std::max<long long>(wave, ((batch + 7) / 8 + wave - 1) / wave * wave);
    }
    C = std::min<long long>(C, batch);
    const size_t N = (size_t)p.N, nb = (size_t)p.n_big, n = (size_t)p.n;
    const bool lut_per_ct = lut_count == batch && batch > 1;
    const size_t lut_words = (lut_per_ct ? (size_t)C : 1) * 2 * N;
    const size_t slot_words = (size_t)C * nb + C + lut_words + (size_t)C * (n + 1) + (size_t)C * n_lut * N +
                              (size_t)C * n_lut;
    uint32_t* scratch = nullptr;
    TFHE_TRY(check_cuda(cudaMallocAsync(&scratch, 2 * slot_words * sizeof(uint32_t), stream),
                        "cudaMallocAsync(host pipeline)"));
    struct Slot {
        uint32_t *a, *b, *lut, *ks, *oa, *ob;
    } slot[2];
    for (int s = 0; s < 2; ++s) {
        uint32_t* base = scratch + s * slot_words;
        slot[s].a = base;
        slot[s].b = slot[s].a + (size_t)C * nb;
        slot[s].lut = slot[s].b + C;
        slot[s].ks = slot[s].lut + lut_words;
        slot[s].oa = slot[s].ks + (size_t)C * (n + 1);
        slot[s].ob = slot[s].oa + (size_t)C * n_lut * N;
    }
    cudaStream_t h2d = nullptr, d2h = nullptr;
    cudaEvent_t ready = nullptr, h2d_end = nullptr, d2h_end = nullptr;
    cudaEvent_t h2d_done[2] = {}, comp_done[2] = {}, d2h_done[2] = {};
    int rc = check_cuda(cudaStreamCreateWithFlags(&h2d, cudaStreamNonBlocking), "cudaStreamCreate");
    if (rc == TFHE_OK) rc = check_cuda(cudaStreamCreateWithFlags(&d2h, cudaStreamNonBlocking), "cudaStreamCreate");
    for (cudaEvent_t* e : {&ready, &h2d_end, &d2h_end, &h2d_done[0], &h2d_done[1], &comp_done[0], &comp_done[1],
                           &d2h_done[0], &d2h_done[1]})
        if (rc == TFHE_OK) rc = check_cuda(cudaEventCreateWithFlags(e, cudaEventDisableTiming), "cudaEventCreate");
    if (rc == TFHE_OK) rc = check_cuda(cudaEventRecord(ready, stream), "event record");
    if (rc == TFHE_OK) rc = check_cuda(cudaStreamWaitEvent(h2d, ready, 0), "stream wait");
    if (rc == TFHE_OK) rc = check_cuda(cudaStreamWaitEvent(d2h, ready, 0), "stream wait");
    if (rc == TFHE_OK && !lut_per_ct)
        for (int s = 0; s < 2 && rc == TFHE_OK; ++s)
            rc = check_cuda(cudaMemcpyAsync(slot[s].lut, lut_host, 2 * N * sizeof(uint32_t), cudaMemcpyHostToDevice,
                                            h2d), "LUT upload");
    const long long nchunks = (batch + C - 1) / C;
    for (long long i = 0; i < nchunks && rc == TFHE_OK; ++i) {
        const int s = (int)(i & 1);
        const long long c0 = i * C;
        const long long cb = std::min<long long>(C, batch - c0);
        Slot& sl = slot[s];
        if (i >= 2) rc = check_cuda(cudaStreamWaitEvent(h2d, comp_done[s], 0), "stream wait");
        if (rc == TFHE_OK)
            rc = check_cuda(cudaMemcpyAsync(sl.a, a_host + c0 * nb, (size_t)cb * nb * sizeof(uint32_t),
                                            cudaMemcpyHostToDevice, h2d), "input upload");
        if (rc == TFHE_OK)
            rc = check_cuda(cudaMemcpyAsync(sl.b, b_host + c0, (size_t)cb * sizeof(uint32_t), cudaMemcpyHostToDevice,
                                            h2d), "input upload");
        if (rc == TFHE_OK && lut_per_ct)
            rc = check_cuda(cudaMemcpyAsync(sl.lut, lut_host + (size_t)c0 * 2 * N, (size_t)cb * 2 * N * sizeof(uint32_t),
                                            cudaMemcpyHostToDevice, h2d), "LUT upload");
        if (rc == TFHE_OK) rc = check_cuda(cudaEventRecord(h2d_done[s], h2d), "event record");
        if (rc == TFHE_OK) rc = check_cuda(cudaStreamWaitEvent(stream, h2d_done[s], 0), "stream wait");
        if (rc == TFHE_OK && i >= 2) rc = check_cuda(cudaStreamWaitEvent(stream, d2h_done[s], 0), "stream wait");
        uint32_t* ks_b = sl.ks + (size_t)cb * n;
        if (rc == TFHE_OK) rc = launch_ks(keys, sl.a, sl.b, sl.ks, ks_b, cb, stream);
        if (rc == TFHE_OK)
            rc = br_native(keys, sl.ks, ks_b, sl.lut, lut_per_ct ? cb : 1, n_lut, nullptr, sl.oa, sl.ob, cb, stream);
        if (rc == TFHE_OK) rc = check_cuda(cudaEventRecord(comp_done[s], stream), "event record");
        if (rc == TFHE_OK) rc = check_cuda(cudaStreamWaitEvent(d2h, comp_done[s], 0), "stream wait");
        if (rc == TFHE_OK)
            rc = check_cuda(cudaMemcpyAsync(out_a_host + (size_t)c0 * n_lut * N, sl.oa,
                                            (size_t)cb * n_lut * N * sizeof(uint32_t), cudaMemcpyDeviceToHost, d2h),
                            "output download");
        if (rc == TFHE_OK)
            rc = check_cuda(cudaMemcpyAsync(out_b_host + (size_t)c0 * n_lut, sl.ob, (size_t)cb * n_lut * sizeof(uint32_t),
                                            cudaMemcpyDeviceToHost, d2h), "output download");
        if (rc == TFHE_OK) rc = check_cuda(cudaEventRecord(d2h_done[s], d2h), "event record");
    }
    // the caller's stream resumes after every copy; then the scratch is released
    if (h2d && h2d_end) {
        cudaEventRecord(h2d_end, h2d);
        cudaStreamWaitEvent(stream, h2d_end, 0);
    }
    if (d2h && d2h_end) {
        cudaEventRecord(d2h_end, d2h);
        cudaStreamWaitEvent(stream, d2h_end, 0);
    }
    const int rc2 = check_cuda(cudaFreeAsync(scratch, stream), "cudaFreeAsync(host pipeline)");
    for (cudaEvent_t e : {ready, h2d_end, d2h_end, h2d_done[0], h2d_done[1], comp_done[0], comp_done[1], d2h_done[0],
                          d2h_done[1]})
        if (e) cudaEventDestroy(e);
    if (h2d) cudaStreamDestroy(h2d);
    if (d2h) cudaStreamDestroy(d2h);
    return rc != TFHE_OK ? rc : rc2;
}

int tfhe_probe_fp64_fma(int32_t blocks, int32_t threads, int32_t iters, double* scratch, double* flops,
                        void* stream) {
    if (blocks < 1 || threads < 1 || threads > 1024 || iters < 1 || !scratch || !flops)
        return fail(TFHE_ERR_INVALID_ARGUMENT, "invalid probe shape");
    *flops = 2.0 * 8.0 * (double)blocks * threads * iters;
    count_launch();
    fp64_fma_probe_kernel<<<blocks, threads, 0, static_cast<cudaStream_t>(stream)>>>(iters, scratch);
    return check_cuda(cudaGetLastError(), "fp64 probe launch");
}

int tfhe_keys_set_tuning(tfhe_keys* keys, const tfhe_tuning* tuning) {
    if (!keys) return fail(TFHE_ERR_INVALID_ARGUMENT, "keys is NULL");
    if (!tuning) {
        keys->tune = tfhe_tuning{0, -1, -1, -1, -1};
        return TFHE_OK;
    }
    if (tuning->ciphertexts_per_cta < 0 || tuning->ciphertexts_per_cta > 64 || tuning->prefetch < -1 ||
        tuning->prefetch > 1 || tuning->persistent < -1 || tuning->persistent > 1 ||
        tuning->ks_tensor_cores < -1 || tuning->ks_tensor_cores > 1 || tuning->l2_prefetch < -1 ||
        tuning->l2_prefetch > 1)
        return fail(TFHE_ERR_INVALID_ARGUMENT, "tuning out of range");
    keys->tune = *tuning;
    return TFHE_OK;
}

int tfhe_keys_launch_shape(const tfhe_keys* keys, int64_t batch, int32_t* ciphertexts_per_cta,
                           int32_t* threads, int64_t* shared_bytes) {
    if (!keys || !ciphertexts_per_cta || !threads || !shared_bytes)
        return fail(TFHE_ERR_INVALID_ARGUMENT, "NULL argument");
    const tfhe_params& p = keys->p;
    const BrShape sh = keys->ring_kr > 0 ? ring_shape(p.N, p.l_bs, keys->M)
                                         : br_shape(p.N, p.l_bs, keys->M, std::max<int64_t>(batch, 1),
                                                    keys->tune.ciphertexts_per_cta, true);
    *ciphertexts_per_cta = sh.K;
    *threads = sh.nt;
    *shared_bytes = (int64_t)sh.smem;
    return sh.K > 0 ? TFHE_OK : fail(TFHE_ERR_INVALID_ARGUMENT, "no launch shape fits");
}

int32_t tfhe_keys_cluster_size(const tfhe_keys* keys, int64_t batch) {
    if (!keys) return 0;
    const tfhe_params& p = keys->p;
    const bool t64 = p.log2_q == 64;
    if (const int S = cluster_form(p.N, p.l_bs, keys->G, keys->M, batch, false, keys->ring_kr, &keys->tune, t64))
        return 2 * S;
    return split_applies(p.N, p.l_bs, keys->G, keys->M, batch, false, keys->ring_kr, &keys->tune, t64) ? 2 : 1;
}

int64_t tfhe_launch_count(void) { return launch_count(); }

int tfhe_device_status(int32_t* status_out, int32_t clear) {
    if (!status_out) return fail(TFHE_ERR_INVALID_ARGUMENT, "status_out is NULL");
    int* w = device_status_word();
    if (!w) return fail(TFHE_ERR_INTERNAL, "device status word unavailable");
    int v = 0;
    TFHE_TRY(check_cuda(cudaMemcpy(&v, w, sizeof(int), cudaMemcpyDeviceToHost), "read device status"));
    *status_out = v;
    if (clear) TFHE_TRY(check_cuda(cudaMemset(w, 0, sizeof(int)), "clear device status"));
    return TFHE_OK;
}

int tfhe_probe_wait_timeout(int64_t limit_cycles, int32_t* waited_out) {
    if (limit_cycles < 1 || limit_cycles > 4000000000LL || !waited_out)
        return fail(TFHE_ERR_INVALID_ARGUMENT, "limit must be in [1, 4e9] cycles");
    int* w = device_status_word();
    if (!w) return fail(TFHE_ERR_INTERNAL, "device status word unavailable");
    int* res = nullptr;
    TFHE_TRY(check_cuda(cudaMalloc(&res, sizeof(int)), "cudaMalloc(probe)"));
    count_launch();
    wait_timeout_probe_kernel<<<1, 32>>>(limit_cycles, w, res);
    int rc = check_cuda(cudaGetLastError(), "timeout probe launch");
    int v = -1;
    if (rc == TFHE_OK) rc = check_cuda(cudaMemcpy(&v, res, sizeof(int), cudaMemcpyDeviceToHost), "timeout probe");
    cudaFree(res);
    *waited_out = v;
    return rc;
}

int tfhe_keyswitch_ref(const uint32_t* a_in, const uint32_t* b_in, const uint32_t* ksk_a, const uint32_t* ksk_b,
                       int32_t n_big, int32_t n, int32_t l_ks, int32_t log2_beta_ks, uint32_t* a_out,
                       uint32_t* b_out, int64_t batch, void* stream) {
    if (n_big <= 0 || n <= 0) return fail(TFHE_ERR_INVALID_ARGUMENT, "dimensions must be positive");
    if (l_ks < 1 || l_ks > KS_LMAX || log2_beta_ks < 1 || log2_beta_ks * l_ks > 32)
        return fail(TFHE_ERR_INVALID_ARGUMENT, "unsupported key-switch base / levels");
    if (batch < 0) return fail(TFHE_ERR_INVALID_ARGUMENT, "negative batch");
    if (batch == 0) return TFHE_OK;
    if (!a_in || !b_in || !ksk_a || !ksk_b || !a_out || !b_out) return fail(TFHE_ERR_INVALID_ARGUMENT, "NULL buffer");
    const KsKey key{ksk_a, ksk_b, n, (long long)n_big * n, 1, n_big};
    return launch_ks_key(key, n_big, n, l_ks, log2_beta_ks, a_in, b_in, a_out, b_out, batch,
                         static_cast<cudaStream_t>(stream));
}

int tfhe_rotate_extract_i64(const int64_t* acc, const double* b, int32_t N, int32_t n_lut, int64_t log2_q,
                            int64_t* out_acc, int64_t* out_a, int64_t* out_b, int64_t batch, void* stream) {
    if (!is_pow2(N) || N < 2) return fail(TFHE_ERR_INVALID_ARGUMENT, "N must be a power of two");
    if (n_lut < 1 || n_lut > N) return fail(TFHE_ERR_INVALID_ARGUMENT, "n_lut must be in [1, N]");
    if (log2_q < 2 || log2_q > 64) return fail(TFHE_ERR_INVALID_ARGUMENT, "unsupported log2_q");
    if (batch < 0) return fail(TFHE_ERR_INVALID_ARGUMENT, "negative batch");
    if (batch == 0) return TFHE_OK;
    if (!acc || !b || (!out_acc && !out_a && !out_b) || ((out_a == nullptr) != (out_b == nullptr)))
        return fail(TFHE_ERR_INVALID_ARGUMENT, "NULL buffer");
    const long long total = batch * (2LL * N + (long long)n_lut * N + n_lut);
    const int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 32);
    count_launch();
    rotate_extract_i64_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        acc, b, N, n_lut, std::ldexp(1.0, (int)log2_q), out_acc, out_a, out_b, batch);
    return check_cuda(cudaGetLastError(), "rotate/extract launch");
}

// ---------------------------------------------------------------------------
// Programmable bootstrap without any allocation.  The key-switched LWEs that
// tfhe_pbs keeps in a stream-ordered allocation live here in a fixed static
// device array instead, for callers that must not allocate device memory:
// an XLA custom call whose runtime has preallocated most of the GPU, a
// serving loop that forbids allocation on its latency path, or code running
// under an external memory manager.  Every GPU that loads the library holds
// this array until the process exits.  Bounded-wait timeouts of both kernels
// of the call go to the device status word (itself a static device
// variable), read with tfhe_device_status like those of every other entry.
// ---------------------------------------------------------------------------
constexpr size_t NOALLOC_SCRATCH_WORDS = (size_t(8) << 20) / 4;   // 8 MiB of key-switched LWEs
static __device__ __align__(256) uint32_t g_pbs_noalloc_scratch[NOALLOC_SCRATCH_WORDS];

static std::mutex g_noalloc_mu;
static std::map<int, uint32_t*> g_noalloc_base;   // device -> address of the array

// device address of the static array for the current device (looked up
// once per device; the host-side symbol itself is not a device address)
static int noalloc_base(uint32_t** out) {
    int dev = 0;
    TFHE_TRY(check_cuda(cudaGetDevice(&dev), "cudaGetDevice"));
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    auto it = g_noalloc_base.find(dev);
    if (it == g_noalloc_base.end()) {
        uint32_t* ptr = nullptr;
        TFHE_TRY(check_cuda(cudaGetSymbolAddress((void**)&ptr, g_pbs_noalloc_scratch),
                            "cudaGetSymbolAddress(no-allocation scratch)"));
        it = g_noalloc_base.emplace(dev, ptr).first;
    }
    *out = it->second;
    return TFHE_OK;
}

int tfhe_pbs_noalloc(const tfhe_keys* keys, const uint32_t* a_in, const uint32_t* b_in, const uint32_t* lut,
                     int64_t lut_count, int32_t n_lut, uint32_t* out_a, uint32_t* out_b, int64_t batch,
                     void* stream_v) {
    TFHE_TRY(check_keys(keys));
    if (batch < 0) return fail(TFHE_ERR_INVALID_ARGUMENT, "negative batch");
    if (batch == 0) return TFHE_OK;
    if (!a_in || !b_in || !lut || !out_a || !out_b) return fail(TFHE_ERR_INVALID_ARGUMENT, "NULL buffer");
    const size_t n = (size_t)keys->p.n;
    const size_t max_batch = NOALLOC_SCRATCH_WORDS / (n + 1);
    if ((size_t)batch > max_batch)
        return fail(TFHE_ERR_INVALID_ARGUMENT,
                    "tfhe_pbs_noalloc: batch " + std::to_string(batch) + " exceeds the static scratch of " +
                        std::to_string(NOALLOC_SCRATCH_WORDS * 4) + " bytes (at most " + std::to_string(max_batch) +
                        " ciphertexts for n = " + std::to_string(n) + "); split the batch or use tfhe_pbs");
    cudaStream_t stream = static_cast<cudaStream_t>(stream_v);
    uint32_t* ks = nullptr;
    TFHE_TRY(noalloc_base(&ks));
    uint32_t* ks_b = ks + (size_t)batch * n;
    TFHE_TRY(launch_ks(keys, a_in, b_in, ks, ks_b, batch, stream));
    return br_native(keys, ks, ks_b, lut, lut_count, n_lut, nullptr, out_a, out_b, batch, stream, nullptr);
}

}  // extern "C"
