/*
 * tfhe_b200.h - C ABI of the B200 (sm_100a) TFHE programmable-bootstrapping
 * engine: LWE key switching, collapsed blind rotation and many-LUT sample
 * extraction for the encrypted Spike-LSTM of AMIAD-Research/Blind-Spiking-LSTM.
 *
 * Conventions
 *  - Every compute entry point takes DEVICE pointers, runs asynchronously on
 *    the given CUDA stream (cudaStream_t passed as void*, NULL = legacy
 *    default stream) and returns a status code (TFHE_OK = 0).  The message
 *    of the last failing call on the calling thread is tfhe_last_error().
 *  - Native entry points carry torus values as uint32 (q = 2^32), the
 *    reference's float64 values centred in [-q/2, q/2] reduced modulo 2^32.
 *  - tfhe_mul_bootstrap keeps the reference's int64 / complex128 buffers.
 *  - No torch, JAX or C++ types cross this boundary.
 */
#ifndef TFHE_B200_H
#define TFHE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TFHE_B200_ABI_VERSION 2

/* status codes: the reference handler returns ffi::Error::InvalidArgument
 * for unsupported degree / l and ffi::Error::Internal for launch failures
 * (csrc/mul_bootstrap.cuh:183-188, 211-223). */
enum {
    TFHE_OK = 0,
    TFHE_ERR_INVALID_ARGUMENT = 1,
    TFHE_ERR_INTERNAL = 2,
    TFHE_ERR_OUT_OF_MEMORY = 3,
    TFHE_ERR_NO_DEVICE = 4
};

/* Parameter set of one bootstrapping key (the reference keeps these in the
 * dict_params* globals of parameters_crypto.py:6-84). */
typedef struct tfhe_params {
    int32_t N;             /* GLWE degree: 128 .. 4096, power of two            */
    int32_t n;             /* LWE dimension of the blind rotation               */
    int32_t n_big;         /* LWE dimension entering the key switch (usually N) */
    int32_t log2_beta_bs;  /* blind-rotation gadget base, log2                  */
    int32_t l_bs;          /* blind-rotation gadget levels: 1 .. 4              */
    int32_t collapse;      /* collapse factor c (n % c == 0): 1 .. 4            */
    int32_t log2_beta_ks;  /* key-switch gadget base, log2                      */
    int32_t l_ks;          /* key-switch gadget levels: 1 .. 8                  */
    int32_t log2_q;        /* must be 32 for the native entry points            */
} tfhe_params;

typedef struct tfhe_keys tfhe_keys;   /* device-resident key material */

/* Launch shape of the blind rotation for one key set (no counterpart in
 * the reference; chosen by an autotuner or left automatic). */
typedef struct tfhe_tuning {
    int32_t ciphertexts_per_cta;  /* 0: as many as shared memory and 512 threads allow */
    int32_t prefetch;             /* L1 prefetch of key words: -1 automatic (off), 0 off, 1 on */
    int32_t persistent;           /* CTAs loop over ciphertext sets: -1 automatic (on), 0, 1 */
    int32_t ks_tensor_cores;      /* key switch on tcgen05 int8 tensor cores: -1 automatic (on
                                     where the parameters allow), 0 off (CUDA cores), 1 on */
    int32_t l2_prefetch;          /* each group's key block brought into L2 during the group
                                     before it: -1 automatic (on), 0 off, 1 on */
} tfhe_tuning;

/* library identification and the last error of the calling thread */
const char* tfhe_version(void);
const char* tfhe_last_error(void);

/*
 * Drop-in for the reference's XLA FFI handler "mul_bootstrap"
 * (csrc/mul_bootstrap.cuh:192-243, registered at cuTFHE/multiply.py:10-14,
 * called at cuTFHE/multiply.py:17-51): the collapsed CMux chain
 * (multiply_seq_monomial's kernel) on reference-layout buffers.
 *   ct_init      int64 (..., 2, N); ct_elems == 2N broadcasts one ACC
 *                (batch stride 0, mul_bootstrap.cuh:162-164)
 *   bsk          complex128, last six dims (G, 2, L, 2, M, N/2)
 *                (multiply.py:81-86); bsk_dims = those six extents
 *   all_rot_fft  complex128 (2N, N/2): row r = jax_fourier(X^r)
 *   indices      int32 (batch, G, M)
 *   out          int64 (batch, 2, N)
 * degree in {128..4096}, l in {1..4}; other values -> INVALID_ARGUMENT.
 * log2_q: 2..64 with the reference's float64 semantics (exact for <= 53).
 */
int tfhe_mul_bootstrap(void* stream,
                       const int64_t* ct_init, int64_t ct_elems,
                       const void* bsk, const int64_t* bsk_dims,
                       const void* all_rot_fft, int64_t all_rot_rows,
                       const int32_t* indices,
                       int64_t log2_beta, int64_t log2_q, int64_t l, int64_t degree,
                       int64_t* out, int64_t batch);

/*
 * Upload key material (HOST pointers) and convert it to the device layout;
 * returns after the upload has finished.  Replaces the key arrays the
 * reference passes into every call (HeavysideBoostrapper's
 * bootstrapping_key / key_switching_key_bs, nn_tfhe/activation.py:88-97).
 *   bsk_coeff  uint32 (2 left/right, 2 mask/body, G*M, l_bs, N): the
 *              coefficient-domain key of get_boostrapping_key_collapse
 *              (schemas/RLWE_jax.py:162-197) modulo 2^32
 *   ksk_a      uint32 (l_ks, n_big, n), ksk_b uint32 (l_ks, n_big): the key
 *              of get_keyswitch_sk_LWE (schemas/LWE_jax.py:86-93)
 */
int tfhe_keys_create(const tfhe_params* params, const uint32_t* bsk_coeff,
                     const uint32_t* ksk_a, const uint32_t* ksk_b,
                     void* stream, tfhe_keys** keys_out);

/* Same, from the reference's Fourier key ``bsk_ordered`` (complex128
 * (2, 2, l_bs, G*M, N/2), nn_tfhe/activation.py:49-53) as interleaved
 * doubles. */
int tfhe_keys_create_fourier(const tfhe_params* params, const double* bsk_ordered,
                             const uint32_t* ksk_a, const uint32_t* ksk_b,
                             void* stream, tfhe_keys** keys_out);

void tfhe_keys_destroy(tfhe_keys* keys);

/* Set (NULL: reset to automatic) the launch shape used by this key set's
 * blind rotations, and query the shape a batch would get.  Tuning only
 * changes speed, never results (no counterpart in the reference). */
int tfhe_keys_set_tuning(tfhe_keys* keys, const tfhe_tuning* tuning);
int tfhe_keys_launch_shape(const tfhe_keys* keys, int64_t batch, int32_t* ciphertexts_per_cta,
                           int32_t* threads, int64_t* shared_bytes);

/* CTAs per ciphertext a batch's blind rotation takes: 8 where one
 * ciphertext runs on a cluster of eight CTAs (N = 1024 or 2048, collapse
 * <= 3, at N = 1024 collapse >= 2; batches of at most an eighth of the SM
 * count; TFHE_B200_OCTET=0 turns it off), 4 on a cluster of four (N = 1024
 * or 2048, at most a quarter;
 * TFHE_B200_QUAD=0 turns both off), 2 on a cluster of two (at most half the
 * SM count), else 1 (automatic shapes only; TFHE_B200_SPLIT=0 turns every
 * cluster form off); 0 for NULL keys.  Speed only: every form gives
 * identical outputs. */
int32_t tfhe_keys_cluster_size(const tfhe_keys* keys, int64_t batch);
int64_t tfhe_keys_device_bytes(const tfhe_keys* keys);

/* Batched LWE key switch: key_switch_LWE vmapped over ciphertexts
 * (schemas/LWE_jax.py:97-117 as called at nn_tfhe/activation.py:150).
 * a_in (batch, n_big), b_in (batch) -> a_out (batch, n), b_out (batch). */
int tfhe_keyswitch(const tfhe_keys* keys, const uint32_t* a_in, const uint32_t* b_in,
                   uint32_t* a_out, uint32_t* b_out, int64_t batch, void* stream);

/* Blind rotation then rotation by -b~: BR (schemas/RLWE_jax.py:305-315).
 * lwe_a (batch, n), lwe_b (batch): key-switched LWEs; lut (lut_count, 2, N)
 * with lut_count == 1 (shared) or == batch; acc_out (batch, 2, N). */
int tfhe_blind_rotate(const tfhe_keys* keys, const uint32_t* lwe_a, const uint32_t* lwe_b,
                      const uint32_t* lut, int64_t lut_count, int32_t n_lut,
                      uint32_t* acc_out, int64_t batch, void* stream);

/* Many-LUT sample extraction at alpha = 0 .. n_lut-1
 * (schemas/text_jax.py:191-208 vmapped as in schemas/RLWE_jax.py:301-303).
 * acc (batch, 2, N) -> out_a (batch, n_lut, N), out_b (batch, n_lut). */
int tfhe_sample_extract(const uint32_t* acc, int32_t N, int32_t n_lut,
                        uint32_t* out_a, uint32_t* out_b, int64_t batch, void* stream);

/* The steps of cuboot_merge (schemas/RLWE_jax.py:288-303) from
 * key-switched LWEs: blind rotation from the LUT, rotation by -b~, many-LUT
 * extraction.  lwe_a (batch, n), lwe_b (batch), lut (lut_count, 2, N)
 * -> out_a (batch, n_lut, N), out_b (batch, n_lut). */
int tfhe_cuboot_merge(const tfhe_keys* keys, const uint32_t* lwe_a, const uint32_t* lwe_b,
                      const uint32_t* lut, int64_t lut_count, int32_t n_lut,
                      uint32_t* out_a, uint32_t* out_b, int64_t batch, void* stream);

/* Full programmable bootstrap: key switch, blind rotation, rotation by -b~
 * and many-LUT extraction, HeavysideBoostrapper.cuboot
 * (nn_tfhe/activation.py:148-162) = cuboot_merge(key_switch_LWE(h)).
 * a_in (batch, n_big), b_in (batch), lut (lut_count, 2, N)
 * -> out_a (batch, n_lut, N), out_b (batch, n_lut).
 * The key-switched intermediate is allocated stream-ordered on `stream`. */
int tfhe_pbs(const tfhe_keys* keys, const uint32_t* a_in, const uint32_t* b_in,
             const uint32_t* lut, int64_t lut_count, int32_t n_lut,
             uint32_t* out_a, uint32_t* out_b, int64_t batch, void* stream);

/* tfhe_pbs without any device allocation (no counterpart in the
 * reference).  For callers that cannot call cudaMalloc: an XLA custom call
 * (XLA preallocates most of the GPU for its own allocator), a serving loop
 * that forbids allocation on its latency path, code under an external
 * memory manager.  The key-switched intermediate lives in a static 8 MiB
 * device array of the library, so batch * (n + 1) * 4 bytes must fit in it
 * (at most 2822 ciphertexts for n = 742, 3323 for n = 630); larger batches
 * return TFHE_ERR_INVALID_ARGUMENT.  The array's device address, and that of
 * the device status word, are looked up on the first call on each device
 * (make that first call before any stream capture).  Every call shares the
 * one array: calls that overlap on the GPU (other streams, other threads)
 * race and corrupt each other's results.  Bounded-wait timeouts of the call
 * are reported by tfhe_device_status.  Same arguments and results as
 * tfhe_pbs. */
int tfhe_pbs_noalloc(const tfhe_keys* keys, const uint32_t* a_in, const uint32_t* b_in,
                     const uint32_t* lut, int64_t lut_count, int32_t n_lut,
                     uint32_t* out_a, uint32_t* out_b, int64_t batch, void* stream);

/* key_switch_LWE (schemas/LWE_jax.py:97-117) with the key in the
 * reference's own layout, as DEVICE uint32 arrays: ksk_a (l_ks, n_big, n)
 * and ksk_b (l_ks, n_big) (the pk / b of get_keyswitch_sk_LWE modulo 2^32).
 * a_in (batch, n_big), b_in (batch) -> a_out (batch, n), b_out (batch). */
int tfhe_keyswitch_ref(const uint32_t* a_in, const uint32_t* b_in,
                       const uint32_t* ksk_a, const uint32_t* ksk_b,
                       int32_t n_big, int32_t n, int32_t l_ks, int32_t log2_beta_ks,
                       uint32_t* a_out, uint32_t* b_out, int64_t batch, void* stream);

/* The steps of cuboot_merge / BR after the kernel (schemas/RLWE_jax.py:
 * 295-303 and 305-315) on the reference's int64 values, keeping its
 * +-q/2 representatives: b~ = round(2N b / (q n_lut)) n_lut, ACC rotated by
 * X^(-b~), then sample_extract at alpha = 0 .. n_lut-1.
 *   acc (batch, 2, N) int64 (tfhe_mul_bootstrap's output), b (batch) float64
 *   out_acc (batch, 2, N) and/or out_a (batch, n_lut, N) + out_b
 *   (batch, n_lut), all int64; pass NULL for outputs not wanted. */
int tfhe_rotate_extract_i64(const int64_t* acc, const double* b, int32_t N, int32_t n_lut,
                            int64_t log2_q, int64_t* out_acc, int64_t* out_a, int64_t* out_b,
                            int64_t batch, void* stream);

/* Status word of the current device: kernels that wait on an mbarrier
 * give up after a bounded time and record TFHE_DEVICE_TIMEOUT here instead
 * of hanging (no counterpart in the reference).  It is a static device
 * variable of the library (no allocation), shared by every entry point,
 * tfhe_pbs_noalloc included.  Synchronous; clear != 0 resets it. */
#define TFHE_DEVICE_TIMEOUT 1
int tfhe_device_status(int32_t* status_out, int32_t clear);

/* Kernels this library has launched in this process, all devices (no
 * counterpart in the reference): the difference across a region of calls is
 * the number of the library's kernel launches in it. */
int64_t tfhe_launch_count(void);

/* Diagnostics (no counterpart in the reference): runs one bounded mbarrier
 * wait that nothing completes, with a limit of limit_cycles clock cycles;
 * *waited_out = 0 when it gave up (the device status then reads
 * TFHE_DEVICE_TIMEOUT).  Synchronous. */
int tfhe_probe_wait_timeout(int64_t limit_cycles, int32_t* waited_out);

/* tfhe_pbs from HOST buffers (pinned, for overlap): the batch is processed
 * in chunks of `chunk` ciphertexts (0: automatic); each chunk's upload,
 * compute and download run on separate streams so the copies overlap the
 * compute of neighbouring chunks.  Same layouts and results as tfhe_pbs
 * (HeavysideBoostrapper.cuboot, nn_tfhe/activation.py:148-162); the
 * caller's stream resumes after the last download. */
int tfhe_pbs_host(const tfhe_keys* keys, const uint32_t* a_host, const uint32_t* b_host,
                  const uint32_t* lut_host, int64_t lut_count, int32_t n_lut,
                  uint32_t* out_a_host, uint32_t* out_b_host, int64_t batch, int64_t chunk,
                  void* stream);

/* Diagnostics (no counterpart in the reference): FP64 FMA throughput
 * probe for the roofline denominator.  Launches blocks x threads threads,
 * each running 8 independent FMA chains of `iters` steps; *flops receives
 * the flop count of the launch (host pointer); scratch is one device
 * double.  Time it with events on `stream`. */
int tfhe_probe_fp64_fma(int32_t blocks, int32_t threads, int32_t iters, double* scratch,
                        double* flops, void* stream);

/* ------------------------------------------------------------------------
 * Spike-LSTM timestep operators (nn_tfhe/Spike_LSTM.py:15-62, 103-184).
 * Integer plaintexts times ciphertexts are exact modulo 2^32; the reference
 * rounds FP64 FFT products that are exact at these sizes.
 * ---------------------------------------------------------------------- */

/* Linear.__call__ (nn_tfhe/Spike_LSTM.py:48-58): for every ciphertext s and
 * output j, W_j(X) * rlwe_s (multiply_plaintext_ciphertext), sample_extract
 * at 0 (schemas/text_jax.py:191-208), + bias_j.
 *   weights (J, N) int32 in the layout of Linear.set_weights (:28-41),
 *   bias (J) int32, rlwe (S, 2, N) -> out_a (S, J, N), out_b (S, J). */
int tfhe_linear_extract(const int32_t* weights, const int32_t* bias, int32_t J,
                        const uint32_t* rlwe, int64_t S, int32_t N,
                        uint32_t* out_a, uint32_t* out_b, void* stream);

/* prepare_LUT's product (nn_tfhe/activation.py:103-106) summed over the
 * packed sub-LUTs (nn_tfhe/Spike_LSTM.py:129-132):
 *   out[s][k] = sum_{g < groups} luts[g][k](X) * rlwe[s][g][k]
 *   luts (groups, per_group, N) int32, rlwe (S, groups, per_group, 2, N)
 *   -> out (S, per_group, 2, N). */
int tfhe_lut_mul_sum(const int32_t* luts, int32_t groups, int32_t per_group,
                     const uint32_t* rlwe, int64_t S, int32_t N,
                     uint32_t* out, void* stream);

typedef struct tfhe_galois_keys tfhe_galois_keys;

/* Galois keys of pack_lwe_to_rlwe (get_galois_key, schemas/RLWE_jax.py:
 * 218-226): keys (log2 N, l, 2, N) uint32 on the device, step i switching
 * from the automorphism X -> X^(2^(log2 N - i) + 1) of the secret back to
 * it, l levels of base 2^log2_beta.  Converted once to the FP64 Fourier
 * domain. */
int tfhe_galois_keys_create(int32_t N, int32_t log2_beta, int32_t l, const uint32_t* keys,
                            void* stream, tfhe_galois_keys** out);
int tfhe_galois_keys_destroy(tfhe_galois_keys* keys);

/* pack_lwe_to_rlwe (schemas/text_jax.py:316-345): modulus switch to q/N,
 * trivial embedding, log2 N automorphism + key-switch trace steps.
 *   lwe_a (R, N), lwe_b (R) -> out (R, 2, N), reduced modulo 2^32. */
int tfhe_pack_lwe_to_rlwe(const tfhe_galois_keys* keys, const uint32_t* lwe_a,
                          const uint32_t* lwe_b, int64_t R, uint32_t* out, void* stream);

/* packing (schemas/text_jax.py:211-239): T LWEs of dimension n_dim per
 * output into one RLWE of degree N with the packing key
 * (get_packing_KSK, schemas/RLWE_jax.py:205-215) laid out as
 * ksp (n_dim, l, 2, N) uint32.
 *   lwe_a (S, T, n_dim), lwe_b (S, T) -> out (S, 2, N); T <= N, l <= 4. */
int tfhe_pack_lwes(const uint32_t* ksp, int32_t n_dim, int32_t N, int32_t log2_beta, int32_t l,
                   const uint32_t* lwe_a, const uint32_t* lwe_b, int32_t T, int64_t S,
                   uint32_t* out, void* stream);

/* Device-resident packing key for repeated packings: a copy of ksp
 * (n_dim, l, 2, N) and, where the digits fit 8 bits (log2_beta <= 7) and the
 * int32 sums cannot overflow, its int8 limbs for the tcgen05 tensor cores. */
typedef struct tfhe_packing_key tfhe_packing_key;
int tfhe_packing_key_create(const uint32_t* ksp, int32_t n_dim, int32_t N, int32_t log2_beta, int32_t l,
                            void* stream, tfhe_packing_key** out);
int tfhe_packing_key_destroy(tfhe_packing_key* key);
/* 1 when the key carries tensor-core limbs, else 0. */
int tfhe_packing_key_uses_tensor_cores(const tfhe_packing_key* key);
/* tfhe_pack_lwes with a packing key (packing, schemas/text_jax.py:211-239):
 * on the tensor cores when the key has limbs, tensor_cores != 0 and lwe_a is
 * 16-byte aligned, else on CUDA cores; same result either way. */
int tfhe_pack_lwes_with_key(const tfhe_packing_key* key, const uint32_t* lwe_a, const uint32_t* lwe_b,
                            int32_t T, int64_t S, uint32_t* out, int32_t tensor_cores, void* stream);

/* out[s] = X^rot * x[s] + y[s] for RLWEs (S, 2, N); y may be NULL
 * (rotate_ciphertext, schemas/text_jax.py:348-362, and
 * sum_ciphertext_ciphertext, :24-41).  out may alias y, and x only if
 * rot == 0 mod 2N. */
int tfhe_rlwe_rotate_add(const uint32_t* x, int32_t rot, const uint32_t* y, int64_t S,
                         int32_t N, uint32_t* out, void* stream);

/* out = x + y modulo 2^32 over n words (sums of LWE ciphertexts). */
int tfhe_u32_add(const uint32_t* x, const uint32_t* y, int64_t n, uint32_t* out, void* stream);

/* ------------------------------------------------------------------------
 * The FP32 split-limb form of the blind rotation (the precision ablation of
 * the external product; no counterpart in the reference, whose kernel is
 * FP64, csrc/mul_bootstrap.cuh:20-95).  Every FFT runs in FP32 and the
 * bootstrapping key is split into `limbs` (2..4) signed limbs of
 * ceil(32 / limbs) bits whose FP32 products are rounded to integers and
 * recombined exactly modulo 2^32.  bsk_coeff as for tfhe_keys_create
 * (HOST pointer); N in {256, 1024, 2048}, l_bs <= 3 (<= 2 at N = 2048),
 * collapse <= 3.
 * ---------------------------------------------------------------------- */
typedef struct tfhe_fp32_keys tfhe_fp32_keys;
int tfhe_fp32_keys_create(const tfhe_params* params, const uint32_t* bsk_coeff, int32_t limbs, void* stream,
                          tfhe_fp32_keys** keys_out);
void tfhe_fp32_keys_destroy(tfhe_fp32_keys* keys);

/* cuboot_merge (schemas/RLWE_jax.py:288-303) with the FP32 split-limb chain:
 * lwe_a (batch, n), lwe_b (batch), lut (lut_count, 2, N) -> out_a
 * (batch, n_lut, N), out_b (batch, n_lut); or, when acc_out is not NULL,
 * the accumulator after the chain (batch, 2, N), not rotated by -b~.
 * ciphertexts_per_cta: 1 or 2 (0: 2). */
int tfhe_fp32_cuboot_merge(const tfhe_fp32_keys* keys, const uint32_t* lwe_a, const uint32_t* lwe_b,
                           const uint32_t* lut, int64_t lut_count, int32_t n_lut, uint32_t* out_a,
                           uint32_t* out_b, uint32_t* acc_out, int64_t batch, int32_t ciphertexts_per_cta,
                           void* stream);

/* ------------------------------------------------------------------------
 * The reference's own torus, q = 2^64 (parameters_crypto.py:6), where the
 * reference holds values in float64.  Torus values are uint64 words and
 * every integer step is exact modulo 2^64; gadget digits are the
 * reference's decomposition (schemas/polynomial_jax.py:90-111: round half
 * to even) evaluated exactly on the integer.  The blind rotation is the
 * FP64 chain at q = 2^64, as the reference's: natively (tfhe64_keys_create,
 * tfhe64_cuboot_merge) or through tfhe_mul_bootstrap at log2_q = 64.
 * ---------------------------------------------------------------------- */

/* Bootstrapping keys on Z/2^64 (KeyGen, schemas/RLWE_jax.py:162-197):
 * params as for tfhe_keys_create with log2_q = 64 and l_bs <= 3; bsk_coeff
 * (host) (2, 2, G M, l_bs, N) uint64 = RLWE encryptions of the collapsed
 * CMux key as for tfhe_keys_create.  The key is converted to its FP64
 * spectra on the device; free with tfhe_keys_destroy.  The key switch on
 * this torus takes its key directly (tfhe64_keyswitch*). */
int tfhe64_keys_create(const tfhe_params* params, const uint64_t* bsk_coeff, void* stream, tfhe_keys** keys_out);

/* cuboot_merge (schemas/RLWE_jax.py:281-303) on Z/2^64 in one kernel: the
 * rotation indices of multiply_seq_monomial from the masks (exact integer
 * sums, round half to even), the collapsed CMux chain from ACC = lut, the
 * rotation by X^(-b~) and the extraction of n_lut LWEs.  lwe_a (batch, n),
 * lwe_b (batch) uint64; lut (lut_count, 2, N) int64, lut_count 1 or batch;
 * n_lut a power of two <= N -> out_a (batch, n_lut, N), out_b (batch,
 * n_lut) uint64.  tfhe64_blind_rotate: the rotated ACC (batch, 2, N)
 * instead of the extraction. */
int tfhe64_cuboot_merge(const tfhe_keys* keys, const uint64_t* lwe_a, const uint64_t* lwe_b, const int64_t* lut,
                        int64_t lut_count, int32_t n_lut, uint64_t* out_a, uint64_t* out_b, int64_t batch,
                        void* stream);
int tfhe64_blind_rotate(const tfhe_keys* keys, const uint64_t* lwe_a, const uint64_t* lwe_b, const int64_t* lut,
                        int64_t lut_count, int32_t n_lut, uint64_t* acc_out, int64_t batch, void* stream);

/* key_switch_LWE (schemas/LWE_jax.py:97-117) on Z/2^64: ksk (n_big l_ks,
 * n + 1) uint64, row i l_ks + j = LWE(-s_big[i] q / beta^(j+1)) as n mask
 * words then the body; a_in (batch, n_big), b_in (batch) -> a_out
 * (batch, n), b_out (batch).  l_ks <= 8, log2_beta_ks <= 16. */
int tfhe64_keyswitch(const uint64_t* ksk, int32_t n_big, int32_t n, int32_t l_ks, int32_t log2_beta_ks,
                     const uint64_t* a_in, const uint64_t* b_in, uint64_t* a_out, uint64_t* b_out,
                     int64_t batch, void* stream);

/* Rotation indices of multiply_seq_monomial (cuTFHE/multiply.py:67-79)
 * from 64-bit masks: indices (batch, n / collapse, 2^collapse) int32,
 * round(2N <a_g, p> / (q n_lut)) n_lut mod 2N, ready for
 * tfhe_mul_bootstrap.  n_lut a power of two. */
int tfhe64_rotation_indices(const uint64_t* lwe_a, int32_t n, int32_t collapse, int32_t N, int32_t n_lut,
                            int32_t* indices, int64_t batch, void* stream);

/* The steps of cuboot_merge after the chain (schemas/RLWE_jax.py:295-303)
 * on Z/2^64: b~ = round(2N b / (q n_lut)) n_lut, ACC rotated by X^(-b~),
 * sample_extract at 0 .. n_lut-1.  acc (batch, 2, N) int64 (the output of
 * tfhe_mul_bootstrap at log2_q = 64), b (batch) -> out_a (batch, n_lut, N),
 * out_b (batch, n_lut). */
int tfhe64_rotate_extract(const int64_t* acc, const uint64_t* b, int32_t N, int32_t n_lut, uint64_t* out_a,
                          uint64_t* out_b, int64_t batch, void* stream);

/* Linear.__call__ (nn_tfhe/Spike_LSTM.py:48-58) on Z/2^64: weights (J, N)
 * int32, bias (J) int64, rlwe (S, 2, N) -> out_a (S, J, N), out_b (S, J). */
int tfhe64_linear_extract(const int32_t* weights, const int64_t* bias, int32_t J, const uint64_t* rlwe,
                          int64_t S, int32_t N, uint64_t* out_a, uint64_t* out_b, void* stream);

/* prepare_LUT's product summed over the packed sub-LUTs
 * (nn_tfhe/activation.py:103-106, nn_tfhe/Spike_LSTM.py:129-132) on
 * Z/2^64: luts (groups, per_group, N) int64, rlwe (S, groups, per_group,
 * 2, N) -> out (S, per_group, 2, N). */
int tfhe64_lut_mul_sum(const int64_t* luts, int32_t groups, int32_t per_group, const uint64_t* rlwe, int64_t S,
                       int32_t N, uint64_t* out, void* stream);

/* Galois keys of pack_lwe_to_rlwe (get_galois_key, schemas/RLWE_jax.py:
 * 218-226) on Z/2^64: keys (log2 N, l, 2, N) uint64 on the device, kept as
 * the FP64 Fourier transforms of their four 16-bit limbs so that every key
 * product is an exact integer. */
typedef struct tfhe64_galois_keys tfhe64_galois_keys;
int tfhe64_galois_keys_create(int32_t N, int32_t log2_beta, int32_t l, const uint64_t* keys, void* stream,
                              tfhe64_galois_keys** out);
int tfhe64_galois_keys_destroy(tfhe64_galois_keys* keys);

/* pack_lwe_to_rlwe (schemas/text_jax.py:316-345) on Z/2^64: lwe_a (R, N),
 * lwe_b (R) -> out (R, 2, N). */
int tfhe64_pack_lwe_to_rlwe(const tfhe64_galois_keys* keys, const uint64_t* lwe_a, const uint64_t* lwe_b,
                            int64_t R, uint64_t* out, void* stream);

/* packing (schemas/text_jax.py:211-239) on Z/2^64 with ksp (n_dim, l, 2, N)
 * uint64 (get_packing_KSK, schemas/RLWE_jax.py:205-215): lwe_a
 * (S, T, n_dim), lwe_b (S, T) -> out (S, 2, N); T <= N, l <= 8. */
int tfhe64_pack_lwes(const uint64_t* ksp, int32_t n_dim, int32_t N, int32_t log2_beta, int32_t l,
                     const uint64_t* lwe_a, const uint64_t* lwe_b, int32_t T, int64_t S, uint64_t* out,
                     void* stream);

/* The key switch and the packing on Z/2^64 on the tcgen05 tensor cores
 * (kind::i8): every 64-bit key word split into eight signed 8-bit limbs,
 * int8 digits x limbs -> int32 sums recombined modulo 2^64 (exact: the sums
 * cannot overflow, checked).  Needs log2_beta <= 7, n_big (n_dim) a multiple
 * of 32 and 16-byte aligned masks.
 *   tfhe64_tc_limb_rows(cols): rows of the limb matrix of a key with `cols`
 *     columns (8 cols rounded up to the CTA tile);
 *   tfhe64_tc_limbs: key (K, cols) uint64 row-major -> limbs (rows, K) int8
 *     (the key switch: K = n_big l_ks, cols = n + 1; the packing key
 *     (n_dim, l, 2, N): K = n_dim l, cols = 2N);
 *   tfhe64_keyswitch_tc / tfhe64_pack_lwes_tc: tfhe64_keyswitch and
 *     tfhe64_pack_lwes (key_switch_LWE, schemas/LWE_jax.py:97-117; packing,
 *     schemas/text_jax.py:211-239) from those limbs, same results. */
int64_t tfhe64_tc_limb_rows(int32_t cols);
int tfhe64_tc_limbs(const uint64_t* key, int64_t K, int32_t cols, int8_t* limbs, void* stream);
int tfhe64_keyswitch_tc(const int8_t* limbs, int32_t n_big, int32_t n, int32_t l_ks, int32_t log2_beta_ks,
                        const uint64_t* a_in, const uint64_t* b_in, uint64_t* a_out, uint64_t* b_out,
                        int64_t batch, void* stream);
int tfhe64_pack_lwes_tc(const int8_t* limbs, int32_t n_dim, int32_t N, int32_t log2_beta, int32_t l,
                        const uint64_t* lwe_a, const uint64_t* lwe_b, int32_t T, int64_t S, uint64_t* out,
                        void* stream);

/* out[s] = X^rot x[s] + y[s] (y may be NULL), out = x + y, and the LWEs of
 * coefficients 0 .. count-1 of RLWEs (rotate_ciphertext, sum_ciphertext_
 * ciphertext, sample_extract: schemas/text_jax.py:24-41, 191-208, 348-362)
 * on Z/2^64. */
int tfhe64_rlwe_rotate_add(const uint64_t* x, int32_t rot, const uint64_t* y, int64_t S, int32_t N,
                           uint64_t* out, void* stream);
int tfhe64_add(const uint64_t* x, const uint64_t* y, int64_t n, uint64_t* out, void* stream);
int tfhe64_sample_extract(const uint64_t* rlwe, int32_t N, int32_t count, uint64_t* out_a, uint64_t* out_b,
                          int64_t S, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* TFHE_B200_H */
