/*
 * lattice_cuda.h -- C ABI of the B200 (sm_100a) commitment hot path of LZX.
 *
 * Drop-in GPU backend for the negacyclic NTT over Z_q[X]/(X^n+1) and the Ajtai
 * commitment c = A.w of idrees2516/lzx (Rust crates lattice-ring and
 * lattice-commitment).  Every result is an exact residue, bit-identical to the
 * reference's scalar code.  Plain C types only: pointers, sizes, status codes.
 *
 * Conventions
 *   - Ring degree n = 2^log_n.  A batch of polynomials is coefficient-
 *     contiguous and element-major ([count][n]); a plan with several u32
 *     moduli (a CRT set) takes [modulus][count][n].
 *   - u32 plans hold residues as uint32_t in [0,q); Goldilocks plans as
 *     uint64_t in [0,p), p = 2^64 - 2^32 + 1.  Inputs must be canonical.
 *   - "Device" entry points take device pointers (16-byte aligned) and an
 *     optional cudaStream_t (NULL = legacy default stream); they only enqueue
 *     work.  "Host" entry points take host pointers, are synchronous and move
 *     the data themselves.
 *   - Status codes map 1:1 onto the reference's error enums where one exists
 *     (NttError, lattice-ring/src/ntt.rs:38-42; RingError, ring.rs:17-21;
 *     AjtaiError, lattice-commitment/src/ajtai.rs:43-49).  No entry point
 *     aborts or prints.
 *   - There is no CPU fallback: without a usable sm_100 device every compute
 *     entry point returns LC_ERR_NO_DEVICE.
 */
#ifndef LATTICE_CUDA_H
#define LATTICE_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LC_API __attribute__((visibility("default")))

typedef enum lc_status {
  LC_OK = 0,
  LC_ERR_LENGTH_MISMATCH = 1,     /* NttError::LengthMismatch (ntt.rs:40), RingError::LengthMismatch (ring.rs:20) */
  LC_ERR_ADICITY_TOO_SMALL = 2,   /* NttError::AdicityTooSmall (ntt.rs:41) */
  LC_ERR_DIMENSION_MISMATCH = 3,  /* AjtaiError::DimensionMismatch (ajtai.rs:45) */
  LC_ERR_NORM_EXCEEDED = 4,       /* AjtaiError::NormExceeded (ajtai.rs:46) */
  LC_ERR_COMMITMENT_MISMATCH = 5, /* AjtaiError::CommitmentMismatch (ajtai.rs:47) */
  LC_ERR_NON_CANONICAL = 6,       /* RingElement::from_bytes rejection (ring.rs:394-400) */
  LC_ERR_INVALID_ARGUMENT = 7,    /* null/misaligned pointer, bad modulus, bad sizes */
  LC_ERR_UNSUPPORTED = 8,         /* valid in the reference but not built here (e.g. log_n) */
  LC_ERR_CUDA = 9,                /* a CUDA runtime call failed */
  LC_ERR_OUT_OF_MEMORY = 10,
  LC_ERR_TIMEOUT = 11,            /* a bounded device-side wait expired */
  LC_ERR_NO_DEVICE = 12,          /* no sm_100 device available */
  LC_ERR_LOG_N_OUT_OF_RANGE = 13, /* Mod50Error::LogNOutOfRange (lattice-ring/src/modulus50.rs:418) */
  LC_ERR_GENERATOR_INVALID = 14   /* Mod50Error::GeneratorInvalid (modulus50.rs:420) */
} lc_status;

typedef void *lc_stream; /* cudaStream_t */

typedef struct lc_ntt_plan lc_ntt_plan;

/* Library version ("major.minor.patch") and a static string for a status. */
LC_API const char *lc_version(void);
LC_API const char *lc_status_string(int status);
/* 1 when a CUDA device of compute capability 10.x is usable, else 0. */
LC_API int lc_device_available(void);

/* ------------------------------------------------------------------------
 * NTT plans.  Replace NttTables::new(Modulus32, log_n)
 * (lattice-ring/src/ntt.rs:46-106): psi = g^((q-1) >> (log_n+1)) exactly as
 * Modulus32::root_of_unity_order_2n (modulus.rs:149-161).  The plan keeps
 * its twiddle tables resident on the current device.
 *   - lc_ntt_plan_create_u32: num_moduli (1..8) u32 primes sharing log_n;
 *     q odd, 2 < q < 2^32; returns LC_ERR_ADICITY_TOO_SMALL when
 *     log_n + 1 > two_adicity (ntt.rs:47-50) and LC_ERR_INVALID_ARGUMENT when
 *     psi does not have order exactly 2n.  Supported log_n: 1..11.
 *   - lc_ntt_plan_create_goldilocks: the same transform over Goldilocks
 *     (lattice-core/src/field.rs), generator 7 (field.rs:195-200), log_n 1..10.
 * ---------------------------------------------------------------------- */
LC_API int lc_ntt_plan_create_u32(uint32_t log_n, const uint32_t *q, const uint32_t *two_adicity,
                                  const uint32_t *generator, uint32_t num_moduli,
                                  lc_ntt_plan **out);
LC_API int lc_ntt_plan_create_goldilocks(uint32_t log_n, lc_ntt_plan **out);
LC_API void lc_ntt_plan_destroy(lc_ntt_plan *plan);
/* n, number of moduli, element size in bytes (4 or 8). */
LC_API int lc_ntt_plan_info(const lc_ntt_plan *plan, uint32_t *log_n, uint32_t *num_moduli,
                            uint32_t *elem_bytes);

/* Tuning hook (no counterpart in the reference, which has no kernels): picks
 * one of the instantiated tile shapes / pipeline depths of this plan's
 * transform kernels, 0 = the default.  Results are identical for every
 * variant; only the speed changes.  LC_ERR_INVALID_ARGUMENT outside
 * 0 .. LC_NTT_NUM_VARIANTS - 1. */
#define LC_NTT_NUM_VARIANTS 7
LC_API int lc_ntt_plan_set_variant(lc_ntt_plan *plan, int variant);

/* Batched forward transform, device pointers.  Replaces
 * NttTables::forward_fast / RingElement::to_ntt (ntt.rs:118-146,
 * ring.rs:344-351) applied to `count` polynomials per modulus; output in the
 * reference's natural order out[j] = a(psi^(2j+1)).  in == out is allowed;
 * count <= 2^29 (LC_ERR_INVALID_ARGUMENT above). */
LC_API int lc_ntt_forward(const lc_ntt_plan *plan, const void *in, void *out, size_t count,
                          lc_stream stream);
/* Batched inverse, device pointers.  Replaces NttTables::inverse_fast /
 * RingElement::from_ntt (ntt.rs:187-216, ring.rs:354-367). */
LC_API int lc_ntt_inverse(const lc_ntt_plan *plan, const void *in, void *out, size_t count,
                          lc_stream stream);

/* Incomplete transform, device pointers: NttTables::forward_partial
 * (ntt.rs:252-286) -- psi^i pre-scale, bit reversal, then only the first
 * `levels` Cooley-Tukey levels -- and NttTables::complete_partial
 * (ntt.rs:288-316), which applies the levels after `already`; the output is
 * the reference's own intermediate order, and complete_partial(
 * forward_partial(a, L), L) equals lc_ntt_forward(a).  u32 plans only
 * (LC_ERR_UNSUPPORTED for Goldilocks); levels/already > log_n gives
 * LC_ERR_LENGTH_MISMATCH as in the reference.  in == out is allowed. */
LC_API int lc_ntt_forward_partial(lc_ntt_plan *plan, const void *in, void *out, size_t count, uint32_t levels,
                                  lc_stream stream);
LC_API int lc_ntt_complete_partial(lc_ntt_plan *plan, const void *in, void *out, size_t count, uint32_t already,
                                   lc_stream stream);

/* Host-buffer variants: synchronous; copy in, transform, copy out (pipelined
 * in chunks over two streams).  in == out is allowed.  Pinned host memory
 * gives the full PCIe rate; pageable memory works at a lower rate. */
LC_API int lc_ntt_forward_host(lc_ntt_plan *plan, const void *in, void *out, size_t count);
LC_API int lc_ntt_inverse_host(lc_ntt_plan *plan, const void *in, void *out, size_t count);

/* Wait for `stream`, then report (and clear) any device-side error recorded
 * by this plan's kernels since the last check (LC_ERR_TIMEOUT), or a pending
 * CUDA error (LC_ERR_CUDA). */
LC_API int lc_ntt_plan_check(lc_ntt_plan *plan, lc_stream stream);

/* ------------------------------------------------------------------------
 * Ajtai commitment keys and commits (lattice-commitment/src/ajtai.rs).
 * A key holds the cached forward NTT of A resident on the device, as
 * AjtaiPublicKey::from_seed does (ajtai.rs:87-103), for one modulus: a u32
 * plan with num_moduli == 1 (e.g. Modulus32::Q_32) or a Goldilocks plan.
 * Supported: log_n 1..10 (u32) / 1..9 (Goldilocks), k <= 16 rows, any m.
 * A key is used by one thread
 * at a time (it owns its scratch buffers).
 * ---------------------------------------------------------------------- */
typedef struct lc_ajtai_key lc_ajtai_key;

/* `matrix`: the k*m entries A[i][j] in coefficient form, row-major
 * (entry (i,j) at (i*m + j)*n), residues of the plan's element type; host
 * memory, or device memory when matrix_on_device != 0.  Replaces the
 * cached-NTT part of AjtaiPublicKey::from_seed (ajtai.rs:91-96); the seed
 * expansion (uniform_from_seed, ring.rs:102-180) runs on the device in
 * lc_ajtai_key_from_seed, or on the host before this call. */
LC_API int lc_ajtai_key_create(const lc_ntt_plan *plan, uint32_t k, uint32_t m, const void *matrix,
                               int matrix_on_device, lc_ajtai_key **out);
LC_API void lc_ajtai_key_destroy(lc_ajtai_key *key);
LC_API int lc_ajtai_key_info(const lc_ajtai_key *key, uint32_t *k, uint32_t *m, uint32_t *log_n);

/* Commit `batch` witnesses, device pointers: s = [batch][m][n] canonical
 * residues, out = [batch][k][n].  For each witness this is
 * AjtaiPublicKey::commit (ajtai.rs:118-153): forward NTT of every s_j,
 * pointwise multiply-accumulate against the cached NTT(A), one inverse NTT
 * per row.  Bit-identical to the reference. */
LC_API int lc_ajtai_commit(lc_ajtai_key *key, const void *s, size_t batch, void *out,
                           lc_stream stream);
/* Same with witness coefficients given as int8 digits in [-128, 127] (a digit
 * x < 0 stands for the residue q - |x|, as NeoRing::small does,
 * lattice-folding/src/neo.rs:98-109). */
LC_API int lc_ajtai_commit_i8(lc_ajtai_key *key, const int8_t *s, size_t batch, void *out,
                              lc_stream stream);
/* Same with unsigned byte digits in [0, 255] (the rows of decomp_b with
 * b <= 8, lattice-folding/src/neo.rs:253-266, each row one witness). */
LC_API int lc_ajtai_commit_u8(lc_ajtai_key *key, const uint8_t *s, size_t batch, void *out,
                              lc_stream stream);
/* Host-buffer variants (synchronous).  Small commitments (those the
 * single-launch kernel takes: at most 4 witnesses, 2048 ring elements, with
 * a witness of at most 256 KiB) run that kernel directly on page-locked host
 * memory -- the caller's buffers
 * when they are pinned (output 16-byte aligned), else the key's pinned
 * staging buffers -- with no copies queued; larger ones upload, commit on
 * the device and download. */
LC_API int lc_ajtai_commit_host(lc_ajtai_key *key, const void *s, size_t batch, void *out);
LC_API int lc_ajtai_commit_i8_host(lc_ajtai_key *key, const int8_t *s, size_t batch, void *out);
LC_API int lc_ajtai_commit_u8_host(lc_ajtai_key *key, const uint8_t *s, size_t batch, void *out);
/* Wait for `stream` and report device-side errors of this key's kernels
 * (LC_ERR_TIMEOUT).  The error word is cleared by the report, except when a
 * timed-out kernel could not confirm that its own copies had landed: that
 * state stays set and every later check reports it. */
LC_API int lc_ajtai_key_check(lc_ajtai_key *key, lc_stream stream);

/* A view of the first k rows and m columns of `parent`'s A: commits through
 * it equal commits with a key created from that sub-matrix (rows and columns
 * of A enter the commitment independently), without copying the cached
 * NTT(A).  No counterpart in the reference, where an AjtaiPublicKey is built
 * per shape; it lets callers with many commitment shapes share one resident
 * key.  The view owns its scratch; `parent` must outlive it; NTT engine only. */
LC_API int lc_ajtai_key_view(const lc_ajtai_key *parent, uint32_t k, uint32_t m, lc_ajtai_key **out);

/* RingConfig::uniform_from_seed (lattice-ring/src/ring.rs:102-180) on the
 * device for `count` consecutive indices index0, index0+1, ...: out (device)
 * = [count][n] residues of the plan's single u32 modulus, byte-identical to
 * the reference (SHAKE256 via Transcript::xof, transcript.rs:229-237;
 * rejection of windows >= 2^32 - 2^32 mod q).  The framed message
 * (domain and seed plus 27 bytes) must fit 4 SHAKE blocks: domain_len +
 * seed_len <= 516, else LC_ERR_INVALID_ARGUMENT. */
LC_API int lc_uniform_from_seed(const lc_ntt_plan *plan, const uint8_t *domain, size_t domain_len,
                                const uint8_t *seed, size_t seed_len, uint64_t index0, size_t count,
                                uint32_t *out, lc_stream stream);

/* AjtaiPublicKey::from_seed (lattice-commitment/src/ajtai.rs:87-103) on the
 * device: A[i][j] = uniform_from_seed(b"ajtai-A", seed, i*m + j), then the
 * cached NTT as lc_ajtai_key_create.  Synchronous. */
LC_API int lc_ajtai_key_from_seed(const lc_ntt_plan *plan, uint32_t k, uint32_t m, const uint8_t seed[32],
                                  lc_ajtai_key **out);

/* Key creation flags. */
#define LC_KEY_TENSOR_I8 1u /* also build the INT8 tensor-core commit tables */

/* lc_ajtai_key_create with flags.  LC_KEY_TENSOR_I8 (Goldilocks plans with
 * log_n == 6 only, else LC_ERR_UNSUPPORTED) additionally stores every entry
 * of A as byte limbs of its negacyclic rotation (16 KiB per j for every 16
 * rows i, twice the size of A) for the tensor-core engine of
 * lc_ajtai_commit_i8, and makes that engine the key's default.  This is the
 * limb-split form of the coefficient-domain commit
 * (lattice-folding/src/neo.rs:138-158, 419-441); the results are identical
 * to the NTT engine's. */
LC_API int lc_ajtai_key_create_ex(const lc_ntt_plan *plan, uint32_t k, uint32_t m, const void *matrix,
                                  int matrix_on_device, uint32_t flags, lc_ajtai_key **out);

/* Which engine the byte-digit commits (lc_ajtai_commit_i8 / _u8 and their
 * host variants) use: LC_ENGINE_NTT (cached-NTT multiply-accumulate, every
 * key) or LC_ENGINE_TENSOR_I8 (keys created with LC_KEY_TENSOR_I8; exact
 * s8 x u8 (u8 x u8) products on the tensor cores, per-limb int32 sums of at
 * most 1024 (512) ring elements, exact 128-bit reduction).  Residue
 * witnesses (lc_ajtai_commit) always use the NTT engine. */
#define LC_ENGINE_NTT 0
#define LC_ENGINE_TENSOR_I8 1
LC_API int lc_ajtai_key_set_engine(lc_ajtai_key *key, int engine);
LC_API int lc_ajtai_key_get_engine(const lc_ajtai_key *key);

/* Measured INT8 tensor rate (no counterpart in the reference): one CTA per
 * SM issues `iters` x 4 tcgen05.mma.kind::i8 (M = 128, N = 256, K = 32, the
 * shape of the tensor-core engines; s8 != 0: signed x unsigned operands,
 * else unsigned x unsigned) on operands resident in shared memory, timed
 * with CUDA events after a warm-up launch.  *ops_per_s = integer operations
 * (2 per multiply-add) per second over the whole GPU; *ms (optional) the
 * timed launch.  The roofline denominator of the INT8 engines. */
LC_API int lc_tc_i8_rate(uint32_t iters, int s8, double *ops_per_s, float *ms);

/* Single-launch form of the NTT engine, on by default: a commitment of at
 * most 4 witnesses, at most 2048 ring elements and at most 2^20
 * multiply-adds (batch * m * n * k), log_n 6..8, runs as one kernel -- the
 * witness forward transforms, the pointwise products against the cached
 * NTT(A), their sum over the whole witness and the row inverse transforms,
 * i.e. the whole body of AjtaiPublicKey::commit (ajtai.rs:118-153) -- rather
 * than the staged launches.  Larger commits whose per-slot products run on
 * the CUDA cores (LC_PRODUCTS_INT64), log_n 6..8, can run their products,
 * the modular sum of the K splits and the row inverse transforms as one
 * cooperative launch after the witness transforms (grid barriers between the
 * three phases; ajtai.rs:139-150).  enable = 1 (the default) uses the one-
 * launch forms where they measured faster -- the single launch above and,
 * for batches of at most 3 witnesses, the one-launch products + inverse
 * NTT; enable = 2 uses the one-launch products + inverse NTT for every
 * batch shape as well; enable = 0 runs every commit staged (products, split
 * sum, inverse NTT as separate launches).  Identical results.
 * lc_ajtai_key_get_fused returns 0, 1 or 2 (-1 for a null key). */
LC_API int lc_ajtai_key_set_fused(lc_ajtai_key *key, int enable);
LC_API int lc_ajtai_key_get_fused(const lc_ajtai_key *key);

/* How the NTT engine forms its per-slot products C_t = A_t^T W_t (staged
 * commits): LC_PRODUCTS_TENSOR (default) as exact byte-limb GEMMs on the INT8
 * tensor cores -- both residues split into unsigned byte limbs (8 for
 * Goldilocks, 4 for u32 moduli), read in place from the cached NTT(A) and the
 * witness transforms, int32 sums of at most 32768 ring elements, limbs
 * recombined and reduced mod q -- whenever a witness row of the transforms
 * (limbs x padded batch) is 32, 64, 128, 256 or a multiple of 512 bytes (other
 * paddings use the integer form); LC_PRODUCTS_INT64 with 160-bit integer
 * multiply-accumulates on the CUDA cores.  Identical results.
 * lc_ajtai_key_get_slot_products returns the mode (-1 for a null key). */
#define LC_PRODUCTS_INT64 0
#define LC_PRODUCTS_TENSOR 1
LC_API int lc_ajtai_key_set_slot_products(lc_ajtai_key *key, int mode);
LC_API int lc_ajtai_key_get_slot_products(const lc_ajtai_key *key);

/* Commit without allocating any device memory.  No counterpart in the
 * reference: it exists for callers that cannot call cudaMalloc while they
 * commit -- processes whose device memory is already handed out by another
 * allocator under a fixed budget, and latency-critical verifiers that cannot
 * afford cudaMalloc's implicit device synchronisation.  It computes exactly
 * what lc_ajtai_commit computes for the same key and residues (device
 * pointers s = [batch][m][n], out = [batch][k][n]), but its scratch is one
 * fixed 16 MiB array compiled into this library, which every GPU that loads
 * the library keeps for the life of the process.  The key (created
 * beforehand, which does allocate) is only read.
 * Limits: log_n 6..8, and three regions must fit in 16 MiB together: the
 * witness transforms (n*m*b_pad elements) and the summed rows (batch*k*n
 * elements), each rounded up to a multiple of 256 bytes, plus one K-split of
 * partial sums (n*16*b_pad elements); b_pad = batch below 64, else batch
 * rounded up to 128.  A larger request returns LC_ERR_INVALID_ARGUMENT
 * without touching the GPU.
 * The first call on each device looks up the array's device address through
 * the CUDA runtime (later calls reuse it); make that first call on a device
 * before any stream capture begins.  All calls share the one array, so
 * calls whose kernels overlap on the GPU (different streams, or different host
 * threads on one device) race with each other: serialise them.  The array
 * keeps the previous call's contents; no part of it needs to start at zero,
 * because every word a call reads is written earlier in the same call. */
LC_API int lc_ajtai_commit_noalloc(const lc_ajtai_key *key, const void *s, size_t batch, void *out,
                                   lc_stream stream);

/* ------------------------------------------------------------------------
 * Digit decompositions of Goldilocks vectors (device pointers).
 * ---------------------------------------------------------------------- */

/* decomp_b (lattice-folding/src/neo.rs:253-266): for each of the `count`
 * residues z[e] (reduced to canonical first, as to_canonical_u64 does), its
 * unsigned base-2^b_bits digits; out = [rows][count] bytes with
 * rows = ceil(64 / b_bits), row r holding digit r of every element.
 * b_bits in 1..8. */
LC_API int lc_decomp_b(const uint64_t *z, size_t count, uint32_t b_bits, uint8_t *out, lc_stream stream);

/* GadgetDecomposition::decompose (lattice-core/src/decomposition.rs:48-70) of
 * each u64 z[e] in base 2^log_base (1..15) into num_digits balanced digits
 * (a digit t > base/2 becomes t - base and borrows); out = [num_digits][count]
 * int16.  The reference returns ValueTooLarge for a value whose remainder is
 * not zero after num_digits digits: here the digits are still written and the
 * number of such values is added to *too_large (a device counter; may be
 * NULL). */
LC_API int lc_gadget_decompose(const uint64_t *z, size_t count, uint32_t log_base, uint32_t num_digits,
                               int16_t *out, uint32_t *too_large, lc_stream stream);

/* ------------------------------------------------------------------------
 * CRT residues and the folding-step pipeline.
 * ---------------------------------------------------------------------- */

/* out[i][e] = z[e] mod q_i for every u32 modulus q_i of `plan`
 * (Modulus32::reduce_u64, lattice-ring/src/modulus.rs:65, per prime): maps
 * 64-bit coefficients into the plan's CRT set ([num_moduli][count] u32, the
 * layout lc_ntt_forward takes). */
LC_API int lc_crt_residues(const lc_ntt_plan *plan, const uint64_t *z, size_t count, uint32_t *out,
                           lc_stream stream);

/* One folding step over d = 64 Goldilocks as a single graph launch.  No
 * single counterpart in the reference: it chains decomp_b(z, 8)
 * (lattice-folding/src/neo.rs:253-266), the commitment of the 8 digit rows
 * with `key` (AjtaiPublicKey::commit, ajtai.rs:118-153, as a batch of 8
 * witnesses through lc_ajtai_commit_u8), and the forward NTT of z over the
 * CRT set of `crt_plan` (lc_crt_residues + lc_ntt_forward).  `key`: Goldilocks,
 * log_n 6, m ring elements; `crt_plan`: u32 moduli, log_n 6.  The pipeline owns
 * its buffers (lc_fold_pipeline_buffers): z = [m][64] residues (written by the
 * caller), digits = [8][m][64] bytes, commits = [8][k][64] residues,
 * crt_ntt = [num_moduli][m][64] u32.  With use_graph != 0 the first run is
 * eager (it sizes the key's scratch) and the second captures the four stages
 * into a CUDA graph that every later run replays; if another commit on the
 * same key reallocates that scratch, the next run captures again.  Runs of
 * one pipeline, and other commits on its key, must not overlap on the GPU. */
typedef struct lc_fold_pipeline lc_fold_pipeline;
LC_API int lc_fold_pipeline_create(lc_ajtai_key *key, const lc_ntt_plan *crt_plan, int use_graph,
                                   lc_fold_pipeline **out);
LC_API int lc_fold_pipeline_buffers(lc_fold_pipeline *pipe, uint64_t **z, uint8_t **digits,
                                    uint64_t **commits, uint32_t **crt_ntt);
LC_API int lc_fold_pipeline_run(lc_fold_pipeline *pipe, lc_stream stream);
/* Wait for `stream` and report device-side errors of the pipeline's kernels. */
LC_API int lc_fold_pipeline_check(lc_fold_pipeline *pipe, lc_stream stream);
LC_API void lc_fold_pipeline_destroy(lc_fold_pipeline *pipe);

/* ------------------------------------------------------------------------
 * Batches of uneven commitment jobs in persistent launches.
 * No single counterpart in the reference (which commits one witness per
 * AjtaiPublicKey::commit call, ajtai.rs:118-153): every job's result equals
 * that call on its key's first `kappa` rows and first `n` columns.
 * ---------------------------------------------------------------------- */

/* A class: one Goldilocks key, or 1..4 u32 keys (one per prime of a CRT set),
 * all with the same log_n (6, 7 or 8).  A job of the class is committed under
 * every key of the class. */
typedef struct lc_commit_class {
  const lc_ajtai_key *keys[4];
  uint32_t num_keys;
} lc_commit_class;

/* A job: int8 digit witness w = [n][d] (device), committed with the first
 * kappa rows and n columns of its class's keys; out (device) = [num_keys][kappa][d]
 * residues (uint64 for Goldilocks, uint32 per prime). */
typedef struct lc_commit_job {
  uint32_t cls;
  uint32_t kappa;
  uint32_t n;
  const int8_t *w;
  void *out;
} lc_commit_job;

typedef struct lc_batch lc_batch;

/* Plan a batch: jobs of one key are grouped into lanes of at most 128 jobs
 * sorted by n, so the key's cached NTT(A) is read once per block of jobs of a
 * lane, not once per job.  Three launches run it: the witness NTTs
 * (persistent, fed by a device work counter), the products (see
 * lc_batch_set_products), and per job the sum over chunks plus the inverse
 * NTT.
 * flags: LC_BATCH_GRAPH captures the three launches into a CUDA graph on
 * the second run and replays it afterwards.  The keys must outlive the batch;
 * runs of one batch must not overlap on the GPU. */
#define LC_BATCH_GRAPH 1u
LC_API int lc_batch_create(const lc_commit_class *classes, uint32_t num_classes, const lc_commit_job *jobs,
                           uint32_t num_jobs, uint32_t flags, lc_batch **out);
/* Tuning: ring elements per product work item (chunk, a power of two in
 * 1024..16384), CTAs per SM of the persistent launches (1..4) and work items
 * claimed per counter increment (1..16).  Results do not depend on them. */
LC_API int lc_batch_set_config(lc_batch *batch, uint32_t chunk, uint32_t ctas_per_sm, uint32_t claim);
LC_API int lc_batch_get_config(const lc_batch *batch, uint32_t *chunk, uint32_t *ctas_per_sm, uint32_t *claim);
/* How the products run (the same per-slot sums as the keys' commits,
 * ajtai.rs:139-148): LC_PRODUCTS_TENSOR (the default wherever it can run) as
 * exact byte-limb GEMMs on the INT8 tensor cores -- one work item per lane,
 * NTT slot, block of 32 jobs and chunk of at most 32768 ring elements, the
 * staircase of transformed witnesses gathered with its inactive jobs as
 * zeros -- or LC_PRODUCTS_INT64 with 160-bit / 64-bit multiply-accumulates on
 * the CUDA cores (one item per slot, chunk and 16-job block; `chunk` of
 * lc_batch_set_config applies to this form only).  Identical results.
 * In the tensor mode the witness NTTs run on the tensor cores too, for
 * Goldilocks lanes and lanes of a 30-bit modulus q = 2^30 - c, c <= 2^20
 * (the 4-prime CRT set): per tile of 128 witness polynomials the product
 * with the fixed matrix V[t][k] = psi^((2t+1)k) split into byte limbs (the
 * values ntt.rs:118-146 computes); lanes of other moduli keep the CUDA-core
 * transforms.
 * lc_batch_set_products returns LC_ERR_UNSUPPORTED when the tensor form
 * cannot run (no tensor-map encoder in the driver); lc_batch_get_products
 * returns the mode (-1 for a null batch). */
LC_API int lc_batch_set_products(lc_batch *batch, int mode);
LC_API int lc_batch_get_products(const lc_batch *batch);
/* Work items of the launches (items_ntt counts the tensor-core witness
 * tiles too in the tensor mode), and the lanes of the plan. */
LC_API int lc_batch_info(const lc_batch *batch, uint64_t *items_ntt, uint64_t *items_product,
                         uint64_t *items_finish, uint32_t *lanes);
LC_API int lc_batch_run(lc_batch *batch, lc_stream stream);
/* Wait for `stream` and report device-side errors of the batch's kernels. */
LC_API int lc_batch_check(lc_batch *batch, lc_stream stream);
LC_API void lc_batch_destroy(lc_batch *batch);

/* pack_field_elements (lattice-ring/src/packing.rs:30-52): each of the
 * `count` Goldilocks values (device, reduced to canonical first) becomes the
 * three 22-bit limbs raw & (2^22-1), (raw >> 22) & (2^22-1), raw >> 44 in
 * consecutive coefficients of out = [out_elems][n] u32 (device), zero beyond;
 * out_elems must be at least max(1, ceil(3*count/n)) (else
 * LC_ERR_DIMENSION_MISMATCH), so passing the key's m gives pad_to_m
 * (ajtai.rs:245-257) and the result is the witness AkitaPcs::commit
 * (lattice-akita/src/pcs.rs:66-76) commits with lc_ajtai_commit. */
LC_API int lc_pack_field_elements(const uint64_t *values, size_t count, uint32_t log_n, size_t out_elems,
                                  uint32_t *out, lc_stream stream);

/* ---------------------------------------------------------------------------
 * Modulus50 quadratic-slot ring (lattice-ring/src/modulus50.rs).
 *
 * A plan is QuadSlotTables::new(Modulus50::new(q, two_adicity, generator),
 * log_n) (modulus50.rs:250-301): q an odd prime in (2^49, 2^50) -- the
 * "~2^50" class, e.g. Q_50 = 2^50 - 2687 with generator 3 (:44-51); other q give
 * LC_ERR_INVALID_ARGUMENT -- and log_n in [1, 7].  Errors in the reference's
 * order: LC_ERR_LOG_N_OUT_OF_RANGE, LC_ERR_ADICITY_TOO_SMALL (two_adicity < 7),
 * LC_ERR_GENERATOR_INVALID (zeta = g^((q-1)/128) not of order 128).
 * Polynomials are contiguous [count][n] canonical u64 residues on the device;
 * out may alias an input. */
typedef struct lc_quad50_plan lc_quad50_plan;
LC_API int lc_quad50_plan_create(uint64_t q, uint32_t two_adicity, uint64_t generator, uint32_t log_n,
                                 lc_quad50_plan **out);
LC_API void lc_quad50_plan_destroy(lc_quad50_plan *plan);
/* zeta (QuadSlotTables::zeta) and, if non-null, the n/2 leaf constants
 * gamma_p (RingConfig50::slot_constants, :446-448) into host memory. */
LC_API int lc_quad50_plan_info(const lc_quad50_plan *plan, uint64_t *zeta, uint64_t *slot_constants);
/* QuadSlotTables::forward (:313-334) / inverse (:338-364) of count polynomials */
LC_API int lc_quad50_forward(const lc_quad50_plan *plan, const uint64_t *in, uint64_t *out, size_t count,
                             lc_stream stream);
LC_API int lc_quad50_inverse(const lc_quad50_plan *plan, const uint64_t *in, uint64_t *out, size_t count,
                             lc_stream stream);
/* QuadSlotTables::slotwise_mul (:368-392) of slot-form operands */
LC_API int lc_quad50_slotwise_mul(const lc_quad50_plan *plan, const uint64_t *a, const uint64_t *b,
                                  uint64_t *out, size_t count, lc_stream stream);
/* QuadSlotTables::mul / RingConfig50::mul (:395-411, :450-453): count
 * products in Z_q[X]/(X^n + 1), both forwards, the slot products and the
 * inverse in one launch. */
LC_API int lc_quad50_mul(const lc_quad50_plan *plan, const uint64_t *a, const uint64_t *b, uint64_t *out,
                         size_t count, lc_stream stream);
/* The same product over host buffers (synchronous; copies overlap kernels). */
LC_API int lc_quad50_mul_host(lc_quad50_plan *plan, const uint64_t *a, const uint64_t *b, uint64_t *out,
                              size_t count);

/* ---------------------------------------------------------------------------
 * labinius Ajtai commitment over R_648 = Z_q[X]/(X^648 - X^324 + 1)
 * (crates/lattice-labinius).  Limb primes: 3889, 9721, 17497, 19441 (fully
 * splitting, params.rs:20-30) and 2917, 4861, 12637 (quadratic slots,
 * params.rs:306-315); the first listed is the base limb.
 *
 * A key holds A: per limb nr = len_f162 / 4 rows of 648 transform-domain
 * residues (CommitmentKey::a, key.rs:45-57), centered int16 on the host
 * side.  len_f162 must be a positive multiple of 4 (at most 2^18) and no
 * prime may repeat (key.rs:96-106), else LC_ERR_INVALID_ARGUMENT. */
typedef struct lc_lb_key lc_lb_key;
/* CommitmentKey::random (key.rs:94-137), bit-identical rows */
LC_API int lc_lb_key_random(size_t len_f162, uint64_t seed, const uint16_t *primes, uint32_t limbs,
                            lc_lb_key **out);
/* a key from explicit centered rows a = [limbs][nr][648] (host) */
LC_API int lc_lb_key_create(size_t len_f162, const uint16_t *primes, uint32_t limbs, const int16_t *a,
                            lc_lb_key **out);
LC_API void lc_lb_key_destroy(lc_lb_key *key);
/* len_f162, limbs, primes[limbs] and the centered rows [limbs][nr][648] (host), each if non-null */
LC_API int lc_lb_key_info(const lc_lb_key *key, size_t *len_f162, uint32_t *limbs, uint16_t *primes, int16_t *a);
/* ntt_of (ring.rs:322-333) with limb `limb`'s prime: count elements [count][648] u32 (device) */
LC_API int lc_lb_ntt(const lc_lb_key *key, uint32_t limb, const uint32_t *in, uint32_t *out, size_t count,
                     lc_stream stream);
/* CommitmentKey::commit_with (key.rs:237-474): witness = r * len_f162 F162
 * elements as [..][3] u64 (device), r a power of two in [2, 2^15].  Outputs
 * (device): raw = [limbs][r][648] u32 in [0, q) (AuxData::raw), matrix =
 * [4][r][limbs][162] centered int16 (CommitmentMatrix::value[row][column]
 * [modulus]), batches = [r * nr][648] u32, the base limb's transform of every
 * lifted ring element (AuxData::batches), or null to skip it. */
LC_API int lc_lb_commit(lc_lb_key *key, const uint64_t *witness, uint32_t r, uint32_t *raw, int16_t *matrix,
                        uint32_t *batches, lc_stream stream);
/* the same over host buffers, synchronous */
LC_API int lc_lb_commit_host(lc_lb_key *key, const uint64_t *witness, uint32_t r, uint32_t *raw, int16_t *matrix,
                             uint32_t *batches);
/* random_elems (binfield.rs:177-189): n F162 elements [n][3] u64 into host memory */
LC_API int lc_lb_random_elems(size_t n, uint64_t seed, uint64_t *out);

/* Benchmark/test utility, no counterpart in the reference: fill `count`
 * elements of `out` (device) with the seeded counter-based synthetic stream
 * x_i = H(seed, stream, offset + i): kind 0 raw u64, 1 u32 residues mod q
 * (rejection below 2^32 - 2^32 mod q, as ring.rs:123), 2 Goldilocks residues,
 * 3 int8 digits.  Bit-identical to lzx_b200/synth.py. */
LC_API int lc_synth_fill(int kind, uint64_t seed, uint64_t stream, uint32_t q, void *out,
                         size_t count, size_t offset, lc_stream stream_handle);

#ifdef __cplusplus
}
#endif

#endif /* LATTICE_CUDA_H */
