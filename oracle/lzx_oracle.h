/*
 * lzx_oracle.h -- CPU restatement of the LZX commitment hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the correctness oracle and the
 * timed CPU baseline.  Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline / reference arm may load it.  The product (lzx_b200 and the
 * lattice_cuda C ABI) never links or calls it.
 *
 * Every function restates a function of idrees2516/lzx (Rust) and cites the
 * file:line it follows.  The reference cannot be compiled in this image (it is
 * Rust; there is no cargo/rustc), so the restatement is pinned instead by:
 *   - the reference's own numeric known-answer tests (Goldilocks add/sub/mul
 *     KATs, crates/lattice-core/src/field.rs:267-313; FIPS-202 digests,
 *     crates/lattice-core/src/keccak.rs:415-448), see tests/golden/;
 *   - the reference's identity tests re-run against this code (Barrett vs %,
 *     NTT round trip, NTT product == schoolbook, fast == generic, cached-NTT
 *     commit == naive commit, linearity, zero-skip);
 *   - direct evaluation out[j] = a(psi^(2j+1)) of the forward transform, which
 *     fixes the reference's natural output order independently of the loop.
 * No NTT or commitment digests are committed in the reference (its KAT
 * manifest is generated at run time), so those digests are reproduced from
 * the restated code, not checked against stored reference output.
 */
#ifndef LZX_ORACLE_H
#define LZX_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------- Modulus32 (crates/lattice-ring/src/modulus.rs) ---------- */

typedef struct {
  uint32_t q;
  uint32_t two_adicity;
  uint32_t generator;
  uint64_t barrett_recip; /* floor(2^64 / q), modulus.rs:15-17 */
} orc_mod32;

orc_mod32 orc_mod32_new(uint32_t q, uint32_t two_adicity, uint32_t generator);
uint32_t orc_mod32_reduce_u64(const orc_mod32 *m, uint64_t x);
uint32_t orc_mod32_reduce_i64(const orc_mod32 *m, int64_t x);
uint32_t orc_mod32_mul(const orc_mod32 *m, uint32_t a, uint32_t b);
uint32_t orc_mod32_add(const orc_mod32 *m, uint32_t a, uint32_t b);
uint32_t orc_mod32_sub(const orc_mod32 *m, uint32_t a, uint32_t b);
uint32_t orc_mod32_neg(const orc_mod32 *m, uint32_t a);
uint32_t orc_mod32_pow(const orc_mod32 *m, uint32_t base, uint64_t exp);
/* returns 0 when a == 0 (the reference returns None) */
uint32_t orc_mod32_inv(const orc_mod32 *m, uint32_t a);
/* returns 0 when k > two_adicity (the reference returns None) */
uint32_t orc_mod32_root_of_unity(const orc_mod32 *m, uint32_t k);

/* ---------------- Goldilocks (crates/lattice-core/src/field.rs) ----------- */

#define ORC_GL_P 0xFFFFFFFF00000001ull

uint64_t orc_gl_from_u64(uint64_t x);
uint64_t orc_gl_from_u128(uint64_t hi, uint64_t lo);
uint64_t orc_gl_add(uint64_t a, uint64_t b);
uint64_t orc_gl_sub(uint64_t a, uint64_t b);
uint64_t orc_gl_neg(uint64_t a);
uint64_t orc_gl_mul(uint64_t a, uint64_t b);
uint64_t orc_gl_pow(uint64_t a, uint64_t e);
uint64_t orc_gl_inv(uint64_t a);

/* ---------------- NTT tables (crates/lattice-ring/src/ntt.rs) ------------- */

/* status codes shared with the product ABI (NttError, ntt.rs:38-42) */
#define ORC_OK 0
#define ORC_ERR_LENGTH_MISMATCH 1
#define ORC_ERR_ADICITY_TOO_SMALL 2

typedef struct {
  orc_mod32 modulus;
  uint32_t log_n;
  uint32_t n_inv;
  uint32_t *pow_psi;       /* [n]   */
  uint32_t *pow_psi_inv;   /* [n]   */
  uint32_t *pow_omega;     /* [max(n/2,1)] */
  uint32_t *pow_omega_inv; /* [max(n/2,1)] */
  uint32_t *level_tw;      /* concatenated per-level tables, level j has 2^j entries */
  uint32_t *level_tw_inv;
} orc_ntt32;

int orc_ntt32_new(orc_mod32 m, uint32_t log_n, orc_ntt32 *out);
void orc_ntt32_free(orc_ntt32 *t);
int orc_ntt32_forward(const orc_ntt32 *t, uint32_t *a, size_t len);
int orc_ntt32_forward_fast(const orc_ntt32 *t, uint32_t *a, size_t len);
int orc_ntt32_inverse(const orc_ntt32 *t, uint32_t *a, size_t len);
int orc_ntt32_inverse_fast(const orc_ntt32 *t, uint32_t *a, size_t len);
int orc_ntt32_forward_partial(const orc_ntt32 *t, uint32_t *a, size_t len, uint32_t levels);
int orc_ntt32_complete_partial(const orc_ntt32 *t, uint32_t *a, size_t len, uint32_t already);

/* Batched helpers (CPU baseline): count polynomials of n coefficients,
 * contiguous; nthreads <= 0 means "all cores" (OpenMP). */
int orc_ntt32_forward_batch(const orc_ntt32 *t, uint32_t *a, size_t count, int nthreads);
int orc_ntt32_inverse_batch(const orc_ntt32 *t, uint32_t *a, size_t count, int nthreads);

/* Goldilocks instantiation of the same ntt.rs algorithm, psi from generator 7
 * (field.rs:195-200).  Output order identical to ntt.rs (natural). */
typedef struct {
  uint32_t log_n;
  uint64_t n_inv;
  uint64_t *pow_psi, *pow_psi_inv;
  uint64_t *level_tw, *level_tw_inv;
} orc_nttgl;

int orc_nttgl_new(uint32_t log_n, orc_nttgl *out);
void orc_nttgl_free(orc_nttgl *t);
int orc_nttgl_forward_fast(const orc_nttgl *t, uint64_t *a, size_t len);
int orc_nttgl_inverse_fast(const orc_nttgl *t, uint64_t *a, size_t len);
int orc_nttgl_forward_batch(const orc_nttgl *t, uint64_t *a, size_t count, int nthreads);
int orc_nttgl_inverse_batch(const orc_nttgl *t, uint64_t *a, size_t count, int nthreads);

/* ---------------- Ajtai commit (crates/lattice-commitment/src/ajtai.rs) --- */

/* Cached-NTT commit, ajtai.rs:118-153.  matrix_ntt: k*m*n row-major (entry
 * (i,j) at (i*m+j)*n), s: m*n coefficients, out: k*n. Zero s_j skipped. */
int orc_ajtai32_commit(const orc_ntt32 *t, const uint32_t *matrix_ntt, size_t k, size_t m,
                       const uint32_t *s, uint32_t *out);
/* Per-product naive path, ajtai.rs:158-180 (matrix in coefficient form). */
int orc_ajtai32_commit_naive(const orc_ntt32 *t, const uint32_t *matrix, size_t k, size_t m,
                             const uint32_t *s, uint32_t *out);
/* Ring multiply via NTT, ring.rs:309-340. */
int orc_ring32_mul(const orc_ntt32 *t, const uint32_t *a, const uint32_t *b, uint32_t *out);

/* Goldilocks instantiation of the cached-NTT commit for a batch of witnesses.
 * matrix_ntt: kappa*m*d (entry (i,j) at (i*m+j)*d), w: batch*m*d residues,
 * out: batch*kappa*d.  nthreads<=0: all cores.  simd!=0: use the AVX-512
 * Goldilocks MAC restated from field_simd.rs where the CPU has avx512f. */
int orc_ajtaigl_commit_batch(const orc_nttgl *t, const uint64_t *matrix_ntt, size_t kappa,
                             size_t m, const uint64_t *w, size_t batch, uint64_t *out,
                             int nthreads, int simd);
/* same with int8 witness digits (w_i8[b][j][c] in [-128,127] mapped into F_p) */
int orc_ajtaigl_commit_batch_i8(const orc_nttgl *t, const uint64_t *matrix_ntt, size_t kappa,
                                size_t m, const int8_t *w, size_t batch, uint64_t *out,
                                int nthreads, int simd);
int orc_avx512_available(void);

/* ---------------- Neo ring / coefficient-domain commit (neo.rs) ----------- */

/* NeoRing::mul, crates/lattice-folding/src/neo.rs:138-158 */
void orc_neo_mul(size_t d, const uint64_t *a, const uint64_t *b, uint64_t *out);
/* NeoAjtaiKey::commit_naive, neo.rs:419-441.  matrix: kappa*m*d, cols: ncols*d */
int orc_neo_commit_naive(size_t d, size_t kappa, size_t m, const uint64_t *matrix,
                         const uint64_t *cols, size_t ncols, uint64_t *out);
/* NeoAjtaiKey::commit_pay_per_bit, neo.rs:374-415; column_adds counted */
int orc_neo_commit_pay_per_bit(size_t d, size_t kappa, size_t m, const uint64_t *matrix,
                               const uint64_t *cols, size_t ncols, uint64_t *out,
                               uint64_t *column_adds);
/* decomp_b, neo.rs:253-266: rows = ceil(64/b_bits); out[row*len + j] */
void orc_decomp_b(const uint64_t *z, size_t len, uint32_t b_bits, uint64_t *out);
/* pack_field_elements, lattice-ring/src/packing.rs:30-52: out = [elems][n] residues mod q */
size_t orc_pack_field_elements(uint32_t q, uint32_t log_n, const uint64_t *values, size_t count, uint32_t *out);
/* GadgetDecomposition::decompose, lattice-core/src/decomposition.rs:48-70;
 * returns 0 ok, 1 ValueTooLarge */
int orc_gadget_decompose(uint64_t base, size_t num_digits, uint64_t x, int64_t *out);

/* ---------------- Modulus50 + quadratic-slot incomplete NTT --------------
 * (crates/lattice-ring/src/modulus50.rs) */

#define ORC_ERR_LOG_N_OUT_OF_RANGE 13 /* Mod50Error::LogNOutOfRange (modulus50.rs:418) */
#define ORC_ERR_GENERATOR_INVALID 14  /* Mod50Error::GeneratorInvalid (modulus50.rs:420) */

typedef struct {
  uint64_t q;
  uint64_t recip; /* floor((2^64-1) / q), modulus50.rs:69 */
  uint32_t two_adicity;
  uint64_t generator;
} orc_mod50;

orc_mod50 orc_mod50_new(uint64_t q, uint32_t two_adicity, uint64_t generator);
uint64_t orc_mod50_reduce_u128(const orc_mod50 *m, uint64_t hi, uint64_t lo);
uint64_t orc_mod50_mul(const orc_mod50 *m, uint64_t a, uint64_t b);
uint64_t orc_mod50_add(const orc_mod50 *m, uint64_t a, uint64_t b);
uint64_t orc_mod50_sub(const orc_mod50 *m, uint64_t a, uint64_t b);
uint64_t orc_mod50_pow(const orc_mod50 *m, uint64_t base, uint64_t exp);

/* QuadSlotTables (modulus50.rs:206-301): level d (blocks 2^d) at offset 2^d - 1 */
typedef struct {
  orc_mod50 modulus;
  uint32_t log_n;
  uint64_t zeta;
  uint64_t *level_tw;     /* [n/2 - 1] */
  uint64_t *level_tw_inv; /* [n/2 - 1] */
  uint64_t *leaf_gamma;   /* [n/2] */
} orc_quad50;

/* ORC_ERR_LOG_N_OUT_OF_RANGE, ORC_ERR_ADICITY_TOO_SMALL, ORC_ERR_GENERATOR_INVALID */
int orc_quad50_new(orc_mod50 m, uint32_t log_n, orc_quad50 *out);
void orc_quad50_free(orc_quad50 *t);
int orc_quad50_forward(const orc_quad50 *t, uint64_t *a, size_t len);
int orc_quad50_inverse(const orc_quad50 *t, uint64_t *a, size_t len);
int orc_quad50_slotwise_mul(const orc_quad50 *t, const uint64_t *a, const uint64_t *b, uint64_t *out,
                            size_t len);
int orc_quad50_mul(const orc_quad50 *t, const uint64_t *a, const uint64_t *b, uint64_t *out, size_t len);
/* count independent ring products (CPU baseline); nthreads <= 0: all cores */
int orc_quad50_mul_batch(const orc_quad50 *t, const uint64_t *a, const uint64_t *b, uint64_t *out,
                         size_t count, int nthreads);

/* ---------------- labinius commitment over R_648 (labinius.c) --------------
 * (crates/lattice-labinius: params.rs, scalar.rs, ring.rs, binfield.rs, key.rs) */

int orc_lb_quadratic(uint32_t q);
uint32_t orc_lb_psi(uint32_t q); /* psi (order 1944) or psi' (order 972) */
/* SLOT_EXP[648], QUAD_SLOT_EXP[324], POW3_SLOT_EXP[162], SLOT_648[4][162], QUAD_CLASS_SLOT[2][162] */
void orc_lb_tables(uint16_t *slot_exp, uint16_t *quad_slot_exp, uint16_t *pow3_slot_exp, uint16_t *slot_648,
                   uint16_t *quad_class_slot);
void orc_lb_ntt(uint32_t q, const uint32_t *a, uint32_t *out);
uint32_t orc_lb_eval_at(uint32_t q, const uint32_t *a, uint32_t u);
void orc_lb_eval_quad_at(uint32_t q, const uint32_t *a, uint32_t u, uint32_t out[2]);
void orc_lb_mul_mod_phi(uint32_t q, const uint32_t *a, const uint32_t *b, uint32_t *out);
void orc_lb_mul_quad_slots(uint32_t q, const uint32_t *a, const uint32_t *b, uint32_t *out);
void orc_lb_components(uint32_t q, const uint32_t *y, int16_t *out);
void orc_lb_r162_from_coeffs(uint32_t q, const int64_t *c, int16_t *out);
void orc_lb_random_elems(size_t n, uint64_t seed, uint64_t *out);
void orc_lb_lift(const uint64_t *elems, size_t r, uint32_t *out);
void orc_lb_key_random(size_t len_f162, uint64_t seed, const uint32_t *primes, size_t limbs, int16_t *a);
int orc_lb_commit(const int16_t *a, const uint32_t *primes, size_t limbs, size_t len_f162, const uint64_t *witness,
                  size_t r, uint32_t *raw, int16_t *matrix, uint32_t *batches, int nthreads);

/* ---------------- Keccak / transcript (keccak.rs, transcript.rs) ---------- */

void orc_keccak_f1600(uint64_t st[25]);
void orc_sha3_256(const uint8_t *in, size_t len, uint8_t out[32]);
void orc_shake256(const uint8_t *in, size_t len, uint8_t *out, size_t out_len);
/* Transcript::xof, transcript.rs:229-237 */
void orc_xof(const uint8_t *domain, size_t dlen, const uint8_t *msg, size_t mlen, uint8_t *out,
             size_t out_len);
/* Transcript::hash_domain, transcript.rs:218-226 */
void orc_hash_domain(const uint8_t *domain, size_t dlen, const uint8_t *msg, size_t mlen,
                     uint8_t out[32]);

/* RingConfig::uniform_from_seed, ring.rs:102-180 */
void orc_uniform_from_seed(const orc_mod32 *m, uint32_t log_n, const uint8_t *domain, size_t dlen,
                           const uint8_t *seed, size_t slen, uint64_t index, uint32_t *out);
/* RingConfig::random, ring.rs:83-98 */
void orc_ring_random(const orc_mod32 *m, uint32_t log_n, const uint8_t *seed, size_t slen,
                     uint32_t *out);
/* AjtaiPublicKey::from_seed, ajtai.rs:87-103: matrix (coeffs) and cached NTT */
int orc_ajtai32_from_seed(const orc_ntt32 *t, size_t k, size_t m, const uint8_t seed[32],
                          uint32_t *matrix, uint32_t *matrix_ntt);
/* sample_small_secret, ajtai.rs:307-348 */
void orc_sample_small_secret(const orc_mod32 *mod, uint32_t log_n, size_t m, uint32_t bound,
                             const uint8_t *seed, size_t slen, uint32_t *out);

/* ---------------- Synthetic inputs (counter-based, prefix-consistent) ------ */

/* x = H(seed, stream, index): SplitMix64 finaliser over a counter. */
uint64_t orc_synth_u64(uint64_t seed, uint64_t stream, uint64_t index);
/* uniform residues mod q (rejection on the counter's retry lane) */
void orc_synth_mod32(uint64_t seed, uint64_t stream, uint32_t q, uint32_t *out, size_t count,
                     size_t offset);
void orc_synth_gl(uint64_t seed, uint64_t stream, uint64_t *out, size_t count, size_t offset);
/* int8 digits: low byte of H reinterpreted as signed */
void orc_synth_i8(uint64_t seed, uint64_t stream, int8_t *out, size_t count, size_t offset);

#ifdef __cplusplus
}
#endif

#endif
