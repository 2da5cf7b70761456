/*
 * labinius.c -- CPU restatement of the labinius Ajtai commitment
 * (crates/lattice-labinius) for R_648 = Z_q[X]/(X^648 - X^324 + 1).
 *
 * TEST INFRASTRUCTURE ONLY (see lzx_oracle.h): the checker and CPU baseline
 * of the lattice_cuda labinius entry points, never linked by the product.
 *
 * Restated from the scalar reference path, which the reference itself names
 * its specification:
 *   params.rs:20-392  the two NTT trees (split: radix 2,2,2,3,3,3,3 with
 *                     psi of order 1944; quadratic: 2,2,3,3,3,3 with psi' of
 *                     order 972 ending in 324 leaves X^2 - psi'^u)
 *   scalar.rs:11-246  schoolbook product, ntt, eval_at, ntt_quad,
 *                     eval_quad_at, mul_quad_slots
 *   ring.rs:68-307    slot order of R_162 and the 648 -> 4 x 162 decomposition
 *   binfield.rs:118-189  lift of an F162 stream, xorshift64* Rng, random F162
 *   key.rs:94-137, 382-474  CommitmentKey::random and commit_scalar
 * All arithmetic is exact (values below 2^15, products below 2^30), so
 * outputs are determined by the mathematics and the table orders above.
 */
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "lzx_oracle.h"

#define LB_N 648
#define LB_N162 162
#define LB_COND 1944
#define LB_COND_Q 972
#define LB_QSLOTS 324

static const int RADIX[7] = {2, 2, 2, 3, 3, 3, 3};
static const int SUBRINGS[8] = {1, 2, 4, 8, 24, 72, 216, 648};
static const int DEGREE[8] = {648, 324, 162, 81, 27, 9, 3, 1};
static const int RADIX_Q[6] = {2, 2, 3, 3, 3, 3};
static const int SUBRINGS_Q[7] = {1, 2, 4, 12, 36, 108, 324};
static const int DEGREE_Q[7] = {648, 324, 162, 54, 18, 6, 2};

static uint64_t lb_pow(uint64_t b, uint64_t e, uint64_t q) {
  uint64_t r = 1;
  b %= q;
  while (e) {
    if (e & 1) r = r * b % q;
    b = b * b % q;
    e >>= 1;
  }
  return r;
}

static uint64_t lb_inv(uint64_t a, uint64_t q) { return lb_pow(a, q - 2, q); }

/* params.rs:61-70 and :262-270: smallest element of order exactly 1944 / 972 */
static uint64_t find_psi(uint64_t q) {
  for (uint64_t x = 2;; x++)
    if (lb_pow(x, 1944, q) == 1 && lb_pow(x, 972, q) != 1 && lb_pow(x, 648, q) != 1) return x;
}

static uint64_t find_psi972(uint64_t q) {
  for (uint64_t x = 2;; x++)
    if (lb_pow(x, 972, q) == 1 && lb_pow(x, 486, q) != 1 && lb_pow(x, 324, q) != 1) return x;
}

/* params.rs:73-85 */
static uint32_t subring_exp(int level, int k) {
  if (level == 1) return k == 0 ? 324 : 1620;
  uint32_t p = (uint32_t)RADIX[level - 1];
  return (subring_exp(level - 1, k / (int)p) + LB_COND * ((uint32_t)k % p)) / p;
}

static uint32_t twiddle_exp(int level, int k) { return subring_exp(level, k) / (uint32_t)RADIX[level]; }

/* params.rs:273-285 */
static uint32_t subring_exp_quad(int level, int k) {
  if (level == 1) return k == 0 ? 162 : 810;
  uint32_t p = (uint32_t)RADIX_Q[level - 1];
  return (subring_exp_quad(level - 1, k / (int)p) + LB_COND_Q * ((uint32_t)k % p)) / p;
}

static uint32_t twiddle_exp_quad(int level, int k) {
  return subring_exp_quad(level, k) / (uint32_t)RADIX_Q[level];
}

/* params.rs:311-315 */
int orc_lb_quadratic(uint32_t q) { return (q - 1) % LB_COND_Q == 0 && (q - 1) % LB_COND != 0; }

/* ---- slot-order tables (params.rs:88-97, ring.rs:68-99, params.rs:297-355) ---- */

static uint16_t SLOT_EXP[LB_N];
static uint16_t QUAD_SLOT_EXP[LB_QSLOTS];
static uint16_t POW3_SLOT_EXP[LB_N162];
static uint16_t SLOT_648[4][LB_N162];
static uint16_t QUAD_CLASS_SLOT[2][LB_N162];
static int tables_ready = 0;

static void build_tables(void) {
  if (tables_ready) return;
  for (int j = 0; j < LB_N; j++) SLOT_EXP[j] = (uint16_t)subring_exp(7, j);
  for (int j = 0; j < LB_QSLOTS; j++) QUAD_SLOT_EXP[j] = (uint16_t)subring_exp_quad(6, j);
  int pos[486];
  for (int v = 0; v < 486; v++) pos[v] = -1;
  int n = 0;
  for (int j = 0; j < LB_N; j++) {
    int u = SLOT_EXP[j], v = u % 486, t = (u - v) / 486;
    if (pos[v] < 0) {
      pos[v] = n;
      POW3_SLOT_EXP[n] = (uint16_t)v;
      n++;
    }
    SLOT_648[t][pos[v]] = (uint16_t)j;
  }
  for (int s = 0; s < LB_N162; s++) {
    int v = POW3_SLOT_EXP[s];
    for (int j = 0; j < LB_QSLOTS; j++) {
      if (QUAD_SLOT_EXP[j] == v) QUAD_CLASS_SLOT[0][s] = (uint16_t)j;
      if (QUAD_SLOT_EXP[j] == v + 486) QUAD_CLASS_SLOT[1][s] = (uint16_t)j;
    }
  }
  tables_ready = 1;
}

void orc_lb_tables(uint16_t *slot_exp, uint16_t *quad_slot_exp, uint16_t *pow3_slot_exp, uint16_t *slot_648,
                   uint16_t *quad_class_slot) {
  build_tables();
  if (slot_exp) memcpy(slot_exp, SLOT_EXP, sizeof(SLOT_EXP));
  if (quad_slot_exp) memcpy(quad_slot_exp, QUAD_SLOT_EXP, sizeof(QUAD_SLOT_EXP));
  if (pow3_slot_exp) memcpy(pow3_slot_exp, POW3_SLOT_EXP, sizeof(POW3_SLOT_EXP));
  if (slot_648) memcpy(slot_648, SLOT_648, sizeof(SLOT_648));
  if (quad_class_slot) memcpy(quad_class_slot, QUAD_CLASS_SLOT, sizeof(QUAD_CLASS_SLOT));
}

uint32_t orc_lb_psi(uint32_t q) {
  return (uint32_t)(orc_lb_quadratic(q) ? find_psi972(q) : find_psi(q));
}

/* ---- transforms (scalar.rs) ---- */

/* ntt, scalar.rs:37-86: out[j] = a(psi^SLOT_EXP[j]) */
static void ntt_split(uint64_t q, const uint32_t *a, uint32_t *out) {
  uint64_t psi = find_psi(q), w = lb_pow(psi, 648, q), w2 = w * w % q, z6 = lb_pow(psi, 324, q);
  uint64_t v[LB_N];
  for (int i = 0; i < LB_N; i++) v[i] = a[i] % q;
  for (int i = 0; i < 324; i++) {
    uint64_t a0 = v[i], a1 = v[i + 324], t = a1 * z6 % q;
    v[i] = (a0 + t) % q;
    v[i + 324] = (a0 + a1 + q - t) % q;
  }
  for (int level = 1; level <= 6; level++) {
    int n = DEGREE[level], p = RADIX[level], m = n / p;
    for (int k = 0; k < SUBRINGS[level]; k++) {
      int base = k * n;
      uint64_t zeta = lb_pow(psi, twiddle_exp(level, k), q);
      if (p == 2) {
        for (int i = 0; i < m; i++) {
          uint64_t a0 = v[base + i], a1 = v[base + m + i], t = a1 * zeta % q;
          v[base + i] = (a0 + t) % q;
          v[base + m + i] = (a0 + q - t) % q;
        }
      } else {
        uint64_t zeta2 = zeta * zeta % q;
        for (int i = 0; i < m; i++) {
          uint64_t a0 = v[base + i], t1 = v[base + m + i] * zeta % q, t2 = v[base + 2 * m + i] * zeta2 % q;
          v[base + i] = (a0 + t1 + t2) % q;
          v[base + m + i] = (a0 + w * t1 + w2 * t2) % q;
          v[base + 2 * m + i] = (a0 + w2 * t1 + w * t2) % q;
        }
      }
    }
  }
  for (int i = 0; i < LB_N; i++) out[i] = (uint32_t)v[i];
}

/* ntt_quad, scalar.rs:165-213: leaf j in rows 2j (constant) and 2j+1 (X) */
static void ntt_quad(uint64_t q, const uint32_t *a, uint32_t *out) {
  uint64_t psi = find_psi972(q), w = lb_pow(psi, 324, q), w2 = w * w % q, z6 = lb_pow(psi, 162, q);
  uint64_t v[LB_N];
  for (int i = 0; i < LB_N; i++) v[i] = a[i] % q;
  for (int i = 0; i < 324; i++) {
    uint64_t a0 = v[i], a1 = v[i + 324], t = a1 * z6 % q;
    v[i] = (a0 + t) % q;
    v[i + 324] = (a0 + a1 + q - t) % q;
  }
  for (int level = 1; level <= 5; level++) {
    int n = DEGREE_Q[level], p = RADIX_Q[level], m = n / p;
    for (int k = 0; k < SUBRINGS_Q[level]; k++) {
      int base = k * n;
      uint64_t zeta = lb_pow(psi, twiddle_exp_quad(level, k), q);
      if (p == 2) {
        for (int i = 0; i < m; i++) {
          uint64_t a0 = v[base + i], a1 = v[base + m + i], t = a1 * zeta % q;
          v[base + i] = (a0 + t) % q;
          v[base + m + i] = (a0 + q - t) % q;
        }
      } else {
        uint64_t zeta2 = zeta * zeta % q;
        for (int i = 0; i < m; i++) {
          uint64_t a0 = v[base + i], t1 = v[base + m + i] * zeta % q, t2 = v[base + 2 * m + i] * zeta2 % q;
          v[base + i] = (a0 + t1 + t2) % q;
          v[base + m + i] = (a0 + w * t1 + w2 * t2) % q;
          v[base + 2 * m + i] = (a0 + w2 * t1 + w * t2) % q;
        }
      }
    }
  }
  for (int i = 0; i < LB_N; i++) out[i] = (uint32_t)v[i];
}

/* ring.rs:322-333 ntt_of */
void orc_lb_ntt(uint32_t q, const uint32_t *a, uint32_t *out) {
  if (orc_lb_quadratic(q))
    ntt_quad(q, a, out);
  else
    ntt_split(q, a, out);
}

/* eval_at, scalar.rs:89-97 (split) / eval_quad_at, scalar.rs:216-226 (quadratic) */
uint32_t orc_lb_eval_at(uint32_t q, const uint32_t *a, uint32_t u) {
  uint64_t x = lb_pow(find_psi(q), u, q), acc = 0;
  for (int i = LB_N - 1; i >= 0; i--) acc = (acc * x + a[i]) % q;
  return (uint32_t)acc;
}

void orc_lb_eval_quad_at(uint32_t q, const uint32_t *a, uint32_t u, uint32_t out[2]) {
  uint64_t c = lb_pow(find_psi972(q), u, q), r0 = 0, r1 = 0;
  for (int i = LB_N - 1; i >= 0; i--) {
    uint64_t n0 = (r1 * c + a[i]) % q, n1 = r0;
    r0 = n0;
    r1 = n1;
  }
  out[0] = (uint32_t)r0;
  out[1] = (uint32_t)r1;
}

/* mul_mod_phi, scalar.rs:11-34 */
void orc_lb_mul_mod_phi(uint32_t q32, const uint32_t *a, const uint32_t *b, uint32_t *out) {
  uint64_t q = q32;
  uint64_t *c = (uint64_t *)calloc(2 * LB_N, sizeof(uint64_t));
  for (int i = 0; i < LB_N; i++) {
    if (!a[i]) continue;
    for (int j = 0; j < LB_N; j++) c[i + j] += (uint64_t)a[i] * b[j];
  }
  for (int k = 2 * LB_N - 1; k >= LB_N; k--) {
    uint64_t v = c[k] % q;
    c[k] = 0;
    c[k - 324] += v;
    c[k - 648] += q * q - v;
  }
  for (int i = 0; i < LB_N; i++) out[i] = (uint32_t)(c[i] % q);
  free(c);
}

/* mul_quad_slots, scalar.rs:229-243 */
void orc_lb_mul_quad_slots(uint32_t q32, const uint32_t *a, const uint32_t *b, uint32_t *out) {
  uint64_t q = q32, psi = find_psi972(q);
  build_tables();
  for (int j = 0; j < LB_QSLOTS; j++) {
    uint64_t cj = lb_pow(psi, QUAD_SLOT_EXP[j], q);
    uint64_t a0 = a[2 * j] % q, a1 = a[2 * j + 1] % q, b0 = b[2 * j] % q, b1 = b[2 * j + 1] % q;
    out[2 * j] = (uint32_t)((a0 * b0 + cj * (a1 * b1 % q)) % q);
    out[2 * j + 1] = (uint32_t)((a0 * b1 + a1 * b0) % q);
  }
}

/* ---- 648 -> 4 x 162 (ring.rs:167-307) ---- */

static int16_t center(uint64_t r, uint64_t q) { return r > (q - 1) / 2 ? (int16_t)((int64_t)r - (int64_t)q) : (int16_t)r; }

/* decompose_components, ring.rs:193-245: Y_k(v_s) = 4^-1 psi^{-v_s k} sum_t i^{-tk} y(psi^{v_s + 486 t}) */
static void decompose_split(uint64_t q, const uint32_t *y, int16_t out[4][LB_N162]) {
  uint64_t psi = find_psi(q), inv4 = lb_inv(4, q), i_root = lb_pow(psi, 486, q);
  for (int s = 0; s < LB_N162; s++) {
    uint64_t v = POW3_SLOT_EXP[s], e[4];
    for (int t = 0; t < 4; t++) e[t] = y[SLOT_648[t][s]] % q;
    uint64_t a = e[0] + e[2], d0 = e[0] + q - e[2], c = e[1] + e[3], d1 = e[1] + q - e[3];
    uint64_t id = (d1 % q) * i_root % q;
    uint64_t m[4] = {a + c, d0 + q - id, a + 2 * q - c, d0 + id};
    for (int k = 0; k < 4; k++) {
      uint64_t tw = inv4 * lb_pow(psi, (LB_COND - v * k % LB_COND) % LB_COND, q) % q;
      out[k][s] = center((m[k] % q) * tw % q, q);
    }
  }
}

/* decompose_components_quad, ring.rs:264-306 */
static void decompose_quad(uint64_t q, const uint32_t *y, int16_t out[4][LB_N162]) {
  uint64_t psi = find_psi972(q), inv2 = lb_inv(2, q);
  for (int s = 0; s < LB_N162; s++) {
    uint64_t v = POW3_SLOT_EXP[s];
    int jp = QUAD_CLASS_SLOT[0][s], jm = QUAD_CLASS_SLOT[1][s];
    uint64_t tws = inv2 * lb_pow(psi, (LB_COND_Q - v) % LB_COND_Q, q) % q;
    for (int k = 0; k < 2; k++) {
      uint64_t ep = y[2 * jp + k] % q, em = y[2 * jm + k] % q;
      out[k][s] = center((ep + em) % q * inv2 % q, q);
      out[k + 2][s] = center((ep + q - em) % q * tws % q, q);
    }
  }
}

/* components_of, ring.rs:308-319; out = [4][162] centered */
void orc_lb_components(uint32_t q, const uint32_t *y, int16_t *out) {
  build_tables();
  if (orc_lb_quadratic(q))
    decompose_quad(q, y, (int16_t(*)[LB_N162])out);
  else
    decompose_split(q, y, (int16_t(*)[LB_N162])out);
}

/* PowerOfThreeRing::from_coeffs, ring.rs:131-149 (theta = psi^4 of the split tree) */
void orc_lb_r162_from_coeffs(uint32_t q, const int64_t *c, int16_t *out) {
  build_tables();
  uint64_t theta = lb_pow(find_psi(q), 4, q);
  for (int s = 0; s < LB_N162; s++) {
    uint64_t x = lb_pow(theta, POW3_SLOT_EXP[s], q), acc = 0;
    for (int k = LB_N162 - 1; k >= 0; k--) {
      int64_t r = c[k] % (int64_t)q;
      if (r < 0) r += q;
      acc = (acc * x + (uint64_t)r) % q;
    }
    out[s] = center(acc, q);
  }
}

/* ---- witnesses and keys (binfield.rs, key.rs) ---- */

/* Rng, binfield.rs:158-175 (xorshift64*) */
typedef struct {
  uint64_t s;
} lb_rng;

static lb_rng rng_new(uint64_t seed) {
  lb_rng r = {seed * 0x9E3779B97F4A7C15ull | 1};
  return r;
}

static uint64_t rng_next(lb_rng *r) {
  uint64_t x = r->s;
  x ^= x >> 12;
  x ^= x << 25;
  x ^= x >> 27;
  r->s = x;
  return x * 0x2545F4914F6CDD1Dull;
}

static uint32_t rng_below(lb_rng *r, uint32_t n) { return (uint32_t)(((rng_next(r) >> 32) * n) >> 32); }

/* random_elems, binfield.rs:177-189: out = n x [3] u64 */
void orc_lb_random_elems(size_t n, uint64_t seed, uint64_t *out) {
  lb_rng r = rng_new(seed);
  for (size_t i = 0; i < n; i++) {
    out[3 * i] = rng_next(&r);
    out[3 * i + 1] = rng_next(&r);
    out[3 * i + 2] = rng_next(&r) & ((1ull << 34) - 1);
  }
}

/* lift4 / lift_elem, binfield.rs:128-143: coefficient 4m + k = bit m of element 4r + k */
void orc_lb_lift(const uint64_t *elems, size_t r, uint32_t *out) {
  const uint64_t *e = elems + 12 * r;
  for (int m = 0; m < LB_N162; m++)
    for (int k = 0; k < 4; k++) out[4 * m + k] = (uint32_t)((e[3 * k + (m >> 6)] >> (m & 63)) & 1);
}

/* CommitmentKey::random, key.rs:94-137: a = [limbs][nr][648] centered NTT-domain rows */
void orc_lb_key_random(size_t len_f162, uint64_t seed, const uint32_t *primes, size_t limbs, int16_t *a) {
  size_t nr = len_f162 / 4;
  uint32_t coeffs[LB_N], t[LB_N];
  for (size_t k = 0; k < limbs; k++) {
    uint32_t q = primes[k];
    int32_t half = (int32_t)((q - 1) / 2);
    lb_rng r = rng_new(seed ^ (0x9E3779B9ull * (uint64_t)(k + 1)));
    for (size_t i = 0; i < nr; i++) {
      for (int c = 0; c < LB_N; c++) coeffs[c] = rng_below(&r, q);
      orc_lb_ntt(q, coeffs, t);
      for (int u = 0; u < LB_N; u++)
        a[(k * nr + i) * LB_N + u] = (int16_t)((int32_t)t[u] > half ? (int32_t)t[u] - (int32_t)q : (int32_t)t[u]);
    }
  }
}

/* commit_scalar, key.rs:382-474.  witness: r * len_f162 F162 ([3] u64 each);
 * raw = [limbs][r][648]; matrix = [4][r][limbs][162] centered; batches =
 * [r * nr][648] (base limb transform) or NULL.  nthreads <= 0: all cores. */
int orc_lb_commit(const int16_t *a, const uint32_t *primes, size_t limbs, size_t len_f162, const uint64_t *witness,
                  size_t r, uint32_t *raw, int16_t *matrix, uint32_t *batches, int nthreads) {
  build_tables();
  size_t nr = len_f162 / 4;
  int nt = nthreads > 0 ? nthreads : omp_get_num_procs();
  for (size_t k = 0; k < limbs; k++) {
    uint32_t q = primes[k];
    int quad = orc_lb_quadratic(q);
#pragma omp parallel for schedule(static) num_threads(nt)
    for (long long cc = 0; cc < (long long)r; cc++) {
      size_t c = (size_t)cc;
      uint64_t y[LB_N];
      uint32_t w[LB_N], t[LB_N], acoef[LB_N], prod[LB_N];
      memset(y, 0, sizeof(y));
      for (size_t i = 0; i < nr; i++) {
        orc_lb_lift(witness + 3 * c * len_f162, i, w);
        orc_lb_ntt(q, w, t);
        if (k == 0 && batches) memcpy(batches + (c * nr + i) * LB_N, t, sizeof(t));
        const int16_t *arow = a + (k * nr + i) * LB_N;
        if (quad) {
          for (int u = 0; u < LB_N; u++) {
            int32_t x = arow[u] % (int32_t)q;
            acoef[u] = (uint32_t)(x < 0 ? x + (int32_t)q : x);
          }
          orc_lb_mul_quad_slots(q, acoef, t, prod);
          for (int u = 0; u < LB_N; u++) y[u] += prod[u];
        } else {
          for (int u = 0; u < LB_N; u++) {
            int32_t x = arow[u] % (int32_t)q;
            y[u] += (uint64_t)(x < 0 ? x + (int32_t)q : x) * t[u];
          }
        }
      }
      uint32_t *yc = raw + (k * r + c) * LB_N;
      for (int u = 0; u < LB_N; u++) yc[u] = (uint32_t)(y[u] % q);
      int16_t comps[4][LB_N162];
      orc_lb_components(q, yc, &comps[0][0]);
      for (int row = 0; row < 4; row++)
        memcpy(matrix + ((row * r + c) * limbs + k) * LB_N162, comps[row], sizeof(comps[row]));
    }
  }
  return 0;
}
