/*
 * lzx_oracle.c -- CPU restatement of the LZX commitment hot path.
 *
 * TEST INFRASTRUCTURE ONLY (correctness oracle and timed CPU baseline); the
 * product never links it.  See lzx_oracle.h for what pins it.  Each function
 * cites the reference (idrees2516/lzx, Rust) file:line that it restates.
 */
#include "lzx_oracle.h"

#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#if defined(__x86_64__)
#include <immintrin.h>
#endif

typedef unsigned __int128 u128;

/* ======================= Modulus32 (modulus.rs) ========================== */

/* Modulus32::new + barrett_recip, modulus.rs:15-17, 37-44 */
orc_mod32 orc_mod32_new(uint32_t q, uint32_t two_adicity, uint32_t generator) {
  orc_mod32 m;
  m.q = q;
  m.two_adicity = two_adicity;
  m.generator = generator;
  m.barrett_recip = UINT64_MAX / (uint64_t)q;
  return m;
}

/* Modulus32::reduce_u64, modulus.rs:64-76 (Barrett, <= 2 corrections) */
uint32_t orc_mod32_reduce_u64(const orc_mod32 *m, uint64_t x) {
  u128 q = m->q;
  u128 qhat = ((u128)x * (u128)m->barrett_recip) >> 64;
  u128 r = (u128)x - qhat * q; /* never negative: qhat <= floor(x/q) */
  if (r >= q) r -= q;
  if (r >= q) r -= q;
  return (uint32_t)r;
}

/* Modulus32::reduce_i64, modulus.rs:79-83 (rem_euclid) */
uint32_t orc_mod32_reduce_i64(const orc_mod32 *m, int64_t x) {
  int64_t q = (int64_t)m->q;
  int64_t r = x % q;
  if (r < 0) r += q;
  return (uint32_t)r;
}

/* modulus.rs:86-89 */
uint32_t orc_mod32_mul(const orc_mod32 *m, uint32_t a, uint32_t b) {
  return orc_mod32_reduce_u64(m, (uint64_t)a * (uint64_t)b);
}

/* modulus.rs:92-100 */
uint32_t orc_mod32_add(const orc_mod32 *m, uint32_t a, uint32_t b) {
  uint64_t s = (uint64_t)a + (uint64_t)b;
  return s >= m->q ? (uint32_t)(s - m->q) : (uint32_t)s;
}

/* modulus.rs:103-112 */
uint32_t orc_mod32_sub(const orc_mod32 *m, uint32_t a, uint32_t b) {
  return a >= b ? a - b : a + (m->q - b);
}

/* modulus.rs:115-122 */
uint32_t orc_mod32_neg(const orc_mod32 *m, uint32_t a) { return a == 0 ? 0 : m->q - a; }

/* modulus.rs:125-137 */
uint32_t orc_mod32_pow(const orc_mod32 *m, uint32_t base, uint64_t exp) {
  uint32_t acc = 1;
  uint32_t b = orc_mod32_reduce_u64(m, base);
  uint64_t e = exp;
  while (e > 0) {
    if (e & 1) acc = orc_mod32_mul(m, acc, b);
    b = orc_mod32_mul(m, b, b);
    e >>= 1;
  }
  return acc;
}

/* modulus.rs:140-146 */
uint32_t orc_mod32_inv(const orc_mod32 *m, uint32_t a) {
  if (a == 0) return 0;
  return orc_mod32_pow(m, a, (uint64_t)m->q - 2);
}

/* modulus.rs:149-156 */
uint32_t orc_mod32_root_of_unity(const orc_mod32 *m, uint32_t k) {
  if (k > m->two_adicity) return 0;
  uint64_t e = ((uint64_t)m->q - 1) >> k;
  return orc_mod32_pow(m, m->generator, e);
}

/* ======================= Goldilocks (field.rs) =========================== */

/* Goldilocks::from_u64, field.rs:28-36 */
uint64_t orc_gl_from_u64(uint64_t x) { return x >= ORC_GL_P ? x - ORC_GL_P : x; }

/* Goldilocks::from_u128, field.rs:42-55: fold hi*2^64 == hi*(2^32-1) */
uint64_t orc_gl_from_u128(uint64_t hi, uint64_t lo) {
  u128 acc = ((u128)hi << 64) | lo;
  for (int i = 0; i < 6; i++) {
    if ((acc >> 64) == 0) break;
    uint64_t h = (uint64_t)(acc >> 64);
    uint64_t l = (uint64_t)acc;
    acc = (u128)h * 0xFFFFFFFFull + (u128)l;
  }
  return orc_gl_from_u64((uint64_t)acc);
}

/* Goldilocks::add, field.rs:69-77 */
uint64_t orc_gl_add(uint64_t a, uint64_t b) {
  uint64_t s = a + b;
  if (s < a) s += 0xFFFFFFFFull; /* dropped 2^64 == 2^32-1 */
  return orc_gl_from_u64(s);
}

/* Goldilocks::sub, field.rs:81-89 */
uint64_t orc_gl_sub(uint64_t a, uint64_t b) {
  uint64_t d = a - b;
  if (a < b) d -= 0xFFFFFFFFull;
  return orc_gl_from_u64(d);
}

/* Goldilocks::neg, field.rs:92-99 */
uint64_t orc_gl_neg(uint64_t a) { return a == 0 ? 0 : orc_gl_from_u64(ORC_GL_P - a); }

/* Goldilocks::mul, field.rs:102-105 */
uint64_t orc_gl_mul(uint64_t a, uint64_t b) {
  u128 p = (u128)a * (u128)b;
  return orc_gl_from_u128((uint64_t)(p >> 64), (uint64_t)p);
}

/* Goldilocks::pow (square-and-multiply), field.rs:119-134 */
uint64_t orc_gl_pow(uint64_t a, uint64_t e) {
  uint64_t acc = 1;
  for (int i = 63; i >= 0; i--) {
    acc = orc_gl_mul(acc, acc);
    if ((e >> i) & 1) acc = orc_gl_mul(acc, a);
  }
  return acc;
}

/* Goldilocks::inverse, field.rs:137-143 (0 -> 0) */
uint64_t orc_gl_inv(uint64_t a) { return a == 0 ? 0 : orc_gl_pow(a, ORC_GL_P - 2); }

/* ======================= NTT over Modulus32 (ntt.rs) ===================== */

/* bit_reverse / reverse_bits, ntt.rs:320-342 */
static uint32_t reverse_bits(uint32_t x, uint32_t bits) {
  uint32_t r = 0;
  for (uint32_t i = 0; i < bits; i++) {
    r = (r << 1) | (x & 1);
    x >>= 1;
  }
  return r;
}

static void bit_reverse32(uint32_t *a, size_t n) {
  if (n <= 1) return;
  uint32_t bits = (uint32_t)__builtin_ctzll(n);
  for (size_t i = 0; i < n; i++) {
    size_t j = reverse_bits((uint32_t)i, bits);
    if (i < j) {
      uint32_t t = a[i];
      a[i] = a[j];
      a[j] = t;
    }
  }
}

static void bit_reverse64(uint64_t *a, size_t n) {
  if (n <= 1) return;
  uint32_t bits = (uint32_t)__builtin_ctzll(n);
  for (size_t i = 0; i < n; i++) {
    size_t j = reverse_bits((uint32_t)i, bits);
    if (i < j) {
      uint64_t t = a[i];
      a[i] = a[j];
      a[j] = t;
    }
  }
}

/* NttTables::new, ntt.rs:46-106 */
int orc_ntt32_new(orc_mod32 m, uint32_t log_n, orc_ntt32 *out) {
  memset(out, 0, sizeof(*out));
  if (log_n + 1 > m.two_adicity) return ORC_ERR_ADICITY_TOO_SMALL;
  size_t n = (size_t)1 << log_n;
  uint32_t psi = orc_mod32_root_of_unity(&m, log_n + 1);
  if (psi == 0) return ORC_ERR_ADICITY_TOO_SMALL;
  uint32_t psi_inv = orc_mod32_inv(&m, psi);
  uint32_t omega = orc_mod32_mul(&m, psi, psi);
  uint32_t omega_inv = orc_mod32_inv(&m, omega);
  out->modulus = m;
  out->log_n = log_n;
  out->n_inv = orc_mod32_pow(&m, (uint32_t)n, (uint64_t)m.q - 2);
  size_t half = n / 2 > 1 ? n / 2 : 1;
  out->pow_psi = (uint32_t *)malloc(n * 4);
  out->pow_psi_inv = (uint32_t *)malloc(n * 4);
  out->pow_omega = (uint32_t *)malloc(half * 4);
  out->pow_omega_inv = (uint32_t *)malloc(half * 4);
  out->level_tw = (uint32_t *)malloc((n > 1 ? n : 2) * 4);
  out->level_tw_inv = (uint32_t *)malloc((n > 1 ? n : 2) * 4);
  uint32_t p = 1, pi = 1;
  for (size_t i = 0; i < n; i++) {
    out->pow_psi[i] = p;
    out->pow_psi_inv[i] = pi;
    p = orc_mod32_mul(&m, p, psi);
    pi = orc_mod32_mul(&m, pi, psi_inv);
  }
  uint32_t w = 1, wi = 1;
  for (size_t i = 0; i < half; i++) {
    out->pow_omega[i] = w;
    out->pow_omega_inv[i] = wi;
    w = orc_mod32_mul(&m, w, omega);
    wi = orc_mod32_mul(&m, wi, omega_inv);
  }
  /* level j (len = 2^(j+1)) stores len/2 = 2^j entries at offset 2^j - 1 */
  for (uint32_t level = 0; level < log_n; level++) {
    size_t len = (size_t)1 << (level + 1);
    size_t stride = n / len;
    size_t off = ((size_t)1 << level) - 1;
    for (size_t t = 0; t < len / 2; t++) {
      out->level_tw[off + t] = out->pow_omega[t * stride];
      out->level_tw_inv[off + t] = out->pow_omega_inv[t * stride];
    }
  }
  return ORC_OK;
}

void orc_ntt32_free(orc_ntt32 *t) {
  free(t->pow_psi);
  free(t->pow_psi_inv);
  free(t->pow_omega);
  free(t->pow_omega_inv);
  free(t->level_tw);
  free(t->level_tw_inv);
  memset(t, 0, sizeof(*t));
}

/* NttTables::forward, ntt.rs:152-182 */
int orc_ntt32_forward(const orc_ntt32 *t, uint32_t *a, size_t len) {
  size_t n = (size_t)1 << t->log_n;
  if (len != n) return ORC_ERR_LENGTH_MISMATCH;
  const orc_mod32 *q = &t->modulus;
  for (size_t i = 0; i < n; i++) a[i] = orc_mod32_mul(q, a[i], t->pow_psi[i]);
  bit_reverse32(a, n);
  for (size_t l = 2; l <= n; l <<= 1) {
    size_t stride = n / l;
    for (size_t start = 0; start < n; start += l) {
      for (size_t j = 0; j < l / 2; j++) {
        uint32_t w = t->pow_omega[stride * j];
        uint32_t u = a[start + j];
        uint32_t v = orc_mod32_mul(q, a[start + j + l / 2], w);
        a[start + j] = orc_mod32_add(q, u, v);
        a[start + j + l / 2] = orc_mod32_sub(q, u, v);
      }
    }
  }
  return ORC_OK;
}

/* NttTables::forward_fast, ntt.rs:118-146 */
int orc_ntt32_forward_fast(const orc_ntt32 *t, uint32_t *a, size_t len) {
  size_t n = (size_t)1 << t->log_n;
  if (len != n) return ORC_ERR_LENGTH_MISMATCH;
  const orc_mod32 *q = &t->modulus;
  for (size_t i = 0; i < n; i++) a[i] = orc_mod32_mul(q, a[i], t->pow_psi[i]);
  bit_reverse32(a, n);
  for (uint32_t level = 0; level < t->log_n; level++) {
    const uint32_t *tw = t->level_tw + (((size_t)1 << level) - 1);
    size_t sl = (size_t)1 << level;
    size_t l = sl << 1;
    for (size_t start = 0; start < n; start += l) {
      for (size_t k = 0; k < sl; k++) {
        uint32_t w = tw[k];
        uint32_t u = a[start + k];
        uint32_t v = orc_mod32_mul(q, a[start + k + sl], w);
        a[start + k] = orc_mod32_add(q, u, v);
        a[start + k + sl] = orc_mod32_sub(q, u, v);
      }
    }
  }
  return ORC_OK;
}

/* NttTables::inverse_fast, ntt.rs:187-216 */
int orc_ntt32_inverse_fast(const orc_ntt32 *t, uint32_t *a, size_t len) {
  size_t n = (size_t)1 << t->log_n;
  if (len != n) return ORC_ERR_LENGTH_MISMATCH;
  const orc_mod32 *q = &t->modulus;
  for (int level = (int)t->log_n - 1; level >= 0; level--) {
    const uint32_t *tw = t->level_tw_inv + (((size_t)1 << level) - 1);
    size_t sl = (size_t)1 << level;
    size_t l = sl << 1;
    for (size_t start = 0; start < n; start += l) {
      for (size_t k = 0; k < sl; k++) {
        uint32_t w = tw[k];
        uint32_t u = a[start + k];
        uint32_t v = a[start + k + sl];
        a[start + k] = orc_mod32_add(q, u, v);
        a[start + k + sl] = orc_mod32_mul(q, orc_mod32_sub(q, u, v), w);
      }
    }
  }
  bit_reverse32(a, n);
  for (size_t i = 0; i < n; i++)
    a[i] = orc_mod32_mul(q, orc_mod32_mul(q, a[i], t->pow_psi_inv[i]), t->n_inv);
  return ORC_OK;
}

/* NttTables::inverse, ntt.rs:219-250 */
int orc_ntt32_inverse(const orc_ntt32 *t, uint32_t *a, size_t len) {
  size_t n = (size_t)1 << t->log_n;
  if (len != n) return ORC_ERR_LENGTH_MISMATCH;
  const orc_mod32 *q = &t->modulus;
  for (size_t l = n; l >= 2; l >>= 1) {
    size_t stride = n / l;
    for (size_t start = 0; start < n; start += l) {
      for (size_t j = 0; j < l / 2; j++) {
        uint32_t w = t->pow_omega_inv[stride * j];
        uint32_t u = a[start + j];
        uint32_t v = a[start + j + l / 2];
        a[start + j] = orc_mod32_add(q, u, v);
        a[start + j + l / 2] = orc_mod32_mul(q, orc_mod32_sub(q, u, v), w);
      }
    }
  }
  bit_reverse32(a, n);
  for (size_t i = 0; i < n; i++)
    a[i] = orc_mod32_mul(q, orc_mod32_mul(q, a[i], t->pow_psi_inv[i]), t->n_inv);
  return ORC_OK;
}

/* NttTables::forward_partial, ntt.rs:256-286 */
int orc_ntt32_forward_partial(const orc_ntt32 *t, uint32_t *a, size_t len, uint32_t levels) {
  size_t n = (size_t)1 << t->log_n;
  if (len != n || levels > t->log_n) return ORC_ERR_LENGTH_MISMATCH;
  const orc_mod32 *q = &t->modulus;
  for (size_t i = 0; i < n; i++) a[i] = orc_mod32_mul(q, a[i], t->pow_psi[i]);
  bit_reverse32(a, n);
  uint32_t applied = 0;
  for (size_t l = 2; l <= n && applied < levels; l <<= 1, applied++) {
    size_t stride = n / l;
    for (size_t start = 0; start < n; start += l) {
      for (size_t j = 0; j < l / 2; j++) {
        uint32_t w = t->pow_omega[stride * j];
        uint32_t u = a[start + j];
        uint32_t v = orc_mod32_mul(q, a[start + j + l / 2], w);
        a[start + j] = orc_mod32_add(q, u, v);
        a[start + j + l / 2] = orc_mod32_sub(q, u, v);
      }
    }
  }
  return ORC_OK;
}

/* NttTables::complete_partial, ntt.rs:290-316 */
int orc_ntt32_complete_partial(const orc_ntt32 *t, uint32_t *a, size_t len, uint32_t already) {
  size_t n = (size_t)1 << t->log_n;
  if (len != n || already > t->log_n) return ORC_ERR_LENGTH_MISMATCH;
  const orc_mod32 *q = &t->modulus;
  for (size_t l = (size_t)1 << (already + 1); l <= n; l <<= 1) {
    size_t stride = n / l;
    for (size_t start = 0; start < n; start += l) {
      for (size_t j = 0; j < l / 2; j++) {
        uint32_t w = t->pow_omega[stride * j];
        uint32_t u = a[start + j];
        uint32_t v = orc_mod32_mul(q, a[start + j + l / 2], w);
        a[start + j] = orc_mod32_add(q, u, v);
        a[start + j + l / 2] = orc_mod32_sub(q, u, v);
      }
    }
  }
  return ORC_OK;
}

static int resolve_threads(int nthreads) {
#ifdef _OPENMP
  return nthreads > 0 ? nthreads : omp_get_max_threads();
#else
  (void)nthreads;
  return 1;
#endif
}

int orc_ntt32_forward_batch(const orc_ntt32 *t, uint32_t *a, size_t count, int nthreads) {
  size_t n = (size_t)1 << t->log_n;
  int nt = resolve_threads(nthreads);
  (void)nt;
#pragma omp parallel for schedule(static) num_threads(nt)
  for (long long i = 0; i < (long long)count; i++) orc_ntt32_forward_fast(t, a + (size_t)i * n, n);
  return ORC_OK;
}

int orc_ntt32_inverse_batch(const orc_ntt32 *t, uint32_t *a, size_t count, int nthreads) {
  size_t n = (size_t)1 << t->log_n;
  int nt = resolve_threads(nthreads);
  (void)nt;
#pragma omp parallel for schedule(static) num_threads(nt)
  for (long long i = 0; i < (long long)count; i++) orc_ntt32_inverse_fast(t, a + (size_t)i * n, n);
  return ORC_OK;
}

/* ============== Goldilocks instantiation of ntt.rs ======================= */

/* NttTables::new over field.rs: psi = 7^((p-1)/2^(log_n+1)) (field.rs:195-200,
 * adicity 32, field.rs:12) */
int orc_nttgl_new(uint32_t log_n, orc_nttgl *out) {
  memset(out, 0, sizeof(*out));
  if (log_n + 1 > 32) return ORC_ERR_ADICITY_TOO_SMALL;
  size_t n = (size_t)1 << log_n;
  uint64_t psi = orc_gl_pow(7, (ORC_GL_P - 1) >> (log_n + 1));
  uint64_t psi_inv = orc_gl_inv(psi);
  uint64_t omega = orc_gl_mul(psi, psi);
  uint64_t omega_inv = orc_gl_inv(omega);
  out->log_n = log_n;
  out->n_inv = orc_gl_pow((uint64_t)n, ORC_GL_P - 2);
  size_t half = n / 2 > 1 ? n / 2 : 1;
  uint64_t *pw = (uint64_t *)malloc(half * 8), *pwi = (uint64_t *)malloc(half * 8);
  out->pow_psi = (uint64_t *)malloc(n * 8);
  out->pow_psi_inv = (uint64_t *)malloc(n * 8);
  out->level_tw = (uint64_t *)malloc((n > 1 ? n : 2) * 8);
  out->level_tw_inv = (uint64_t *)malloc((n > 1 ? n : 2) * 8);
  uint64_t p = 1, pi = 1;
  for (size_t i = 0; i < n; i++) {
    out->pow_psi[i] = p;
    out->pow_psi_inv[i] = pi;
    p = orc_gl_mul(p, psi);
    pi = orc_gl_mul(pi, psi_inv);
  }
  uint64_t w = 1, wi = 1;
  for (size_t i = 0; i < half; i++) {
    pw[i] = w;
    pwi[i] = wi;
    w = orc_gl_mul(w, omega);
    wi = orc_gl_mul(wi, omega_inv);
  }
  for (uint32_t level = 0; level < log_n; level++) {
    size_t len = (size_t)1 << (level + 1);
    size_t stride = n / len;
    size_t off = ((size_t)1 << level) - 1;
    for (size_t t = 0; t < len / 2; t++) {
      out->level_tw[off + t] = pw[t * stride];
      out->level_tw_inv[off + t] = pwi[t * stride];
    }
  }
  free(pw);
  free(pwi);
  return ORC_OK;
}

void orc_nttgl_free(orc_nttgl *t) {
  free(t->pow_psi);
  free(t->pow_psi_inv);
  free(t->level_tw);
  free(t->level_tw_inv);
  memset(t, 0, sizeof(*t));
}

/* forward_fast (ntt.rs:118-146) over Goldilocks */
int orc_nttgl_forward_fast(const orc_nttgl *t, uint64_t *a, size_t len) {
  size_t n = (size_t)1 << t->log_n;
  if (len != n) return ORC_ERR_LENGTH_MISMATCH;
  for (size_t i = 0; i < n; i++) a[i] = orc_gl_mul(a[i], t->pow_psi[i]);
  bit_reverse64(a, n);
  for (uint32_t level = 0; level < t->log_n; level++) {
    const uint64_t *tw = t->level_tw + (((size_t)1 << level) - 1);
    size_t sl = (size_t)1 << level;
    for (size_t start = 0; start < n; start += 2 * sl) {
      for (size_t k = 0; k < sl; k++) {
        uint64_t u = a[start + k];
        uint64_t v = orc_gl_mul(a[start + k + sl], tw[k]);
        a[start + k] = orc_gl_add(u, v);
        a[start + k + sl] = orc_gl_sub(u, v);
      }
    }
  }
  return ORC_OK;
}

/* inverse_fast (ntt.rs:187-216) over Goldilocks */
int orc_nttgl_inverse_fast(const orc_nttgl *t, uint64_t *a, size_t len) {
  size_t n = (size_t)1 << t->log_n;
  if (len != n) return ORC_ERR_LENGTH_MISMATCH;
  for (int level = (int)t->log_n - 1; level >= 0; level--) {
    const uint64_t *tw = t->level_tw_inv + (((size_t)1 << level) - 1);
    size_t sl = (size_t)1 << level;
    for (size_t start = 0; start < n; start += 2 * sl) {
      for (size_t k = 0; k < sl; k++) {
        uint64_t u = a[start + k];
        uint64_t v = a[start + k + sl];
        a[start + k] = orc_gl_add(u, v);
        a[start + k + sl] = orc_gl_mul(orc_gl_sub(u, v), tw[k]);
      }
    }
  }
  bit_reverse64(a, n);
  for (size_t i = 0; i < n; i++) a[i] = orc_gl_mul(orc_gl_mul(a[i], t->pow_psi_inv[i]), t->n_inv);
  return ORC_OK;
}

int orc_nttgl_forward_batch(const orc_nttgl *t, uint64_t *a, size_t count, int nthreads) {
  size_t n = (size_t)1 << t->log_n;
  int nt = resolve_threads(nthreads);
  (void)nt;
#pragma omp parallel for schedule(static) num_threads(nt)
  for (long long i = 0; i < (long long)count; i++) orc_nttgl_forward_fast(t, a + (size_t)i * n, n);
  return ORC_OK;
}

int orc_nttgl_inverse_batch(const orc_nttgl *t, uint64_t *a, size_t count, int nthreads) {
  size_t n = (size_t)1 << t->log_n;
  int nt = resolve_threads(nthreads);
  (void)nt;
#pragma omp parallel for schedule(static) num_threads(nt)
  for (long long i = 0; i < (long long)count; i++) orc_nttgl_inverse_fast(t, a + (size_t)i * n, n);
  return ORC_OK;
}

/* ======================= Ajtai commit (ajtai.rs) ========================= */

static int all_zero32(const uint32_t *a, size_t n) {
  for (size_t i = 0; i < n; i++)
    if (a[i]) return 0;
  return 1;
}

static int all_zero64(const uint64_t *a, size_t n) {
  for (size_t i = 0; i < n; i++)
    if (a[i]) return 0;
  return 1;
}

/* AjtaiPublicKey::commit, ajtai.rs:118-153 */
int orc_ajtai32_commit(const orc_ntt32 *t, const uint32_t *matrix_ntt, size_t k, size_t m,
                       const uint32_t *s, uint32_t *out) {
  size_t n = (size_t)1 << t->log_n;
  const orc_mod32 *q = &t->modulus;
  uint32_t *s_ntt = (uint32_t *)malloc(m * n * 4);
  unsigned char *nz = (unsigned char *)malloc(m ? m : 1);
  for (size_t j = 0; j < m; j++) {
    nz[j] = !all_zero32(s + j * n, n); /* RingElement::is_zero, ring.rs:253 */
    if (nz[j]) {
      memcpy(s_ntt + j * n, s + j * n, n * 4);
      orc_ntt32_forward_fast(t, s_ntt + j * n, n);
    }
  }
  for (size_t i = 0; i < k; i++) {
    uint32_t *acc = out + i * n;
    memset(acc, 0, n * 4);
    for (size_t j = 0; j < m; j++) {
      if (!nz[j]) continue;
      const uint32_t *a = matrix_ntt + (i * m + j) * n;
      const uint32_t *b = s_ntt + j * n;
      for (size_t x = 0; x < n; x++) acc[x] = orc_mod32_add(q, acc[x], orc_mod32_mul(q, a[x], b[x]));
    }
    orc_ntt32_inverse_fast(t, acc, n); /* RingElement::from_ntt, ring.rs:354-367 */
  }
  free(s_ntt);
  free(nz);
  return ORC_OK;
}

/* RingElement::mul, ring.rs:309-340 */
int orc_ring32_mul(const orc_ntt32 *t, const uint32_t *a, const uint32_t *b, uint32_t *out) {
  size_t n = (size_t)1 << t->log_n;
  uint32_t *x = (uint32_t *)malloc(n * 4), *y = (uint32_t *)malloc(n * 4);
  memcpy(x, a, n * 4);
  memcpy(y, b, n * 4);
  orc_ntt32_forward_fast(t, x, n);
  orc_ntt32_forward_fast(t, y, n);
  for (size_t i = 0; i < n; i++) x[i] = orc_mod32_mul(&t->modulus, x[i], y[i]);
  orc_ntt32_inverse_fast(t, x, n);
  memcpy(out, x, n * 4);
  free(x);
  free(y);
  return ORC_OK;
}

/* AjtaiPublicKey::commit_naive_reference, ajtai.rs:158-180 */
int orc_ajtai32_commit_naive(const orc_ntt32 *t, const uint32_t *matrix, size_t k, size_t m,
                             const uint32_t *s, uint32_t *out) {
  size_t n = (size_t)1 << t->log_n;
  uint32_t *prod = (uint32_t *)malloc(n * 4);
  for (size_t i = 0; i < k; i++) {
    uint32_t *acc = out + i * n;
    memset(acc, 0, n * 4);
    for (size_t j = 0; j < m; j++) {
      if (all_zero32(s + j * n, n)) continue;
      orc_ring32_mul(t, matrix + (i * m + j) * n, s + j * n, prod);
      for (size_t x = 0; x < n; x++) acc[x] = orc_mod32_add(&t->modulus, acc[x], prod[x]);
    }
  }
  free(prod);
  return ORC_OK;
}

/* ---- AVX-512 Goldilocks multiply-accumulate (restates the derivation of
 * lattice-core/src/field_simd.rs:11-56: 32-bit half products, three folds of
 * 2^64 == 2^32-1, masked compensation, canonical subtraction). ----------- */
#if defined(__x86_64__)
__attribute__((target("avx512f"))) static inline __m512i gl_reduce128_v(__m512i hi, __m512i lo) {
  const __m512i M32 = _mm512_set1_epi64(0xFFFFFFFFll);
  for (int f = 0; f < 3; f++) {
    /* sum = lo + ((hi & M32) << 32), carry cA */
    __m512i t = _mm512_slli_epi64(_mm512_and_si512(hi, M32), 32);
    __m512i sum = _mm512_add_epi64(lo, t);
    __mmask8 cA = _mm512_cmplt_epu64_mask(sum, lo);
    __m512i q64 = _mm512_mask_add_epi64(_mm512_srli_epi64(hi, 32), cA, _mm512_srli_epi64(hi, 32),
                                        _mm512_set1_epi64(1));
    /* lo' = sum - hi with borrow b */
    __m512i lo2 = _mm512_sub_epi64(sum, hi);
    __mmask8 b = _mm512_cmplt_epu64_mask(sum, hi);
    hi = _mm512_mask_sub_epi64(q64, b, q64, _mm512_set1_epi64(1));
    lo = lo2;
  }
  /* hi in {0,1}: add 2^32-1 where hi == 1 (cannot wrap) */
  __mmask8 h1 = _mm512_test_epi64_mask(hi, hi);
  lo = _mm512_mask_add_epi64(lo, h1, lo, M32);
  const __m512i P = _mm512_set1_epi64((long long)ORC_GL_P);
  __mmask8 ge = _mm512_cmpge_epu64_mask(lo, P);
  return _mm512_mask_sub_epi64(lo, ge, lo, P);
}

__attribute__((target("avx512f"))) static inline __m512i gl_mul_v(__m512i a, __m512i b) {
  const __m512i M32 = _mm512_set1_epi64(0xFFFFFFFFll);
  __m512i ah = _mm512_srli_epi64(a, 32), bh = _mm512_srli_epi64(b, 32);
  __m512i ll = _mm512_mul_epu32(a, b);
  __m512i lh = _mm512_mul_epu32(a, bh);
  __m512i hl = _mm512_mul_epu32(ah, b);
  __m512i hh = _mm512_mul_epu32(ah, bh);
  __m512i mid = _mm512_add_epi64(lh, hl);
  __mmask8 c1 = _mm512_cmplt_epu64_mask(mid, lh);
  __m512i lo = _mm512_add_epi64(ll, _mm512_slli_epi64(mid, 32));
  __mmask8 c2 = _mm512_cmplt_epu64_mask(lo, ll);
  __m512i hi = _mm512_add_epi64(hh, _mm512_srli_epi64(mid, 32));
  hi = _mm512_mask_add_epi64(hi, c2, hi, _mm512_set1_epi64(1));
  hi = _mm512_mask_add_epi64(hi, c1, hi, _mm512_set1_epi64(1ll << 32));
  (void)M32;
  return gl_reduce128_v(hi, lo);
}

__attribute__((target("avx512f"))) static inline __m512i gl_add_v(__m512i a, __m512i b) {
  __m512i s = _mm512_add_epi64(a, b);
  __mmask8 c = _mm512_cmplt_epu64_mask(s, a);
  s = _mm512_mask_add_epi64(s, c, s, _mm512_set1_epi64(0xFFFFFFFFll));
  const __m512i P = _mm512_set1_epi64((long long)ORC_GL_P);
  __mmask8 ge = _mm512_cmpge_epu64_mask(s, P);
  return _mm512_mask_sub_epi64(s, ge, s, P);
}

/* acc[x] = acc[x] + a[x]*b[x] (mul_add_slices, field_simd.rs:214) */
__attribute__((target("avx512f"))) static void gl_mac_avx512(uint64_t *acc, const uint64_t *a,
                                                             const uint64_t *b, size_t n) {
  size_t x = 0;
  for (; x + 8 <= n; x += 8) {
    __m512i va = _mm512_loadu_si512((const void *)(a + x));
    __m512i vb = _mm512_loadu_si512((const void *)(b + x));
    __m512i vc = _mm512_loadu_si512((const void *)(acc + x));
    _mm512_storeu_si512((void *)(acc + x), gl_add_v(gl_mul_v(va, vb), vc));
  }
  for (; x < n; x++) acc[x] = orc_gl_add(acc[x], orc_gl_mul(a[x], b[x]));
}
#endif

int orc_avx512_available(void) {
#if defined(__x86_64__)
  __builtin_cpu_init();
  return __builtin_cpu_supports("avx512f") ? 1 : 0;
#else
  return 0;
#endif
}

static void gl_mac_scalar(uint64_t *acc, const uint64_t *a, const uint64_t *b, size_t n) {
  for (size_t x = 0; x < n; x++) acc[x] = orc_gl_add(acc[x], orc_gl_mul(a[x], b[x]));
}

/* One witness of the Goldilocks cached-NTT commit (ajtai.rs:118-153 over
 * field.rs).  s_ntt: scratch m*d. */
static void ajtaigl_commit_one(const orc_nttgl *t, const uint64_t *matrix_ntt, size_t kappa,
                               size_t m, const uint64_t *w, uint64_t *s_ntt, unsigned char *nz,
                               uint64_t *out, int use_simd) {
  size_t d = (size_t)1 << t->log_n;
  for (size_t j = 0; j < m; j++) {
    nz[j] = !all_zero64(w + j * d, d);
    if (nz[j]) {
      memcpy(s_ntt + j * d, w + j * d, d * 8);
      orc_nttgl_forward_fast(t, s_ntt + j * d, d);
    }
  }
  for (size_t i = 0; i < kappa; i++) {
    uint64_t *acc = out + i * d;
    memset(acc, 0, d * 8);
    for (size_t j = 0; j < m; j++) {
      if (!nz[j]) continue;
#if defined(__x86_64__)
      if (use_simd)
        gl_mac_avx512(acc, matrix_ntt + (i * m + j) * d, s_ntt + j * d, d);
      else
#endif
        gl_mac_scalar(acc, matrix_ntt + (i * m + j) * d, s_ntt + j * d, d);
    }
    orc_nttgl_inverse_fast(t, acc, d);
  }
}

int orc_ajtaigl_commit_batch(const orc_nttgl *t, const uint64_t *matrix_ntt, size_t kappa,
                             size_t m, const uint64_t *w, size_t batch, uint64_t *out,
                             int nthreads, int simd) {
  size_t d = (size_t)1 << t->log_n;
  int use_simd = simd && orc_avx512_available();
  int nt = resolve_threads(nthreads);
  (void)nt;
#pragma omp parallel num_threads(nt)
  {
    uint64_t *s_ntt = (uint64_t *)malloc(m * d * 8);
    unsigned char *nz = (unsigned char *)malloc(m ? m : 1);
#pragma omp for schedule(dynamic, 1)
    for (long long b = 0; b < (long long)batch; b++)
      ajtaigl_commit_one(t, matrix_ntt, kappa, m, w + (size_t)b * m * d, s_ntt, nz,
                         out + (size_t)b * kappa * d, use_simd);
    free(s_ntt);
    free(nz);
  }
  return ORC_OK;
}

int orc_ajtaigl_commit_batch_i8(const orc_nttgl *t, const uint64_t *matrix_ntt, size_t kappa,
                                size_t m, const int8_t *w, size_t batch, uint64_t *out,
                                int nthreads, int simd) {
  size_t d = (size_t)1 << t->log_n;
  int use_simd = simd && orc_avx512_available();
  int nt = resolve_threads(nthreads);
  (void)nt;
#pragma omp parallel num_threads(nt)
  {
    uint64_t *s_ntt = (uint64_t *)malloc(m * d * 8);
    uint64_t *wf = (uint64_t *)malloc(m * d * 8);
    unsigned char *nz = (unsigned char *)malloc(m ? m : 1);
#pragma omp for schedule(dynamic, 1)
    for (long long b = 0; b < (long long)batch; b++) {
      const int8_t *src = w + (size_t)b * m * d;
      /* NeoRing::small (neo.rs:98-109): negative digits map to p - |x| */
      for (size_t x = 0; x < m * d; x++)
        wf[x] = src[x] >= 0 ? (uint64_t)src[x] : ORC_GL_P - (uint64_t)(-(int64_t)src[x]);
      ajtaigl_commit_one(t, matrix_ntt, kappa, m, wf, s_ntt, nz, out + (size_t)b * kappa * d,
                         use_simd);
    }
    free(s_ntt);
    free(wf);
    free(nz);
  }
  return ORC_OK;
}

/* ======================= Neo ring (neo.rs) =============================== */

/* NeoRing::mul, neo.rs:138-158 (zero coefficients of b skipped) */
void orc_neo_mul(size_t d, const uint64_t *a, const uint64_t *b, uint64_t *out) {
  uint64_t *acc = (uint64_t *)calloc(d, 8);
  for (size_t bi = 0; bi < d; bi++) {
    uint64_t bv = b[bi];
    if (bv == 0) continue;
    for (size_t aj = 0; aj < d; aj++) {
      size_t dst = aj + bi;
      uint64_t term = orc_gl_mul(a[aj], bv);
      if (dst < d)
        acc[dst] = orc_gl_add(acc[dst], term);
      else
        acc[dst - d] = orc_gl_sub(acc[dst - d], term);
    }
  }
  memcpy(out, acc, d * 8);
  free(acc);
}

/* NeoAjtaiKey::commit_naive, neo.rs:419-441; returns 1 on Shape error */
int orc_neo_commit_naive(size_t d, size_t kappa, size_t m, const uint64_t *matrix,
                         const uint64_t *cols, size_t ncols, uint64_t *out) {
  if (ncols > m) return 1;
  uint64_t *prod = (uint64_t *)malloc(d * 8);
  for (size_t i = 0; i < kappa; i++) {
    uint64_t *acc = out + i * d;
    memset(acc, 0, d * 8);
    for (size_t j = 0; j < ncols; j++) {
      orc_neo_mul(d, matrix + (i * m + j) * d, cols + j * d, prod);
      for (size_t x = 0; x < d; x++) acc[x] = orc_gl_add(acc[x], prod[x]);
    }
  }
  free(prod);
  return 0;
}

/* NeoAjtaiKey::commit_pay_per_bit, neo.rs:374-415 */
int orc_neo_commit_pay_per_bit(size_t d, size_t kappa, size_t m, const uint64_t *matrix,
                               const uint64_t *cols, size_t ncols, uint64_t *out,
                               uint64_t *column_adds) {
  if (ncols > m) return 1;
  uint64_t adds = 0;
  uint64_t *rot = (uint64_t *)malloc(d * 8);
  for (size_t i = 0; i < kappa; i++) {
    uint64_t *acc = out + i * d;
    memset(acc, 0, d * 8);
    for (size_t j = 0; j < ncols; j++) {
      const uint64_t *mij = matrix + (i * m + j) * d;
      for (size_t l = 0; l < d; l++) {
        uint64_t zl = cols[j * d + l];
        if (zl == 0) continue;
        adds++;
        for (size_t r = 0; r < d; r++) {
          size_t dst = r + l;
          if (dst < d)
            rot[dst] = mij[r];
          else
            rot[dst - d] = orc_gl_neg(mij[r]);
        }
        for (size_t x = 0; x < d; x++) acc[x] = orc_gl_add(acc[x], orc_gl_mul(zl, rot[x]));
      }
    }
  }
  free(rot);
  if (column_adds) *column_adds = adds;
  return 0;
}

/* decomp_b, neo.rs:253-266 */
void orc_decomp_b(const uint64_t *z, size_t len, uint32_t b_bits, uint64_t *out) {
  uint64_t b = (uint64_t)1 << b_bits;
  size_t rows = (64 + b_bits - 1) / b_bits;
  for (size_t j = 0; j < len; j++) {
    uint64_t x = z[j];
    for (size_t r = 0; r < rows; r++) {
      out[r * len + j] = orc_gl_from_u64(x % b);
      x /= b;
    }
  }
}

/* pack_field_elements, packing.rs:30-52: three 22-bit limbs per canonical
 * value (the top one < 2^20), chunked into ring elements of n coefficients
 * with zero padding, at least one element; RingElement::from_signed maps the
 * (non-negative) limbs to residues.  Returns the number of elements. */
size_t orc_pack_field_elements(uint32_t q, uint32_t log_n, const uint64_t *values, size_t count, uint32_t *out) {
  size_t n = (size_t)1 << log_n;
  size_t nl = 3 * count;
  size_t elems = (nl + n - 1) / n;
  if (elems == 0) elems = 1;
  uint64_t mask = ((uint64_t)1 << 22) - 1;
  for (size_t i = 0; i < elems * n; i++) {
    int64_t limb = 0;
    if (i < nl) {
      uint64_t raw = orc_gl_from_u64(values[i / 3]);
      size_t part = i % 3;
      limb = (int64_t)(part == 0 ? raw & mask : part == 1 ? (raw >> 22) & mask : raw >> 44);
    }
    out[i] = (uint32_t)(((limb % (int64_t)q) + (int64_t)q) % (int64_t)q);
  }
  return elems;
}

/* ============== Modulus50 + QuadSlotTables (modulus50.rs) ================= */

/* Modulus50::new, modulus50.rs:75-83 */
orc_mod50 orc_mod50_new(uint64_t q, uint32_t two_adicity, uint64_t generator) {
  orc_mod50 m;
  m.q = q;
  m.recip = UINT64_MAX / q;
  m.two_adicity = two_adicity;
  m.generator = generator;
  return m;
}

/* Modulus50::reduce_u128, modulus50.rs:90-118: fold 2^50 == 2^50 mod q (once
 * more if the result reaches 2^62), then one Barrett pass, <= 2 corrections. */
uint64_t orc_mod50_reduce_u128(const orc_mod50 *m, uint64_t xhi, uint64_t xlo) {
  u128 x = ((u128)xhi << 64) | xlo;
  u128 q = m->q;
  if (x < q) return (uint64_t)x;
  u128 fold = ((u128)1 << 50) % q;
  u128 mask = ((u128)1 << 50) - 1;
  u128 y = (x >> 50) * fold + (x & mask);
  if ((y >> 62) != 0) y = (y >> 50) * fold + (y & mask);
  u128 qhat = (y * (u128)m->recip) >> 64;
  u128 r = y - qhat * q;
  if (r >= q) r -= q;
  if (r >= q) r -= q;
  return (uint64_t)r;
}

/* mul :126-128, add :131-139, sub :142-149, pow :168-180 */
uint64_t orc_mod50_mul(const orc_mod50 *m, uint64_t a, uint64_t b) {
  u128 x = (u128)a * b;
  return orc_mod50_reduce_u128(m, (uint64_t)(x >> 64), (uint64_t)x);
}

uint64_t orc_mod50_add(const orc_mod50 *m, uint64_t a, uint64_t b) {
  uint64_t s = a + b;
  return s >= m->q ? s - m->q : s;
}

uint64_t orc_mod50_sub(const orc_mod50 *m, uint64_t a, uint64_t b) {
  return a >= b ? a - b : a + (m->q - b);
}

uint64_t orc_mod50_pow(const orc_mod50 *m, uint64_t base, uint64_t exp) {
  uint64_t acc = 1, b = base % m->q;
  while (exp > 0) {
    if (exp & 1) acc = orc_mod50_mul(m, acc, b);
    b = orc_mod50_mul(m, b, b);
    exp >>= 1;
  }
  return acc;
}

static size_t rev_bits50(size_t x, uint32_t bits) {
  size_t r = 0;
  for (uint32_t b = 0; b < bits; b++) r |= ((x >> b) & 1) << (bits - 1 - b);
  return r;
}

/* QuadSlotTables::new, modulus50.rs:250-301 */
int orc_quad50_new(orc_mod50 m, uint32_t log_n, orc_quad50 *out) {
  memset(out, 0, sizeof(*out));
  if (log_n == 0 || log_n > 7) return ORC_ERR_LOG_N_OUT_OF_RANGE;
  if (m.two_adicity < 7) return ORC_ERR_ADICITY_TOO_SMALL;
  uint64_t zeta = orc_mod50_pow(&m, m.generator, (m.q - 1) >> 7); /* root_of_unity(7), :191-197 */
  if (orc_mod50_pow(&m, zeta, 64) != m.q - 1) return ORC_ERR_GENERATOR_INVALID;
  size_t slots = (size_t)1 << (log_n - 1);
  out->modulus = m;
  out->log_n = log_n;
  out->zeta = zeta;
  out->level_tw = (uint64_t *)calloc(slots, sizeof(uint64_t));
  out->level_tw_inv = (uint64_t *)calloc(slots, sizeof(uint64_t));
  out->leaf_gamma = (uint64_t *)calloc(slots, sizeof(uint64_t));
  for (uint32_t d = 0; d + 1 < log_n; d++) {
    uint32_t shift = 5 - d;
    for (size_t i = 0; i < ((size_t)1 << d); i++) {
      uint64_t e = ((2 * (uint64_t)rev_bits50(i, d) + 1) << shift) % 128;
      uint64_t w = orc_mod50_pow(&m, zeta, e);
      out->level_tw[((size_t)1 << d) - 1 + i] = w;
      out->level_tw_inv[((size_t)1 << d) - 1 + i] = orc_mod50_pow(&m, w, m.q - 2); /* inv, :183-189 */
    }
  }
  uint32_t leaf_shift = 7 - log_n;
  for (size_t p = 0; p < slots; p++) {
    uint64_t e = ((2 * (uint64_t)rev_bits50(p, log_n - 1) + 1) << leaf_shift) % 128;
    out->leaf_gamma[p] = orc_mod50_pow(&m, zeta, e);
  }
  return ORC_OK;
}

void orc_quad50_free(orc_quad50 *t) {
  free(t->level_tw);
  free(t->level_tw_inv);
  free(t->leaf_gamma);
  memset(t, 0, sizeof(*t));
}

/* forward, modulus50.rs:313-334 */
int orc_quad50_forward(const orc_quad50 *t, uint64_t *a, size_t len) {
  size_t n = (size_t)1 << t->log_n;
  if (len != n) return ORC_ERR_LENGTH_MISMATCH;
  const orc_mod50 *q = &t->modulus;
  for (uint32_t d = 0; d + 1 < t->log_n; d++) {
    size_t span = n >> d, half = span / 2;
    for (size_t i = 0; i < ((size_t)1 << d); i++) {
      uint64_t w = t->level_tw[((size_t)1 << d) - 1 + i];
      size_t start = i * span;
      for (size_t j = 0; j < half; j++) {
        uint64_t lo = a[start + j], hi = a[start + j + half];
        a[start + j] = orc_mod50_add(q, lo, orc_mod50_mul(q, w, hi));
        a[start + j + half] = orc_mod50_sub(q, lo, orc_mod50_mul(q, w, hi));
      }
    }
  }
  return ORC_OK;
}

/* inverse, modulus50.rs:338-364 */
int orc_quad50_inverse(const orc_quad50 *t, uint64_t *a, size_t len) {
  size_t n = (size_t)1 << t->log_n;
  if (len != n) return ORC_ERR_LENGTH_MISMATCH;
  const orc_mod50 *q = &t->modulus;
  uint64_t inv2 = orc_mod50_pow(q, 2, q->q - 2);
  for (int d = (int)t->log_n - 2; d >= 0; d--) {
    size_t span = n >> d, half = span / 2;
    for (size_t i = 0; i < ((size_t)1 << d); i++) {
      uint64_t w_inv = t->level_tw_inv[((size_t)1 << d) - 1 + i];
      size_t start = i * span;
      for (size_t j = 0; j < half; j++) {
        uint64_t lo = a[start + j], hi = a[start + j + half];
        uint64_t sum = orc_mod50_add(q, lo, hi);
        uint64_t diff = orc_mod50_sub(q, lo, hi);
        uint64_t half_diff = orc_mod50_mul(q, diff, inv2);
        a[start + j] = orc_mod50_mul(q, sum, inv2);
        a[start + j + half] = orc_mod50_mul(q, half_diff, w_inv);
      }
    }
  }
  return ORC_OK;
}

/* slotwise_mul, modulus50.rs:368-392 (Karatsuba per quadratic slot) */
int orc_quad50_slotwise_mul(const orc_quad50 *t, const uint64_t *a, const uint64_t *b, uint64_t *out,
                            size_t len) {
  size_t n = (size_t)1 << t->log_n;
  if (len != n) return ORC_ERR_LENGTH_MISMATCH;
  const orc_mod50 *q = &t->modulus;
  for (size_t p = 0; p < n / 2; p++) {
    uint64_t u0 = a[2 * p], u1 = a[2 * p + 1], v0 = b[2 * p], v1 = b[2 * p + 1];
    uint64_t g = t->leaf_gamma[p];
    uint64_t p0 = orc_mod50_mul(q, u0, v0);
    uint64_t p1 = orc_mod50_mul(q, u1, v1);
    uint64_t cross = orc_mod50_mul(q, orc_mod50_add(q, u0, u1), orc_mod50_add(q, v0, v1));
    out[2 * p] = orc_mod50_add(q, p0, orc_mod50_mul(q, g, p1));
    out[2 * p + 1] = orc_mod50_sub(q, cross, orc_mod50_add(q, p0, p1));
  }
  return ORC_OK;
}

/* mul, modulus50.rs:395-411 */
int orc_quad50_mul(const orc_quad50 *t, const uint64_t *a, const uint64_t *b, uint64_t *out, size_t len) {
  size_t n = (size_t)1 << t->log_n;
  if (len != n) return ORC_ERR_LENGTH_MISMATCH;
  uint64_t ta[128], tb[128];
  memcpy(ta, a, n * 8);
  memcpy(tb, b, n * 8);
  orc_quad50_forward(t, ta, n);
  orc_quad50_forward(t, tb, n);
  orc_quad50_slotwise_mul(t, ta, tb, out, n);
  return orc_quad50_inverse(t, out, n);
}

int orc_quad50_mul_batch(const orc_quad50 *t, const uint64_t *a, const uint64_t *b, uint64_t *out,
                         size_t count, int nthreads) {
  size_t n = (size_t)1 << t->log_n;
  int nt = resolve_threads(nthreads);
  (void)nt;
#pragma omp parallel for schedule(static) num_threads(nt)
  for (long long i = 0; i < (long long)count; i++)
    orc_quad50_mul(t, a + (size_t)i * n, b + (size_t)i * n, out + (size_t)i * n, n);
  return ORC_OK;
}

/* GadgetDecomposition::decompose, decomposition.rs:48-70 */
int orc_gadget_decompose(uint64_t base, size_t num_digits, uint64_t x, int64_t *out) {
  u128 rem = x;
  int64_t half = (int64_t)(base / 2);
  for (size_t i = 0; i < num_digits; i++) {
    int64_t digit = (int64_t)(rem % base);
    int64_t dd = digit > half ? digit - (int64_t)base : digit;
    __int128 r = (__int128)rem - dd;
    rem = (u128)(r / (__int128)base);
    out[i] = dd;
  }
  return rem != 0 ? 1 : 0;
}

/* ======================= Keccak (keccak.rs; FIPS 202) ==================== */

/* Round constants and rho offsets are generated from their FIPS 202
 * definitions (the rc(t) LFSR and the (x,y) -> (y, 2x+3y) walk). */
static uint64_t K_RC[24];
static unsigned K_RHO[25];
static int k_init_done = 0;

static int rc_bit(unsigned t) {
  unsigned m = t % 255;
  if (m == 0) return 1;
  unsigned r = 0x80; /* R = 10000000 with R[0] the MSB of this byte */
  for (unsigned i = 1; i <= m; i++) {
    /* R = 0 || R (9 bits); R[0]^=R[8]; R[4]^=R[8]; R[5]^=R[8]; R[6]^=R[8]; truncate */
    unsigned r9 = r; /* bit positions: R[k] is bit (7-k) of r before shift */
    unsigned bits[9];
    bits[0] = 0;
    for (int k = 0; k < 8; k++) bits[k + 1] = (r9 >> (7 - k)) & 1;
    unsigned r8 = bits[8];
    bits[0] ^= r8;
    bits[4] ^= r8;
    bits[5] ^= r8;
    bits[6] ^= r8;
    r = 0;
    for (int k = 0; k < 8; k++) r |= bits[k] << (7 - k);
  }
  return (r >> 7) & 1;
}

static void keccak_init(void) {
  if (k_init_done) return;
  for (unsigned ir = 0; ir < 24; ir++) {
    uint64_t rc = 0;
    for (unsigned j = 0; j <= 6; j++)
      if (rc_bit(j + 7 * ir)) rc |= (uint64_t)1 << ((1u << j) - 1);
    K_RC[ir] = rc;
  }
  K_RHO[0] = 0;
  unsigned x = 1, y = 0;
  for (unsigned t = 0; t < 24; t++) {
    K_RHO[x + 5 * y] = ((t + 1) * (t + 2) / 2) % 64;
    unsigned nx = y, ny = (2 * x + 3 * y) % 5;
    x = nx;
    y = ny;
  }
  k_init_done = 1;
}

static inline uint64_t rotl64(uint64_t v, unsigned r) { return r ? (v << r) | (v >> (64 - r)) : v; }

/* keccak_f1600, keccak.rs:52 (theta, rho, pi, chi, iota; 24 rounds) */
void orc_keccak_f1600(uint64_t a[25]) {
  keccak_init();
  for (int round = 0; round < 24; round++) {
    uint64_t c[5], d[5], b[25];
    for (int x = 0; x < 5; x++) c[x] = a[x] ^ a[x + 5] ^ a[x + 10] ^ a[x + 15] ^ a[x + 20];
    for (int x = 0; x < 5; x++) d[x] = c[(x + 4) % 5] ^ rotl64(c[(x + 1) % 5], 1);
    for (int i = 0; i < 25; i++) a[i] ^= d[i % 5];
    /* rho + pi: B[y, 2x+3y] = rot(A[x,y], r[x,y]) */
    for (int x = 0; x < 5; x++)
      for (int y = 0; y < 5; y++) b[y + 5 * ((2 * x + 3 * y) % 5)] = rotl64(a[x + 5 * y], K_RHO[x + 5 * y]);
    for (int y = 0; y < 5; y++)
      for (int x = 0; x < 5; x++)
        a[x + 5 * y] = b[x + 5 * y] ^ (~b[(x + 1) % 5 + 5 * y] & b[(x + 2) % 5 + 5 * y]);
    a[0] ^= K_RC[round];
  }
}

/* KeccakSponge absorb / pad10*1 / squeeze, keccak.rs:250-340 */
static void sponge(const uint8_t *in, size_t len, uint8_t suffix, size_t rate, uint8_t *out,
                   size_t out_len) {
  uint64_t st[25];
  memset(st, 0, sizeof(st));
  size_t pos = 0;
  for (size_t i = 0; i < len; i++) {
    st[pos / 8] ^= (uint64_t)in[i] << (8 * (pos % 8));
    if (++pos == rate) {
      orc_keccak_f1600(st);
      pos = 0;
    }
  }
  st[pos / 8] ^= (uint64_t)suffix << (8 * (pos % 8));
  st[(rate - 1) / 8] ^= (uint64_t)0x80 << (8 * ((rate - 1) % 8));
  orc_keccak_f1600(st);
  size_t done = 0;
  while (done < out_len) {
    size_t take = rate < out_len - done ? rate : out_len - done;
    for (size_t i = 0; i < take; i++) out[done + i] = (uint8_t)(st[i / 8] >> (8 * (i % 8)));
    done += take;
    if (done < out_len) orc_keccak_f1600(st);
  }
}

void orc_sha3_256(const uint8_t *in, size_t len, uint8_t out[32]) { sponge(in, len, 0x06, 136, out, 32); }

void orc_shake256(const uint8_t *in, size_t len, uint8_t *out, size_t out_len) {
  sponge(in, len, 0x1f, 136, out, out_len);
}

static size_t frame(uint8_t *buf, const char *tag, const uint8_t *domain, size_t dlen,
                    const uint8_t *msg, size_t mlen) {
  size_t p = 0;
  memcpy(buf, tag, 4);
  p += 4;
  uint32_t dl = (uint32_t)dlen, ml = (uint32_t)mlen;
  for (int i = 0; i < 4; i++) buf[p++] = (uint8_t)(dl >> (8 * i));
  memcpy(buf + p, domain, dlen);
  p += dlen;
  for (int i = 0; i < 4; i++) buf[p++] = (uint8_t)(ml >> (8 * i));
  memcpy(buf + p, msg, mlen);
  p += mlen;
  return p;
}

/* Transcript::xof, transcript.rs:229-237 */
void orc_xof(const uint8_t *domain, size_t dlen, const uint8_t *msg, size_t mlen, uint8_t *out,
             size_t out_len) {
  uint8_t *buf = (uint8_t *)malloc(12 + dlen + mlen);
  size_t l = frame(buf, "LZXX", domain, dlen, msg, mlen);
  orc_shake256(buf, l, out, out_len);
  free(buf);
}

/* Transcript::hash_domain, transcript.rs:218-226 */
void orc_hash_domain(const uint8_t *domain, size_t dlen, const uint8_t *msg, size_t mlen,
                     uint8_t out[32]) {
  uint8_t *buf = (uint8_t *)malloc(12 + dlen + mlen);
  size_t l = frame(buf, "LZXD", domain, dlen, msg, mlen);
  orc_sha3_256(buf, l, out);
  free(buf);
}

static uint32_t le32(const uint8_t *p) {
  return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}

/* RingConfig::uniform_from_seed, ring.rs:102-180 (one squeeze of
 * 8 + 4(n + slack) bytes, windows from offset 8; counter fallback) */
void orc_uniform_from_seed(const orc_mod32 *m, uint32_t log_n, const uint8_t *domain, size_t dlen,
                           const uint8_t *seed, size_t slen, uint64_t index, uint32_t *out) {
  size_t n = (size_t)1 << log_n;
  uint8_t *salt = (uint8_t *)malloc(dlen + slen + 8);
  memcpy(salt, domain, dlen);
  memcpy(salt + dlen, seed, slen);
  for (int i = 0; i < 8; i++) salt[dlen + slen + i] = (uint8_t)(index >> (8 * i));
  size_t saltlen = dlen + slen + 8;
  uint64_t q = m->q;
  uint64_t limit = ((uint64_t)1 << 32) - (((uint64_t)1 << 32) % q);
  size_t slack = n > 16 ? n : 16;
  size_t slen_total = 8 + 4 * (n + slack);
  uint8_t *stream = (uint8_t *)malloc(slen_total);
  orc_xof((const uint8_t *)"uniform", 7, salt, saltlen, stream, slen_total);
  size_t got = 0;
  for (size_t w = 0; w < n + slack && got < n; w++) {
    uint64_t cand = le32(stream + 8 + 4 * w);
    if (cand < limit) out[got++] = (uint32_t)(cand % q);
  }
  size_t counter = (slen_total - 8) / 4;
  while (got < n) {
    size_t l = 8 + counter * 4 + 4;
    uint8_t *bytes = (uint8_t *)malloc(l);
    orc_xof((const uint8_t *)"uniform", 7, salt, saltlen, bytes, l);
    uint64_t cand = le32(bytes + l - 4);
    if (cand < limit) out[got++] = (uint32_t)(cand % q);
    counter++;
    free(bytes);
  }
  free(stream);
  free(salt);
}

/* RingConfig::random, ring.rs:83-98 */
void orc_ring_random(const orc_mod32 *m, uint32_t log_n, const uint8_t *seed, size_t slen,
                     uint32_t *out) {
  size_t n = (size_t)1 << log_n;
  uint8_t *bytes = (uint8_t *)malloc(n * 4);
  orc_xof((const uint8_t *)"ring-random", 11, seed, slen, bytes, n * 4);
  for (size_t i = 0; i < n; i++) out[i] = orc_mod32_reduce_u64(m, le32(bytes + 4 * i));
  free(bytes);
}

/* AjtaiPublicKey::from_seed, ajtai.rs:87-103 */
int orc_ajtai32_from_seed(const orc_ntt32 *t, size_t k, size_t m, const uint8_t seed[32],
                          uint32_t *matrix, uint32_t *matrix_ntt) {
  size_t n = (size_t)1 << t->log_n;
  for (size_t i = 0; i < k * m; i++) {
    orc_uniform_from_seed(&t->modulus, t->log_n, (const uint8_t *)"ajtai-A", 7, seed, 32, i,
                          matrix + i * n);
    memcpy(matrix_ntt + i * n, matrix + i * n, n * 4);
    orc_ntt32_forward_fast(t, matrix_ntt + i * n, n);
  }
  return ORC_OK;
}

/* sample_small_secret, ajtai.rs:307-348 */
void orc_sample_small_secret(const orc_mod32 *mod, uint32_t log_n, size_t m, uint32_t bound,
                             const uint8_t *seed, size_t slen, uint32_t *out) {
  size_t n = (size_t)1 << log_n;
  uint64_t span = 2 * (uint64_t)bound + 1;
  uint64_t limit = ((uint64_t)UINT32_MAX / span) * span;
  size_t blen = n * 16 > 64 ? n * 16 : 64;
  uint8_t *input = (uint8_t *)malloc(slen + 16);
  uint8_t *bytes = (uint8_t *)malloc(blen);
  for (size_t i = 0; i < m; i++) {
    size_t got = 0;
    uint64_t sc = 0;
    while (got < n) {
      memcpy(input, seed, slen);
      for (int b = 0; b < 8; b++) input[slen + b] = (uint8_t)((uint64_t)i >> (8 * b));
      for (int b = 0; b < 8; b++) input[slen + 8 + b] = (uint8_t)(sc >> (8 * b));
      orc_xof((const uint8_t *)"ajtai-secret", 12, input, slen + 16, bytes, blen);
      for (size_t c = 0; c + 4 <= blen && got < n; c += 4) {
        uint64_t v = le32(bytes + c);
        if (v < limit) {
          uint64_t bb = v % span;
          out[i * n + got++] = orc_mod32_reduce_i64(mod, (int64_t)bb - (int64_t)bound);
        }
      }
      sc++;
    }
  }
  free(input);
  free(bytes);
}

/* ======================= Synthetic inputs ================================ */

static inline uint64_t mix64(uint64_t z) {
  z ^= z >> 30;
  z *= 0xBF58476D1CE4E5B9ull;
  z ^= z >> 27;
  z *= 0x94D049BB133111EBull;
  z ^= z >> 31;
  return z;
}

uint64_t orc_synth_u64(uint64_t seed, uint64_t stream, uint64_t index) {
  uint64_t base = mix64(seed * 0x9E3779B97F4A7C15ull + stream * 0xC2B2AE3D27D4EB4Full +
                        0x165667B19E3779F9ull);
  return mix64(base + index * 0x9E3779B97F4A7C15ull);
}

/* retry r of element i reads stream + (r << 40) */
void orc_synth_mod32(uint64_t seed, uint64_t stream, uint32_t q, uint32_t *out, size_t count,
                     size_t offset) {
  uint64_t limit = ((uint64_t)1 << 32) - (((uint64_t)1 << 32) % q);
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < count; i++) {
    for (uint64_t r = 0;; r++) {
      uint64_t c = orc_synth_u64(seed, stream + (r << 40), offset + i) & 0xFFFFFFFFull;
      if (c < limit) {
        out[i] = (uint32_t)(c % q);
        break;
      }
    }
  }
}

void orc_synth_gl(uint64_t seed, uint64_t stream, uint64_t *out, size_t count, size_t offset) {
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < count; i++) {
    for (uint64_t r = 0;; r++) {
      uint64_t c = orc_synth_u64(seed, stream + (r << 40), offset + i);
      if (c < ORC_GL_P) {
        out[i] = c;
        break;
      }
    }
  }
}

void orc_synth_i8(uint64_t seed, uint64_t stream, int8_t *out, size_t count, size_t offset) {
  for (size_t i = 0; i < count; i++) out[i] = (int8_t)(uint8_t)orc_synth_u64(seed, stream, offset + i);
}
