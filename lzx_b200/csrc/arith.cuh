// arith.cuh -- exact modular arithmetic for the NTT butterflies (device side).
//
// Three policies share one interface so that one kernel template serves every
// modulus family of the reference's NTT (lattice-ring/src/ntt.rs) :
//
//   ShoupLazy  : u32 primes q < 2^30 (the CRT set).  Harvey butterflies with
//                operands kept lazily in [0,4q) (forward) / [0,2q) (inverse);
//                twiddle products by Shoup's method with a precomputed
//                floor(w*2^32/q).  4q < 2^32, so nothing overflows.
//   MontCanon  : any odd u32 prime (Modulus32::Q_32 = 3*2^30+1 has no lazy
//                headroom).  Signed Montgomery reduction with R = 2^32 and
//                twiddles stored as w*R mod q; every value stays in [0,q).
//   Goldilocks : p = 2^64 - 2^32 + 1 with 2^64 == 2^32 - 1 folding
//                (lattice-core/src/field.rs:38-55); values in [0,p).
//
// All three return canonical residues, so the transforms are bit-identical to
// the reference's Barrett / u128 arithmetic (ntt.rs:118-216).
#pragma once

#include <stdint.h>

#include "common.cuh"

namespace lc {

// ------------------------------------------------------------- u32, lazy

struct ShoupLazy {
  using T = uint32_t;
  using Tw = uint2;  // {w, floor(w * 2^32 / q)}
  uint32_t q, q2;

  LC_D explicit ShoupLazy(uint32_t q_) : q(q_), q2(2 * q_) {}

  // a*w mod q in [0, 2q) for any a < 2^32 (q < 2^31).
  LC_D uint32_t mulw(uint32_t a, Tw w) const {
    uint32_t qh = __umulhi(a, w.y);
    return a * w.x - qh * q;
  }
  // Cooley-Tukey (forward) butterfly: X,Y in [0,4q) -> [0,4q).
  LC_D void fwd(uint32_t& x, uint32_t& y, Tw w) const {
    uint32_t X = min(x, x - q2);  // [0,2q)
    uint32_t t = mulw(y, w);      // [0,2q)
    x = X + t;
    y = X - t + q2;
  }
  // First forward level: canonical inputs need no correction of X.
  LC_D void fwd_first(uint32_t& x, uint32_t& y, Tw w) const {
    uint32_t X = x;
    uint32_t t = mulw(y, w);
    x = X + t;
    y = X - t + q2;
  }
  // Gentleman-Sande (inverse) butterfly: X,Y in [0,2q) -> [0,2q).
  LC_D void inv(uint32_t& x, uint32_t& y, Tw w) const {
    uint32_t s = x + y;
    uint32_t d = x - y + q2;
    x = min(s, s - q2);
    y = mulw(d, w);
  }
  // First inverse level: canonical inputs, so X + Y < 2q already.
  LC_D void inv_first(uint32_t& x, uint32_t& y, Tw w) const {
    uint32_t s = x + y;
    uint32_t d = x - y + q2;
    x = s;
    y = mulw(d, w);
  }
  // Last inverse level fused with the n^{-1} scaling: X,Y in [0,2q).
  LC_D void inv_last(uint32_t& x, uint32_t& y, Tw ninv, Tw wninv) const {
    uint32_t s = x + y;        // [0,4q)
    uint32_t d = x - y + q2;   // (0,4q)
    x = mulw(s, ninv);
    y = mulw(d, wninv);
  }
  LC_D void scale(uint32_t& x, Tw c) const { x = mulw(x, c); }
  LC_D uint32_t fwd_final(uint32_t x) const {
    x = min(x, x - q2);
    return min(x, x - q);
  }
  LC_D uint32_t inv_final(uint32_t x) const { return min(x, x - q); }
};

// ------------------------------------------------------------- u32, canonical Montgomery

struct MontCanon {
  using T = uint32_t;
  using Tw = uint2;  // {w * 2^32 mod q, unused}
  uint32_t q, qinv;  // qinv = q^{-1} mod 2^32

  LC_D MontCanon(uint32_t q_, uint32_t qinv_) : q(q_), qinv(qinv_) {}

  // a * wR * 2^-32 mod q, canonical, for a, wR < q.
  LC_D uint32_t mont(uint32_t a, uint32_t wR) const {
    uint64_t t = (uint64_t)a * wR;
    uint32_t m = (uint32_t)t * qinv;
    uint32_t th = (uint32_t)(t >> 32);
    uint32_t mh = __umulhi(m, q);
    uint32_t r = th - mh;
    return th < mh ? r + q : r;
  }
  LC_D uint32_t add(uint32_t a, uint32_t b) const {
    uint32_t s = a + b;
    return (s < a || s >= q) ? s - q : s;
  }
  LC_D uint32_t sub(uint32_t a, uint32_t b) const {
    uint32_t d = a - b;
    return a < b ? d + q : d;
  }
  LC_D void fwd(uint32_t& x, uint32_t& y, Tw w) const {
    uint32_t t = mont(y, w.x);
    uint32_t X = x;
    x = add(X, t);
    y = sub(X, t);
  }
  LC_D void inv(uint32_t& x, uint32_t& y, Tw w) const {
    uint32_t X = x, Y = y;
    x = add(X, Y);
    y = mont(sub(X, Y), w.x);
  }
  LC_D void fwd_first(uint32_t& x, uint32_t& y, Tw w) const { fwd(x, y, w); }
  LC_D void inv_first(uint32_t& x, uint32_t& y, Tw w) const { inv(x, y, w); }
  LC_D void inv_last(uint32_t& x, uint32_t& y, Tw ninv, Tw wninv) const {
    uint32_t X = x, Y = y;
    x = mont(add(X, Y), ninv.x);
    y = mont(sub(X, Y), wninv.x);
  }
  LC_D void scale(uint32_t& x, Tw c) const { x = mont(x, c.x); }
  LC_D uint32_t fwd_final(uint32_t x) const { return x; }
  LC_D uint32_t inv_final(uint32_t x) const { return x; }
};

// ------------------------------------------------------------- Goldilocks

constexpr uint64_t kGlP = 0xFFFFFFFF00000001ull;
constexpr uint64_t kGlEps = 0xFFFFFFFFull;  // 2^64 mod p

// 128-bit product a*b as (hi, lo).
LC_D void mul64x64(uint64_t a, uint64_t b, uint64_t& hi, uint64_t& lo) {
  lo = a * b;
  hi = __umul64hi(a, b);
}

// Reduce hi*2^64 + lo into [0, 2^64) (congruent mod p, not yet canonical):
// hi = hh*2^32 + hl, 2^64 == 2^32-1, 2^96 == -1.
LC_D uint64_t gl_reduce128_lazy(uint64_t hi, uint64_t lo) {
  uint32_t hh = (uint32_t)(hi >> 32);
  uint32_t hl = (uint32_t)hi;
  uint64_t t0 = lo - hh;
  if (lo < hh) t0 -= kGlEps;                  // borrowed 2^64 == 2^32-1
  uint64_t t1 = ((uint64_t)hl << 32) - hl;    // hl * (2^32-1)
  uint64_t r = t0 + t1;
  if (r < t1) r += kGlEps;                    // carried 2^64 == 2^32-1
  return r;
}

LC_D uint64_t gl_canon(uint64_t x) { return x >= kGlP ? x - kGlP : x; }

// a * b mod p, canonical, for any a, b < 2^64: the 128-bit product from four
// 32x32 partial products, then p3:p2:p1:p0 == (p1:p0) - p3 + p2 (2^32 - 1),
// each wrap of 2^64 folded as 2^64 == 2^32 - 1, and r >= p  <=>  r + eps
// carries out of 64 bits (that sum minus 2^64 is r - p).
LC_D uint64_t gl_mul(uint64_t a, uint64_t b) {
  uint32_t r0, r1;
  asm("{\n\t"
      ".reg .u32 a0, a1, b0, b1, p0, p1, p2, p3, m, u0, u1, c, t0, t1, e;\n\t"
      ".reg .pred q;\n\t"
      "mov.b64 {a0, a1}, %2;\n\t"
      "mov.b64 {b0, b1}, %3;\n\t"
      "mov.u32 e, 0xFFFFFFFF;\n\t"
      "mul.lo.u32 p0, a0, b0;\n\t"
      "mul.hi.u32 p1, a0, b0;\n\t"
      "mul.lo.u32 p2, a1, b1;\n\t"
      "mul.hi.u32 p3, a1, b1;\n\t"
      "mad.lo.cc.u32 p1, a0, b1, p1;\n\t"
      "madc.hi.cc.u32 p2, a0, b1, p2;\n\t"
      "addc.u32 p3, p3, 0;\n\t"
      "mad.lo.cc.u32 p1, a1, b0, p1;\n\t"
      "madc.hi.cc.u32 p2, a1, b0, p2;\n\t"
      "addc.u32 p3, p3, 0;\n\t"
      // (p1:p0) - p3; a borrow wrapped by +2^64, so subtract eps
      "sub.cc.u32 p0, p0, p3;\n\t"
      "subc.cc.u32 p1, p1, 0;\n\t"
      "subc.u32 m, 0, 0;\n\t"
      "sub.cc.u32 p0, p0, m;\n\t"
      "subc.u32 p1, p1, 0;\n\t"
      // + p2 * 2^32 - p2; a carry lost 2^64, so add eps
      "sub.cc.u32 u0, 0, p2;\n\t"
      "subc.u32 u1, p2, 0;\n\t"
      "add.cc.u32 p0, p0, u0;\n\t"
      "addc.cc.u32 p1, p1, u1;\n\t"
      "addc.u32 c, 0, 0;\n\t"
      "mad.lo.cc.u32 p0, c, e, p0;\n\t"
      "addc.u32 p1, p1, 0;\n\t"
      // canonical
      "add.cc.u32 t0, p0, e;\n\t"
      "addc.cc.u32 t1, p1, 0;\n\t"
      "addc.u32 c, 0, 0;\n\t"
      "setp.ne.u32 q, c, 0;\n\t"
      "selp.b32 %0, t0, p0, q;\n\t"
      "selp.b32 %1, t1, p1, q;\n\t"
      "}"
      : "=r"(r0), "=r"(r1)
      : "l"(a), "l"(b));
  return ((uint64_t)r1 << 32) | r0;
}

// Canonical inputs -> canonical output.
LC_D uint64_t gl_add(uint64_t a, uint64_t b) {
  uint64_t s = a + b;
  if (s < a) s += kGlEps;  // cannot carry again for a, b < p
  return gl_canon(s);
}

LC_D uint64_t gl_sub(uint64_t a, uint64_t b) {
  uint64_t d = a - b;
  if (a < b) d -= kGlEps;  // == d + p (mod 2^64); no second borrow for b < p
  return d;                // a, b < p  =>  result < p; any a  =>  congruent, in [0, 2^64)
}

// a + b for any a and b < p: congruent, in [0, 2^64) -- a + b - 2^64 + eps = a + b - p < a
LC_D uint64_t gl_add_lazy(uint64_t a, uint64_t b) {
  uint32_t r0, r1;
  asm("{\n\t"
      ".reg .u32 a0, a1, b0, b1, c, e;\n\t"
      "mov.b64 {a0, a1}, %2;\n\t"
      "mov.b64 {b0, b1}, %3;\n\t"
      "mov.u32 e, 0xFFFFFFFF;\n\t"
      "add.cc.u32 %0, a0, b0;\n\t"
      "addc.cc.u32 %1, a1, b1;\n\t"
      "addc.u32 c, 0, 0;\n\t"
      "mad.lo.cc.u32 %0, c, e, %0;\n\t"
      "addc.u32 %1, %1, 0;\n\t"
      "}"
      : "=r"(r0), "=r"(r1)
      : "l"(a), "l"(b));
  return ((uint64_t)r1 << 32) | r0;
}

// a - b for any a and b < p: congruent, in [0, 2^64) (a borrow wrapped by
// +2^64 == eps, so eps is taken off again; that cannot borrow for b < p)
LC_D uint64_t gl_sub_lazy(uint64_t a, uint64_t b) {
  uint32_t r0, r1;
  asm("{\n\t"
      ".reg .u32 a0, a1, b0, b1, m;\n\t"
      "mov.b64 {a0, a1}, %2;\n\t"
      "mov.b64 {b0, b1}, %3;\n\t"
      "sub.cc.u32 %0, a0, b0;\n\t"
      "subc.cc.u32 %1, a1, b1;\n\t"
      "subc.u32 m, 0, 0;\n\t"
      "sub.cc.u32 %0, %0, m;\n\t"
      "subc.u32 %1, %1, 0;\n\t"
      "}"
      : "=r"(r0), "=r"(r1)
      : "l"(a), "l"(b));
  return ((uint64_t)r1 << 32) | r0;
}

struct Goldilocks {
  using T = uint64_t;
  using Tw = uint64_t;

  LC_D Goldilocks() {}
  // Forward values are lazy (any u64 congruent to the canonical one): the
  // product t = y * w is canonical, so x + t and x - t need one fold each,
  // and fwd_final makes the output canonical.
  LC_D void fwd(uint64_t& x, uint64_t& y, Tw w) const {
    const uint64_t t = gl_mul(y, w);
    const uint64_t X = x;
    x = gl_add_lazy(X, t);
    y = gl_sub_lazy(X, t);
  }
  LC_D void inv(uint64_t& x, uint64_t& y, Tw w) const {
    uint64_t X = x, Y = y;
    x = gl_add(X, Y);
    y = gl_mul(gl_sub(X, Y), w);
  }
  LC_D void fwd_first(uint64_t& x, uint64_t& y, Tw w) const { fwd(x, y, w); }
  LC_D void inv_first(uint64_t& x, uint64_t& y, Tw w) const { inv(x, y, w); }
  LC_D void inv_last(uint64_t& x, uint64_t& y, Tw ninv, Tw wninv) const {
    uint64_t X = x, Y = y;
    x = gl_mul(gl_add(X, Y), ninv);
    y = gl_mul(gl_sub(X, Y), wninv);
  }
  LC_D void scale(uint64_t& x, Tw c) const { x = gl_mul(x, c); }
  LC_D uint64_t fwd_final(uint64_t x) const { return gl_canon(x); }
  LC_D uint64_t inv_final(uint64_t x) const { return x; }
};

}  // namespace lc
