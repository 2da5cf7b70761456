// mac.cuh -- exact multiply-accumulate of residues for the commit products.
//
// A 160-bit accumulator takes up to 2^32 products of 64-bit (Goldilocks) or
// 32-bit residues without overflow; acc_reduce folds it to a canonical
// residue once per sum.  Shared by the cached-NTT commit (commit.cu) and the
// batch engine (batch.cu).
#pragma once

#include "arith.cuh"
#include "common.cuh"

namespace lc {

constexpr int kIPad = 16;  // rows of A per product tile (padded with zero rows)

// ------------------------------------------------------------------ element traits

template <class E>
struct Field;

template <>
struct Field<uint64_t> {  // Goldilocks
  LC_D static uint64_t reduce160(uint32_t r0, uint32_t r1, uint32_t r2, uint32_t r3, uint32_t r4,
                                 uint32_t) {
    // x = (r3 r2)*2^64 + (r1 r0) + r4*2^128;  2^128 == -2^32 (mod p)
    uint64_t lo = ((uint64_t)r1 << 32) | r0;
    uint64_t hi = ((uint64_t)r3 << 32) | r2;
    uint64_t y = gl_canon(gl_reduce128_lazy(hi, lo));
    uint64_t z = gl_canon(((uint64_t)r4 << 32) % kGlP);  // r4 * 2^32 < 2^64
    return gl_sub(y, z);
  }
  LC_D static uint64_t add(uint64_t a, uint64_t b, uint32_t) { return gl_add(a, b); }
};

template <>
struct Field<uint32_t> {  // any odd u32 modulus q
  LC_D static uint32_t reduce160(uint32_t r0, uint32_t r1, uint32_t r2, uint32_t r3, uint32_t r4,
                                 uint32_t q) {
    // products are < 2^64 and at most 2^32 of them are summed: r3 = r4 = 0 is
    // not assumed; fold limb by limb from the top with 64-bit remainders.
    uint64_t acc = r4 % q;
    acc = ((acc << 32) | r3) % q;
    acc = ((acc << 32) | r2) % q;
    acc = ((acc << 32) | r1) % q;
    acc = ((acc << 32) | r0) % q;
    return (uint32_t)acc;
  }
  LC_D static uint32_t add(uint32_t a, uint32_t b, uint32_t q) {
    uint32_t s = a + b;
    return (s < a || s >= q) ? s - q : s;
  }
};

// 160-bit accumulator: outer products a0*b0 and a1*b1 into r0..r4, the two
// middle products into m0..m2 (added at 2^32 when the sum is reduced).
struct Acc160 {
  uint32_t r0 = 0, r1 = 0, r2 = 0, r3 = 0, r4 = 0, m0 = 0, m1 = 0, m2 = 0;
};

LC_D void mac64(Acc160& c, uint64_t a, uint64_t b) {
  const uint32_t a0 = (uint32_t)a, a1 = (uint32_t)(a >> 32);
  const uint32_t b0 = (uint32_t)b, b1 = (uint32_t)(b >> 32);
  asm("mad.lo.cc.u32 %0, %5, %7, %0;\n\t"
      "madc.hi.cc.u32 %1, %5, %7, %1;\n\t"
      "madc.lo.cc.u32 %2, %6, %8, %2;\n\t"
      "madc.hi.cc.u32 %3, %6, %8, %3;\n\t"
      "addc.u32 %4, %4, 0;"
      : "+r"(c.r0), "+r"(c.r1), "+r"(c.r2), "+r"(c.r3), "+r"(c.r4)
      : "r"(a0), "r"(a1), "r"(b0), "r"(b1));
  asm("mad.lo.cc.u32 %0, %3, %6, %0;\n\t"
      "madc.hi.cc.u32 %1, %3, %6, %1;\n\t"
      "addc.u32 %2, %2, 0;\n\t"
      "mad.lo.cc.u32 %0, %4, %5, %0;\n\t"
      "madc.hi.cc.u32 %1, %4, %5, %1;\n\t"
      "addc.u32 %2, %2, 0;"
      : "+r"(c.m0), "+r"(c.m1), "+r"(c.m2)
      : "r"(a0), "r"(a1), "r"(b0), "r"(b1));
}

LC_D void mac32(Acc160& c, uint32_t a, uint32_t b) {
  asm("mad.lo.cc.u32 %0, %3, %4, %0;\n\t"
      "madc.hi.cc.u32 %1, %3, %4, %1;\n\t"
      "addc.u32 %2, %2, 0;"
      : "+r"(c.r0), "+r"(c.r1), "+r"(c.r2)
      : "r"(a), "r"(b));
}

template <class E>
LC_D void mac(Acc160& c, E a, E b);
template <>
LC_D void mac<uint64_t>(Acc160& c, uint64_t a, uint64_t b) {
  mac64(c, a, b);
}
template <>
LC_D void mac<uint32_t>(Acc160& c, uint32_t a, uint32_t b) {
  mac32(c, a, b);
}

template <class E>
LC_D E acc_reduce(const Acc160& c, uint32_t q) {
  uint32_t r1, r2, r3, r4;
  asm("add.cc.u32 %0, %4, %7;\n\t"
      "addc.cc.u32 %1, %5, %8;\n\t"
      "addc.cc.u32 %2, %6, %9;\n\t"
      "addc.u32 %3, %10, 0;"
      : "=r"(r1), "=r"(r2), "=r"(r3), "=r"(r4)
      : "r"(c.r1), "r"(c.r2), "r"(c.r3), "r"(c.m0), "r"(c.m1), "r"(c.m2), "r"(c.r4));
  return Field<E>::reduce160(c.r0, r1, r2, r3, r4, q);
}

}  // namespace lc
