// small_field.cuh -- device arithmetic for the 64-bit-word fields of zig-field's
// SmallField backend (libs/field/src/field.zig:89-849): Goldilocks
// (p = 2^64 - 2^32 + 1) and BabyBear (p = 15 * 2^27 + 1).
//
// SmallField stores the canonical value in [0, p) as one u64 (field.zig:141),
// so data vectors are 8 bytes per element and every kernel input and output
// is canonical.  Products follow one rule, mul(a, b) = a * b * R^-1 mod p, with
// R = 1 for Goldilocks (a direct reduction) and R = 2^32 for BabyBear (a 32-bit
// Montgomery reduction).  Twiddles and scale factors are kept in "twiddle
// form" w * R mod p, so mul(w_form, x) = w * x mod p stays canonical, and
// mul of two twiddle-form values is the twiddle form of their product.
// Canonical values are unique, so results equal the reference's bit for bit.
#pragma once

#include <cstdint>

namespace zntt {

// 1 in constant memory: the compiler cannot fold it, so x * one + y issues on
// the multiply-add pipe.
static __constant__ uint32_t kOpaqueOne = 1;

struct Goldilocks {
  static constexpr int kId = 2;
  static constexpr uint64_t P = 0xFFFFFFFF00000001ull;
  static constexpr uint64_t EPS = 0xFFFFFFFFull;  // 2^64 mod p = 2^32 - 1

  // The arithmetic runs on 32-bit halves with carry chains: a 64-bit compare
  // and select costs several ALU instructions, a carry flag none.  The add
  // chains of add() and of the product's accumulation issue as multiply-adds
  // by kOpaqueOne, moving them from the ALU to the multiply-add pipe (the
  // subtractions and selects stay on the ALU).
  __device__ __forceinline__ static uint64_t join(uint32_t lo, uint32_t hi) {
    return ((uint64_t)hi << 32) | lo;
  }
  // x - p when x >= p, else x, for x = (hi:lo) below 2^64.
  __device__ __forceinline__ static uint64_t reduce_once(uint32_t lo, uint32_t hi) {
    uint32_t d0, d1, br;
    asm("sub.cc.u32  %0, %3, 1;\n\t"
        "subc.cc.u32 %1, %4, 0xFFFFFFFF;\n\t"
        "subc.u32    %2, 0, 0;"
        : "=r"(d0), "=r"(d1), "=r"(br)
        : "r"(lo), "r"(hi));
    return br ? join(lo, hi) : join(d0, d1);
  }
  // a + b < 2p: the 65-bit sum less p, unless that borrows.
  __device__ __forceinline__ static uint64_t add(uint64_t a, uint64_t b) {
    uint32_t s0, s1, c, d0, d1, br;
    const uint32_t one = kOpaqueOne;
    asm("mad.lo.cc.u32  %0, %3, %7, %5;\n\t"
        "madc.lo.cc.u32 %1, %4, %7, %6;\n\t"
        "madc.lo.u32    %2, %7, 0, 0;"
        : "=r"(s0), "=r"(s1), "=r"(c)
        : "r"((uint32_t)a), "r"((uint32_t)(a >> 32)), "r"((uint32_t)b), "r"((uint32_t)(b >> 32)), "r"(one));
    asm("sub.cc.u32  %0, %3, 1;\n\t"
        "subc.cc.u32 %1, %4, 0xFFFFFFFF;\n\t"
        "subc.u32    %2, %5, 0;"
        : "=r"(d0), "=r"(d1), "=r"(br)
        : "r"(s0), "r"(s1), "r"(c));
    return br ? join(s0, s1) : join(d0, d1);
  }
  // a - b, plus p (low word 1, high word 2^32 - 1) when it borrows.
  __device__ __forceinline__ static uint64_t sub(uint64_t a, uint64_t b) {
    uint32_t d0, d1, br;
    asm("sub.cc.u32  %0, %3, %5;\n\t"
        "subc.cc.u32 %1, %4, %6;\n\t"
        "subc.u32    %2, 0, 0;"
        : "=r"(d0), "=r"(d1), "=r"(br)
        : "r"((uint32_t)a), "r"((uint32_t)(a >> 32)), "r"((uint32_t)b), "r"((uint32_t)(b >> 32)));
    asm("add.cc.u32  %0, %0, %2;\n\t"
        "addc.u32    %1, %1, %3;"
        : "+r"(d0), "+r"(d1)
        : "r"(br & 1u), "r"(br));
    return join(d0, d1);
  }
  __device__ __forceinline__ static uint64_t neg(uint64_t a) { return a == 0 ? 0 : P - a; }
  // a * b mod p.  The 128-bit product is z3:z2:z1:z0 (32-bit words); with
  // 2^64 = 2^32 - 1 and 2^96 = -1 (mod p) it is (z1:z0) + z2 * 2^32 - z2 - z3.
  // That sum is c * 2^64 + t with c in {-1, 0, 1}; c * 2^64 = c * (2^32 - 1),
  // added to t as a 64-bit two's-complement term (lo -c, hi c >> 31), cannot
  // leave [0, 2^64): for c = 1, t <= 2^64 - 2^32 - 1; for c = -1, t >= 2^64 - 2^33.
  __device__ __forceinline__ static uint64_t mul(uint64_t a, uint64_t b) {
    const uint32_t a0 = (uint32_t)a, a1 = (uint32_t)(a >> 32), b0 = (uint32_t)b, b1 = (uint32_t)(b >> 32);
    uint32_t z0, z1, z2, z3;
    asm("mul.lo.u32     %0, %4, %6;\n\t"
        "mul.hi.u32     %1, %4, %6;\n\t"
        "mul.lo.u32     %2, %5, %7;\n\t"
        "mul.hi.u32     %3, %5, %7;\n\t"
        "mad.lo.cc.u32  %1, %4, %7, %1;\n\t"
        "madc.hi.cc.u32 %2, %4, %7, %2;\n\t"
        "madc.lo.u32    %3, %8, 0, %3;\n\t"
        "mad.lo.cc.u32  %1, %5, %6, %1;\n\t"
        "madc.hi.cc.u32 %2, %5, %6, %2;\n\t"
        "madc.lo.u32    %3, %8, 0, %3;"
        : "=r"(z0), "=r"(z1), "=r"(z2), "=r"(z3)
        : "r"(a0), "r"(a1), "r"(b0), "r"(b1), "r"(kOpaqueOne));
    uint32_t t0, t1, c, w0, w1;
    const uint32_t one = kOpaqueOne;
    asm("mad.lo.cc.u32  %0, %2, %4, %3;\n\t"   // w = z2 + z3 (33 bits)
        "madc.lo.u32    %1, %4, 0, 0;"
        : "=r"(w0), "=r"(w1)
        : "r"(z2), "r"(z3), "r"(one));
    asm("mad.lo.cc.u32  %1, %4, %8, %5;\n\t"   // (c:t1:t0) = (z1:z0) + z2 * 2^32 ...
        "madc.lo.u32    %2, %8, 0, 0;\n\t"
        "sub.cc.u32  %0, %3, %6;\n\t"   // ... - w
        "subc.cc.u32 %1, %1, %7;\n\t"
        "subc.u32    %2, %2, 0;"
        : "=r"(t0), "=r"(t1), "=r"(c)
        : "r"(z0), "r"(z1), "r"(z2), "r"(w0), "r"(w1), "r"(one));
    asm("add.cc.u32  %0, %0, %2;\n\t"
        "addc.u32    %1, %1, %3;"
        : "+r"(t0), "+r"(t1)
        : "r"(0u - c), "r"((uint32_t)((int32_t)c >> 31)));
    return reduce_once(t0, t1);
  }
};

// p^-1 mod 2^32 for odd p by Newton's iteration x <- x (2 - p x), which
// doubles the correct low bits: exact after five steps from x = 1.
constexpr uint32_t inverse_mod_2_32(uint32_t p) {
  uint32_t x = 1;
  for (int i = 0; i < 5; i++) x *= 2u - p * x;
  return x;
}

struct BabyBear {
  static constexpr int kId = 3;
  static constexpr uint64_t P = 0x78000001ull;
  static constexpr uint32_t P32 = 0x78000001u;
  static constexpr uint32_t N0 = 0u - inverse_mod_2_32(P32);  // -p^-1 mod 2^32

  // s < 2p: min(s, s - p) is s - p when s >= p and s otherwise (s - p wraps above s).
  __device__ __forceinline__ static uint64_t add(uint64_t a, uint64_t b) {
    uint32_t s;
    asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(s) : "r"((uint32_t)a), "r"(kOpaqueOne), "r"((uint32_t)b));
    return min(s, s - P32);
  }
  // d = x - y wraps above 2^31 > p when y > x; then d + p (mod 2^32) is the smaller.
  __device__ __forceinline__ static uint64_t sub(uint64_t a, uint64_t b) {
    const uint32_t d = (uint32_t)a - (uint32_t)b;
    uint32_t dp;
    asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(dp) : "r"(P32), "r"(kOpaqueOne), "r"(d));
    return min(d, dp);
  }
  __device__ __forceinline__ static uint64_t neg(uint64_t a) { return a == 0 ? 0 : P - a; }
  // Montgomery: z = a * b < p^2; m = z * N0 mod 2^32; (z + m p) / 2^32 < 2p.
  __device__ __forceinline__ static uint64_t mul(uint64_t a, uint64_t b) {
    const uint64_t z = (uint64_t)(uint32_t)a * (uint32_t)b;
    const uint32_t m = (uint32_t)z * N0;
    const uint32_t t = (uint32_t)((z + (uint64_t)m * P32) >> 32);  // < 2p < 2^32
    return min(t, t - P32);
  }
};

}  // namespace zntt
