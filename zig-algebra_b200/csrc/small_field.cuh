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

struct Goldilocks {
  static constexpr int kId = 2;
  static constexpr uint64_t P = 0xFFFFFFFF00000001ull;
  static constexpr uint64_t EPS = 0xFFFFFFFFull;  // 2^64 mod p = 2^32 - 1

  __device__ __forceinline__ static uint64_t add(uint64_t a, uint64_t b) {
    uint64_t s = a + b;
    // a + b < 2p: a carry out of 64 bits means s + 2^64 = s + EPS (mod p),
    // which is then below p; otherwise subtract p once if needed.
    if (s < a) return s + EPS;
    return s >= P ? s - P : s;
  }
  __device__ __forceinline__ static uint64_t sub(uint64_t a, uint64_t b) {
    const uint64_t d = a - b;
    // a < b: the wrapped difference is a - b + 2^64; adding p is subtracting EPS.
    return a < b ? d - EPS : d;
  }
  __device__ __forceinline__ static uint64_t neg(uint64_t a) { return a == 0 ? 0 : P - a; }
  // a * b mod p from the 128-bit product hi * 2^64 + lo with hi = h1 * 2^32 + h0:
  // 2^64 = 2^32 - 1 and 2^96 = -1 (mod p), so the product is
  // lo - h1 + h0 * (2^32 - 1) (mod p).
  __device__ __forceinline__ static uint64_t mul(uint64_t a, uint64_t b) {
    const uint64_t lo = a * b, hi = __umul64hi(a, b);
    const uint64_t h0 = hi & 0xFFFFFFFFull, h1 = hi >> 32;
    uint64_t t = lo - h1;
    if (lo < h1) t -= EPS;  // borrow: add p
    const uint64_t u = (h0 << 32) - h0;
    uint64_t r = t + u;
    if (r < t) r += EPS;  // carry: 2^64 = EPS (mod p); cannot carry again
    return r >= P ? r - P : r;
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

  __device__ __forceinline__ static uint64_t add(uint64_t a, uint64_t b) {
    const uint32_t s = (uint32_t)a + (uint32_t)b;  // < 2p < 2^32
    return s >= P32 ? s - P32 : s;
  }
  __device__ __forceinline__ static uint64_t sub(uint64_t a, uint64_t b) {
    const uint32_t x = (uint32_t)a, y = (uint32_t)b;
    return x >= y ? x - y : x + P32 - y;
  }
  __device__ __forceinline__ static uint64_t neg(uint64_t a) { return a == 0 ? 0 : P - a; }
  // Montgomery: z = a * b < p^2; m = z * N0 mod 2^32; (z + m p) / 2^32 < 2p.
  __device__ __forceinline__ static uint64_t mul(uint64_t a, uint64_t b) {
    const uint64_t z = (uint64_t)(uint32_t)a * (uint32_t)b;
    const uint32_t m = (uint32_t)z * N0;
    const uint64_t t = (z + (uint64_t)m * P32) >> 32;
    return t >= P ? t - P : t;
  }
};

}  // namespace zntt
