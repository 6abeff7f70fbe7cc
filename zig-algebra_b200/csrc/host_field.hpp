// host_field.hpp -- host-side scalar arithmetic for transform set-up.
//
// Set-up needs a handful of scalar field operations per call: root inverses
// (zig-ntt intt, libs/ntt/src/root.zig:100), n^-1 (:103, :208), the power
// tables the twiddle kernel expands, and fromInt
// (libs/field/src/field.zig:911-921).  Elements are the reference's [4]u64
// Montgomery limbs.  Multiplication is a separated-operand-scanning Montgomery
// product on unsigned __int128 (full 512-bit product, then word-by-word
// reduction); inversion is Fermat's little theorem (a^(p-2)), which returns 0
// for 0 exactly like the reference's total `inv`.  All results are fully
// reduced, hence equal to the reference's.
#pragma once

#include <cstdint>
#include <cstring>

namespace zntt {

typedef unsigned __int128 u128;

struct HostField {
  uint64_t p[4];
  uint64_t one[4];  // 2^256 mod p
  uint64_t r2[4];   // 2^512 mod p
  uint64_t n0;      // -p^-1 mod 2^64
  uint32_t two_adicity;

  static bool geq(const uint64_t* a, const uint64_t* b) {
    for (int i = 3; i >= 0; i--) {
      if (a[i] != b[i]) return a[i] > b[i];
    }
    return true;
  }
  void sub_p(uint64_t* a) const {
    uint64_t br = 0;
    for (int i = 0; i < 4; i++) {
      u128 d = (u128)a[i] - p[i] - br;
      a[i] = (uint64_t)d;
      br = (uint64_t)(d >> 127);
    }
  }

  void add(const uint64_t* a, const uint64_t* b, uint64_t* r) const {
    uint64_t s[4];
    uint64_t c = 0;
    for (int i = 0; i < 4; i++) {
      u128 t = (u128)a[i] + b[i] + c;
      s[i] = (uint64_t)t;
      c = (uint64_t)(t >> 64);
    }
    if (c || geq(s, p)) sub_p(s);
    std::memcpy(r, s, sizeof(s));
  }

  void mul(const uint64_t* a, const uint64_t* b, uint64_t* r) const {
    uint64_t t[9] = {0};
    for (int i = 0; i < 4; i++) {  // schoolbook 4x4 -> 8 words
      uint64_t c = 0;
      for (int j = 0; j < 4; j++) {
        u128 z = (u128)a[i] * b[j] + t[i + j] + c;
        t[i + j] = (uint64_t)z;
        c = (uint64_t)(z >> 64);
      }
      t[i + 4] = c;
    }
    for (int i = 0; i < 4; i++) {  // reduce one word at a time
      uint64_t m = t[i] * n0;
      uint64_t c = 0;
      for (int j = 0; j < 4; j++) {
        u128 z = (u128)m * p[j] + t[i + j] + c;
        t[i + j] = (uint64_t)z;
        c = (uint64_t)(z >> 64);
      }
      for (int k = i + 4; c && k < 9; k++) {
        u128 z = (u128)t[k] + c;
        t[k] = (uint64_t)z;
        c = (uint64_t)(z >> 64);
      }
    }
    uint64_t out[4] = {t[4], t[5], t[6], t[7]};
    if (t[8] || geq(out, p)) sub_p(out);
    std::memcpy(r, out, sizeof(out));
  }

  void pow_u64(const uint64_t* a, uint64_t e, uint64_t* r) const {
    uint64_t acc[4], base[4];
    std::memcpy(acc, one, sizeof(acc));
    std::memcpy(base, a, sizeof(base));
    while (e) {
      if (e & 1) mul(acc, base, acc);
      mul(base, base, base);
      e >>= 1;
    }
    std::memcpy(r, acc, sizeof(acc));
  }

  // a^e for a 256-bit exponent: left-to-right square-and-multiply.
  void pow_limbs(const uint64_t* a, const uint64_t* e, uint64_t* r) const {
    uint64_t acc[4], base[4];
    std::memcpy(acc, one, sizeof(acc));
    std::memcpy(base, a, sizeof(base));
    for (int i = 255; i >= 0; i--) {
      mul(acc, acc, acc);
      if ((e[i / 64] >> (i % 64)) & 1) mul(acc, base, acc);
    }
    std::memcpy(r, acc, sizeof(acc));
  }

  // a^(p-2) (Fermat); 0 maps to 0 like the reference's total inverse.
  void inv(const uint64_t* a, uint64_t* r) const {
    uint64_t e[4];
    std::memcpy(e, p, sizeof(e));
    e[0] -= 2;  // p is odd and > 2, no borrow
    pow_limbs(a, e, r);
  }

  void from_u64(uint64_t x, uint64_t* r) const {
    uint64_t v[4] = {x, 0, 0, 0};  // x < 2^64 < p: already reduced
    mul(v, r2, r);
  }

  bool is_one(const uint64_t* a) const { return std::memcmp(a, one, 32) == 0; }
};

inline const HostField& host_field(int id) {
  static const HostField bn254 = {
      {0x43e1f593f0000001ULL, 0x2833e84879b97091ULL, 0xb85045b68181585dULL, 0x30644e72e131a029ULL},
      {0xac96341c4ffffffbULL, 0x36fc76959f60cd29ULL, 0x666ea36f7879462eULL, 0x0e0a77c19a07df2fULL},
      {0x1bb8e645ae216da7ULL, 0x53fe3ab1e35c59e3ULL, 0x8c49833d53bb8085ULL, 0x0216d0b17f4e44a5ULL},
      0xc2e1f593efffffffULL,
      28};
  static const HostField bls = {
      {0xffffffff00000001ULL, 0x53bda402fffe5bfeULL, 0x3339d80809a1d805ULL, 0x73eda753299d7d48ULL},
      {0x00000001fffffffeULL, 0x5884b7fa00034802ULL, 0x998c4fefecbc4ff5ULL, 0x1824b159acc5056fULL},
      {0xc999e990f3f29c6dULL, 0x2b6cedcb87925c23ULL, 0x05d314967254398fULL, 0x0748d9d99f59ff11ULL},
      0xfffffffeffffffffULL,
      32};
  return id == 0 ? bn254 : bls;
}

}  // namespace zntt
