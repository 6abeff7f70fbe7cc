// field.cuh -- device arithmetic for 256-bit Montgomery prime fields (sm_100a).
//
// Mirrors libs/field/src/montgomery.zig (add :197-217, sub :220-240, neg
// :243-245, CIOS mul :252-297) for the two scalar fields the transform serves,
// BN254-Fr (libs/curve/src/bn254.zig:67) and BLS12-381-Fr
// (libs/curve/src/bls12_381.zig:66).  An element is the reference's
// `[4]u64` Montgomery limbs (x * 2^256 mod p, always fully reduced to [0, p)),
// viewed here as 8 little-endian u32 limbs; the bytes are identical, so host
// buffers move to the device with a plain copy.  Because every result is fully
// reduced and the reduced representative is unique, equal inputs give
// bit-identical outputs to the reference's u64 CIOS.
//
// Multiplication is CIOS (Koc, Acar, Kaliski 1996) over 32-bit words with the
// running sum split into two accumulators so that each row is two independent
// carry chains of mad.lo/madc.hi:
//   T (aligned)        collects the products a_j * w for even j (and m * p_j),
//                      whose lo/hi halves tile words j, j+1 without overlap;
//   U (one word up)    collects the products for odd j.
// After the reduction word m is added the low word of T is zero; the shift by
// one word is T[1..8] + U[0..8], one add chain.  With a, b < p and 2p < 2^256
// (true for both fields) the running value stays below 2p, so nine words
// suffice and one conditional subtraction gives the canonical result.
// Multiply-class instructions per product: 8 rows x (8 + 8 + 1 + 8 + 8) = 264.
#pragma once

#include <cstdint>

namespace zntt {

// kRed selects the reduction step of the field product:
//   0  generic: m = T0 * N0, then m * p with 8 products per row
//   1  BN254-Fr: N0 = -(2^28 + 1) and p0 = 2^32 - 2^28 + 1, so m and m * p0
//      come from shifts and adds (7 products per row instead of 9)
//   2  BLS12-381-Fr: N0 = -1, p0 = 1 and p1 = 2^32 - 1, so m, m * p0 and
//      m * p1 come from adds (6 products per row instead of 9)
struct Bn254Fr {
  static constexpr int kId = 0;
  static constexpr int kRed = 1;
  static constexpr uint32_t P0 = 0xf0000001u, P1 = 0x43e1f593u, P2 = 0x79b97091u, P3 = 0x2833e848u,
                            P4 = 0x8181585du, P5 = 0xb85045b6u, P6 = 0xe131a029u, P7 = 0x30644e72u;
  static constexpr uint32_t N0 = 0xefffffffu;  // -p^-1 mod 2^32
  static constexpr uint32_t ONE0 = 0x4ffffffbu, ONE1 = 0xac96341cu, ONE2 = 0x9f60cd29u,
                            ONE3 = 0x36fc7695u, ONE4 = 0x7879462eu, ONE5 = 0x666ea36fu,
                            ONE6 = 0x9a07df2fu, ONE7 = 0x0e0a77c1u;
  static constexpr uint32_t R2_0 = 0xae216da7u, R2_1 = 0x1bb8e645u, R2_2 = 0xe35c59e3u,
                            R2_3 = 0x53fe3ab1u, R2_4 = 0x53bb8085u, R2_5 = 0x8c49833du,
                            R2_6 = 0x7f4e44a5u, R2_7 = 0x0216d0b1u;  // 2^512 mod p
};

struct Bls12381Fr {
  static constexpr int kId = 1;
  static constexpr int kRed = 2;
  static constexpr uint32_t P0 = 0x00000001u, P1 = 0xffffffffu, P2 = 0xfffe5bfeu, P3 = 0x53bda402u,
                            P4 = 0x09a1d805u, P5 = 0x3339d808u, P6 = 0x299d7d48u, P7 = 0x73eda753u;
  static constexpr uint32_t N0 = 0xffffffffu;
  static constexpr uint32_t ONE0 = 0xfffffffeu, ONE1 = 0x00000001u, ONE2 = 0x00034802u,
                            ONE3 = 0x5884b7fau, ONE4 = 0xecbc4ff5u, ONE5 = 0x998c4fefu,
                            ONE6 = 0xacc5056fu, ONE7 = 0x1824b159u;
  static constexpr uint32_t R2_0 = 0xf3f29c6du, R2_1 = 0xc999e990u, R2_2 = 0x87925c23u,
                            R2_3 = 0x2b6cedcbu, R2_4 = 0x7254398fu, R2_5 = 0x05d31496u,
                            R2_6 = 0x9f59ff11u, R2_7 = 0x0748d9d9u;
};

// A field element in registers.
struct fe {
  uint32_t v[8];
};

template <class F>
__device__ __forceinline__ fe fe_one() {
  fe r;
  r.v[0] = F::ONE0; r.v[1] = F::ONE1; r.v[2] = F::ONE2; r.v[3] = F::ONE3;
  r.v[4] = F::ONE4; r.v[5] = F::ONE5; r.v[6] = F::ONE6; r.v[7] = F::ONE7;
  return r;
}

template <class F>
__device__ __forceinline__ fe fe_r2() {
  fe r;
  r.v[0] = F::R2_0; r.v[1] = F::R2_1; r.v[2] = F::R2_2; r.v[3] = F::R2_3;
  r.v[4] = F::R2_4; r.v[5] = F::R2_5; r.v[6] = F::R2_6; r.v[7] = F::R2_7;
  return r;
}

// a < p (canonical limbs), as a branch-free borrow chain.
template <class F>
__device__ __forceinline__ bool fe_lt_p(const fe& a) {
  uint32_t br;
  asm("sub.cc.u32  %0, %1, %9;\n\t"
      "subc.cc.u32 %0, %2, %10;\n\t"
      "subc.cc.u32 %0, %3, %11;\n\t"
      "subc.cc.u32 %0, %4, %12;\n\t"
      "subc.cc.u32 %0, %5, %13;\n\t"
      "subc.cc.u32 %0, %6, %14;\n\t"
      "subc.cc.u32 %0, %7, %15;\n\t"
      "subc.cc.u32 %0, %8, %16;\n\t"
      "subc.u32    %0, 0, 0;"
      : "=r"(br)
      : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]), "r"(a.v[6]),
        "r"(a.v[7]), "n"(F::P0), "n"(F::P1), "n"(F::P2), "n"(F::P3), "n"(F::P4), "n"(F::P5),
        "n"(F::P6), "n"(F::P7));
  return br != 0;
}

__device__ __forceinline__ bool fe_is_zero(const fe& a) {
  uint32_t acc = a.v[0] | a.v[1] | a.v[2] | a.v[3] | a.v[4] | a.v[5] | a.v[6] | a.v[7];
  return acc == 0;
}

// a + b mod p.  a + b < 2p < 2^256, so the sum needs no ninth word; subtract p
// and keep the difference unless it borrowed.
template <class F>
__device__ __forceinline__ fe fe_add(const fe& a, const fe& b) {
  uint32_t s0, s1, s2, s3, s4, s5, s6, s7;
  uint32_t d0, d1, d2, d3, d4, d5, d6, d7, br;
  asm("add.cc.u32  %0, %8, %16;\n\t"
      "addc.cc.u32 %1, %9, %17;\n\t"
      "addc.cc.u32 %2, %10, %18;\n\t"
      "addc.cc.u32 %3, %11, %19;\n\t"
      "addc.cc.u32 %4, %12, %20;\n\t"
      "addc.cc.u32 %5, %13, %21;\n\t"
      "addc.cc.u32 %6, %14, %22;\n\t"
      "addc.u32    %7, %15, %23;"
      : "=r"(s0), "=r"(s1), "=r"(s2), "=r"(s3), "=r"(s4), "=r"(s5), "=r"(s6), "=r"(s7)
      : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]), "r"(a.v[6]),
        "r"(a.v[7]), "r"(b.v[0]), "r"(b.v[1]), "r"(b.v[2]), "r"(b.v[3]), "r"(b.v[4]), "r"(b.v[5]),
        "r"(b.v[6]), "r"(b.v[7]));
  asm("sub.cc.u32  %0, %9, %17;\n\t"
      "subc.cc.u32 %1, %10, %18;\n\t"
      "subc.cc.u32 %2, %11, %19;\n\t"
      "subc.cc.u32 %3, %12, %20;\n\t"
      "subc.cc.u32 %4, %13, %21;\n\t"
      "subc.cc.u32 %5, %14, %22;\n\t"
      "subc.cc.u32 %6, %15, %23;\n\t"
      "subc.cc.u32 %7, %16, %24;\n\t"
      "subc.u32    %8, 0, 0;"
      : "=r"(d0), "=r"(d1), "=r"(d2), "=r"(d3), "=r"(d4), "=r"(d5), "=r"(d6), "=r"(d7), "=r"(br)
      : "r"(s0), "r"(s1), "r"(s2), "r"(s3), "r"(s4), "r"(s5), "r"(s6), "r"(s7), "n"(F::P0),
        "n"(F::P1), "n"(F::P2), "n"(F::P3), "n"(F::P4), "n"(F::P5), "n"(F::P6), "n"(F::P7));
  fe r;
  // br == 0xffffffff when s < p: keep s.
  r.v[0] = br ? s0 : d0; r.v[1] = br ? s1 : d1; r.v[2] = br ? s2 : d2; r.v[3] = br ? s3 : d3;
  r.v[4] = br ? s4 : d4; r.v[5] = br ? s5 : d5; r.v[6] = br ? s6 : d6; r.v[7] = br ? s7 : d7;
  return r;
}

// a - b mod p: subtract, and add p back when the subtraction borrowed.
template <class F>
__device__ __forceinline__ fe fe_sub(const fe& a, const fe& b) {
  uint32_t d0, d1, d2, d3, d4, d5, d6, d7, br;
  asm("sub.cc.u32  %0, %9, %17;\n\t"
      "subc.cc.u32 %1, %10, %18;\n\t"
      "subc.cc.u32 %2, %11, %19;\n\t"
      "subc.cc.u32 %3, %12, %20;\n\t"
      "subc.cc.u32 %4, %13, %21;\n\t"
      "subc.cc.u32 %5, %14, %22;\n\t"
      "subc.cc.u32 %6, %15, %23;\n\t"
      "subc.cc.u32 %7, %16, %24;\n\t"
      "subc.u32    %8, 0, 0;"
      : "=r"(d0), "=r"(d1), "=r"(d2), "=r"(d3), "=r"(d4), "=r"(d5), "=r"(d6), "=r"(d7), "=r"(br)
      : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]), "r"(a.v[6]),
        "r"(a.v[7]), "r"(b.v[0]), "r"(b.v[1]), "r"(b.v[2]), "r"(b.v[3]), "r"(b.v[4]), "r"(b.v[5]),
        "r"(b.v[6]), "r"(b.v[7]));
  fe r;
  asm("add.cc.u32  %0, %8, %16;\n\t"
      "addc.cc.u32 %1, %9, %17;\n\t"
      "addc.cc.u32 %2, %10, %18;\n\t"
      "addc.cc.u32 %3, %11, %19;\n\t"
      "addc.cc.u32 %4, %12, %20;\n\t"
      "addc.cc.u32 %5, %13, %21;\n\t"
      "addc.cc.u32 %6, %14, %22;\n\t"
      "addc.u32    %7, %15, %23;"
      : "=r"(r.v[0]), "=r"(r.v[1]), "=r"(r.v[2]), "=r"(r.v[3]), "=r"(r.v[4]), "=r"(r.v[5]),
        "=r"(r.v[6]), "=r"(r.v[7])
      : "r"(d0), "r"(d1), "r"(d2), "r"(d3), "r"(d4), "r"(d5), "r"(d6), "r"(d7), "r"(F::P0 & br),
        "r"(F::P1 & br), "r"(F::P2 & br), "r"(F::P3 & br), "r"(F::P4 & br), "r"(F::P5 & br),
        "r"(F::P6 & br), "r"(F::P7 & br));
  return r;
}

// -a mod p (0 stays 0), as montgomery.zig:243-245 (0 - a).
template <class F>
__device__ __forceinline__ fe fe_neg(const fe& a) {
  fe z;
#pragma unroll
  for (int i = 0; i < 8; i++) z.v[i] = 0;
  return fe_sub<F>(z, a);
}

// One CIOS row: accumulate a * w into (T, U), then reduce one word.
// On entry T[0..7] holds the running value (< 2p) and U is dead; on exit the
// same.  `first` skips the accumulate-into-T for the first row (T == 0).
template <class F, bool kFirst>
__device__ __forceinline__ void cios_row(uint32_t (&T)[9], const fe& a, uint32_t w) {
  uint32_t U0, U1, U2, U3, U4, U5, U6, U7, U8, m;
  if (kFirst) {
    asm("mul.lo.u32 %0, %8, %12;\n\t"
        "mul.hi.u32 %1, %8, %12;\n\t"
        "mul.lo.u32 %2, %9, %12;\n\t"
        "mul.hi.u32 %3, %9, %12;\n\t"
        "mul.lo.u32 %4, %10, %12;\n\t"
        "mul.hi.u32 %5, %10, %12;\n\t"
        "mul.lo.u32 %6, %11, %12;\n\t"
        "mul.hi.u32 %7, %11, %12;"
        : "=r"(T[0]), "=r"(T[1]), "=r"(T[2]), "=r"(T[3]), "=r"(T[4]), "=r"(T[5]), "=r"(T[6]),
          "=r"(T[7])
        : "r"(a.v[0]), "r"(a.v[2]), "r"(a.v[4]), "r"(a.v[6]), "r"(w));
    T[8] = 0;
  } else {
    asm("mad.lo.cc.u32  %0, %9, %13, %0;\n\t"
        "madc.hi.cc.u32 %1, %9, %13, %1;\n\t"
        "madc.lo.cc.u32 %2, %10, %13, %2;\n\t"
        "madc.hi.cc.u32 %3, %10, %13, %3;\n\t"
        "madc.lo.cc.u32 %4, %11, %13, %4;\n\t"
        "madc.hi.cc.u32 %5, %11, %13, %5;\n\t"
        "madc.lo.cc.u32 %6, %12, %13, %6;\n\t"
        "madc.hi.cc.u32 %7, %12, %13, %7;\n\t"
        "addc.u32       %8, 0, 0;"
        : "+r"(T[0]), "+r"(T[1]), "+r"(T[2]), "+r"(T[3]), "+r"(T[4]), "+r"(T[5]), "+r"(T[6]),
          "+r"(T[7]), "=r"(T[8])
        : "r"(a.v[0]), "r"(a.v[2]), "r"(a.v[4]), "r"(a.v[6]), "r"(w));
  }
  asm("mul.lo.u32 %0, %8, %12;\n\t"
      "mul.hi.u32 %1, %8, %12;\n\t"
      "mul.lo.u32 %2, %9, %12;\n\t"
      "mul.hi.u32 %3, %9, %12;\n\t"
      "mul.lo.u32 %4, %10, %12;\n\t"
      "mul.hi.u32 %5, %10, %12;\n\t"
      "mul.lo.u32 %6, %11, %12;\n\t"
      "mul.hi.u32 %7, %11, %12;"
      : "=r"(U0), "=r"(U1), "=r"(U2), "=r"(U3), "=r"(U4), "=r"(U5), "=r"(U6), "=r"(U7)
      : "r"(a.v[1]), "r"(a.v[3]), "r"(a.v[5]), "r"(a.v[7]), "r"(w));
  if constexpr (F::kRed == 1) {
    // m = T0 * N0 = -(T0 + T0 * 2^28) mod 2^32.
    m = 0u - T[0] - (T[0] << 28);
    // Words 0 and 1 of T + m * p0 with p0 = 2^32 - D/m, D = m * (2^28 - 1):
    // word 0 becomes zero and word 1 gains m - floor(D / 2^32) (the carry out
    // of word 0 and the rounding of the high half cancel).
    // floor(D / 2^32) = (m >> 4) - [((m << 28) mod 2^32) < m].
    uint32_t a;
    asm("{\n\t.reg .u32 x, d;\n\t"
        "shl.b32     x, %1, 28;\n\t"
        "sub.cc.u32  x, x, %1;\n\t"
        "shr.b32     d, %1, 4;\n\t"
        "subc.u32    d, d, 0;\n\t"
        "sub.u32     %0, %1, d;\n\t}"
        : "=r"(a)
        : "r"(m));
    asm("add.cc.u32     %0, %0, %8;\n\t"
        "madc.lo.cc.u32 %1, %9, %10, %1;\n\t"
        "madc.hi.cc.u32 %2, %9, %10, %2;\n\t"
        "madc.lo.cc.u32 %3, %9, %11, %3;\n\t"
        "madc.hi.cc.u32 %4, %9, %11, %4;\n\t"
        "madc.lo.cc.u32 %5, %9, %12, %5;\n\t"
        "madc.hi.cc.u32 %6, %9, %12, %6;\n\t"
        "addc.u32       %7, %7, 0;"
        : "+r"(T[1]), "+r"(T[2]), "+r"(T[3]), "+r"(T[4]), "+r"(T[5]), "+r"(T[6]), "+r"(T[7]), "+r"(T[8])
        : "r"(a), "r"(m), "n"(F::P2), "n"(F::P4), "n"(F::P6));
  } else if constexpr (F::kRed == 2) {
    // m = -T0 mod 2^32.  With p0 = 1: T0 + m = 0 with carry [T0 != 0] and a
    // zero high half.  With p1 = 2^32 - 1: m * p1 = (m - [m != 0]) * 2^32 +
    // (-m mod 2^32) and -m mod 2^32 = T0.
    m = 0u - T[0];
    const uint32_t c0 = T[0] != 0u ? 1u : 0u;
    asm("add.cc.u32     %0, %0, %8;\n\t"
        "madc.lo.cc.u32 %1, %9, %10, %1;\n\t"
        "madc.hi.cc.u32 %2, %9, %10, %2;\n\t"
        "madc.lo.cc.u32 %3, %9, %11, %3;\n\t"
        "madc.hi.cc.u32 %4, %9, %11, %4;\n\t"
        "madc.lo.cc.u32 %5, %9, %12, %5;\n\t"
        "madc.hi.cc.u32 %6, %9, %12, %6;\n\t"
        "addc.u32       %7, %7, 0;"
        : "+r"(T[1]), "+r"(T[2]), "+r"(T[3]), "+r"(T[4]), "+r"(T[5]), "+r"(T[6]), "+r"(T[7]), "+r"(T[8])
        : "r"(c0), "r"(m), "n"(F::P2), "n"(F::P4), "n"(F::P6));
    asm("add.cc.u32     %0, %0, %9;\n\t"
        "addc.cc.u32    %1, %1, %10;\n\t"
        "madc.lo.cc.u32 %2, %11, %12, %2;\n\t"
        "madc.hi.cc.u32 %3, %11, %12, %3;\n\t"
        "madc.lo.cc.u32 %4, %11, %13, %4;\n\t"
        "madc.hi.cc.u32 %5, %11, %13, %5;\n\t"
        "madc.lo.cc.u32 %6, %11, %14, %6;\n\t"
        "madc.hi.cc.u32 %7, %11, %14, %7;\n\t"
        "addc.u32       %8, 0, 0;"
        : "+r"(U0), "+r"(U1), "+r"(U2), "+r"(U3), "+r"(U4), "+r"(U5), "+r"(U6), "+r"(U7), "=r"(U8)
        : "r"(T[0]), "r"(m - c0), "r"(m), "n"(F::P3), "n"(F::P5), "n"(F::P7));
  } else {
    m = T[0] * F::N0;
    asm("mad.lo.cc.u32  %0, %9, %10, %0;\n\t"
        "madc.hi.cc.u32 %1, %9, %10, %1;\n\t"
        "madc.lo.cc.u32 %2, %9, %11, %2;\n\t"
        "madc.hi.cc.u32 %3, %9, %11, %3;\n\t"
        "madc.lo.cc.u32 %4, %9, %12, %4;\n\t"
        "madc.hi.cc.u32 %5, %9, %12, %5;\n\t"
        "madc.lo.cc.u32 %6, %9, %13, %6;\n\t"
        "madc.hi.cc.u32 %7, %9, %13, %7;\n\t"
        "addc.u32       %8, %8, 0;"
        : "+r"(T[0]), "+r"(T[1]), "+r"(T[2]), "+r"(T[3]), "+r"(T[4]), "+r"(T[5]), "+r"(T[6]),
          "+r"(T[7]), "+r"(T[8])
        : "r"(m), "n"(F::P0), "n"(F::P2), "n"(F::P4), "n"(F::P6));
  }
  if constexpr (F::kRed != 2) {
    asm("mad.lo.cc.u32  %0, %9, %10, %0;\n\t"
        "madc.hi.cc.u32 %1, %9, %10, %1;\n\t"
        "madc.lo.cc.u32 %2, %9, %11, %2;\n\t"
        "madc.hi.cc.u32 %3, %9, %11, %3;\n\t"
        "madc.lo.cc.u32 %4, %9, %12, %4;\n\t"
        "madc.hi.cc.u32 %5, %9, %12, %5;\n\t"
        "madc.lo.cc.u32 %6, %9, %13, %6;\n\t"
        "madc.hi.cc.u32 %7, %9, %13, %7;\n\t"
        "addc.u32       %8, 0, 0;"
        : "+r"(U0), "+r"(U1), "+r"(U2), "+r"(U3), "+r"(U4), "+r"(U5), "+r"(U6), "+r"(U7), "=r"(U8)
        : "r"(m), "n"(F::P1), "n"(F::P3), "n"(F::P5), "n"(F::P7));
  }
  // T[0] is now zero: shift down one word and fold U in.  The result is below
  // 2p < 2^256, so the ninth word of the sum is zero and is not kept.
  asm("add.cc.u32  %0, %0, %8;\n\t"
      "addc.cc.u32 %1, %1, %9;\n\t"
      "addc.cc.u32 %2, %2, %10;\n\t"
      "addc.cc.u32 %3, %3, %11;\n\t"
      "addc.cc.u32 %4, %4, %12;\n\t"
      "addc.cc.u32 %5, %5, %13;\n\t"
      "addc.cc.u32 %6, %6, %14;\n\t"
      "addc.u32    %7, %7, %15;"
      : "+r"(T[1]), "+r"(T[2]), "+r"(T[3]), "+r"(T[4]), "+r"(T[5]), "+r"(T[6]), "+r"(T[7]),
        "+r"(T[8])
      : "r"(U0), "r"(U1), "r"(U2), "r"(U3), "r"(U4), "r"(U5), "r"(U6), "r"(U7));
  (void)U8;
#pragma unroll
  for (int k = 0; k < 8; k++) T[k] = T[k + 1];
}

// a * b * 2^-256 mod p, canonical.
template <class F>
__device__ __forceinline__ fe fe_mul(const fe& a, const fe& b) {
  uint32_t T[9];
  cios_row<F, true>(T, a, b.v[0]);
  cios_row<F, false>(T, a, b.v[1]);
  cios_row<F, false>(T, a, b.v[2]);
  cios_row<F, false>(T, a, b.v[3]);
  cios_row<F, false>(T, a, b.v[4]);
  cios_row<F, false>(T, a, b.v[5]);
  cios_row<F, false>(T, a, b.v[6]);
  cios_row<F, false>(T, a, b.v[7]);
  uint32_t d0, d1, d2, d3, d4, d5, d6, d7, br;
  asm("sub.cc.u32  %0, %9, %17;\n\t"
      "subc.cc.u32 %1, %10, %18;\n\t"
      "subc.cc.u32 %2, %11, %19;\n\t"
      "subc.cc.u32 %3, %12, %20;\n\t"
      "subc.cc.u32 %4, %13, %21;\n\t"
      "subc.cc.u32 %5, %14, %22;\n\t"
      "subc.cc.u32 %6, %15, %23;\n\t"
      "subc.cc.u32 %7, %16, %24;\n\t"
      "subc.u32    %8, 0, 0;"
      : "=r"(d0), "=r"(d1), "=r"(d2), "=r"(d3), "=r"(d4), "=r"(d5), "=r"(d6), "=r"(d7), "=r"(br)
      : "r"(T[0]), "r"(T[1]), "r"(T[2]), "r"(T[3]), "r"(T[4]), "r"(T[5]), "r"(T[6]), "r"(T[7]),
        "n"(F::P0), "n"(F::P1), "n"(F::P2), "n"(F::P3), "n"(F::P4), "n"(F::P5), "n"(F::P6),
        "n"(F::P7));
  fe r;
  r.v[0] = br ? T[0] : d0; r.v[1] = br ? T[1] : d1; r.v[2] = br ? T[2] : d2; r.v[3] = br ? T[3] : d3;
  r.v[4] = br ? T[4] : d4; r.v[5] = br ? T[5] : d5; r.v[6] = br ? T[6] : d6; r.v[7] = br ? T[7] : d7;
  return r;
}

// Global-memory element access: an element is 32 bytes = two uint4.
__device__ __forceinline__ fe fe_load(const uint4* p) {
  uint4 lo = p[0], hi = p[1];
  fe r;
  r.v[0] = lo.x; r.v[1] = lo.y; r.v[2] = lo.z; r.v[3] = lo.w;
  r.v[4] = hi.x; r.v[5] = hi.y; r.v[6] = hi.z; r.v[7] = hi.w;
  return r;
}
__device__ __forceinline__ fe fe_load_nc(const uint4* p) {
  uint4 lo = __ldg(p), hi = __ldg(p + 1);
  fe r;
  r.v[0] = lo.x; r.v[1] = lo.y; r.v[2] = lo.z; r.v[3] = lo.w;
  r.v[4] = hi.x; r.v[5] = hi.y; r.v[6] = hi.z; r.v[7] = hi.w;
  return r;
}
__device__ __forceinline__ void fe_store(uint4* p, const fe& a) {
  p[0] = make_uint4(a.v[0], a.v[1], a.v[2], a.v[3]);
  p[1] = make_uint4(a.v[4], a.v[5], a.v[6], a.v[7]);
}

}  // namespace zntt
