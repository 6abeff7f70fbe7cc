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
// Multiplication is CIOS (Koc, Acar, Kaliski 1996) over 32-bit words.  The
// running value is two accumulators so that each row is independent carry
// chains of mad.lo/madc.hi:
//   even (aligned)     collects the products a_j * w for even j (and m * p_j),
//                      whose lo/hi halves tile words j, j+1 without overlap;
//   odd (one word up)  collects the products for odd j.
// Two forms, chosen per field (F::kSplit):
//   merged rows: each row adds the odd accumulator into the even one while
//     shifting down a word, so only one accumulator lives across rows;
//   split: both accumulators live for the whole product; the shift is a
//     renaming, the odd accumulator's low word (left at word 0) joins the even
//     one in the next row with its carry entering the odd chain, and one add
//     chain merges them after the last row.
// The reduction word is m = T0 * N0 with eight products m * p_j per row.  With
// a < p, b < 2^256 and 2p < 2^256 (true for both fields) the running value
// stays below 2p, so nine words suffice and one conditional subtraction gives
// the canonical result.
#pragma once

#include <cstdint>

namespace zntt {

// Per-field choices, measured on B200 inside the transform's pass kernel
// (80 registers per thread):
//   kLazy   4p < 2^256, so butterflies keep values in [0, 2p) (sums below 4p
//           fit in eight words) and skip the final subtraction of each
//           product; Q0..Q7 are the limbs of 2p.
//   kSplit  product form: split accumulators (fe_mul_split) or merged rows
//           (fe_mul_merged).
//   kScaleCompiled  the pass kernel keeps its output-scaling code in every
//           pass, also where no pass scales: the register allocation it gets
//           times faster for this field (B200).
// The special low limbs of both primes (BN254-Fr: p0 = 2^32 - 2^28 + 1;
// BLS12-381-Fr: p0 = 1, p1 = 2^32 - 1) allow a reduction from shifts and adds
// with fewer products.  It times faster alone but slower in the pass kernel,
// whose register budget its extra live values exceed, so it is not used.
struct Bn254Fr {
  static constexpr int kId = 0;
  static constexpr bool kLazy = true;
  static constexpr bool kSplit = false;
  static constexpr bool kScaleCompiled = false;
  static constexpr uint32_t P0 = 0xf0000001u, P1 = 0x43e1f593u, P2 = 0x79b97091u, P3 = 0x2833e848u,
                            P4 = 0x8181585du, P5 = 0xb85045b6u, P6 = 0xe131a029u, P7 = 0x30644e72u;
  static constexpr uint32_t Q0 = P0 << 1, Q1 = (P1 << 1) | (P0 >> 31), Q2 = (P2 << 1) | (P1 >> 31),
                            Q3 = (P3 << 1) | (P2 >> 31), Q4 = (P4 << 1) | (P3 >> 31),
                            Q5 = (P5 << 1) | (P4 >> 31), Q6 = (P6 << 1) | (P5 >> 31),
                            Q7 = (P7 << 1) | (P6 >> 31);
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
  static constexpr bool kLazy = false;  // 4p > 2^256
  static constexpr bool kSplit = true;
  static constexpr bool kScaleCompiled = true;
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

// p - a for a in [0, p]: the negation of a twiddle factor as a multiplier.  For
// a != 0 it is -a mod p; for a = 0 it is p, which is not canonical but is a
// valid left operand of fe_mul (the CIOS bound needs a <= p: the running value
// stays below 2p) and gives the same reduced product as 0.  One subtraction
// chain, no select: cheaper than fe_neg on the inverse transform's hot path.
template <class F>
__device__ __forceinline__ fe fe_p_minus(const fe& a) {
  fe r;
  asm("sub.cc.u32  %0, %8, %16;\n\t"
      "subc.cc.u32 %1, %9, %17;\n\t"
      "subc.cc.u32 %2, %10, %18;\n\t"
      "subc.cc.u32 %3, %11, %19;\n\t"
      "subc.cc.u32 %4, %12, %20;\n\t"
      "subc.cc.u32 %5, %13, %21;\n\t"
      "subc.cc.u32 %6, %14, %22;\n\t"
      "subc.u32    %7, %15, %23;"
      : "=r"(r.v[0]), "=r"(r.v[1]), "=r"(r.v[2]), "=r"(r.v[3]), "=r"(r.v[4]), "=r"(r.v[5]), "=r"(r.v[6]),
        "=r"(r.v[7])
      : "n"(F::P0), "n"(F::P1), "n"(F::P2), "n"(F::P3), "n"(F::P4), "n"(F::P5), "n"(F::P6), "n"(F::P7),
        "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]), "r"(a.v[6]), "r"(a.v[7]));
  return r;
}

// x in [0, 2p) -> [0, p): one conditional subtraction of p.
template <class F>
__device__ __forceinline__ fe fe_reduce(const fe& x) {
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
      : "r"(x.v[0]), "r"(x.v[1]), "r"(x.v[2]), "r"(x.v[3]), "r"(x.v[4]), "r"(x.v[5]), "r"(x.v[6]),
        "r"(x.v[7]), "n"(F::P0), "n"(F::P1), "n"(F::P2), "n"(F::P3), "n"(F::P4), "n"(F::P5), "n"(F::P6),
        "n"(F::P7));
  fe r;
  // br == 0xffffffff when x < p: keep x.
  r.v[0] = br ? x.v[0] : d0; r.v[1] = br ? x.v[1] : d1; r.v[2] = br ? x.v[2] : d2; r.v[3] = br ? x.v[3] : d3;
  r.v[4] = br ? x.v[4] : d4; r.v[5] = br ? x.v[5] : d5; r.v[6] = br ? x.v[6] : d6; r.v[7] = br ? x.v[7] : d7;
  return r;
}

// Lazy butterfly arithmetic for fields with 4p < 2^256 (F::kLazy): inputs and
// outputs in [0, 2p).
// a + b, less 2p when the sum reaches 2p.
template <class F>
__device__ __forceinline__ fe fe_add2p(const fe& a, const fe& b) {
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
      : "r"(s0), "r"(s1), "r"(s2), "r"(s3), "r"(s4), "r"(s5), "r"(s6), "r"(s7), "n"(F::Q0),
        "n"(F::Q1), "n"(F::Q2), "n"(F::Q3), "n"(F::Q4), "n"(F::Q5), "n"(F::Q6), "n"(F::Q7));
  fe r;
  r.v[0] = br ? s0 : d0; r.v[1] = br ? s1 : d1; r.v[2] = br ? s2 : d2; r.v[3] = br ? s3 : d3;
  r.v[4] = br ? s4 : d4; r.v[5] = br ? s5 : d5; r.v[6] = br ? s6 : d6; r.v[7] = br ? s7 : d7;
  return r;
}

// a - b, plus 2p when the difference is negative.
template <class F>
__device__ __forceinline__ fe fe_sub2p(const fe& a, const fe& b) {
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
      : "r"(d0), "r"(d1), "r"(d2), "r"(d3), "r"(d4), "r"(d5), "r"(d6), "r"(d7), "r"(F::Q0 & br),
        "r"(F::Q1 & br), "r"(F::Q2 & br), "r"(F::Q3 & br), "r"(F::Q4 & br), "r"(F::Q5 & br),
        "r"(F::Q6 & br), "r"(F::Q7 & br));
  return r;
}

// acc[0..7] = x_j * w for the four x_j given, lo/hi halves at consecutive
// words (no carries: the eight halves tile the words).
#define ZNTT_MUL8(A0, A1, A2, A3, A4, A5, A6, A7, X0, X1, X2, X3, W)                                  \
  asm("mul.lo.u32 %0, %8, %12;\n\t"                                                                   \
      "mul.hi.u32 %1, %8, %12;\n\t"                                                                   \
      "mul.lo.u32 %2, %9, %12;\n\t"                                                                   \
      "mul.hi.u32 %3, %9, %12;\n\t"                                                                   \
      "mul.lo.u32 %4, %10, %12;\n\t"                                                                  \
      "mul.hi.u32 %5, %10, %12;\n\t"                                                                  \
      "mul.lo.u32 %6, %11, %12;\n\t"                                                                  \
      "mul.hi.u32 %7, %11, %12;"                                                                      \
      : "=r"(A0), "=r"(A1), "=r"(A2), "=r"(A3), "=r"(A4), "=r"(A5), "=r"(A6), "=r"(A7)                \
      : "r"(X0), "r"(X1), "r"(X2), "r"(X3), "r"(W))
// acc += x * w over eight words; TOP is the ninth word: "=r" with addc 0, 0
// (a new word) or "+r" with addc TOP, 0 (an existing one).
#define ZNTT_MAD8(TOPC, TOPI, A0, A1, A2, A3, A4, A5, A6, A7, A8, X0, X1, X2, X3, W)                  \
  asm("mad.lo.cc.u32  %0, %9, %13, %0;\n\t"                                                           \
      "madc.hi.cc.u32 %1, %9, %13, %1;\n\t"                                                           \
      "madc.lo.cc.u32 %2, %10, %13, %2;\n\t"                                                          \
      "madc.hi.cc.u32 %3, %10, %13, %3;\n\t"                                                          \
      "madc.lo.cc.u32 %4, %11, %13, %4;\n\t"                                                          \
      "madc.hi.cc.u32 %5, %11, %13, %5;\n\t"                                                          \
      "madc.lo.cc.u32 %6, %12, %13, %6;\n\t"                                                          \
      "madc.hi.cc.u32 %7, %12, %13, %7;\n\t"                                                          \
      "addc.u32       %8, " TOPI ", 0;"                                                               \
      : "+r"(A0), "+r"(A1), "+r"(A2), "+r"(A3), "+r"(A4), "+r"(A5), "+r"(A6), "+r"(A7), TOPC(A8)      \
      : "r"(X0), "r"(X1), "r"(X2), "r"(X3), "r"(W))

// acc += m * (P0, P1, P2, P3) over eight words with the limbs as immediates.
#define ZNTT_MADP8(TOPC, TOPI, A0, A1, A2, A3, A4, A5, A6, A7, A8, P0, P1, P2, P3, M)                \
  asm("mad.lo.cc.u32  %0, %9, %10, %0;\n\t"                                                           \
      "madc.hi.cc.u32 %1, %9, %10, %1;\n\t"                                                           \
      "madc.lo.cc.u32 %2, %9, %11, %2;\n\t"                                                           \
      "madc.hi.cc.u32 %3, %9, %11, %3;\n\t"                                                           \
      "madc.lo.cc.u32 %4, %9, %12, %4;\n\t"                                                           \
      "madc.hi.cc.u32 %5, %9, %12, %5;\n\t"                                                           \
      "madc.lo.cc.u32 %6, %9, %13, %6;\n\t"                                                           \
      "madc.hi.cc.u32 %7, %9, %13, %7;\n\t"                                                           \
      "addc.u32       %8, " TOPI ", 0;"                                                               \
      : "+r"(A0), "+r"(A1), "+r"(A2), "+r"(A3), "+r"(A4), "+r"(A5), "+r"(A6), "+r"(A7), TOPC(A8)      \
      : "r"(M), "n"(P0), "n"(P1), "n"(P2), "n"(P3))

// The reduction's half of ZNTT_MADP8 for the accumulator that holds the word
// being cleared: m = A0 * N0 makes A0 + lo(m * p0) = 0 mod 2^32, so that low
// product need not be formed -- the sum carries exactly when A0 != 0, which
// A0 + (2^32 - 1) reproduces on the ALU.  A0 is dead afterwards.  Used by
// the split form (2^24 BLS12-381-Fr 4.101 -> 4.072 ms) and fe_from_mont.
#define ZNTT_REDP8(A0, A1, A2, A3, A4, A5, A6, A7, A8, P0, P1, P2, P3, M)                              \
  asm("add.cc.u32     %0, %0, 0xFFFFFFFF;\n\t"                                                         \
      "madc.hi.cc.u32 %1, %9, %10, %1;\n\t"                                                           \
      "madc.lo.cc.u32 %2, %9, %11, %2;\n\t"                                                           \
      "madc.hi.cc.u32 %3, %9, %11, %3;\n\t"                                                           \
      "madc.lo.cc.u32 %4, %9, %12, %4;\n\t"                                                           \
      "madc.hi.cc.u32 %5, %9, %12, %5;\n\t"                                                           \
      "madc.lo.cc.u32 %6, %9, %13, %6;\n\t"                                                           \
      "madc.hi.cc.u32 %7, %9, %13, %7;\n\t"                                                           \
      "addc.u32       %8, %8, 0;"                                                                     \
      : "+r"(A0), "+r"(A1), "+r"(A2), "+r"(A3), "+r"(A4), "+r"(A5), "+r"(A6), "+r"(A7), "+r"(A8)      \
      : "r"(M), "n"(P0), "n"(P1), "n"(P2), "n"(P3))

// ---- merged rows ----

// One CIOS row: accumulate a * w into (T, U), reduce one word, and merge U
// into T while shifting.  On entry T[0..7] holds the running value (< 2p) and
// U is dead; on exit the same.  kFirst: T == 0 on entry.
template <class F, bool kFirst>
__device__ __forceinline__ void cios_row_merged(uint32_t (&T)[9], const fe& a, uint32_t w) {
  uint32_t U[9];
  if (kFirst) {
    ZNTT_MUL8(T[0], T[1], T[2], T[3], T[4], T[5], T[6], T[7], a.v[0], a.v[2], a.v[4], a.v[6], w);
    T[8] = 0;
  } else {
    ZNTT_MAD8("=r", "0", T[0], T[1], T[2], T[3], T[4], T[5], T[6], T[7], T[8], a.v[0], a.v[2], a.v[4], a.v[6], w);
  }
  ZNTT_MUL8(U[0], U[1], U[2], U[3], U[4], U[5], U[6], U[7], a.v[1], a.v[3], a.v[5], a.v[7], w);
  const uint32_t m = T[0] * F::N0;
  // The full first product here, not ZNTT_REDP8: measured in the pass kernel,
  // the merged rows run slower with it (2^24 BN254-Fr 3.848 -> 3.879 ms).
  ZNTT_MADP8("+r", "%8", T[0], T[1], T[2], T[3], T[4], T[5], T[6], T[7], T[8], F::P0, F::P2, F::P4, F::P6, m);
  ZNTT_MADP8("=r", "0", U[0], U[1], U[2], U[3], U[4], U[5], U[6], U[7], U[8], F::P1, F::P3, F::P5, F::P7, m);
  // T[0] is now zero: shift down one word and fold U in.  The result is below
  // 2p < 2^256, so the ninth word of the sum (with U[8]) is zero and not kept.
  asm("add.cc.u32  %0, %0, %8;\n\t"
      "addc.cc.u32 %1, %1, %9;\n\t"
      "addc.cc.u32 %2, %2, %10;\n\t"
      "addc.cc.u32 %3, %3, %11;\n\t"
      "addc.cc.u32 %4, %4, %12;\n\t"
      "addc.cc.u32 %5, %5, %13;\n\t"
      "addc.cc.u32 %6, %6, %14;\n\t"
      "addc.u32    %7, %7, %15;"
      : "+r"(T[1]), "+r"(T[2]), "+r"(T[3]), "+r"(T[4]), "+r"(T[5]), "+r"(T[6]), "+r"(T[7]), "+r"(T[8])
      : "r"(U[0]), "r"(U[1]), "r"(U[2]), "r"(U[3]), "r"(U[4]), "r"(U[5]), "r"(U[6]), "r"(U[7]));
#pragma unroll
  for (int k = 0; k < 8; k++) T[k] = T[k + 1];
}

// Merged-row product, not yet reduced (below 2p).
template <class F>
__device__ __forceinline__ fe fe_mul_merged(const fe& a, const fe& b) {
  uint32_t T[9];
  cios_row_merged<F, true>(T, a, b.v[0]);
#pragma unroll
  for (int i = 1; i < 8; i++) cios_row_merged<F, false>(T, a, b.v[i]);
  fe r;
#pragma unroll
  for (int q = 0; q < 8; q++) r.v[q] = T[q];
  return r;
}

// x * 2^-256 mod p: Montgomery form to the canonical value (REDC of x), the
// merged-row product with multiplier one but no multiplier products -- eight
// reduction rows, about half the products of fe_mul.  For x < p the value
// stays below p + 1, so one conditional subtraction finishes.
template <class F>
__device__ __forceinline__ fe fe_from_mont(const fe& x) {
  uint32_t T[9], U[9];
#pragma unroll
  for (int q = 0; q < 8; q++) T[q] = x.v[q];
  T[8] = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const uint32_t m = T[0] * F::N0;
    ZNTT_REDP8(T[0], T[1], T[2], T[3], T[4], T[5], T[6], T[7], T[8], F::P0, F::P2, F::P4, F::P6, m);
    asm("mul.lo.u32 %0, %8, %9;\n\t"
        "mul.hi.u32 %1, %8, %9;\n\t"
        "mul.lo.u32 %2, %8, %10;\n\t"
        "mul.hi.u32 %3, %8, %10;\n\t"
        "mul.lo.u32 %4, %8, %11;\n\t"
        "mul.hi.u32 %5, %8, %11;\n\t"
        "mul.lo.u32 %6, %8, %12;\n\t"
        "mul.hi.u32 %7, %8, %12;"
        : "=r"(U[0]), "=r"(U[1]), "=r"(U[2]), "=r"(U[3]), "=r"(U[4]), "=r"(U[5]), "=r"(U[6]), "=r"(U[7])
        : "r"(m), "n"(F::P1), "n"(F::P3), "n"(F::P5), "n"(F::P7));
    asm("add.cc.u32  %0, %0, %8;\n\t"
        "addc.cc.u32 %1, %1, %9;\n\t"
        "addc.cc.u32 %2, %2, %10;\n\t"
        "addc.cc.u32 %3, %3, %11;\n\t"
        "addc.cc.u32 %4, %4, %12;\n\t"
        "addc.cc.u32 %5, %5, %13;\n\t"
        "addc.cc.u32 %6, %6, %14;\n\t"
        "addc.u32    %7, %7, %15;"
        : "+r"(T[1]), "+r"(T[2]), "+r"(T[3]), "+r"(T[4]), "+r"(T[5]), "+r"(T[6]), "+r"(T[7]), "+r"(T[8])
        : "r"(U[0]), "r"(U[1]), "r"(U[2]), "r"(U[3]), "r"(U[4]), "r"(U[5]), "r"(U[6]), "r"(U[7]));
#pragma unroll
    for (int k = 0; k < 8; k++) T[k] = T[k + 1];
    T[8] = 0;
  }
  fe r;
#pragma unroll
  for (int q = 0; q < 8; q++) r.v[q] = T[q];
  return fe_reduce<F>(r);
}

// ---- split accumulators ----

// Reduction of one row: add m * p with m = A0 * N0, which zeroes the low word
// of A + 2^32 * B.  Even limbs of p go into A, odd ones into B.
template <class F>
__device__ __forceinline__ void cios_reduce_split(uint32_t (&A)[9], uint32_t (&B)[9]) {
  const uint32_t m = A[0] * F::N0;
  ZNTT_REDP8(A[0], A[1], A[2], A[3], A[4], A[5], A[6], A[7], A[8], F::P0, F::P2, F::P4, F::P6, m);
  ZNTT_MADP8("+r", "%8", B[0], B[1], B[2], B[3], B[4], B[5], B[6], B[7], B[8], F::P1, F::P3, F::P5, F::P7, m);
}

// Divide the running value by 2^32: A[0] is zero, so A and B each move down
// one word (a renaming once unrolled); B's low word, now at word 0, is
// returned as the stray word that the next row adds to A[0].
__device__ __forceinline__ uint32_t cios_shift_split(uint32_t (&A)[9], uint32_t (&B)[9]) {
  const uint32_t s = B[0];
#pragma unroll
  for (int k = 0; k < 8; k++) {
    A[k] = A[k + 1];
    B[k] = B[k + 1];
  }
  return s;
}

// Split-accumulator product, not yet reduced (below 2p).  The running value
// is A + 2^32 * B (+ the stray word s at word 0 between rows).
template <class F>
__device__ __forceinline__ fe fe_mul_split(const fe& a, const fe& b) {
  uint32_t A[9], B[9];
  ZNTT_MUL8(A[0], A[1], A[2], A[3], A[4], A[5], A[6], A[7], a.v[0], a.v[2], a.v[4], a.v[6], b.v[0]);
  ZNTT_MUL8(B[0], B[1], B[2], B[3], B[4], B[5], B[6], B[7], a.v[1], a.v[3], a.v[5], a.v[7], b.v[0]);
  A[8] = 0;
  B[8] = 0;
  cios_reduce_split<F>(A, B);
  uint32_t s = cios_shift_split(A, B);
#pragma unroll
  for (int i = 1; i < 8; i++) {
    const uint32_t w = b.v[i];
    // s joins A[0]; the carry of that add, worth one word, enters the odd
    // chain at B[0] (word 1).
    asm("add.cc.u32     %0, %0, %10;\n\t"
        "madc.lo.cc.u32 %1, %11, %15, %1;\n\t"
        "madc.hi.cc.u32 %2, %11, %15, %2;\n\t"
        "madc.lo.cc.u32 %3, %12, %15, %3;\n\t"
        "madc.hi.cc.u32 %4, %12, %15, %4;\n\t"
        "madc.lo.cc.u32 %5, %13, %15, %5;\n\t"
        "madc.hi.cc.u32 %6, %13, %15, %6;\n\t"
        "madc.lo.cc.u32 %7, %14, %15, %7;\n\t"
        "madc.hi.cc.u32 %8, %14, %15, %8;\n\t"
        "addc.u32       %9, 0, 0;"
        : "+r"(A[0]), "+r"(B[0]), "+r"(B[1]), "+r"(B[2]), "+r"(B[3]), "+r"(B[4]), "+r"(B[5]), "+r"(B[6]),
          "+r"(B[7]), "=r"(B[8])
        : "r"(s), "r"(a.v[1]), "r"(a.v[3]), "r"(a.v[5]), "r"(a.v[7]), "r"(w));
    ZNTT_MAD8("=r", "0", A[0], A[1], A[2], A[3], A[4], A[5], A[6], A[7], A[8], a.v[0], a.v[2], a.v[4], a.v[6], w);
    cios_reduce_split<F>(A, B);
    s = cios_shift_split(A, B);
  }
  // The value is A + s + 2^32 * B < 2p < 2^256 (so B[7] plus the last carry
  // is zero): one add chain merges it.
  fe r;
  asm("add.cc.u32  %0, %8, %16;\n\t"
      "addc.cc.u32 %1, %9, %17;\n\t"
      "addc.cc.u32 %2, %10, %18;\n\t"
      "addc.cc.u32 %3, %11, %19;\n\t"
      "addc.cc.u32 %4, %12, %20;\n\t"
      "addc.cc.u32 %5, %13, %21;\n\t"
      "addc.cc.u32 %6, %14, %22;\n\t"
      "addc.u32    %7, %15, %23;"
      : "=r"(r.v[0]), "=r"(r.v[1]), "=r"(r.v[2]), "=r"(r.v[3]), "=r"(r.v[4]), "=r"(r.v[5]), "=r"(r.v[6]),
        "=r"(r.v[7])
      : "r"(A[0]), "r"(A[1]), "r"(A[2]), "r"(A[3]), "r"(A[4]), "r"(A[5]), "r"(A[6]), "r"(A[7]), "r"(s),
        "r"(B[0]), "r"(B[1]), "r"(B[2]), "r"(B[3]), "r"(B[4]), "r"(B[5]), "r"(B[6]));
  return r;
}

#undef ZNTT_MUL8
#undef ZNTT_MAD8
#undef ZNTT_MADP8

// a * b * 2^-256 mod p.  With a < p and b < 2^256 the product is below 2p;
// kCanon (the default) reduces it to [0, p), as the reference's mul does.
template <class F, bool kCanon = true>
__device__ __forceinline__ fe fe_mul(const fe& a, const fe& b) {
  fe r;
  if constexpr (F::kSplit) r = fe_mul_split<F>(a, b);
  else r = fe_mul_merged<F>(a, b);
  if constexpr (kCanon) r = fe_reduce<F>(r);
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
