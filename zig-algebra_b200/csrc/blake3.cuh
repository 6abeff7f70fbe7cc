// blake3.cuh -- BLAKE3 compressions on the device, written from BLAKE3's
// published specification: the quarter-round G, one compression from a
// chaining value, a whole single-block message, and the parent of two
// digests.  Used by the Merkle commitments (merkle_tree.cuh).
#pragma once

#include <cstdint>

namespace zntt {

namespace {

__device__ __forceinline__ uint32_t rotr(uint32_t x, int r) { return __funnelshift_r(x, x, r); }

// x + y as a multiply-add by `one`, a kernel argument equal to 1 that the
// compiler cannot fold: the add then issues on the multiply-add pipe instead
// of the integer ALU, which the XORs and rotations keep busy.
__device__ __forceinline__ uint32_t madd(uint32_t x, uint32_t one, uint32_t y) {
  uint32_t r;
  asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(x), "r"(one), "r"(y));
  return r;
}

// BLAKE3's quarter-round G.  kMulAdd puts its six adds on the multiply-add
// pipe (the node levels and the small fields' leaves, where that pipe is
// otherwise idle); without it they stay on the ALU (the 256-bit fields'
// leaves, whose Montgomery conversions load the multiply pipe).
template <bool kMulAdd>
__device__ __forceinline__ void b3_g(uint32_t& a, uint32_t& b, uint32_t& c, uint32_t& d, uint32_t x, uint32_t y,
                                     uint32_t one) {
  if constexpr (kMulAdd) {
    a = madd(b, one, madd(x, one, a));
    d = rotr(d ^ a, 16);
    c = madd(d, one, c);
    b = rotr(b ^ c, 12);
    a = madd(b, one, madd(y, one, a));
    d = rotr(d ^ a, 8);
    c = madd(d, one, c);
    b = rotr(b ^ c, 7);
  } else {
    a = a + b + x;
    d = rotr(d ^ a, 16);
    c = c + d;
    b = rotr(b ^ c, 12);
    a = a + b + y;
    d = rotr(d ^ a, 8);
    c = c + d;
    b = rotr(b ^ c, 7);
  }
}

// One BLAKE3 compression: chaining value cv, block msg of `len` bytes (zero
// beyond len), counter 0, the given flags; 7 rounds of the G mixes with the
// message words permuted between rounds; out = state words 0..7 XOR 8..15.
template <bool kMulAdd>
__device__ __forceinline__ void b3_compress(const uint32_t (&cv)[8], const uint32_t (&msg)[16], uint32_t len,
                                            uint32_t flags, uint32_t (&out)[8], uint32_t one) {
  constexpr uint32_t IV[8] = {0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au,
                              0x510E527Fu, 0x9B05688Cu, 0x1F83D9ABu, 0x5BE0CD19u};
  constexpr int PERM[16] = {2, 6, 3, 10, 7, 0, 4, 13, 1, 11, 12, 5, 9, 14, 15, 8};
  uint32_t v[16], m[16];
#pragma unroll
  for (int i = 0; i < 8; i++) v[i] = cv[i];
#pragma unroll
  for (int i = 0; i < 4; i++) v[8 + i] = IV[i];
  v[12] = 0;
  v[13] = 0;
  v[14] = len;
  v[15] = flags;
#pragma unroll
  for (int i = 0; i < 16; i++) m[i] = msg[i];
#pragma unroll
  for (int r = 0; r < 7; r++) {
    b3_g<kMulAdd>(v[0], v[4], v[8], v[12], m[0], m[1], one);
    b3_g<kMulAdd>(v[1], v[5], v[9], v[13], m[2], m[3], one);
    b3_g<kMulAdd>(v[2], v[6], v[10], v[14], m[4], m[5], one);
    b3_g<kMulAdd>(v[3], v[7], v[11], v[15], m[6], m[7], one);
    b3_g<kMulAdd>(v[0], v[5], v[10], v[15], m[8], m[9], one);
    b3_g<kMulAdd>(v[1], v[6], v[11], v[12], m[10], m[11], one);
    b3_g<kMulAdd>(v[2], v[7], v[8], v[13], m[12], m[13], one);
    b3_g<kMulAdd>(v[3], v[4], v[9], v[14], m[14], m[15], one);
    if (r < 6) {
      uint32_t t[16];
#pragma unroll
      for (int i = 0; i < 16; i++) t[i] = m[PERM[i]];
#pragma unroll
      for (int i = 0; i < 16; i++) m[i] = t[i];
    }
  }
#pragma unroll
  for (int i = 0; i < 8; i++) out[i] = v[i] ^ v[i + 8];
}

// BLAKE3 of one block of `len` bytes as a whole message: one compression from
// the IV with CHUNK_START | CHUNK_END | ROOT.
template <bool kMulAdd>
__device__ __forceinline__ void b3_hash_block(const uint32_t (&msg)[16], uint32_t len, uint32_t (&out)[8],
                                              uint32_t one) {
  constexpr uint32_t IV[8] = {0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au,
                              0x510E527Fu, 0x9B05688Cu, 0x1F83D9ABu, 0x5BE0CD19u};
  b3_compress<kMulAdd>(IV, msg, len, 1u | 2u | 8u, out, one);
}

// The parent digest of two child digests.
__device__ __forceinline__ void b3_parent(const uint32_t (&l)[8], const uint32_t (&r)[8], uint32_t (&out)[8],
                                          uint32_t one) {
  uint32_t m[16];
#pragma unroll
  for (int q = 0; q < 8; q++) {
    m[q] = l[q];
    m[8 + q] = r[q];
  }
  b3_hash_block<true>(m, 64, out, one);
}

}  // namespace

}  // namespace zntt
