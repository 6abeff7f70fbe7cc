// fri_commit.cu -- the FRI layer commitment on the device: zig-fri's hashPair
// leaves (libs/fri/src/root.zig:286-295) and MerkleTree.initFromHashes
// (libs/merkle/src/merkle_tree.zig:146-180) over BLAKE3.
//
// Every message here fits one 64-byte block (a leaf is two field elements of
// at most 32 bytes; an inner node is two 32-byte digests), so each hash is one
// BLAKE3 compression from the IV with flags CHUNK_START | CHUNK_END | ROOT,
// counter 0 and the message length as the block length -- BLAKE3's published
// definition for a single-block input.  Leaves hash toBytes of the canonical
// values (little-endian, ceil(bits/8) bytes: 32 for the 256-bit fields, 8 for
// Goldilocks, 4 for BabyBear).  The node array is the reference's heap order:
// node 1 the root, node h + j leaf j (h = n/2), node i the hash of nodes 2i
// and 2i + 1; node 0 is zero.
//
// The tree is built bottom-up in subtrees: a thread hashes two siblings and
// their parent in registers, and a CTA of 256 threads takes its 256 parents
// three levels further through shared memory, where every level still fills
// whole warps.  One launch therefore writes five levels of the tree.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <type_traits>

#include "field.cuh"
#include "runtime.hpp"
#include "small.hpp"
#include "small_field.cuh"

namespace zntt {

namespace {

constexpr int kThreads = 256;     // CTA size of the subtree kernels
constexpr int kSharedLevels = 3;  // levels a CTA builds in shared memory (256 -> 32 nodes)
// The 256-bit fields' leaves keep BLAKE3's adds on the ALU (b3_g below).
constexpr bool kWideLeafMulAdd = false;

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

__device__ __forceinline__ void store_digest(uint4* nodes, uint64_t i, const uint32_t (&d)[8]) {
  nodes[2 * i] = make_uint4(d[0], d[1], d[2], d[3]);
  nodes[2 * i + 1] = make_uint4(d[4], d[5], d[6], d[7]);
}

__device__ __forceinline__ void load_digest(const uint4* nodes, uint64_t i, uint32_t (&d)[8]) {
  const uint4 a = nodes[2 * i], b = nodes[2 * i + 1];
  d[0] = a.x; d[1] = a.y; d[2] = a.z; d[3] = a.w;
  d[4] = b.x; d[5] = b.y; d[6] = b.z; d[7] = b.w;
}

// hashPair leaf j of a 256-bit field: the canonical values of f_j and f_{j+h}
// are the Montgomery limbs times 2^-256 (fe_from_mont).
template <class F>
__device__ __forceinline__ void leaf_wide(const uint4* layer, uint64_t h, uint64_t j, uint32_t (&d)[8],
                                          uint32_t one) {
  const fe a = fe_from_mont<F>(fe_load_nc(layer + 2 * j));
  const fe b = fe_from_mont<F>(fe_load_nc(layer + 2 * (j + h)));
  uint32_t m[16];
#pragma unroll
  for (int q = 0; q < 8; q++) {
    m[q] = a.v[q];
    m[8 + q] = b.v[q];
  }
  b3_hash_block<kWideLeafMulAdd>(m, 64, d, one);
}

// hashPair leaf j of a small field: canonical u64 values, `nb` bytes each (8 or 4).
__device__ __forceinline__ void leaf_small(const uint64_t* layer, uint64_t h, uint64_t j, uint32_t nb,
                                           uint32_t (&d)[8], uint32_t one) {
  const uint64_t a = __ldg(layer + j), b = __ldg(layer + j + h);
  uint32_t m[16];
#pragma unroll
  for (int q = 0; q < 16; q++) m[q] = 0;
  if (nb == 8) {
    m[0] = (uint32_t)a;
    m[1] = (uint32_t)(a >> 32);
    m[2] = (uint32_t)b;
    m[3] = (uint32_t)(b >> 32);
  } else {
    m[0] = (uint32_t)a;
    m[1] = (uint32_t)b;
  }
  b3_hash_block<true>(m, 2 * nb, d, one);
}

// Source of a subtree's bottom level.  Leaf sources hash pairs of layer
// values; the node source reads digests an earlier launch wrote.
struct NodeSource {
  const uint4* nodes;
  uint64_t width;  // the level read: nodes [width, 2 width)
  __device__ __forceinline__ void get(uint64_t j, uint32_t (&d)[8], uint32_t) const {
    load_digest(nodes, width + j, d);
  }
};
template <class F>
struct WideLeafSource {
  const uint4* layer;
  uint64_t h;
  __device__ __forceinline__ void get(uint64_t j, uint32_t (&d)[8], uint32_t one) const {
    leaf_wide<F>(layer, h, j, d, one);
  }
};
struct SmallLeafSource {
  const uint64_t* layer;
  uint64_t h;
  uint32_t nb;
  __device__ __forceinline__ void get(uint64_t j, uint32_t (&d)[8], uint32_t one) const {
    leaf_small(layer, h, j, nb, d, one);
  }
};

// Leaves of the layer a fold round makes, made by the fold itself (one FRI
// round's fold fused with the next round's commitment): leaf j of the new
// layer (h leaves, 2h values) hashes its values j and j + h, and the thread
// that hashes it computes both from the previous layer (values m and m + 2h
// for m = j, j + h: (f_m + f_{m+2h}) / 2 + alpha (f_m - f_{m+2h}) g^-m / 2,
// the factor from the resident table at stride 2^stride) and stores them.
template <class F>
struct WideFoldLeafSource {
  const uint4* prev;
  uint4* next;
  const uint4* tab;
  uint64_t h;
  uint32_t stride;
  fe half_inv, alpha;
  __device__ __forceinline__ fe fold(uint64_t m) const {
    const fe a = fe_load_nc(prev + 2 * m), b = fe_load_nc(prev + 2 * (m + 2 * h));
    const fe even = fe_mul<F>(fe_add<F>(a, b), half_inv);
    const fe odd = fe_mul<F>(fe_sub<F>(a, b), fe_load_nc(tab + 2 * (m << stride)));
    return fe_add<F>(even, fe_mul<F>(alpha, odd));
  }
  __device__ __forceinline__ void get(uint64_t j, uint32_t (&d)[8], uint32_t one) const {
    const fe x = fold(j), y = fold(j + h);
    fe_store(next + 2 * j, x);
    fe_store(next + 2 * (j + h), y);
    const fe a = fe_from_mont<F>(x), b = fe_from_mont<F>(y);
    uint32_t m[16];
#pragma unroll
    for (int q = 0; q < 8; q++) {
      m[q] = a.v[q];
      m[8 + q] = b.v[q];
    }
    b3_hash_block<kWideLeafMulAdd>(m, 64, d, one);
  }
};
template <class SF>
struct SmallFoldLeafSource {
  const uint64_t* prev;
  uint64_t* next;
  const uint64_t* tab;
  uint64_t h;
  uint32_t stride, nb;
  uint64_t half_inv, alpha;  // twiddle form
  __device__ __forceinline__ uint64_t fold(uint64_t m) const {
    const uint64_t a = __ldg(prev + m), b = __ldg(prev + m + 2 * h);
    const uint64_t even = SF::mul(half_inv, SF::add(a, b));
    const uint64_t odd = SF::mul(__ldg(tab + (m << stride)), SF::sub(a, b));
    return SF::add(even, SF::mul(alpha, odd));
  }
  __device__ __forceinline__ void get(uint64_t j, uint32_t (&d)[8], uint32_t one) const {
    const uint64_t a = fold(j), b = fold(j + h);
    next[j] = a;
    next[j + h] = b;
    uint32_t m[16];
#pragma unroll
    for (int q = 0; q < 16; q++) m[q] = 0;
    if (nb == 8) {
      m[0] = (uint32_t)a;
      m[1] = (uint32_t)(a >> 32);
      m[2] = (uint32_t)b;
      m[3] = (uint32_t)(b >> 32);
    } else {
      m[0] = (uint32_t)a;
      m[1] = (uint32_t)b;
    }
    b3_hash_block<true>(m, 2 * nb, d, one);
  }
};

// Leaves of a row commitment (MerkleTree.init over rows, libs/merkle/src/
// merkle_tree.zig:70-103): leaf i is BLAKE3 of the row's toBytes values in
// column order, W words per element, 16 / W elements per 64-byte block (an
// element never straddles blocks), at most 1024 bytes (one chunk): the blocks
// chain from the IV, the first flagged CHUNK_START, the last CHUNK_END | ROOT.
template <int FIELD>
struct RowLeafSource {
  static constexpr uint32_t W = (FIELD == kBn254Fr || FIELD == kBls12381Fr) ? 8 : (FIELD == kGoldilocksField ? 2 : 1);
  static constexpr uint32_t kMaxCols = 256 / W;  // 1024 bytes per row
  const void* col[kMaxCols];
  uint32_t m;
  __device__ __forceinline__ void words(uint32_t c, uint64_t i, uint32_t* w) const {
    if constexpr (W == 8) {
      using F = typename std::conditional<FIELD == kBn254Fr, Bn254Fr, Bls12381Fr>::type;
      const fe a = fe_from_mont<F>(fe_load_nc(reinterpret_cast<const uint4*>(col[c]) + 2 * i));
#pragma unroll
      for (int q = 0; q < 8; q++) w[q] = a.v[q];
    } else {
      const uint64_t v = __ldg(reinterpret_cast<const uint64_t*>(col[c]) + i);
      w[0] = (uint32_t)v;
      if constexpr (W == 2) w[1] = (uint32_t)(v >> 32);
    }
  }
  __device__ __forceinline__ void get(uint64_t i, uint32_t (&d)[8], uint32_t one) const {
    constexpr uint32_t PB = 16 / W;
    constexpr uint32_t IV[8] = {0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au,
                                0x510E527Fu, 0x9B05688Cu, 0x1F83D9ABu, 0x5BE0CD19u};
#pragma unroll
    for (int q = 0; q < 8; q++) d[q] = IV[q];
    const uint32_t nblocks = (m + PB - 1) / PB;
    for (uint32_t b = 0; b < nblocks; b++) {
      uint32_t blk[16];
#pragma unroll
      for (uint32_t e = 0; e < PB; e++) {
        const uint32_t c = b * PB + e;
        if (c < m) {
          words(c, i, blk + e * W);
        } else {
#pragma unroll
          for (uint32_t q = 0; q < W; q++) blk[e * W + q] = 0;
        }
      }
      const uint32_t len = min(m - b * PB, PB) * W * 4;
      const uint32_t flags = (b == 0 ? 1u : 0u) | (b + 1 == nblocks ? 2u | 8u : 0u);
      b3_compress<true>(d, blk, len, flags, d, one);
    }
  }
};

// Every leaf j < h on its own (small trees).
template <class Src>
__global__ void leaf_kernel(Src src, uint4* __restrict__ nodes, uint64_t h, uint32_t one) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < h; j += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t d[8];
    src.get(j, d, one);
    store_digest(nodes, h + j, d);
  }
}

// One subtree per CTA over the level of width w (a multiple of 512): thread t
// takes entries 2u and 2u + 1 of that level (u = 256 b + t), hashes their
// parent in registers, and the CTA builds three more levels in shared memory,
// each still whole warps (128, 64, 32 nodes).  Writes the levels of width
// w/2 .. w/16, and the bottom level itself when it is made here (leaves).
template <class Src, bool kStoreBottom>
__global__ void __launch_bounds__(kThreads) subtree_kernel(Src src, uint4* __restrict__ nodes, uint64_t w,
                                                           uint32_t one) {
  __shared__ uint4 buf_a[kThreads][2];
  __shared__ uint4 buf_b[kThreads / 2][2];
  const uint32_t t = threadIdx.x;
  const uint64_t u = (uint64_t)blockIdx.x * kThreads + t;
  uint32_t l[8], r[8], p[8];
  src.get(2 * u, l, one);
  if (kStoreBottom) store_digest(nodes, w + 2 * u, l);
  src.get(2 * u + 1, r, one);
  if (kStoreBottom) store_digest(nodes, w + 2 * u + 1, r);
  b3_parent(l, r, p, one);
  uint64_t wl = w >> 1;  // width of the level p belongs to
  store_digest(nodes, wl + u, p);
  buf_a[t][0] = make_uint4(p[0], p[1], p[2], p[3]);
  buf_a[t][1] = make_uint4(p[4], p[5], p[6], p[7]);
  __syncthreads();
  uint4(*from)[2] = buf_a;
  uint4(*to)[2] = buf_b;
#pragma unroll 1
  for (uint32_t lev = 1, cnt = kThreads / 2; lev <= kSharedLevels; lev++, cnt >>= 1) {
    wl >>= 1;
    if (t < cnt) {
      const uint4 a0 = from[2 * t][0], a1 = from[2 * t][1], b0 = from[2 * t + 1][0], b1 = from[2 * t + 1][1];
      const uint32_t m[16] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w,
                              b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
      uint32_t d[8];
      b3_hash_block<true>(m, 64, d, one);
      store_digest(nodes, wl + (uint64_t)blockIdx.x * cnt + t, d);
      if (lev < kSharedLevels) {
        to[t][0] = make_uint4(d[0], d[1], d[2], d[3]);
        to[t][1] = make_uint4(d[4], d[5], d[6], d[7]);
      }
    }
    __syncthreads();
    uint4(*x)[2] = from;
    from = to;
    to = x;
  }
}

// The levels of width w_top, w_top / 2, ..., 1 in one CTA; the barrier between
// levels orders each level's global writes before the next level's reads.
__global__ void top_levels_kernel(uint4* nodes, uint32_t w_top, uint32_t one) {
  for (uint32_t w = w_top; w >= 1; w >>= 1) {
    for (uint32_t i = threadIdx.x; i < w; i += blockDim.x) {
      uint32_t l[8], r[8], d[8];
      load_digest(nodes, 2 * ((uint64_t)w + i), l);
      load_digest(nodes, 2 * ((uint64_t)w + i) + 1, r);
      b3_parent(l, r, d, one);
      store_digest(nodes, (uint64_t)w + i, d);
    }
    __syncthreads();
  }
}

// Roofline probe: chained single-block compressions in registers, the node
// levels' instruction mix with no memory traffic.  Each compression's message
// starts with the previous digest, so none can be hoisted or skipped.
__global__ void blake3_probe_kernel(uint32_t* sink, uint32_t iters, uint32_t one) {
  uint32_t m[16], d[8];
#pragma unroll
  for (int q = 0; q < 16; q++) m[q] = threadIdx.x * 977u + blockIdx.x * 131u + q;
  for (uint32_t it = 0; it < iters; it++) {
    b3_hash_block<true>(m, 64, d, one);
#pragma unroll
    for (int q = 0; q < 8; q++) m[q] = d[q];
  }
  uint32_t x = 0;
#pragma unroll
  for (int q = 0; q < 8; q++) x ^= m[q];
  if (x == 0x9e3779b9u) sink[0] = x;
}

int grid_for_count(uint64_t count) { return (int)std::min<uint64_t>((count + 255) / 256, 148 * 16); }

// Leaves, then subtrees of five levels while a level has 512 entries or more,
// then the rest in one CTA.
// The 256-bit folding leaves (two folds, two conversions and a hash each) run one
// per thread in leaf_kernel rather than two plus their parent per thread in
// subtree_kernel: 14 rounds from 2^24 BN254-Fr took 3.01 ms that way and 3.19 ms
// in the subtree kernel.
template <class T>
struct OneLeafPerThread {
  static constexpr bool value = false;
};
template <class F>
struct OneLeafPerThread<WideFoldLeafSource<F>> {
  static constexpr bool value = true;
};

template <class Src>
cudaError_t build_tree(const Src& src, uint4* nodes, uint64_t h, cudaStream_t st) {
  uint64_t w = h;
  if (h >= 2 * kThreads && !OneLeafPerThread<Src>::value) {
    subtree_kernel<Src, true><<<(unsigned)(h / (2 * kThreads)), kThreads, 0, st>>>(src, nodes, h, 1u);
    w = h >> (1 + kSharedLevels);
  } else {
    leaf_kernel<Src><<<grid_for_count(h), kThreads, 0, st>>>(src, nodes, h, 1u);
  }
  cudaError_t ce = cudaGetLastError();
  for (; w >= 2 * kThreads && ce == cudaSuccess; w >>= 1 + kSharedLevels) {
    subtree_kernel<NodeSource, false><<<(unsigned)(w / (2 * kThreads)), kThreads, 0, st>>>(NodeSource{nodes, w},
                                                                                           nodes, w, 1u);
    ce = cudaGetLastError();
  }
  if (w >= 2 && ce == cudaSuccess) {
    top_levels_kernel<<<1, 1024, 0, st>>>(nodes, (uint32_t)(w / 2), 1u);
    ce = cudaGetLastError();
  }
  return ce;
}

}  // namespace

}  // namespace zntt

using namespace zntt;

extern "C" int zntt_fri_commit_layer(int field, const uint64_t* d_layer, uint32_t log_n, uint8_t* d_nodes,
                                     uint8_t* root_out, void* stream) {
  clear_error();
  const bool small = is_small_field(field);
  if (!small && field != kBn254Fr && field != kBls12381Fr)
    return set_error(ZNTT_ERR_UNSUPPORTED_FIELD, "unsupported field");
  if (!d_layer || !d_nodes) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null pointer");
  if (log_n < 1 || log_n > 31) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "a layer of 2^1 .. 2^31 evaluations");
  if (reinterpret_cast<uintptr_t>(d_nodes) % 16)
    return set_error(ZNTT_ERR_INVALID_ARGUMENT, "the node array must be 16-byte aligned");
  const uint64_t n = 1ull << log_n, h = n / 2;
  const size_t ew = small ? 8 : 32;
  const char* lo = reinterpret_cast<const char*>(d_layer);
  const char* no = reinterpret_cast<const char*>(d_nodes);
  if (no < lo + n * ew && lo < no + 2 * h * 32) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "nodes overlap the layer");
  Context& c = ctx();
  if (c.device < 0) return set_error(ZNTT_ERR_NOT_INITIALIZED, "zntt_init has not been called");
  std::lock_guard<std::recursive_mutex> lock(c.mu);
  cudaStream_t st = stream ? (cudaStream_t)stream : c.stream;
  uint4* nodes = reinterpret_cast<uint4*>(d_nodes);
  cudaError_t ce = cudaMemsetAsync(nodes, 0, 32, st);  // node 0 is unused and zero
  if (ce == cudaSuccess) {
    const uint4* wide = reinterpret_cast<const uint4*>(d_layer);
    if (field == kBn254Fr)
      ce = build_tree(WideLeafSource<Bn254Fr>{wide, h}, nodes, h, st);
    else if (field == kBls12381Fr)
      ce = build_tree(WideLeafSource<Bls12381Fr>{wide, h}, nodes, h, st);
    else
      ce = build_tree(SmallLeafSource{d_layer, h, field == kGoldilocksField ? 8u : 4u}, nodes, h, st);
  }
  if (ce == cudaSuccess && root_out) {
    ce = cudaMemcpyAsync(root_out, d_nodes + 32, 32, cudaMemcpyDeviceToHost, st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
  }
  if (ce != cudaSuccess) return cuda_fail(ce, "fri layer commitment");
  return ZNTT_OK;
}

extern "C" int zntt_probe_blake3(double* per_second) {
  clear_error();
  if (!per_second) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null pointer");
  Context& c = ctx();
  if (c.device < 0) return set_error(ZNTT_ERR_NOT_INITIALIZED, "zntt_init has not been called");
  std::lock_guard<std::recursive_mutex> lock(c.mu);
  int sms = 0, per_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, blake3_probe_kernel, kThreads, 0);
  const int blocks = sms * std::max(per_sm, 1);  // one full wave
  const uint32_t iters = 2048;
  void* sink = nullptr;
  int rc = pool_get(64, &sink);
  if (rc) return rc;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  blake3_probe_kernel<<<blocks, kThreads, 0, c.stream>>>((uint32_t*)sink, 64, 1u);  // warm-up
  cudaEventRecord(e0, c.stream);
  blake3_probe_kernel<<<blocks, kThreads, 0, c.stream>>>((uint32_t*)sink, iters, 1u);
  cudaEventRecord(e1, c.stream);
  cudaError_t ce = cudaGetLastError();
  if (ce == cudaSuccess) ce = cudaEventSynchronize(e1);
  float ms = 0;
  if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (ce == cudaSuccess) pool_put(sink, 64);  // the probe has finished with it
  if (ce != cudaSuccess) return cuda_fail(ce, "blake3 probe");
  *per_second = (double)blocks * kThreads * iters / (ms * 1e-3);
  return ZNTT_OK;
}

extern "C" int zntt_fri_fold_commit(int field, const uint64_t* d_layer, uint32_t log_n, const uint64_t alpha[4],
                                    uint64_t* d_out, uint32_t log_table, uint8_t* d_nodes, uint8_t* root_out,
                                    void* stream) {
  clear_error();
  const bool small = is_small_field(field);
  if (!small && field != kBn254Fr && field != kBls12381Fr)
    return set_error(ZNTT_ERR_UNSUPPORTED_FIELD, "unsupported field");
  if (!d_layer || !alpha || !d_out || !d_nodes) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null pointer");
  if (log_table == 0) log_table = log_n;
  if (log_n < 2 || log_n > log_table)
    return set_error(ZNTT_ERR_INVALID_ARGUMENT, "a fold and commitment needs 2 <= log_n <= log_table");
  uint32_t two_adicity = 0;
  if (small) small_field_info(field, nullptr, &two_adicity);
  else two_adicity = host_field(field).two_adicity;
  if (log_table > two_adicity) return set_error(ZNTT_ERR_ORDER_TOO_LARGE, "domain larger than the two-adicity");
  if (log_table > 31) return set_error(ZNTT_ERR_OUT_OF_MEMORY, "domain larger than 2^31 elements");
  if (small) {
    uint64_t p[4];
    small_field_info(field, p, nullptr);
    if (alpha[1] || alpha[2] || alpha[3] || alpha[0] >= p[0])
      return set_error(ZNTT_ERR_INVALID_ARGUMENT, "alpha is not a field element");
  } else if (HostField::geq(alpha, host_field(field).p)) {
    return set_error(ZNTT_ERR_INVALID_ARGUMENT, "alpha is not a field element");
  }
  if (reinterpret_cast<uintptr_t>(d_nodes) % 16)
    return set_error(ZNTT_ERR_INVALID_ARGUMENT, "the node array must be 16-byte aligned");
  const uint64_t n = 1ull << log_n, n2 = n / 2, h = n2 / 2;  // layer, new layer, its leaves
  const size_t ew = small ? 8 : 32;
  const char* lo = reinterpret_cast<const char*>(d_layer);
  const char* oo = reinterpret_cast<const char*>(d_out);
  const char* no = reinterpret_cast<const char*>(d_nodes);
  const size_t lb = n * ew, ob = n2 * ew, nbytes = n2 * 32;
  if ((oo < lo + lb && lo < oo + ob) || (no < lo + lb && lo < no + nbytes) || (no < oo + ob && oo < no + nbytes))
    return set_error(ZNTT_ERR_INVALID_ARGUMENT, "the layer, the new layer and the nodes must not overlap");
  Context& c = ctx();
  if (c.device < 0) return set_error(ZNTT_ERR_NOT_INITIALIZED, "zntt_init has not been called");
  std::lock_guard<std::recursive_mutex> lock(c.mu);
  cudaStream_t st = stream ? (cudaStream_t)stream : c.stream;
  uint4* nodes = reinterpret_cast<uint4*>(d_nodes);
  const uint32_t stride = log_table - log_n;
  cudaError_t ce = cudaSuccess;
  if (small) {
    const uint64_t* tab = nullptr;
    uint64_t hv = 0, av = 0;
    int rc = small_fold_params(field, log_table, alpha, &tab, &hv, &av);
    if (rc) return rc;
    ce = cudaMemsetAsync(nodes, 0, 32, st);
    if (ce == cudaSuccess) {
      if (field == kGoldilocksField)
        ce = build_tree(SmallFoldLeafSource<Goldilocks>{d_layer, d_out, tab, h, stride, 8u, hv, av}, nodes, h, st);
      else
        ce = build_tree(SmallFoldLeafSource<BabyBear>{d_layer, d_out, tab, h, stride, 4u, hv, av}, nodes, h, st);
    }
  } else {
    const void* tab = nullptr;
    fe hv, av;
    int rc = wide_fold_params(field, log_table, &tab, hv.v);
    if (rc) return rc;
    std::memcpy(av.v, alpha, 32);
    const uint4* prev = reinterpret_cast<const uint4*>(d_layer);
    uint4* next = reinterpret_cast<uint4*>(d_out);
    const uint4* t4 = reinterpret_cast<const uint4*>(tab);
    ce = cudaMemsetAsync(nodes, 0, 32, st);
    if (ce == cudaSuccess) {
      if (field == kBn254Fr)
        ce = build_tree(WideFoldLeafSource<Bn254Fr>{prev, next, t4, h, stride, hv, av}, nodes, h, st);
      else
        ce = build_tree(WideFoldLeafSource<Bls12381Fr>{prev, next, t4, h, stride, hv, av}, nodes, h, st);
    }
  }
  if (ce == cudaSuccess && root_out) {
    ce = cudaMemcpyAsync(root_out, d_nodes + 32, 32, cudaMemcpyDeviceToHost, st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
  }
  if (ce != cudaSuccess) return cuda_fail(ce, "fri fold and commitment");
  return ZNTT_OK;
}

namespace {

template <int FIELD>
cudaError_t commit_rows_typed(const uint64_t* const* cols, uint32_t m, uint64_t n, uint4* nodes, cudaStream_t st) {
  RowLeafSource<FIELD> src;
  for (uint32_t c = 0; c < m; c++) src.col[c] = cols[c];
  for (uint32_t c = m; c < RowLeafSource<FIELD>::kMaxCols; c++) src.col[c] = nullptr;
  src.m = m;
  return build_tree(src, nodes, n, st);
}

}  // namespace

extern "C" int zntt_merkle_commit_rows(int field, const uint64_t* const* d_columns, uint32_t num_columns,
                                       uint32_t log_n, uint8_t* d_nodes, uint8_t* root_out, void* stream) {
  clear_error();
  const bool small = is_small_field(field);
  if (!small && field != kBn254Fr && field != kBls12381Fr)
    return set_error(ZNTT_ERR_UNSUPPORTED_FIELD, "unsupported field");
  if (!d_columns || !d_nodes) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null pointer");
  const uint32_t nb = small ? (field == kGoldilocksField ? 8u : 4u) : 32u;
  if (num_columns == 0 || num_columns > 1024 / nb)  // a row of at most 1024 bytes (no overflow)
    return set_error(ZNTT_ERR_INVALID_ARGUMENT, "rows of 1 .. 1024 bytes (one BLAKE3 chunk)");
  if (log_n > 30) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "at most 2^30 rows");
  if (reinterpret_cast<uintptr_t>(d_nodes) % 16)
    return set_error(ZNTT_ERR_INVALID_ARGUMENT, "the node array must be 16-byte aligned");
  const uint64_t n = 1ull << log_n;
  const size_t ew = small ? 8 : 32;
  const char* no = reinterpret_cast<const char*>(d_nodes);
  for (uint32_t c = 0; c < num_columns; c++) {
    if (!d_columns[c]) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null column");
    const char* co = reinterpret_cast<const char*>(d_columns[c]);
    if (no < co + n * ew && co < no + 2 * n * 32)
      return set_error(ZNTT_ERR_INVALID_ARGUMENT, "the nodes overlap a column");
  }
  Context& c = ctx();
  if (c.device < 0) return set_error(ZNTT_ERR_NOT_INITIALIZED, "zntt_init has not been called");
  std::lock_guard<std::recursive_mutex> lock(c.mu);
  cudaStream_t st = stream ? (cudaStream_t)stream : c.stream;
  uint4* nodes = reinterpret_cast<uint4*>(d_nodes);
  cudaError_t ce = cudaMemsetAsync(nodes, 0, 32, st);
  if (ce == cudaSuccess) {
    switch (field) {
      case kBn254Fr: ce = commit_rows_typed<kBn254Fr>(d_columns, num_columns, n, nodes, st); break;
      case kBls12381Fr: ce = commit_rows_typed<kBls12381Fr>(d_columns, num_columns, n, nodes, st); break;
      case kGoldilocksField: ce = commit_rows_typed<kGoldilocksField>(d_columns, num_columns, n, nodes, st); break;
      default: ce = commit_rows_typed<kBabyBearField>(d_columns, num_columns, n, nodes, st);
    }
  }
  if (ce == cudaSuccess && root_out) {
    ce = cudaMemcpyAsync(root_out, d_nodes + 32, 32, cudaMemcpyDeviceToHost, st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
  }
  if (ce != cudaSuccess) return cuda_fail(ce, "row commitment");
  return ZNTT_OK;
}
