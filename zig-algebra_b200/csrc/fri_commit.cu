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
#include <cuda_runtime.h>

#include <cstring>

#include "field.cuh"
#include "runtime.hpp"
#include "small.hpp"

namespace zntt {

namespace {

__device__ __forceinline__ uint32_t rotr(uint32_t x, int r) { return __funnelshift_r(x, x, r); }

__device__ __forceinline__ void b3_g(uint32_t& a, uint32_t& b, uint32_t& c, uint32_t& d, uint32_t x, uint32_t y) {
  a = a + b + x;
  d = rotr(d ^ a, 16);
  c = c + d;
  b = rotr(b ^ c, 12);
  a = a + b + y;
  d = rotr(d ^ a, 8);
  c = c + d;
  b = rotr(b ^ c, 7);
}

// BLAKE3 of one block of `len` bytes (m, zero beyond len) as a whole message:
// 7 rounds of the G mixes, the message words permuted between rounds, output
// words 0..7 of state XOR state words 8..15.
__device__ __forceinline__ void b3_hash_block(const uint32_t (&msg)[16], uint32_t len, uint32_t (&out)[8]) {
  constexpr uint32_t IV[8] = {0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au,
                              0x510E527Fu, 0x9B05688Cu, 0x1F83D9ABu, 0x5BE0CD19u};
  constexpr int PERM[16] = {2, 6, 3, 10, 7, 0, 4, 13, 1, 11, 12, 5, 9, 14, 15, 8};
  uint32_t v[16], m[16];
#pragma unroll
  for (int i = 0; i < 8; i++) v[i] = IV[i];
#pragma unroll
  for (int i = 0; i < 4; i++) v[8 + i] = IV[i];
  v[12] = 0;
  v[13] = 0;
  v[14] = len;
  v[15] = 1u | 2u | 8u;  // CHUNK_START | CHUNK_END | ROOT
#pragma unroll
  for (int i = 0; i < 16; i++) m[i] = msg[i];
#pragma unroll
  for (int r = 0; r < 7; r++) {
    b3_g(v[0], v[4], v[8], v[12], m[0], m[1]);
    b3_g(v[1], v[5], v[9], v[13], m[2], m[3]);
    b3_g(v[2], v[6], v[10], v[14], m[4], m[5]);
    b3_g(v[3], v[7], v[11], v[15], m[6], m[7]);
    b3_g(v[0], v[5], v[10], v[15], m[8], m[9]);
    b3_g(v[1], v[6], v[11], v[12], m[10], m[11]);
    b3_g(v[2], v[7], v[8], v[13], m[12], m[13]);
    b3_g(v[3], v[4], v[9], v[14], m[14], m[15]);
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

__device__ __forceinline__ void store_digest(uint4* nodes, uint64_t i, const uint32_t (&d)[8]) {
  nodes[2 * i] = make_uint4(d[0], d[1], d[2], d[3]);
  nodes[2 * i + 1] = make_uint4(d[4], d[5], d[6], d[7]);
}

// Leaves of a 256-bit field: the canonical value is the Montgomery limbs times
// 2^-256 (fe_from_mont).
template <class F>
__global__ void leaf_kernel_wide(const uint4* __restrict__ layer, uint4* __restrict__ nodes, uint64_t h) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < h; j += (uint64_t)gridDim.x * blockDim.x) {
    const fe a = fe_from_mont<F>(fe_load_nc(layer + 2 * j));
    const fe b = fe_from_mont<F>(fe_load_nc(layer + 2 * (j + h)));
    uint32_t m[16], d[8];
#pragma unroll
    for (int q = 0; q < 8; q++) {
      m[q] = a.v[q];
      m[8 + q] = b.v[q];
    }
    b3_hash_block(m, 64, d);
    store_digest(nodes, h + j, d);
  }
}

// Leaves of a small field: canonical u64 values, `nb` bytes each (8 or 4).
__global__ void leaf_kernel_small(const uint64_t* __restrict__ layer, uint4* __restrict__ nodes, uint64_t h,
                                  uint32_t nb) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < h; j += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t a = __ldg(layer + j), b = __ldg(layer + j + h);
    uint32_t m[16], d[8];
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
    b3_hash_block(m, 2 * nb, d);
    store_digest(nodes, h + j, d);
  }
}

__device__ __forceinline__ void hash_node(uint4* nodes, uint64_t i) {
  const uint4 c0 = nodes[4 * i], c1 = nodes[4 * i + 1], c2 = nodes[4 * i + 2], c3 = nodes[4 * i + 3];
  const uint32_t m[16] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w,
                          c2.x, c2.y, c2.z, c2.w, c3.x, c3.y, c3.z, c3.w};
  uint32_t d[8];
  b3_hash_block(m, 64, d);
  store_digest(nodes, i, d);
}

// One level: nodes w .. 2w-1 from their children (nodes 2w .. 4w-1).
__global__ void level_kernel(uint4* nodes, uint64_t w) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < w; i += (uint64_t)gridDim.x * blockDim.x)
    hash_node(nodes, w + i);
}

// The levels of width w_top, w_top / 2, ..., 1 in one CTA; the barrier between
// levels orders each level's global writes before the next level's reads.
__global__ void top_levels_kernel(uint4* nodes, uint32_t w_top) {
  for (uint32_t w = w_top; w >= 1; w >>= 1) {
    for (uint32_t i = threadIdx.x; i < w; i += blockDim.x) hash_node(nodes, (uint64_t)w + i);
    __syncthreads();
  }
}

int grid_for_count(uint64_t count) { return (int)std::min<uint64_t>((count + 255) / 256, 148 * 16); }

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
    if (field == kBn254Fr)
      leaf_kernel_wide<Bn254Fr><<<grid_for_count(h), 256, 0, st>>>(reinterpret_cast<const uint4*>(d_layer), nodes, h);
    else if (field == kBls12381Fr)
      leaf_kernel_wide<Bls12381Fr><<<grid_for_count(h), 256, 0, st>>>(reinterpret_cast<const uint4*>(d_layer), nodes,
                                                                        h);
    else
      leaf_kernel_small<<<grid_for_count(h), 256, 0, st>>>(d_layer, nodes, h, field == kGoldilocksField ? 8u : 4u);
    ce = cudaGetLastError();
  }
  // Wide levels one launch each; the top 2^11 - 1 nodes in one CTA.
  uint64_t w = h / 2;
  for (; w > 2048 && ce == cudaSuccess; w /= 2) {
    level_kernel<<<grid_for_count(w), 256, 0, st>>>(nodes, w);
    ce = cudaGetLastError();
  }
  if (w >= 1 && ce == cudaSuccess) {
    top_levels_kernel<<<1, 1024, 0, st>>>(nodes, (uint32_t)w);
    ce = cudaGetLastError();
  }
  if (ce == cudaSuccess && root_out) {
    ce = cudaMemcpyAsync(root_out, d_nodes + 32, 32, cudaMemcpyDeviceToHost, st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
  }
  if (ce != cudaSuccess) return cuda_fail(ce, "fri layer commitment");
  return ZNTT_OK;
}
