// merkle_tree.cuh -- heap-ordered BLAKE3 Merkle trees on the device, the
// layout of MerkleTree (libs/merkle/src/merkle_tree.zig:70-180): node 1 the
// root, node w + j entry j of the level of width w, node i the hash of nodes
// 2i and 2i + 1, node 0 zero.  A leaf source (layer pairs, folded pairs,
// rows, or digests of an earlier launch) supplies the bottom level.
//
// The tree is built bottom-up in subtrees: a thread hashes two siblings and
// their parent in registers, and a CTA of 256 threads takes its 256 parents
// three levels further through shared memory, where every level still fills
// whole warps.  One launch therefore writes five levels of the tree.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "blake3.cuh"

namespace zntt {

namespace {

constexpr int kThreads = 256;     // CTA size of the subtree kernels
constexpr int kSharedLevels = 3;  // levels a CTA builds in shared memory (256 -> 32 nodes)

__device__ __forceinline__ void store_digest(uint4* nodes, uint64_t i, const uint32_t (&d)[8]) {
  nodes[2 * i] = make_uint4(d[0], d[1], d[2], d[3]);
  nodes[2 * i + 1] = make_uint4(d[4], d[5], d[6], d[7]);
}

__device__ __forceinline__ void load_digest(const uint4* nodes, uint64_t i, uint32_t (&d)[8]) {
  const uint4 a = nodes[2 * i], b = nodes[2 * i + 1];
  d[0] = a.x; d[1] = a.y; d[2] = a.z; d[3] = a.w;
  d[4] = b.x; d[5] = b.y; d[6] = b.z; d[7] = b.w;
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

int grid_for_count(uint64_t count) { return (int)std::min<uint64_t>((count + 255) / 256, 148 * 16); }

// Leaves, then subtrees of five levels while a level has 512 entries or more,
// then the rest in one CTA.
// Sources whose leaves are costly enough to run one per thread in leaf_kernel
// specialize this to true.
template <class T>
struct OneLeafPerThread {
  static constexpr bool value = false;
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
