// merkle_rows.cu -- the row commitment of extended columns:
// MerkleTree.init (libs/merkle/src/merkle_tree.zig:70-103) over the rows of
// device columns, leaf i the BLAKE3 hash of row i's toBytes values in column
// order (at most one 1024-byte chunk), in the trees of merkle_tree.cuh.
#include <cuda_runtime.h>

#include <type_traits>

#include "field.cuh"
#include "merkle_tree.cuh"
#include "runtime.hpp"
#include "small.hpp"

namespace zntt {

namespace {

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

}  // namespace

}  // namespace zntt

using namespace zntt;

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
