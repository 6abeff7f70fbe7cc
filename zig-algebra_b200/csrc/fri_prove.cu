// fri_prove.cu -- zig-fri's prover loop over resident layers: the commit phase
// of proveOn (libs/fri/src/root.zig:372-403: commit layer r, absorb its root,
// draw alpha_r, fold) and the per-query extraction of buildQueries
// (root.zig:551-571, MerkleTree.prove at libs/merkle/src/merkle_tree.zig:206-233).
//
// The layers and their Merkle trees stay in HBM between the phases: the
// reference rebuilds every tree for the queries (root.zig:520-527), here the
// node arrays of the commit phase are read directly.  Only the roots (one per
// round, for the caller's transcript) and the queried values and paths cross
// to the host.
#include <cuda_runtime.h>

#include <cstring>
#include <type_traits>

#include "field.cuh"
#include "runtime.hpp"
#include "small.hpp"

namespace zntt {

namespace {

constexpr uint32_t kMaxRounds = 32;  // layers of at most 2^31 evaluations

struct QueryLayers {
  const void* layer[kMaxRounds];
  const uint4* nodes[kMaxRounds];
};

// toBytes of one element into `words` (nb / 4 little-endian 32-bit words).
template <int FIELD>
__device__ __forceinline__ void element_words(const void* layer, uint64_t i, uint32_t* words) {
  if constexpr (FIELD == kBn254Fr || FIELD == kBls12381Fr) {
    using F = typename std::conditional<FIELD == kBn254Fr, Bn254Fr, Bls12381Fr>::type;
    const fe a = fe_from_mont<F>(fe_load_nc(reinterpret_cast<const uint4*>(layer) + 2 * i));
#pragma unroll
    for (int q = 0; q < 8; q++) words[q] = a.v[q];
  } else if constexpr (FIELD == kGoldilocksField) {
    const uint64_t v = reinterpret_cast<const uint64_t*>(layer)[i];
    words[0] = (uint32_t)v;
    words[1] = (uint32_t)(v >> 32);
  } else {
    words[0] = (uint32_t)reinterpret_cast<const uint64_t*>(layer)[i];
  }
}

// One thread per (query, round): the pair (f_r[j], f_r[j + half]) with
// j = e0 mod half -- the reference's e = j carried between rounds reduces to
// this, the halves being decreasing powers of two -- and the siblings of leaf j
// from the leaf level up (node (half + j) ^ 1, then its parent's sibling, ...).
template <int FIELD>
__global__ void query_kernel(QueryLayers L, const uint64_t* __restrict__ pos, uint32_t nq, uint32_t rounds,
                             uint32_t log_domain, uint32_t* __restrict__ values, uint4* __restrict__ paths) {
  constexpr uint32_t kWords = (FIELD == kBn254Fr || FIELD == kBls12381Fr) ? 8 : (FIELD == kGoldilocksField ? 2 : 1);
  const uint32_t id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= nq * rounds) return;
  const uint32_t q = id / rounds, r = id % rounds;
  const uint32_t log_half = log_domain - r - 1;
  const uint64_t half = 1ull << log_half;
  const uint64_t j = pos[q] & (half - 1);
  uint32_t* v = values + (uint64_t)id * 2 * kWords;
  element_words<FIELD>(L.layer[r], j, v);
  element_words<FIELD>(L.layer[r], j + half, v + kWords);
  // Siblings per query: sum over rounds of log_half = rounds (log_domain - 1) - rounds (rounds - 1) / 2.
  const uint64_t per_query = (uint64_t)rounds * (log_domain - 1) - (uint64_t)rounds * (rounds - 1) / 2;
  const uint64_t before = (uint64_t)r * (log_domain - 1) - (uint64_t)r * (r - 1) / 2;
  uint4* out = paths + 2 * (q * per_query + before);
  const uint4* nodes = L.nodes[r];
  uint64_t p = half + j;
  for (uint32_t level = 0; level < log_half; level++, p >>= 1) {
    out[2 * level] = nodes[2 * (p ^ 1)];
    out[2 * level + 1] = nodes[2 * (p ^ 1) + 1];
  }
}

// Openings of a row commitment (MerkleTree.prove over zntt_merkle_commit_rows'
// tree): one thread per query writes row i's toBytes values in column order and
// the log_n siblings of leaf i from the leaf level up.
struct RowColumns {
  const void* col[256];
};

template <int FIELD>
__global__ void open_rows_kernel(RowColumns C, uint32_t m, uint32_t log_n, const uint4* __restrict__ nodes,
                                 const uint64_t* __restrict__ pos, uint32_t nq, uint32_t* __restrict__ values,
                                 uint4* __restrict__ paths) {
  constexpr uint32_t kWords = (FIELD == kBn254Fr || FIELD == kBls12381Fr) ? 8 : (FIELD == kGoldilocksField ? 2 : 1);
  const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nq) return;
  const uint64_t i = pos[q];
  uint32_t* v = values + (uint64_t)q * m * kWords;
  for (uint32_t c = 0; c < m; c++) element_words<FIELD>(C.col[c], i, v + c * kWords);
  uint4* out = paths + 2 * (uint64_t)q * log_n;
  uint64_t p = (1ull << log_n) + i;
  for (uint32_t level = 0; level < log_n; level++, p >>= 1) {
    out[2 * level] = nodes[2 * (p ^ 1)];
    out[2 * level + 1] = nodes[2 * (p ^ 1) + 1];
  }
}

uint32_t element_bytes(int field) {
  return is_small_field(field) ? (field == kGoldilocksField ? 8u : 4u) : 32u;
}

// alpha is a field element in the layout of `field`: Montgomery limbs below p,
// or a canonical value in word 0 with the other words zero.
bool is_field_element(int field, const uint64_t alpha[4]) {
  if (is_small_field(field)) {
    uint64_t p[4];
    small_field_info(field, p, nullptr);
    return alpha[1] == 0 && alpha[2] == 0 && alpha[3] == 0 && alpha[0] < p[0];
  }
  return !HostField::geq(alpha, host_field(field).p);
}

int check_field_id(int field) {
  if (!is_small_field(field) && field != kBn254Fr && field != kBls12381Fr)
    return set_error(ZNTT_ERR_UNSUPPORTED_FIELD, "unsupported field");
  return ZNTT_OK;
}

}  // namespace

}  // namespace zntt

using namespace zntt;

extern "C" {

int zntt_fri_commit_phase(int field, uint32_t log_domain, uint32_t log_final, uint64_t* const* d_layers,
                          uint8_t* const* d_nodes, uint8_t* roots_out, zntt_fri_challenge_fn challenge, void* user,
                          void* stream) {
  clear_error();
  int rc = check_field_id(field);
  if (rc) return rc;
  // Config.rounds (root.zig:188-195) on the two sizes this call takes.
  if (log_domain == 0 || log_final >= log_domain || log_final > 12)
    return set_error(ZNTT_ERR_INVALID_ARGUMENT, "need 0 <= log_final < log_domain and log_final <= 12");
  if (log_domain > 31) return set_error(ZNTT_ERR_OUT_OF_MEMORY, "a layer of more than 2^31 evaluations");
  const uint32_t rounds = log_domain - log_final;
  if (!d_layers || !d_nodes || !roots_out || !challenge) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null pointer");
  for (uint32_t r = 0; r <= rounds; r++)
    if (!d_layers[r] || (r < rounds && !d_nodes[r]))
      return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null layer or node array");
  Context& c = ctx();
  if (c.device < 0) return set_error(ZNTT_ERR_NOT_INITIALIZED, "zntt_init has not been called");
  // proveOn: log_domain <= F.two_adicity (root.zig:347).
  uint32_t two_adicity = 0;
  if (is_small_field(field)) small_field_info(field, nullptr, &two_adicity);
  else two_adicity = host_field(field).two_adicity;
  if (log_domain > two_adicity) return set_error(ZNTT_ERR_ORDER_TOO_LARGE, "domain larger than the two-adicity");
  std::lock_guard<std::recursive_mutex> lock(c.mu);
  // Round r's fold runs fused with round r + 1's commitment (zntt_fri_fold_commit):
  // alpha_r is known once root r is, and the leaves of layer r + 1 are made from
  // the values the fold computes.  The last fold has no commitment after it.
  uint64_t alpha[4] = {0, 0, 0, 0};
  for (uint32_t r = 0; r < rounds; r++) {
    uint8_t* root = roots_out + 32 * (size_t)r;
    const uint32_t log_n = log_domain - r;
    if (r == 0)
      rc = zntt_fri_commit_layer(field, d_layers[0], log_n, d_nodes[0], root, stream);  // waits for the root
    else
      rc = zntt_fri_fold_commit(field, d_layers[r - 1], log_n + 1, alpha, d_layers[r], log_domain, d_nodes[r], root,
                                stream);
    if (rc) return rc;
    for (int k = 0; k < 4; k++) alpha[k] = 0;
    const int cs = challenge(user, r, root, alpha);
    if (cs != 0) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "the challenge callback reported an error");
    if (!is_field_element(field, alpha)) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "alpha is not a field element");
  }
  rc = zntt_fri_fold_device(field, d_layers[rounds - 1], log_domain - rounds + 1, alpha, d_layers[rounds], log_domain,
                            stream);
  if (rc) return rc;
  cudaStream_t st = stream ? (cudaStream_t)stream : c.stream;
  cudaError_t ce = cudaStreamSynchronize(st);  // the last fold; proveOn returns with every layer made
  if (ce != cudaSuccess) return cuda_fail(ce, "fri commit phase");
  return ZNTT_OK;
}

int zntt_fri_query_extract(int field, uint32_t log_domain, uint32_t rounds, const uint64_t* const* d_layers,
                           const uint8_t* const* d_nodes, const uint64_t* positions, size_t num_queries,
                           uint8_t* values_out, uint8_t* paths_out, void* stream) {
  clear_error();
  int rc = check_field_id(field);
  if (rc) return rc;
  if (rounds == 0 || rounds > log_domain || log_domain > 31)
    return set_error(ZNTT_ERR_INVALID_ARGUMENT, "need 1 <= rounds <= log_domain <= 31");
  if (!d_layers || !d_nodes || !positions || !values_out || !paths_out)
    return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null pointer");
  if (num_queries == 0 || num_queries > (1u << 20))
    return set_error(ZNTT_ERR_INVALID_ARGUMENT, "1 .. 2^20 queries");
  QueryLayers L;
  for (uint32_t r = 0; r < rounds; r++) {
    if (!d_layers[r] || !d_nodes[r]) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null layer or node array");
    L.layer[r] = d_layers[r];
    L.nodes[r] = reinterpret_cast<const uint4*>(d_nodes[r]);
    if (reinterpret_cast<uintptr_t>(d_nodes[r]) % 16)
      return set_error(ZNTT_ERR_INVALID_ARGUMENT, "node arrays must be 16-byte aligned");
  }
  for (size_t q = 0; q < num_queries; q++)
    if (positions[q] >> log_domain) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "a position outside the domain");
  Context& c = ctx();
  if (c.device < 0) return set_error(ZNTT_ERR_NOT_INITIALIZED, "zntt_init has not been called");
  std::lock_guard<std::recursive_mutex> lock(c.mu);
  cudaStream_t st = stream ? (cudaStream_t)stream : c.stream;
  const size_t nb = element_bytes(field);
  const size_t value_bytes = num_queries * rounds * 2 * nb;
  const size_t per_query = (size_t)rounds * (log_domain - 1) - (size_t)rounds * (rounds - 1) / 2;
  const size_t path_bytes = num_queries * per_query * 32;
  const size_t vo = (path_bytes + 15) / 16 * 16;  // paths first (16-byte aligned), then values
  const size_t pos_off = (vo + value_bytes + 15) / 16 * 16;
  const size_t bytes = pos_off + num_queries * 8;
  void* stage = nullptr;
  rc = pool_get(bytes, &stage);
  if (rc) return rc;
  uint8_t* s = static_cast<uint8_t*>(stage);
  uint64_t* d_pos = reinterpret_cast<uint64_t*>(s + pos_off);
  cudaError_t ce = cudaMemcpyAsync(d_pos, positions, num_queries * 8, cudaMemcpyHostToDevice, st);
  if (ce == cudaSuccess) {
    const uint32_t items = (uint32_t)(num_queries * rounds);
    const int grid = (int)((items + 127) / 128);
    uint32_t* vals = reinterpret_cast<uint32_t*>(s + vo);
    uint4* paths = reinterpret_cast<uint4*>(s);
    const uint32_t nq = (uint32_t)num_queries;
    switch (field) {
      case kBn254Fr:
        query_kernel<kBn254Fr><<<grid, 128, 0, st>>>(L, d_pos, nq, rounds, log_domain, vals, paths);
        break;
      case kBls12381Fr:
        query_kernel<kBls12381Fr><<<grid, 128, 0, st>>>(L, d_pos, nq, rounds, log_domain, vals, paths);
        break;
      case kGoldilocksField:
        query_kernel<kGoldilocksField><<<grid, 128, 0, st>>>(L, d_pos, nq, rounds, log_domain, vals, paths);
        break;
      default:
        query_kernel<kBabyBearField><<<grid, 128, 0, st>>>(L, d_pos, nq, rounds, log_domain, vals, paths);
    }
    ce = cudaGetLastError();
  }
  if (ce == cudaSuccess) ce = cudaMemcpyAsync(paths_out, s, path_bytes, cudaMemcpyDeviceToHost, st);
  if (ce == cudaSuccess) ce = cudaMemcpyAsync(values_out, s + vo, value_bytes, cudaMemcpyDeviceToHost, st);
  cudaError_t ce2 = cudaStreamSynchronize(st);  // the staging buffer returns to the pool
  if (ce == cudaSuccess) ce = ce2;
  if (ce2 == cudaSuccess) pool_put(stage, bytes);
  if (ce != cudaSuccess) return cuda_fail(ce, "fri query extraction");
  return ZNTT_OK;
}

}  // extern "C"

extern "C" int zntt_merkle_open_rows(int field, const uint64_t* const* d_columns, uint32_t num_columns,
                                     uint32_t log_n, const uint8_t* d_nodes, const uint64_t* positions,
                                     size_t num_queries, uint8_t* values_out, uint8_t* paths_out, void* stream) {
  clear_error();
  int rc = check_field_id(field);
  if (rc) return rc;
  const uint32_t nb = element_bytes(field);
  if (!d_columns || !d_nodes || !positions || !values_out || (!paths_out && log_n > 0))
    return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null pointer");
  if (num_columns == 0 || num_columns > 1024 / nb)  // a row of at most 1024 bytes (no overflow)
    return set_error(ZNTT_ERR_INVALID_ARGUMENT, "rows of 1 .. 1024 bytes (one BLAKE3 chunk)");
  if (log_n > 30) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "at most 2^30 rows");
  if (num_queries == 0 || num_queries > (1u << 20)) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "1 .. 2^20 queries");
  if (reinterpret_cast<uintptr_t>(d_nodes) % 16)
    return set_error(ZNTT_ERR_INVALID_ARGUMENT, "the node array must be 16-byte aligned");
  RowColumns C;
  for (uint32_t c = 0; c < 256; c++) C.col[c] = nullptr;
  for (uint32_t c = 0; c < num_columns; c++) {
    if (!d_columns[c]) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null column");
    C.col[c] = d_columns[c];
  }
  for (size_t q = 0; q < num_queries; q++)
    if (positions[q] >> log_n) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "a row outside the commitment");
  Context& c = ctx();
  if (c.device < 0) return set_error(ZNTT_ERR_NOT_INITIALIZED, "zntt_init has not been called");
  std::lock_guard<std::recursive_mutex> lock(c.mu);
  cudaStream_t st = stream ? (cudaStream_t)stream : c.stream;
  const size_t path_bytes = num_queries * log_n * 32, value_bytes = num_queries * num_columns * nb;
  const size_t vo = (path_bytes + 15) / 16 * 16, po = (vo + value_bytes + 15) / 16 * 16;
  const size_t bytes = po + num_queries * 8;
  void* stage = nullptr;
  rc = pool_get(bytes, &stage);
  if (rc) return rc;
  uint8_t* s = static_cast<uint8_t*>(stage);
  uint64_t* d_pos = reinterpret_cast<uint64_t*>(s + po);
  cudaError_t ce = cudaMemcpyAsync(d_pos, positions, num_queries * 8, cudaMemcpyHostToDevice, st);
  if (ce == cudaSuccess) {
    const uint32_t nq = (uint32_t)num_queries;
    const int grid = (int)((nq + 127) / 128);
    const uint4* nodes = reinterpret_cast<const uint4*>(d_nodes);
    uint32_t* vals = reinterpret_cast<uint32_t*>(s + vo);
    uint4* paths = reinterpret_cast<uint4*>(s);
    switch (field) {
      case kBn254Fr:
        open_rows_kernel<kBn254Fr><<<grid, 128, 0, st>>>(C, num_columns, log_n, nodes, d_pos, nq, vals, paths);
        break;
      case kBls12381Fr:
        open_rows_kernel<kBls12381Fr><<<grid, 128, 0, st>>>(C, num_columns, log_n, nodes, d_pos, nq, vals, paths);
        break;
      case kGoldilocksField:
        open_rows_kernel<kGoldilocksField><<<grid, 128, 0, st>>>(C, num_columns, log_n, nodes, d_pos, nq, vals, paths);
        break;
      default:
        open_rows_kernel<kBabyBearField><<<grid, 128, 0, st>>>(C, num_columns, log_n, nodes, d_pos, nq, vals, paths);
    }
    ce = cudaGetLastError();
  }
  if (ce == cudaSuccess && path_bytes) ce = cudaMemcpyAsync(paths_out, s, path_bytes, cudaMemcpyDeviceToHost, st);
  if (ce == cudaSuccess) ce = cudaMemcpyAsync(values_out, s + vo, value_bytes, cudaMemcpyDeviceToHost, st);
  cudaError_t ce2 = cudaStreamSynchronize(st);  // the staging buffer returns to the pool
  if (ce == cudaSuccess) ce = ce2;
  if (ce2 == cudaSuccess) pool_put(stage, bytes);
  if (ce != cudaSuccess) return cuda_fail(ce, "row openings");
  return ZNTT_OK;
}
