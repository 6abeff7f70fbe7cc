// fri_commit.cu -- the FRI layer commitment on the device: zig-fri's hashPair
// leaves (libs/fri/src/root.zig:286-295) and MerkleTree.initFromHashes
// (libs/merkle/src/merkle_tree.zig:146-180) over BLAKE3, the fold of one round
// fused with the next round's commitment, and the BLAKE3 roofline probe.
//
// Every message here fits one 64-byte block (a leaf is two field elements of
// at most 32 bytes; an inner node is two 32-byte digests), so each hash is one
// BLAKE3 compression from the IV with flags CHUNK_START | CHUNK_END | ROOT,
// counter 0 and the message length as the block length -- BLAKE3's published
// definition for a single-block input.  Leaves hash toBytes of the canonical
// values (little-endian, ceil(bits/8) bytes: 32 for the 256-bit fields, 8 for
// Goldilocks, 4 for BabyBear).  The trees are built by merkle_tree.cuh.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "field.cuh"
#include "merkle_tree.cuh"
#include "runtime.hpp"
#include "small.hpp"
#include "small_field.cuh"

namespace zntt {

namespace {

// The 256-bit fields' leaves keep BLAKE3's adds on the ALU (b3_g).
constexpr bool kWideLeafMulAdd = false;

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

// The 256-bit folding leaves (two folds, two conversions and a hash each) run one
// per thread in leaf_kernel rather than two plus their parent per thread in
// subtree_kernel: 14 rounds from 2^24 BN254-Fr took 3.01 ms that way and 3.19 ms
// in the subtree kernel.
template <class F>
struct OneLeafPerThread<WideFoldLeafSource<F>> {
  static constexpr bool value = true;
};

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

