// fri.cu -- the data-parallel steps of zig-fri's prover on the device:
// Domain.fill (libs/fri/src/root.zig:155-166) and one fold round of proveOn
// (root.zig:396-403), so an LDE's output can stay in HBM through the folds.
//
// A fold round maps the 2^log_n evaluations f of layer r (natural order on the
// subgroup H = <g>, g of order 2^log_n) to the 2^(log_n - 1) values
//   next[j] = (f_j + f_{j+n/2}) / 2 + alpha * (f_j - f_{j+n/2}) / (2 x_j),
// x_j = g^j.  The factors 1 / (2 x_j) = g^-j / 2 come from one table per
// (field, log_n), kept resident: a later round on the subgroup of order
// 2^(log_n - r) needs g^(-j 2^r) / 2, entry j 2^r of the same table.  Field
// arithmetic is exact, so (f_j - f_{j+n/2}) * (g^-j / 2) equals the
// reference's (f_j - f_{j+n/2}).div(x).mul(half_inv) bit for bit.
#include <cuda_runtime.h>

#include <cstring>
#include <map>
#include <vector>

#include "field.cuh"
#include "runtime.hpp"
#include "small.hpp"

namespace zntt {

namespace {

template <class F>
__global__ void fri_fold_kernel(const uint4* __restrict__ in, uint4* __restrict__ out, const uint4* __restrict__ tab,
                                uint64_t half, uint32_t stride, fe half_inv, fe alpha) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < half;
       j += (uint64_t)gridDim.x * blockDim.x) {
    const fe a = fe_load_nc(in + 2 * j), b = fe_load_nc(in + 2 * (j + half));
    const fe even = fe_mul<F>(fe_add<F>(a, b), half_inv);
    const fe odd = fe_mul<F>(fe_sub<F>(a, b), fe_load_nc(tab + 2 * (j << stride)));
    fe_store(out + 2 * j, fe_add<F>(even, fe_mul<F>(alpha, odd)));
  }
}

struct FoldTable {
  uint4* d = nullptr;
  size_t bytes = 0;
};

std::map<std::pair<int, uint32_t>, FoldTable>& fold_tables() {
  static std::map<std::pair<int, uint32_t>, FoldTable> t;
  return t;
}

int grid_of(uint64_t count) { return (int)std::min<uint64_t>((count + 255) / 256, 148 * 16); }

// c * base^i for i < count into out (device), from host power tables.
int powers_device(int field, const uint64_t* base, const uint64_t* c, uint4* out, uint64_t count, cudaStream_t st) {
  std::vector<uint64_t> pw;
  host_power_tables(field, base, pw);
  void* d_pw = nullptr;
  int rc = pool_get(pw.size() * 8, &d_pw);
  if (rc) return rc;
  cudaError_t ce = cudaMemcpyAsync(d_pw, pw.data(), pw.size() * 8, cudaMemcpyHostToDevice, st);
  if (ce == cudaSuccess) ce = launch_powers(field, (const uint4*)d_pw, c, out, count, st);
  cudaError_t ce2 = cudaStreamSynchronize(st);  // the power tables return to the pool
  pool_put(d_pw, pw.size() * 8);
  if (ce == cudaSuccess) ce = ce2;
  if (ce != cudaSuccess) return cuda_fail(ce, "powers");
  return ZNTT_OK;
}

// The table g^-j / 2 (j < 2^(log_n - 1)) for the subgroup of order 2^log_n.
int fold_table(int field, uint32_t log_n, const uint4** out) {
  auto key = std::make_pair(field, log_n);
  auto& tabs = fold_tables();
  auto it = tabs.find(key);
  if (it != tabs.end()) {
    *out = it->second.d;
    return ZNTT_OK;
  }
  const HostField& F = host_field(field);
  uint64_t g[4], ginv[4], two[4], half_inv[4];
  int rc = zntt_primitive_root(field, log_n, g);
  if (rc) return rc;
  F.inv(g, ginv);
  F.from_u64(2, two);
  F.inv(two, half_inv);
  FoldTable t;
  const uint64_t count = 1ull << (log_n - 1);
  t.bytes = count * 32;
  cudaError_t ce = cudaMalloc((void**)&t.d, t.bytes);
  if (ce != cudaSuccess) return cuda_fail(ce, "fold table");
  rc = powers_device(field, ginv, half_inv, t.d, count, ctx().stream);
  if (rc) {
    cudaFree(t.d);
    return rc;
  }
  tabs[key] = t;
  *out = t.d;
  return ZNTT_OK;
}

}  // namespace

int wide_fold_params(int field, uint32_t log_table, const void** tab_out, uint32_t half_inv[8]) {
  const uint4* tab = nullptr;
  int rc = fold_table(field, log_table, &tab);
  if (rc) return rc;
  const HostField& F = host_field(field);
  uint64_t two[4], hi[4];
  F.from_u64(2, two);
  F.inv(two, hi);
  std::memcpy(half_inv, hi, 32);
  *tab_out = tab;
  return ZNTT_OK;
}

void fri_shutdown() {
  for (auto& kv : fold_tables())
    if (kv.second.d) cudaFree(kv.second.d);
  fold_tables().clear();
}

}  // namespace zntt

using namespace zntt;

extern "C" {

int zntt_fri_domain_fill(int field, uint32_t log_n, uint64_t* d_out, void* stream) {
  clear_error();
  if (is_small_field(field)) {
    if (!d_out) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null pointer");
    return small_domain_fill(field, log_n, d_out, stream);
  }
  if (field != kBn254Fr && field != kBls12381Fr) return set_error(ZNTT_ERR_UNSUPPORTED_FIELD, "unsupported field");
  if (!d_out) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null pointer");
  if (log_n > host_field(field).two_adicity)
    return set_error(ZNTT_ERR_ORDER_TOO_LARGE, "domain larger than the two-adicity (Domain.init)");
  if (log_n > 30) return set_error(ZNTT_ERR_OUT_OF_MEMORY, "domain larger than 2^30 elements");
  Context& c = ctx();
  if (c.device < 0) return set_error(ZNTT_ERR_NOT_INITIALIZED, "zntt_init has not been called");
  std::lock_guard<std::recursive_mutex> lock(c.mu);
  uint64_t g[4];
  int rc = zntt_primitive_root(field, log_n, g);
  if (rc) return rc;
  cudaStream_t st = stream ? (cudaStream_t)stream : c.stream;
  // Domain.fill writes x = one, then x *= g: the powers g^i.
  return powers_device(field, g, host_field(field).one, reinterpret_cast<uint4*>(d_out), 1ull << log_n, st);
}

int zntt_fri_fold_device(int field, const uint64_t* d_layer, uint32_t log_n, const uint64_t alpha[4], uint64_t* d_out,
                         uint32_t log_table, void* stream) {
  clear_error();
  if (is_small_field(field)) {
    if (!d_layer || !alpha || !d_out) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null pointer");
    return small_fri_fold(field, d_layer, log_n, alpha, d_out, log_table, stream);
  }
  if (field != kBn254Fr && field != kBls12381Fr) return set_error(ZNTT_ERR_UNSUPPORTED_FIELD, "unsupported field");
  if (!d_layer || !alpha || !d_out) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null pointer");
  const HostField& F = host_field(field);
  if (log_table == 0) log_table = log_n;
  if (log_n < 1 || log_n > log_table)
    return set_error(ZNTT_ERR_INVALID_ARGUMENT, "a fold needs 1 <= log_n <= log_table");
  if (log_table > F.two_adicity) return set_error(ZNTT_ERR_ORDER_TOO_LARGE, "domain larger than the two-adicity");
  if (log_table > 31) return set_error(ZNTT_ERR_OUT_OF_MEMORY, "domain larger than 2^31 elements");
  const uint64_t n = 1ull << log_n, half = n / 2;
  const char* lo = reinterpret_cast<const char*>(d_layer);
  const char* oo = reinterpret_cast<const char*>(d_out);
  if (oo < lo + n * 32 && lo < oo + half * 32) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "fold output overlaps the layer");
  Context& c = ctx();
  if (c.device < 0) return set_error(ZNTT_ERR_NOT_INITIALIZED, "zntt_init has not been called");
  std::lock_guard<std::recursive_mutex> lock(c.mu);
  const uint4* tab = nullptr;
  int rc = fold_table(field, log_table, &tab);
  if (rc) return rc;
  fe hv, av;
  uint64_t two[4], half_inv[4];
  F.from_u64(2, two);
  F.inv(two, half_inv);
  std::memcpy(hv.v, half_inv, 32);
  std::memcpy(av.v, alpha, 32);
  cudaStream_t st = stream ? (cudaStream_t)stream : c.stream;
  const uint32_t stride = log_table - log_n;
  const uint4* in = reinterpret_cast<const uint4*>(d_layer);
  uint4* out = reinterpret_cast<uint4*>(d_out);
  if (field == kBn254Fr)
    fri_fold_kernel<Bn254Fr><<<grid_of(half), 256, 0, st>>>(in, out, tab, half, stride, hv, av);
  else
    fri_fold_kernel<Bls12381Fr><<<grid_of(half), 256, 0, st>>>(in, out, tab, half, stride, hv, av);
  cudaError_t ce = cudaGetLastError();
  if (ce != cudaSuccess) return cuda_fail(ce, "fri fold");
  return ZNTT_OK;
}

}  // extern "C"
