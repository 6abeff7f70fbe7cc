// poly.cu -- polynomial products through the transform kernels.
//
// Polynomial(F, max_degree).mul (libs/poly/src/poly.zig:197-212) sums
// a_i * b_j into coefficient i + j for every pair: (deg a + 1)(deg b + 1) field
// products.  Here the product takes three transforms of n = 2^L >= deg a +
// deg b + 1 points: forward(a) and forward(b), each reading its zero padding
// implicitly, the pointwise product fused into the last pass of forward(b)
// (its per-position scale table is forward(a)), and the inverse with n^-1
// fused into its last pass, which stores only the deg a + deg b + 1
// coefficients.  Field arithmetic is exact, so each coefficient equals the
// schoolbook sum.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "jobs.hpp"
#include "runtime.hpp"
#include "small.hpp"

using namespace zntt;

namespace {

bool is_zero(const uint64_t* x) { return (x[0] | x[1] | x[2] | x[3]) == 0; }

// Index of the last non-zero coefficient, -1 when all are zero (the degree
// Polynomial.normalize computes, poly.zig:100-104).
int64_t degree_of(const uint64_t* c, size_t len) {
  int64_t d = (int64_t)len - 1;
  while (d >= 0 && is_zero(c + 4 * d)) d--;
  return d;
}

bool overlaps(const void* p, size_t pbytes, const void* q, size_t qbytes) {
  const char* a = static_cast<const char*>(p);
  const char* b = static_cast<const char*>(q);
  return a < b + qbytes && b < a + pbytes;
}

uint32_t ceil_log2(uint64_t x) {
  uint32_t L = 0;
  while ((1ull << L) < x) L++;
  return L;
}

// The product on the device, stream-ordered; scratch returns to the pool
// after the stream has finished with it.
int poly_mul_device(const TwEntry* e, const uint64_t* d_a, size_t len_a, const uint64_t* d_b, size_t len_b,
                    uint64_t* d_out, cudaStream_t st) {
  const uint32_t L = e->log_n;
  const size_t bytes = (size_t)32 << L;
  Plan plan = tuned_plan(e->field, L);
  if (L == 0) plan = batch_plan(e->field, 0, plan.shape);  // one pass of no stage: copy and scale
  void* s1 = nullptr;
  void* s2 = nullptr;
  int rc = pool_get(bytes, &s1);
  if (rc) return rc;
  rc = pool_get(bytes, &s2);
  if (rc) {
    pool_put(s1, bytes);
    return rc;
  }
  JobPlan jp;
  plan_poly_mul(jp, e, plan, reinterpret_cast<const uint4*>(d_a), len_a, reinterpret_cast<const uint4*>(d_b), len_b,
                (uint4*)s1, (uint4*)s2, reinterpret_cast<uint4*>(d_out));
  cudaError_t ce = cudaSuccess;
  for (size_t p = 0; p < jp.passes.size() && ce == cudaSuccess; p++)
    ce = launch_ntt_pass(e->field, plan.shape, jp.passes[p], jp.tiles[p], st);
  cudaError_t ce2 = cudaStreamSynchronize(st);
  pool_put(s1, bytes);
  pool_put(s2, bytes);
  if (ce != cudaSuccess) return cuda_fail(ce, "polynomial product");
  if (ce2 != cudaSuccess) return cuda_fail(ce2, "polynomial product");
  return ZNTT_OK;
}

}  // namespace

extern "C" {

int zntt_poly_mul_device(const zntt_twiddles* tw, const uint64_t* d_a, size_t len_a, const uint64_t* d_b,
                         size_t len_b, uint64_t* d_out, void* stream) {
  clear_error();
  if (!tw || !d_a || !d_b || !d_out) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null pointer");
  Context& c = ctx();
  if (c.device < 0) return set_error(ZNTT_ERR_NOT_INITIALIZED, "zntt_init has not been called");
  if (is_small_table(tw))
    return set_error(ZNTT_ERR_UNSUPPORTED_FIELD, "polynomial products take BN254-Fr or BLS12-381-Fr tables only");
  const TwEntry* e = reinterpret_cast<const TwEntry*>(tw);
  const uint64_t n = 1ull << e->log_n;
  if (len_a < 1 || len_b < 1) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "a factor without coefficients");
  if (len_a > n || len_b > n || len_a + len_b - 1 > n)
    return set_error(ZNTT_ERR_INVALID_ARGUMENT, "the product has more coefficients than the transform size");
  const size_t out_bytes = (len_a + len_b - 1) * 32;
  if (overlaps(d_out, out_bytes, d_a, len_a * 32) || overlaps(d_out, out_bytes, d_b, len_b * 32))
    return set_error(ZNTT_ERR_INVALID_ARGUMENT, "the product overlaps a factor");
  std::lock_guard<std::recursive_mutex> lock(c.mu);
  return poly_mul_device(e, d_a, len_a, d_b, len_b, d_out, stream ? (cudaStream_t)stream : c.stream);
}

int zntt_poly_mul(int field, const uint64_t* a, size_t a_len, const uint64_t* b, size_t b_len, size_t max_degree,
                  uint64_t* out, int64_t* out_degree) {
  clear_error();
  if (is_small_field(field)) return small_poly_mul(field, a, a_len, b, b_len, max_degree, out, out_degree);
  if (field != kBn254Fr && field != kBls12381Fr) return set_error(ZNTT_ERR_UNSUPPORTED_FIELD, "unsupported field");
  if ((a_len && !a) || (b_len && !b) || !out || !out_degree) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null pointer");
  if (max_degree >= ((size_t)1 << 58)) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "max_degree out of range");
  // Polynomial.fromCoeffs: more than max_degree + 1 coefficients do not fit.
  if (a_len > max_degree + 1 || b_len > max_degree + 1)
    return set_error(ZNTT_ERR_DEGREE_TOO_LARGE, "a factor has more than max_degree + 1 coefficients");
  const int64_t da = degree_of(a, a_len), db = degree_of(b, b_len);
  const size_t cap_bytes = (max_degree + 1) * 32;
  if (da < 0 || db < 0) {  // a zero factor: the zero polynomial (poly.zig:198)
    std::memset(out, 0, cap_bytes);
    *out_degree = -1;
    return ZNTT_OK;
  }
  const int64_t d = da + db;
  if ((uint64_t)d > max_degree)
    return set_error(ZNTT_ERR_DEGREE_TOO_LARGE, "the product's degree exceeds max_degree (Polynomial.mul)");
  const uint32_t L = ceil_log2((uint64_t)d + 1);
  Context& c = ctx();
  if (c.device < 0) return set_error(ZNTT_ERR_NOT_INITIALIZED, "zntt_init has not been called");
  uint64_t root[4];
  int rc = zntt_primitive_root(field, L, root);
  if (rc) return rc;
  std::lock_guard<std::recursive_mutex> lock(c.mu);
  TwEntry* e = nullptr;
  rc = acquire_table(field, L, root, &e);
  if (rc) return rc;
  const size_t la = (size_t)da + 1, lb = (size_t)db + 1, lo = (size_t)d + 1;
  void* dev[3] = {nullptr, nullptr, nullptr};
  const size_t sizes[3] = {la * 32, lb * 32, lo * 32};
  for (int i = 0; i < 3 && !rc; i++) rc = pool_get(sizes[i], &dev[i]);
  cudaStream_t st = c.stream;
  cudaError_t ce = cudaSuccess;
  if (!rc) {
    ce = cudaMemcpyAsync(dev[0], a, sizes[0], cudaMemcpyHostToDevice, st);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(dev[1], b, sizes[1], cudaMemcpyHostToDevice, st);
    if (ce != cudaSuccess) rc = cuda_fail(ce, "polynomial upload");
  }
  if (!rc) rc = poly_mul_device(e, (const uint64_t*)dev[0], la, (const uint64_t*)dev[1], lb, (uint64_t*)dev[2], st);
  if (!rc) {
    ce = cudaMemcpyAsync(out, dev[2], sizes[2], cudaMemcpyDeviceToHost, st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess) rc = cuda_fail(ce, "polynomial download");
  }
  if (rc) cudaStreamSynchronize(st);  // no copy may still read or write a pooled buffer
  for (int i = 0; i < 3; i++)
    if (dev[i]) pool_put(dev[i], sizes[i]);
  release_table(e);
  if (rc) return rc;
  std::memset(out + 4 * lo, 0, cap_bytes - sizes[2]);
  *out_degree = degree_of(out, lo);  // normalize (poly.zig:210): the leading product is non-zero
  return ZNTT_OK;
}

}  // extern "C"
