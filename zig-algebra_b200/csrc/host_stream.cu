// host_stream.cu -- many host vectors through the device with copies and
// transforms overlapped.
//
// zntt_ntt_with_twiddles on one host vector is three dependent steps (upload,
// transform, download), so one call keeps at most one of PCIe's two directions
// and the SMs busy at a time.  For a run of vectors, vector i rides stream
// i mod 3 with its own device buffers: while vector i is being transformed,
// vector i+1 uploads on the host-to-device copy engine and vector i-1
// downloads on the device-to-host one.  Each vector's steps stay in order on
// its stream; vectors that share a stream run one after the other.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "runtime.hpp"
#include "small.hpp"

using namespace zntt;

namespace {
constexpr int kDepth = 3;  // streams (and device buffer pairs) in the pipeline
}  // namespace

extern "C" int zntt_ntt_host_many(const zntt_twiddles* tw, uint64_t* const* h_data, size_t count, int mode) {
  clear_error();
  if (!tw || (count && !h_data)) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null pointer");
  if (mode != ZNTT_FORWARD && mode != ZNTT_INVERSE) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "unknown mode");
  for (size_t i = 0; i < count; i++)
    if (!h_data[i]) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null vector");
  Context& c = ctx();
  if (c.device < 0) return set_error(ZNTT_ERR_NOT_INITIALIZED, "zntt_init has not been called");
  if (is_small_table(tw))
    return set_error(ZNTT_ERR_UNSUPPORTED_FIELD, "the pipelined host API takes BN254-Fr or BLS12-381-Fr tables only");
  std::lock_guard<std::recursive_mutex> lock(c.mu);
  const TwEntry* e = reinterpret_cast<const TwEntry*>(tw);
  const uint32_t log_n = e->log_n;
  const size_t bytes = (size_t)32 << log_n;
  const bool inverse = mode == ZNTT_INVERSE;
  uint64_t ninv[4];
  if (inverse) n_inverse(e->field, log_n, ninv);
  const Plan plan = tuned_plan(e->field, log_n);
  const int depth = (int)std::min<size_t>(kDepth, count);
  void* a[kDepth] = {nullptr, nullptr, nullptr};
  void* b[kDepth] = {nullptr, nullptr, nullptr};
  int rc = ZNTT_OK;
  for (int d = 0; d < depth && !rc; d++) {
    if (!c.pipe[d]) {
      cudaError_t ce = cudaStreamCreateWithFlags(&c.pipe[d], cudaStreamNonBlocking);
      if (ce != cudaSuccess) rc = cuda_fail(ce, "stream");
    }
    if (!rc) rc = pool_get(bytes, &a[d]);
    if (!rc) rc = pool_get(bytes, &b[d]);
  }
  cudaError_t ce = cudaSuccess;
  for (size_t i = 0; i < count && !rc && ce == cudaSuccess; i++) {
    const int d = (int)(i % kDepth);
    cudaStream_t st = c.pipe[d];
    ce = cudaMemcpyAsync(a[d], h_data[i], bytes, cudaMemcpyHostToDevice, st);
    if (ce != cudaSuccess) break;
    rc = run_plan(e->field, e, plan, log_n, (const uint4*)a[d], (uint4*)b[d], nullptr, inverse, inverse, ninv, st);
    if (rc) break;
    ce = cudaMemcpyAsync(h_data[i], b[d], bytes, cudaMemcpyDeviceToHost, st);
  }
  for (int d = 0; d < depth; d++) {
    cudaError_t se = c.pipe[d] ? cudaStreamSynchronize(c.pipe[d]) : cudaSuccess;
    if (ce == cudaSuccess) ce = se;
    if (a[d]) pool_put(a[d], bytes);
    if (b[d]) pool_put(b[d], bytes);
  }
  if (rc) return rc;
  if (ce != cudaSuccess) return cuda_fail(ce, "pipelined transform");
  return ZNTT_OK;
}
