// noalloc.cu -- an in-place device transform that allocates no memory.
//
// zntt_ntt_device transforms in place by borrowing a scratch vector from the
// library's pool, which can mean a cudaMalloc on the caller's time.  Some
// callers cannot allow that:
//   * services that reserve all of their device memory up front under a fixed
//     budget (the serving loop admits work against an HBM budget) and must not
//     grow past it one request at a time;
//   * programs whose device memory belongs to another allocator (a framework's
//     caching allocator or a fixed arena), where a cudaMalloc behind its back
//     can fail or fragment memory the owner has already promised elsewhere;
//   * latency-critical paths, where cudaMalloc and cudaFree can block the host
//     and serialise with work already queued on the device.
// For them, zntt_ntt_device_inplace_noalloc uses a scratch vector that lives in
// the library image itself: a file-scope __device__ array of kNoAllocMaxLog
// elements' worth (2^18 elements, 8 MiB).  Every GPU that loads the library
// holds this array until the process exits.
//
// The array's host-side name is only a stand-in for the device symbol, so the
// first call on each device looks up its device address with
// cudaGetSymbolAddress (with that device current) and caches it; make that
// first call before any stream capture.  All calls share the one array and it
// keeps whatever the last call left in it; the transform overwrites every
// element it reads, so nothing needs clearing, but calls that overlap on the
// GPU (concurrent streams, or several host threads) race on the scratch.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "runtime.hpp"
#include "small.hpp"

namespace zntt {

constexpr uint32_t kNoAllocMaxLog = 18;
static __device__ __align__(256) uint4 g_noalloc_scratch[2u << kNoAllocMaxLog];

constexpr int kMaxDevices = 64;
static void* g_noalloc_scratch_addr[kMaxDevices];
static std::mutex g_noalloc_mu;

}  // namespace zntt

using namespace zntt;

// In-place transform of 2^log_n device elements (log_n of the twiddle handle,
// at most 18) without allocating device or host memory.  No counterpart in
// the reference.
extern "C" int zntt_ntt_device_inplace_noalloc(const zntt_twiddles* tw, uint64_t* d_data, int mode, void* stream) {
  clear_error();
  if (!tw || !d_data) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null pointer");
  if (mode != ZNTT_FORWARD && mode != ZNTT_INVERSE) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "unknown mode");
  Context& c = ctx();
  if (c.device < 0) return set_error(ZNTT_ERR_NOT_INITIALIZED, "zntt_init has not been called");
  // Held while the table is read and the passes are enqueued, as zntt_ntt_device does, so
  // that zntt_shutdown or a table eviction on another thread cannot free the table meanwhile.
  // Enqueueing does not block, so the lock costs the call nothing on the device.
  std::lock_guard<std::recursive_mutex> ctx_lock(c.mu);
  if (is_small_table(tw))
    return set_error(ZNTT_ERR_UNSUPPORTED_FIELD, "the allocation-free transform takes BN254-Fr or BLS12-381-Fr tables only");
  const TwEntry* e = reinterpret_cast<const TwEntry*>(tw);
  const uint32_t log_n = e->log_n;
  if (log_n > kNoAllocMaxLog)
    return set_error(ZNTT_ERR_INVALID_ARGUMENT,
                     "zntt_ntt_device_inplace_noalloc handles at most 2^18 elements (its static scratch is 8 MiB)");
  int dev = -1;
  cudaError_t ce = cudaGetDevice(&dev);
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaGetDevice");
  if (dev != c.device)
    return set_error(ZNTT_ERR_INVALID_ARGUMENT, "the current device is not the one zntt_init selected");
  if (dev < 0 || dev >= kMaxDevices)
    return set_error(ZNTT_ERR_INVALID_ARGUMENT, "the allocation-free transform serves device ordinals below 64");
  if (log_n == 0) return ZNTT_OK;  // one element: no stage, and the 1/n scale is by one

  uint4* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_scratch_addr[dev]) {
      void* p = nullptr;
      ce = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (ce != cudaSuccess) return cuda_fail(ce, "cudaGetSymbolAddress(no-alloc scratch)");
      g_noalloc_scratch_addr[dev] = p;
    }
    scratch = static_cast<uint4*>(g_noalloc_scratch_addr[dev]);
  }

  // The library's planner (a plan is a value; planning allocates nothing): with 2^11-element
  // tiles and at most 2^18 elements it gives one pass (log_n <= 11) or two.
  const Plan plan = make_plan(log_n, kDefaultShape, kShapes[kDefaultShape].log_tile - 1);
  const uint32_t np = plan.np;
  const PassDesc* passes = plan.p;

  uint64_t ninv[4] = {0, 0, 0, 0};
  const bool inverse = mode == ZNTT_INVERSE;
  if (inverse) {
    const HostField& F = host_field(e->field);
    uint64_t nf[4];
    F.from_u64((uint64_t)1 << log_n, nf);
    F.inv(nf, ninv);
  }
  cudaStream_t st = stream ? (cudaStream_t)stream : c.stream;
  uint4* data = reinterpret_cast<uint4*>(d_data);
  for (uint32_t p = 0; p < np; p++) {
    const bool first = p == 0, last = p + 1 == np;
    PassParams pp;
    std::memset(&pp, 0, sizeof(pp));
    // One pass: in place on the data.  Several: data -> scratch, scratch in
    // place, scratch -> data (a pass writes exactly the positions it read).
    pp.src = first ? data : scratch;
    pp.dst = (np == 1 || last) ? data : scratch;
    pp.tw = e->d_table;
    pp.log_n = log_n;
    pp.S = passes[p].S;
    pp.k = passes[p].k;
    pp.c = passes[p].c;
    pp.first = first;
    pp.inverse = inverse;
    pp.tw0_one = e->tw0_one;
    pp.scale = last && inverse;
    if (pp.scale) std::memcpy(pp.scale_val, ninv, 32);
    pp.src_len = 1ull << log_n;
    pp.dst_len = 1ull << log_n;
    const uint64_t tiles = (1ull << log_n) >> (pp.k + pp.c);
    ce = launch_ntt_pass(e->field, kDefaultShape, pp, tiles, st);
    if (ce != cudaSuccess) return cuda_fail(ce, "ntt pass launch");
  }
  return ZNTT_OK;
}
