// batch.cu -- many transforms (and coset low-degree extensions) in one
// persistent launch that drains a device work queue.
//
// A job is one zig-ntt transform (nttWithTwiddles / inttWithTwiddles
// semantics, libs/ntt/src/root.zig:148-212) or one FRI-style coset extension
// (inverse transform of 2^log_in evaluations, zero-pad to 2^log_n, scale
// coefficient i by g^i, forward transform; the composition of zig-ntt and
// libs/poly/src/vector.zig:24-32,68-73).  Each job is planned into passes;
// each pass into tiles.  The queue lists every (pass, tile) item level by
// level, so every item's prerequisite pass has a lower queue index: an item
// only waits for tiles already taken by CTAs that are running, and the queue
// cannot deadlock whatever the grid size.  Waits are bounded; on timeout the
// kernel raises an error flag and every CTA stops at its next item.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "field.cuh"
#include "pass_tile.cuh"
#include "runtime.hpp"

namespace zntt {

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// FULL: every pass of the batch has whole tiles (k + c == LOG_TILE), so the
// tile runs without bound checks, as the plain pass kernel does for such passes.
template <class F, int LOG_TILE, int THREADS, int MINB, bool EXT, bool FULL>
__global__ void __launch_bounds__(THREADS, MINB)
    batch_kernel(const BatchPass* __restrict__ passes, const BatchItem* __restrict__ items, uint32_t n_items,
                 uint32_t* ctl, uint32_t spin_limit) {
  extern __shared__ uint4 sm[];
  __shared__ PassParams s_pp;
  __shared__ uint32_t s_item, s_ok, s_last;  // s_last: the pass whose parameters s_pp holds (warp 0)
  constexpr int kWords = sizeof(PassParams) / 4;
  static_assert(kWords <= 32, "one warp copies a pass's parameters");
  if (threadIdx.x == 0) s_last = kNoDep;
  // Per item: warp 0 takes the next item (lane 0: one atomicAdd, and the
  // bounded wait for the job's previous pass), copies the pass's parameters
  // when they differ from the last item's, one barrier publishes both, the tile
  // runs, and one barrier plus lane 0's release (fence, then the count) makes
  // the tile's stores visible to the CTAs that wait for them -- the pattern of
  // a cooperative grid barrier.  Two barriers and one fence per tile.
  for (;;) {
    if (threadIdx.x < 32) {
      uint32_t it = n_items, ok = 1;
      if (threadIdx.x == 0) {
        if (ld_relaxed(&ctl[1]) == 0) it = atomicAdd(&ctl[0], 1u);
        if (it < n_items) {
          const uint32_t dep = passes[items[it].pass].dep;
          if (dep != kNoDep) {
            const uint32_t need = passes[dep].tiles;
            uint32_t spins = 0;
            while (ld_acquire(&ctl[2 + dep]) < need) {
              if (ld_relaxed(&ctl[1]) != 0) {
                ok = 0;
                break;
              }
              if (++spins > spin_limit) {
                atomicExch(&ctl[1], 1u);
                ok = 0;
                break;
              }
              __nanosleep(256);
            }
          }
        }
        s_item = it;
        s_ok = ok;
      }
      it = __shfl_sync(0xffffffffu, it, 0);
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (it < n_items && ok) {
        const uint32_t pass = items[it].pass;
        const uint32_t last = s_last;
        __syncwarp();
        if (pass != last) {
          if (threadIdx.x < kWords)
            reinterpret_cast<uint32_t*>(&s_pp)[threadIdx.x] =
                reinterpret_cast<const uint32_t*>(&passes[pass].pp)[threadIdx.x];
          if (threadIdx.x == 0) s_last = pass;
        }
      }
    }
    __syncthreads();
    const uint32_t it = s_item;
    if (it >= n_items || !s_ok) break;
    const BatchItem item = items[it];
    // A copy by value: read through shared memory, every use of a parameter
    // would be a load re-issued after each of the tile's barriers (the mixed
    // 520-transform batch 2.94 -> 2.80 ms, 64 coset extensions 16.7 -> 16.3 ms,
    // B200).
    const PassParams pp = s_pp;
    ntt_tile<F, LOG_TILE, THREADS, true, EXT, FULL>(pp, item.tile, sm);
    __syncthreads();  // every thread's stores are issued and its shared-memory reads done
    if (threadIdx.x == 0) {
      __threadfence();  // ... and, through the barrier, visible device-wide before the count
      atomicAdd(&ctl[2 + item.pass], 1u);
    }
  }
}

template <class F, int SH, bool EXT, bool FULL>
static void* batch_ptr() {
  return (void*)batch_kernel<F, kShapes[SH].log_tile, kShapes[SH].threads, kShapes[SH].min_blocks, EXT, FULL>;
}

template <class F, int SH>
static void* batch_shape_ptr(bool ext, bool full) {
  if (ext) return full ? batch_ptr<F, SH, true, true>() : batch_ptr<F, SH, true, false>();
  return full ? batch_ptr<F, SH, false, true>() : batch_ptr<F, SH, false, false>();
}

template <class F>
static void* batch_kernel_ptr(int shape, bool ext, bool full) {
  switch (shape) {
    case 0: return batch_shape_ptr<F, 0>(ext, full);
    case 1: return batch_shape_ptr<F, 1>(ext, full);
    case 2: return batch_shape_ptr<F, 2>(ext, full);
    case 3: return batch_shape_ptr<F, 3>(ext, full);
    default: return batch_shape_ptr<F, 4>(ext, full);
  }
}

cudaError_t configure_batch_kernels() {
  for (int sh = 0; sh < kNumShapes; sh++) {
    for (int v = 0; v < 4; v++) {
      const bool ext = v & 1, full = v & 2;
      cudaError_t e = cudaFuncSetAttribute(batch_kernel_ptr<Bn254Fr>(sh, ext, full),
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, shape_smem_bytes(sh));
      if (e != cudaSuccess) return e;
      e = cudaFuncSetAttribute(batch_kernel_ptr<Bls12381Fr>(sh, ext, full), cudaFuncAttributeMaxDynamicSharedMemorySize,
                               shape_smem_bytes(sh));
      if (e != cudaSuccess) return e;
    }
  }
  return cudaSuccess;
}

int batch_grid(int field, int shape, bool ext) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  void* fn = field == kBn254Fr ? batch_kernel_ptr<Bn254Fr>(shape, ext, false) : batch_kernel_ptr<Bls12381Fr>(shape, ext, false);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kShapes[shape].threads, shape_smem_bytes(shape));
  if (per_sm < 1) per_sm = 1;
  return sms * per_sm;
}

template <class F, int SH, bool EXT, bool FULL>
static void launch_batch_k(const BatchPass* passes, const BatchItem* items, uint32_t n_items, uint32_t* ctl,
                           uint32_t spin_limit, int grid, cudaStream_t st) {
  constexpr PassShape S = kShapes[SH];
  batch_kernel<F, S.log_tile, S.threads, S.min_blocks, EXT, FULL>
      <<<grid, S.threads, shape_smem_bytes(SH), st>>>(passes, items, n_items, ctl, spin_limit);
}

template <class F, int SH>
static void launch_batch_shape(bool ext, bool full, const BatchPass* passes, const BatchItem* items, uint32_t n_items,
                               uint32_t* ctl, uint32_t spin_limit, int grid, cudaStream_t st) {
  if (ext) {
    if (full) launch_batch_k<F, SH, true, true>(passes, items, n_items, ctl, spin_limit, grid, st);
    else launch_batch_k<F, SH, true, false>(passes, items, n_items, ctl, spin_limit, grid, st);
  } else {
    if (full) launch_batch_k<F, SH, false, true>(passes, items, n_items, ctl, spin_limit, grid, st);
    else launch_batch_k<F, SH, false, false>(passes, items, n_items, ctl, spin_limit, grid, st);
  }
}

template <class F>
static void launch_batch_typed(int shape, bool ext, bool full, const BatchPass* passes, const BatchItem* items,
                               uint32_t n_items, uint32_t* ctl, uint32_t spin_limit, int grid, cudaStream_t st) {
  switch (shape) {
    case 0: launch_batch_shape<F, 0>(ext, full, passes, items, n_items, ctl, spin_limit, grid, st); break;
    case 1: launch_batch_shape<F, 1>(ext, full, passes, items, n_items, ctl, spin_limit, grid, st); break;
    case 2: launch_batch_shape<F, 2>(ext, full, passes, items, n_items, ctl, spin_limit, grid, st); break;
    case 3: launch_batch_shape<F, 3>(ext, full, passes, items, n_items, ctl, spin_limit, grid, st); break;
    default: launch_batch_shape<F, 4>(ext, full, passes, items, n_items, ctl, spin_limit, grid, st); break;
  }
}

cudaError_t launch_batch(int field, int shape, bool ext, bool full, const BatchPass* passes, const BatchItem* items,
                         uint32_t n_items, uint32_t* ctl, uint32_t spin_limit, int grid, cudaStream_t st) {
  if (field == kBn254Fr)
    launch_batch_typed<Bn254Fr>(shape, ext, full, passes, items, n_items, ctl, spin_limit, grid, st);
  else
    launch_batch_typed<Bls12381Fr>(shape, ext, full, passes, items, n_items, ctl, spin_limit, grid, st);
  return cudaGetLastError();
}

}  // namespace zntt
