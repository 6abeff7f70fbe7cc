// runtime.hpp -- library state shared by the C ABI translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "zntt.h"
#include "host_field.hpp"
#include "kernels.cuh"

namespace zntt {

// A device twiddle table in zig-ntt's flat layout (stage s at entry 2^s - 1).
struct TwEntry {
  int field = 0;
  uint32_t log_n = 0;
  uint64_t root[4] = {0, 0, 0, 0};  // Montgomery form; the key of root-derived tables
  uint4* d_table = nullptr;         // 2^log_n - 1 entries (one entry when log_n == 0)
  size_t bytes = 0;
  int refs = 0;                     // handles + registrations holding it
  bool tw0_one = true;              // every stage's entry 0 equals one
  bool foreign = false;             // uploaded from a caller's table, not derived from a root
  uint64_t last_use = 0;
};

// A host table made by zntt_precompute_twiddles, recognised again by its stage
// addresses; the first two entries of every stage are re-checked on use.
struct Registration {
  int field = 0;
  uint32_t log_n = 0;
  std::vector<const uint64_t*> stage_ptrs;
  std::vector<uint64_t> probe;  // stage s entries 0 and 1 (when present), 4 limbs each
  TwEntry* entry = nullptr;
};

// Pass structure of one transform size.
struct PassDesc {
  uint32_t S, k, c;
};
struct Plan {
  int shape = kDefaultShape;
  uint32_t np = 0;
  PassDesc p[8];
};
// Splits log_n stages into passes of at most kmax stages on tiles of the shape.
Plan make_plan(uint32_t log_n, int shape, uint32_t kmax);
// The plan the tuning table holds for (field, log_n), else the default shape
// with kmax = log_tile - 1.
Plan tuned_plan(int field, uint32_t log_n);
// The tuned stage count for a given shape.
uint32_t tuned_kmax(int field, uint32_t log_n, int shape);

// One measured configuration of the autotuner.
struct TuneEntry {
  int field = 0;
  uint32_t log_n = 0;
  int shape = 0;
  uint32_t kmax = 0;
  double us = 0;
};

// Caching device allocator: freed buffers are kept by exact size for reuse.
// Buffers of at most kSlabMax bytes are carved from kSlabBytes slabs, so a
// burst of small requests (the server's transforms of 2^10..2^15 elements)
// costs one cudaMalloc per slab, not one per buffer: a cudaMalloc issued while
// batches run can stall the host thread that issues it for a long time.
class BufferPool {
 public:
  static constexpr size_t kSlabMax = (size_t)1 << 20;
  static constexpr size_t kSlabBytes = (size_t)64 << 20;
  cudaError_t acquire(size_t bytes, void** out);
  void release(void* p, size_t bytes);
  // Frees the idle buffers that own their memory (slab pieces stay cached).
  void trim();
  // Frees everything, slabs included; no buffer may be in use.
  void release_all();
  size_t cached_bytes() const { return cached_; }
  uint64_t acquires() const { return acquires_; }
  uint64_t device_mallocs() const { return mallocs_; }

 private:
  bool in_slab(const void* p) const;
  std::multimap<size_t, void*> free_;
  std::vector<std::pair<char*, size_t>> slabs_;
  size_t slab_used_ = 0;  // bytes carved from the last slab
  size_t cached_ = 0;
  uint64_t acquires_ = 0;  // acquire() calls
  uint64_t mallocs_ = 0;   // cudaMalloc calls made by acquire()
};

struct Context {
  int device = -1;
  cudaStream_t stream = nullptr;
  std::recursive_mutex mu;
  std::map<std::string, TwEntry*> tw_by_key;  // root-derived tables
  std::vector<TwEntry*> all_tables;
  std::vector<Registration> regs;
  BufferPool pool;
  uint64_t clock = 0;
  size_t table_cache_budget = (size_t)16 << 30;  // unreferenced root tables kept up to this
  std::string gpu_name;
  cudaStream_t pipe[3] = {nullptr, nullptr, nullptr};  // streams of the pipelined host API
  std::vector<TuneEntry> tune;  // best kmax per (field, log_n, shape) on this GPU
};

Context& ctx();
int set_error(int status, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);
void clear_error();

// Root-derived device table for (field, log_n, root); refs incremented.
int acquire_table(int field, uint32_t log_n, const uint64_t* root, TwEntry** out);
void release_table(TwEntry* e);

// Runs the DIT network over 2^log_n device elements: d_src -> d_dst, with
// d_scratch (2^log_n elements) used when d_src == d_dst and there are several
// passes.  `inverse` selects the inttWithTwiddles twiddle mapping; `scale`
// multiplies every output by `scale_val` (Montgomery form) after the last stage.
int run_transform(int field, const TwEntry* tw, uint32_t log_n, const uint4* d_src, uint4* d_dst,
                  uint4* d_scratch, bool inverse, bool scale, const uint64_t* scale_val, cudaStream_t st);
// The same with an explicit plan (used by the autotuner).
int run_plan(int field, const TwEntry* tw, const Plan& plan, uint32_t log_n, const uint4* d_src, uint4* d_dst,
             uint4* d_scratch, bool inverse, bool scale, const uint64_t* scale_val, cudaStream_t st);

// Pool buffer helpers shared by the translation units.
int pool_get(size_t bytes, void** out);
void pool_put(void* p, size_t bytes);
// n^-1 in Montgomery form.
void n_inverse(int field, uint32_t log_n, uint64_t* out);
// The three power tables of `base` the twiddle and powers kernels expand.
void host_power_tables(int field, const uint64_t* base, std::vector<uint64_t>& pw);

}  // namespace zntt
