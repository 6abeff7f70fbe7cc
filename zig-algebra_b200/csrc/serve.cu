// serve.cu -- a continuously batching transform server.
//
// Requests (a forward or inverse transform, or a coset low-degree extension,
// with pinned host input and output buffers) are queued by zntt_server_submit
// from any thread.  One worker thread owns the device side:
//   * admission: requests leave the FIFO queue in order while their device
//     buffers (input, output, extension scratch) fit in the HBM budget;
//   * batching: whenever one of the server's stream slots is free, every
//     admitted request that fits the slot's queue capacity becomes one batch:
//     host->device copies, one persistent launch of the batch kernel over all
//     of their passes, device->host copies, an event;
//   * overlap: several slots run at once, so requests that arrive while
//     others are on the GPU are admitted and launched as soon as a slot and
//     memory free up, and their work overlaps on the device;
//   * completion: the worker polls the slots' events, returns the buffers to
//     the pool (they stay allocated, ready for the next request of that size)
//     and the bytes to the budget, and posts completions with timestamps.
// Twiddle tables for every size served stay resident for the server's life.
// With `serial` set the same engine runs one request at a time with plain
// per-pass launches: the baseline the batching is measured against.
#include <cuda_runtime.h>
#include <time.h>

#include <algorithm>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "jobs.hpp"
#include "runtime.hpp"

namespace zntt {

static uint64_t now_ns() {
  timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (uint64_t)ts.tv_sec * 1000000000ull + (uint64_t)ts.tv_nsec;
}

struct SrvReq {
  zntt_request r;
  uint64_t admit_ns = 0;
  void* d_in = nullptr;
  void* d_out = nullptr;
  void* d_coef = nullptr;
  size_t in_bytes = 0, out_bytes = 0, coef_bytes = 0;
  CosetTab* ct = nullptr;
};

struct Slot {
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  BatchPass* h_passes = nullptr;  // pinned staging for the queue
  BatchItem* h_items = nullptr;
  uint32_t* h_flag = nullptr;     // the kernel's error flag, copied back after the batch
  BatchPass* d_passes = nullptr;
  BatchItem* d_items = nullptr;
  uint32_t* d_ctl = nullptr;
  std::vector<SrvReq> reqs;
  bool busy = false;
  uint64_t launched_ns = 0;
};

}  // namespace zntt

using namespace zntt;

struct zntt_server {
  zntt_server_config cfg;
  std::thread worker;
  std::mutex mu;  // guards pending, done, stop, stats counters touched by callers
  std::condition_variable cv_work, cv_done;
  std::deque<zntt_request> pending;
  std::vector<zntt_completion> done;
  bool stop = false;
  std::vector<Slot> slots;
  size_t budget_left = 0;
  size_t in_use = 0;
  TwEntry* tables[32] = {nullptr};
  uint64_t shift_key[4] = {0, 0, 0, 0};
  zntt_server_stats stats;
  size_t cap_passes = 0, cap_items = 0;
  int grid_plain = 0, grid_ext = 0;
  // Request buffers come from one device arena reserved at creation: freed
  // buffers are reused by exact size, new ones are carved from the unused end,
  // and only when the arena is spent does a buffer come from the pool.  A
  // cudaMalloc issued while batches run stalled the worker for hundreds of
  // milliseconds on B200, so steady serving makes none.
  char* arena = nullptr;
  size_t arena_bytes = 0, arena_used = 0;
  std::multimap<size_t, void*> arena_free;
};

namespace zntt {

static size_t req_bytes(const zntt_request& r, size_t* in, size_t* out, size_t* coef) {
  const bool lde = r.kind == ZNTT_JOB_COSET_LDE;
  *in = (size_t)32 << (lde ? r.log_in : r.log_n);
  *out = (size_t)32 << r.log_n;
  *coef = lde ? ((size_t)32 << r.log_in) : 0;
  return *in + *out + *coef;
}

static uint64_t plan_tiles(const Plan& p, uint32_t log_n) {
  uint64_t t = 0;
  for (uint32_t i = 0; i < p.np; i++) t += (1ull << log_n) >> (p.p[i].k + p.p[i].c);
  return t;
}

static void req_work(zntt_server* s, const zntt_request& r, uint64_t* items, uint32_t* passes) {
  const int f = s->cfg.field, sh = kBatchShape;
  const Plan po = batch_plan(f, r.log_n, sh);
  *items = plan_tiles(po, r.log_n);
  *passes = po.np;
  if (r.kind == ZNTT_JOB_COSET_LDE) {
    const Plan pi = batch_plan(f, r.log_in, sh);
    *items += plan_tiles(pi, r.log_in);
    *passes += pi.np;
  }
}

static int table_for(zntt_server* s, uint32_t log_n, TwEntry** out) {
  if (log_n >= 32) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "size out of range");
  if (!s->tables[log_n]) {
    uint64_t root[4];
    int rc = zntt_primitive_root(s->cfg.field, log_n, root);
    if (rc) return rc;
    rc = acquire_table(s->cfg.field, log_n, root, &s->tables[log_n]);
    if (rc) return rc;
  }
  *out = s->tables[log_n];
  return ZNTT_OK;
}

static void post(zntt_server* s, const SrvReq& q, int status, uint64_t t) {
  zntt_completion c;
  c.user_tag = q.r.user_tag;
  c.status = status;
  c.arrival_ns = q.r.arrival_ns;
  c.admit_ns = q.admit_ns;
  c.done_ns = t;
  std::lock_guard<std::mutex> lk(s->mu);
  s->done.push_back(c);
  s->stats.completed++;
}

constexpr size_t kArenaMax = (size_t)8 << 30;

// A request buffer of `bytes` (worker thread only).
static int srv_get(zntt_server* s, size_t bytes, void** out) {
  auto it = s->arena_free.find(bytes);
  if (it != s->arena_free.end()) {
    *out = it->second;
    s->arena_free.erase(it);
    return ZNTT_OK;
  }
  const size_t need = (bytes + 255) & ~(size_t)255;
  if (s->arena && s->arena_used + need <= s->arena_bytes) {
    *out = s->arena + s->arena_used;
    s->arena_used += need;
    return ZNTT_OK;
  }
  return pool_get(bytes, out);
}

static void srv_put(zntt_server* s, void* p, size_t bytes) {
  if (!p) return;
  const char* c = static_cast<const char*>(p);
  if (s->arena && c >= s->arena && c < s->arena + s->arena_bytes) s->arena_free.emplace(bytes, p);
  else pool_put(p, bytes);
}

static void release_req(zntt_server* s, SrvReq& q) {
  srv_put(s, q.d_in, q.in_bytes);
  srv_put(s, q.d_out, q.out_bytes);
  srv_put(s, q.d_coef, q.coef_bytes);
  if (q.ct) release_coset_tab(q.ct);
  const size_t b = q.in_bytes + q.out_bytes + q.coef_bytes;
  s->budget_left += b;
  s->in_use -= b;
  q.d_in = q.d_out = q.d_coef = nullptr;
  q.ct = nullptr;
}

// Completed slots: post their requests and free their memory.
static bool reap(zntt_server* s) {
  bool any = false;
  for (Slot& sl : s->slots) {
    if (!sl.busy) continue;
    cudaError_t q = cudaEventQuery(sl.done);
    if (q == cudaErrorNotReady) continue;
    const uint64_t t = now_ns();
    int status = ZNTT_OK;
    if (q != cudaSuccess) {
      cudaGetLastError();
      status = ZNTT_ERR_DEVICE;
    } else if (*sl.h_flag) {
      status = ZNTT_ERR_TIMEOUT;
    }
    {
      std::lock_guard<std::recursive_mutex> lock(ctx().mu);
      for (SrvReq& r : sl.reqs) release_req(s, r);
    }
    for (SrvReq& r : sl.reqs) post(s, r, status, t);
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->stats.max_batch_ns = std::max<uint64_t>(s->stats.max_batch_ns, t - sl.launched_ns);
    }
    sl.reqs.clear();
    sl.busy = false;
    any = true;
  }
  if (any) s->cv_done.notify_all();
  return any;
}

// Fails every request of a slot that could not be launched.
static void fail_slot(zntt_server* s, Slot& sl, int status) {
  {
    std::lock_guard<std::recursive_mutex> lock(ctx().mu);
    for (SrvReq& r : sl.reqs) release_req(s, r);
  }
  const uint64_t t = now_ns();
  for (SrvReq& r : sl.reqs) post(s, r, status, t);
  sl.reqs.clear();
  s->cv_done.notify_all();
}

static bool launch_into(zntt_server* s, Slot& sl) {
  const int field = s->cfg.field;
  // Admission: FIFO, while the next request fits the budget and the slot.
  const size_t max_jobs = s->cfg.serial ? 1 : (size_t)std::max(1, s->cfg.max_batch_jobs);
  uint64_t items = 0;
  uint32_t passes = 0;
  size_t io_bytes = 0;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    while (!s->pending.empty() && sl.reqs.size() < max_jobs) {
      const zntt_request& r = s->pending.front();
      size_t in, out, coef;
      const size_t b = req_bytes(r, &in, &out, &coef);
      if (b > s->budget_left) break;
      uint64_t it;
      uint32_t np;
      req_work(s, r, &it, &np);
      // Small requests share a batch; one that would push the batch past its
      // transfer cap waits for the next slot, so it does not hold the others.
      if (!sl.reqs.empty() && (items + it > s->cap_items || passes + np > s->cap_passes ||
                               io_bytes + in + out > s->cfg.max_batch_bytes))
        break;
      io_bytes += in + out;
      SrvReq q;
      q.r = r;
      q.in_bytes = in;
      q.out_bytes = out;
      q.coef_bytes = coef;
      s->pending.pop_front();
      s->budget_left -= b;
      s->in_use += b;
      items += it;
      passes += np;
      sl.reqs.push_back(q);
    }
  }
  if (sl.reqs.empty()) return false;
  const uint64_t t_admit = now_ns();
  for (SrvReq& q : sl.reqs) q.admit_ns = t_admit;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stats.peak_bytes = std::max<uint64_t>(s->stats.peak_bytes, s->in_use);
  }

  std::lock_guard<std::recursive_mutex> lock(ctx().mu);
  std::vector<JobPlan> plans(sl.reqs.size());
  const int shape = kBatchShape;
  // One request alone runs as plain per-pass launches: the persistent launch
  // pays off only when several requests share it (its queue upload and launch
  // cost a lone small request about 60 us of latency).
  const bool plain = s->cfg.serial || sl.reqs.size() == 1;
  for (size_t j = 0; j < sl.reqs.size(); j++) {
    SrvReq& q = sl.reqs[j];
    const zntt_request& r = q.r;
    int rc = srv_get(s, q.in_bytes, &q.d_in);
    if (!rc) rc = srv_get(s, q.out_bytes, &q.d_out);
    if (!rc && q.coef_bytes) rc = srv_get(s, q.coef_bytes, &q.d_coef);
    TwEntry* tw = nullptr;
    if (!rc) rc = table_for(s, r.log_n, &tw);
    if (rc) {
      fail_slot(s, sl, rc);
      return true;
    }
    if (r.kind == ZNTT_JOB_NTT) {
      const bool inv = r.mode == ZNTT_INVERSE;
      uint64_t ninv[4];
      if (inv) n_inverse(field, r.log_n, ninv);
      const Plan plan = batch_plan(field, r.log_n, shape);
      plan_transform(plans[j], tw, plan, r.log_n, (const uint4*)q.d_in, (uint4*)q.d_out, (uint4*)q.d_out, inv,
                     inv ? ninv : nullptr, nullptr, 1ull << r.log_n, 1ull << r.log_n);
    } else {
      TwEntry* twi = nullptr;
      rc = table_for(s, r.log_in, &twi);
      if (!rc) rc = acquire_coset_tab(field, r.log_in, r.shift, &q.ct, ctx().stream);
      if (rc) {
        fail_slot(s, sl, rc);
        return true;
      }
      const Plan pi = batch_plan(field, r.log_in, shape);
      const Plan po = batch_plan(field, r.log_n, shape);
      plan_transform(plans[j], twi, pi, r.log_in, (const uint4*)q.d_in, (uint4*)q.d_coef, (uint4*)q.d_coef, true,
                     nullptr, q.ct->d, 1ull << r.log_in, 1ull << r.log_in);
      plan_transform(plans[j], tw, po, r.log_n, (const uint4*)q.d_coef, (uint4*)q.d_out, (uint4*)q.d_out, false,
                     nullptr, nullptr, 1ull << r.log_in, 1ull << r.log_n);
    }
  }

  cudaStream_t st = sl.stream;
  cudaError_t ce = cudaSuccess;
  for (size_t j = 0; j < sl.reqs.size() && ce == cudaSuccess; j++)
    ce = cudaMemcpyAsync(sl.reqs[j].d_in, sl.reqs[j].r.h_in, sl.reqs[j].in_bytes, cudaMemcpyHostToDevice, st);
  *sl.h_flag = 0;
  if (plain) {
    // Plain launches, one pass after another, with the same plans as the batch
    // kernel's (a length-1 transform is one pass of no stage).
    for (size_t p = 0; p < plans[0].passes.size() && ce == cudaSuccess; p++)
      ce = launch_ntt_pass(field, shape, plans[0].passes[p], plans[0].tiles[p], st);
  } else {
    // One persistent launch over every pass of every request, queued level by level.
    std::vector<uint32_t> first(plans.size());
    uint32_t np = 0;
    bool ext = false;
    for (size_t j = 0; j < plans.size(); j++) {
      first[j] = np;
      for (size_t p = 0; p < plans[j].passes.size(); p++) {
        BatchPass& bp = sl.h_passes[np];
        bp.pp = plans[j].passes[p];
        bp.tiles = (uint32_t)plans[j].tiles[p];
        bp.dep = p == 0 ? kNoDep : np - 1;
        ext = ext || pass_needs_ext(bp.pp);
        np++;
      }
    }
    std::vector<size_t> order(plans.size());
    for (size_t j = 0; j < plans.size(); j++) order[j] = j;
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t z) { return plans[a].work > plans[z].work; });
    size_t levels = 0;
    for (auto& jp : plans) levels = std::max(levels, jp.passes.size());
    uint32_t ni = 0;
    for (size_t lvl = 0; lvl < levels; lvl++)
      for (size_t j : order)
        if (lvl < plans[j].passes.size()) {
          const uint32_t pi = first[j] + (uint32_t)lvl;
          for (uint32_t t = 0; t < sl.h_passes[pi].tiles; t++) sl.h_items[ni++] = {pi, t};
        }
    if (ce == cudaSuccess)
      ce = cudaMemcpyAsync(sl.d_passes, sl.h_passes, np * sizeof(BatchPass), cudaMemcpyHostToDevice, st);
    if (ce == cudaSuccess)
      ce = cudaMemcpyAsync(sl.d_items, sl.h_items, ni * sizeof(BatchItem), cudaMemcpyHostToDevice, st);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(sl.d_ctl, 0, (2 + np) * 4, st);
    if (ce == cudaSuccess) {
      const int grid = std::max(1, std::min<int>(ext ? s->grid_ext : s->grid_plain, (int)ni));
      const bool full = batch_all_full(kBatchShape, sl.h_passes, np);
      ce = launch_batch(field, kBatchShape, ext, full, sl.d_passes, sl.d_items, ni, sl.d_ctl, ZNTT_BATCH_SPIN_LIMIT,
                        grid, st);
    }
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(sl.h_flag, sl.d_ctl + 1, 4, cudaMemcpyDeviceToHost, st);
  }
  for (size_t j = 0; j < sl.reqs.size() && ce == cudaSuccess; j++)
    ce = cudaMemcpyAsync(sl.reqs[j].r.h_out, sl.reqs[j].d_out, sl.reqs[j].out_bytes, cudaMemcpyDeviceToHost, st);
  if (ce == cudaSuccess) ce = cudaEventRecord(sl.done, st);
  if (ce != cudaSuccess) {
    cudaGetLastError();
    cudaStreamSynchronize(st);
    fail_slot(s, sl, ZNTT_ERR_DEVICE);
    return true;
  }
  sl.busy = true;
  sl.launched_ns = now_ns();
  uint64_t inflight = 0;
  for (Slot& o : s->slots)
    if (o.busy) inflight += o.reqs.size();
  std::lock_guard<std::mutex> lk(s->mu);
  s->stats.max_launch_ns = std::max<uint64_t>(s->stats.max_launch_ns, sl.launched_ns - t_admit);
  s->stats.batches++;
  s->stats.max_batch_jobs = std::max<uint64_t>(s->stats.max_batch_jobs, sl.reqs.size());
  s->stats.max_inflight_jobs = std::max<uint64_t>(s->stats.max_inflight_jobs, inflight);
  return true;
}

static bool try_launch(zntt_server* s) {
  bool any = false;
  for (Slot& sl : s->slots) {
    if (sl.busy) continue;
    if (launch_into(s, sl)) any = true;
    else break;  // nothing admissible right now
  }
  return any;
}

static void worker_loop(zntt_server* s) {
  cudaSetDevice(ctx().device);
  for (;;) {
    const bool reaped = reap(s);
    const bool launched = try_launch(s);
    bool busy = false;
    for (Slot& sl : s->slots) busy = busy || sl.busy;
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->stop && s->pending.empty() && !busy) break;
    if (!reaped && !launched) {
      // Sleep until an arrival (when a slot is free) or a short poll interval
      // for the GPU to finish something.
      bool free_slot = false;
      for (Slot& sl : s->slots) free_slot = free_slot || !sl.busy;
      if (busy)
        s->cv_work.wait_for(lk, std::chrono::microseconds(20),
                            [&] { return s->stop || (free_slot && !s->pending.empty()); });
      else
        s->cv_work.wait_for(lk, std::chrono::milliseconds(5), [&] { return s->stop || !s->pending.empty(); });
    }
  }
}

static void destroy_slots(zntt_server* s) {
  for (Slot& sl : s->slots) {
    if (sl.stream) cudaStreamSynchronize(sl.stream);
    if (sl.done) cudaEventDestroy(sl.done);
    if (sl.stream) cudaStreamDestroy(sl.stream);
    if (sl.h_passes) cudaFreeHost(sl.h_passes);
    if (sl.h_items) cudaFreeHost(sl.h_items);
    if (sl.h_flag) cudaFreeHost(sl.h_flag);
    if (sl.d_passes) cudaFree(sl.d_passes);
    if (sl.d_items) cudaFree(sl.d_items);
    if (sl.d_ctl) cudaFree(sl.d_ctl);
  }
  s->slots.clear();
}

}  // namespace zntt

extern "C" {

uint64_t zntt_now_ns(void) { return now_ns(); }

int zntt_server_create(const zntt_server_config* cfg, zntt_server** out) {
  clear_error();
  if (!cfg || !out) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null pointer");
  if (cfg->field != kBn254Fr && cfg->field != kBls12381Fr)
    return set_error(ZNTT_ERR_UNSUPPORTED_FIELD, "unsupported field");
  if (ctx().device < 0) return set_error(ZNTT_ERR_NOT_INITIALIZED, "zntt_init has not been called");
  zntt_server* s = new zntt_server();
  s->cfg = *cfg;
  if (s->cfg.slots < 1) s->cfg.slots = 1;
  if (s->cfg.serial) s->cfg.slots = 1;
  if (s->cfg.max_batch_jobs < 1) s->cfg.max_batch_jobs = 256;
  if (s->cfg.max_items < 1024) s->cfg.max_items = 1u << 20;
  if (s->cfg.max_batch_bytes == 0) s->cfg.max_batch_bytes = (size_t)64 << 20;
  s->budget_left = cfg->hbm_budget_bytes;
  std::memset(&s->stats, 0, sizeof(s->stats));
  s->cap_items = s->cfg.max_items;
  s->cap_passes = (size_t)s->cfg.max_batch_jobs * 8;
  s->grid_plain = batch_grid(cfg->field, kBatchShape, false);
  s->grid_ext = batch_grid(cfg->field, kBatchShape, true);
  s->slots.resize(s->cfg.slots);
  cudaError_t ce = cudaSuccess;
  for (Slot& sl : s->slots) {
    if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking);
    if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming);
    if (ce == cudaSuccess) ce = cudaMallocHost((void**)&sl.h_passes, s->cap_passes * sizeof(BatchPass));
    if (ce == cudaSuccess) ce = cudaMallocHost((void**)&sl.h_items, s->cap_items * sizeof(BatchItem));
    if (ce == cudaSuccess) ce = cudaMallocHost((void**)&sl.h_flag, 64);
    if (ce == cudaSuccess) ce = cudaMalloc((void**)&sl.d_passes, s->cap_passes * sizeof(BatchPass));
    if (ce == cudaSuccess) ce = cudaMalloc((void**)&sl.d_items, s->cap_items * sizeof(BatchItem));
    if (ce == cudaSuccess) ce = cudaMalloc((void**)&sl.d_ctl, (2 + s->cap_passes) * 4);
  }
  if (ce == cudaSuccess) {
    s->arena_bytes = std::min(s->cfg.hbm_budget_bytes, kArenaMax) & ~(size_t)255;
    if (s->arena_bytes) ce = cudaMalloc((void**)&s->arena, s->arena_bytes);
  }
  if (ce != cudaSuccess) {
    destroy_slots(s);
    delete s;
    return cuda_fail(ce, "server set-up");
  }
  s->worker = std::thread(worker_loop, s);
  *out = s;
  return ZNTT_OK;
}

int zntt_server_submit(zntt_server* s, const zntt_request* r) {
  clear_error();
  if (!s || !r || !r->h_in || !r->h_out) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null pointer");
  const bool lde = r->kind == ZNTT_JOB_COSET_LDE;
  if ((r->kind != ZNTT_JOB_NTT && !lde) || r->log_n > 28 || (lde && r->log_in > r->log_n) ||
      (!lde && r->mode != ZNTT_FORWARD && r->mode != ZNTT_INVERSE))
    return set_error(ZNTT_ERR_INVALID_ARGUMENT, "malformed request");
  size_t in, out, coef;
  if (req_bytes(*r, &in, &out, &coef) > s->cfg.hbm_budget_bytes) {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stats.rejected++;
    return set_error(ZNTT_ERR_REJECTED, "request larger than the server's HBM budget");
  }
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "server is shutting down");
    s->pending.push_back(*r);
    s->stats.submitted++;
  }
  s->cv_work.notify_one();
  return ZNTT_OK;
}

int zntt_server_poll(zntt_server* s, zntt_completion* out, size_t cap, size_t* n, int wait_ms) {
  if (!s || !n || (cap && !out)) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null pointer");
  std::unique_lock<std::mutex> lk(s->mu);
  if (s->done.empty() && wait_ms > 0)
    s->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return !s->done.empty(); });
  const size_t m = std::min(cap, s->done.size());
  std::copy(s->done.begin(), s->done.begin() + m, out);
  s->done.erase(s->done.begin(), s->done.begin() + m);
  *n = m;
  return ZNTT_OK;
}

int zntt_server_stats_get(zntt_server* s, zntt_server_stats* st) {
  if (!s || !st) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null pointer");
  std::lock_guard<std::mutex> lk(s->mu);
  *st = s->stats;
  st->pending = s->pending.size();
  return ZNTT_OK;
}

int zntt_server_destroy(zntt_server* s) {
  if (!s) return ZNTT_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  if (s->worker.joinable()) s->worker.join();
  {
    std::lock_guard<std::recursive_mutex> lock(ctx().mu);
    destroy_slots(s);
    if (s->arena) cudaFree(s->arena);
    for (TwEntry*& t : s->tables)
      if (t) {
        release_table(t);
        t = nullptr;
      }
  }
  delete s;
  return ZNTT_OK;
}

}  // extern "C"
