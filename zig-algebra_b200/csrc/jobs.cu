// jobs.cu -- host side of batches, coset low-degree extensions and the
// autotuner.
//
// A batch turns a list of jobs into one persistent launch (batch.cu): every
// job is planned into passes and every pass into tiles, and the tiles are
// queued level by level.  A coset extension job is the composition the
// reference performs with zig-ntt and libs/poly: inttWithTwiddles over the
// 2^log_in evaluations, zero-pad to 2^log_n, multiply coefficient i by g^i,
// nttWithTwiddles over 2^log_n.  Here the 1/n scale and g^i are one table
// (n^-1 g^i) applied in the inverse's last pass, and the zero padding is read
// implicitly by the forward's first pass, so an extension is four passes with
// no extra sweep over memory.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "jobs.hpp"
#include "runtime.hpp"
#include "small.hpp"

namespace zntt {

static std::vector<CosetTab*> g_coset_tabs;

int acquire_coset_tab(int field, uint32_t log_in, const uint64_t* shift, CosetTab** out, cudaStream_t st) {
  for (CosetTab* t : g_coset_tabs) {
    if (t->field == field && t->log_in == log_in && std::memcmp(t->shift, shift, 32) == 0) {
      t->refs++;
      *out = t;
      return ZNTT_OK;
    }
  }
  CosetTab* t = new CosetTab();
  t->field = field;
  t->log_in = log_in;
  std::memcpy(t->shift, shift, 32);
  t->bytes = ((size_t)32) << log_in;
  cudaError_t ce = cudaMalloc((void**)&t->d, t->bytes);
  if (ce != cudaSuccess) {
    delete t;
    return cuda_fail(ce, "coset scale table");
  }
  std::vector<uint64_t> pw;
  host_power_tables(field, shift, pw);
  uint64_t ninv[4];
  n_inverse(field, log_in, ninv);
  void* d_pw = nullptr;
  int rc = pool_get(pw.size() * 8, &d_pw);
  if (rc) {
    cudaFree(t->d);
    delete t;
    return rc;
  }
  ce = cudaMemcpyAsync(d_pw, pw.data(), pw.size() * 8, cudaMemcpyHostToDevice, st);
  if (ce == cudaSuccess) ce = launch_powers(field, (const uint4*)d_pw, ninv, t->d, 1ull << log_in, st);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
  pool_put(d_pw, pw.size() * 8);
  if (ce != cudaSuccess) {
    cudaFree(t->d);
    delete t;
    return cuda_fail(ce, "coset scale table");
  }
  t->refs = 1;
  g_coset_tabs.push_back(t);
  *out = t;
  return ZNTT_OK;
}

// Tables stay resident when their last user lets go (a cudaFree would
// synchronise the device behind work in flight, and the next extension of the
// same size would rebuild the table); zntt_shutdown frees them.
void release_coset_tab(CosetTab* t) {
  if (!t) return;
  if (t->refs > 0) t->refs--;
}

void free_coset_tabs() {
  for (CosetTab* t : g_coset_tabs) {
    if (t->d) cudaFree(t->d);
    delete t;
  }
  g_coset_tabs.clear();
}

static PassParams pass_params(const TwEntry* tw, uint32_t log_n, const PassDesc& d, bool first, bool inverse,
                              const uint4* src, uint4* dst) {
  PassParams pp;
  std::memset(&pp, 0, sizeof(pp));
  pp.src = src;
  pp.dst = dst;
  pp.tw = tw->d_table;
  pp.log_n = log_n;
  pp.S = d.S;
  pp.k = d.k;
  pp.c = d.c;
  pp.first = first;
  pp.inverse = inverse;
  pp.tw0_one = tw->tw0_one;
  pp.src_len = 1ull << log_n;
  pp.dst_len = 1ull << log_n;
  return pp;
}

// A batch plan: the tuned plan, and for a length-1 vector one pass of no stage
// (a copy, scaled by 1/1 for the inverse) so that every job writes its output.
Plan batch_plan(int field, uint32_t log_n, int shape) {
  Plan plan = make_plan(log_n, shape, tuned_kmax(field, log_n, shape));
  if (log_n == 0) {
    plan.np = 1;
    plan.p[0] = {0, 0, 0};
  }
  return plan;
}

// Appends the passes of one transform src -> dst (mid: where passes after the
// first run in place).
void plan_transform(JobPlan& jp, const TwEntry* tw, const Plan& plan, uint32_t log_n, const uint4* src,
                           uint4* mid, uint4* dst, bool inverse, const uint64_t* scale_val, const uint4* scale_tab,
                           uint64_t src_len, uint64_t dst_len) {
  for (uint32_t p = 0; p < plan.np; p++) {
    const bool first = p == 0, last = p + 1 == plan.np;
    PassParams pp = pass_params(tw, log_n, plan.p[p], first, inverse, first ? src : mid, last ? dst : mid);
    if (first) pp.src_len = src_len;
    if (last) pp.dst_len = dst_len;
    if (last && (scale_val || scale_tab)) {
      pp.scale = 1;
      if (scale_val) std::memcpy(pp.scale_val, scale_val, 32);
      pp.scale_tab = scale_tab;
    }
    jp.passes.push_back(pp);
    jp.tiles.push_back((1ull << log_n) >> (plan.p[p].k + plan.p[p].c));
    jp.work += ((size_t)1 << log_n) * plan.p[p].k;
  }
}

// Polynomial.mul (libs/poly/src/poly.zig:197-212) computes the product
// coefficients c_k = sum_{i+j=k} a_i b_j directly.  With 2^log_n >= len_a +
// len_b - 1 points the cyclic convolution of the zero-padded inputs is that
// linear product, and by the convolution theorem it is
// intt(ntt(a) . ntt(b)).  Field arithmetic is exact, so every coefficient is
// the schoolbook sum's canonical value.
void plan_poly_mul(JobPlan& jp, const TwEntry* tw, const Plan& plan, const uint4* a, uint64_t len_a, const uint4* b,
                   uint64_t len_b, uint4* s1, uint4* s2, uint4* dst) {
  const uint32_t L = tw->log_n;
  const uint64_t n = 1ull << L;
  uint64_t ninv[4];
  n_inverse(tw->field, L, ninv);
  plan_transform(jp, tw, plan, L, a, s1, s1, false, nullptr, nullptr, len_a, n);
  plan_transform(jp, tw, plan, L, b, s2, s2, false, nullptr, s1, len_b, n);
  plan_transform(jp, tw, plan, L, s2, s1, dst, true, ninv, nullptr, n, len_a + len_b - 1);
}

}  // namespace zntt

using namespace zntt;

struct zntt_batch {
  int field = 0;
  int shape = 0;
  std::vector<BatchPass> passes;
  std::vector<BatchItem> items;
  BatchPass* d_passes = nullptr;
  BatchItem* d_items = nullptr;
  uint32_t* d_ctl = nullptr;
  size_t ctl_words = 0;
  int grid = 0;
  bool ext = false;   // some pass pads or scales by a table
  bool full = false;  // every pass has whole tiles (the kernel runs without bound checks)
  uint32_t spin_limit = ZNTT_BATCH_SPIN_LIMIT;  // x ~0.25-1 us: a stalled dependency gives up after seconds
  std::vector<std::pair<void*, size_t>> scratch;  // pool buffers owned by the batch
  std::vector<CosetTab*> coset_tabs;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
};

static void free_batch(zntt_batch* b) {
  if (b->graph_exec) cudaGraphExecDestroy(b->graph_exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->d_passes) cudaFree(b->d_passes);
  if (b->d_items) cudaFree(b->d_items);
  if (b->d_ctl) cudaFree(b->d_ctl);
  for (auto& s : b->scratch) pool_put(s.first, s.second);
  for (CosetTab* t : b->coset_tabs) release_coset_tab(t);
  delete b;
}

static const TwEntry* tw_of(const zntt_twiddles* h) { return reinterpret_cast<const TwEntry*>(h); }

extern "C" {

int zntt_batch_create(int field, const zntt_job* jobs, size_t n_jobs, int shape, zntt_batch** out) {
  clear_error();
  if (field != kBn254Fr && field != kBls12381Fr) return set_error(ZNTT_ERR_UNSUPPORTED_FIELD, "unsupported field");
  if (!out || (n_jobs && !jobs)) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null pointer");
  if (shape >= kNumShapes) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "unknown pass shape");
  Context& c = ctx();
  if (c.device < 0) return set_error(ZNTT_ERR_NOT_INITIALIZED, "zntt_init has not been called");
  std::lock_guard<std::recursive_mutex> lock(c.mu);
  // Validate every job before allocating anything.
  for (size_t j = 0; j < n_jobs; j++) {
    const zntt_job& job = jobs[j];
    if (!job.tw || !job.d_src || !job.d_dst) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "job with a null pointer");
    if (tw_of(job.tw)->field != field) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "job table of another field");
    if (job.kind == ZNTT_JOB_NTT) {
      if (job.mode != ZNTT_FORWARD && job.mode != ZNTT_INVERSE)
        return set_error(ZNTT_ERR_INVALID_ARGUMENT, "unknown job mode");
    } else if (job.kind == ZNTT_JOB_COSET_LDE) {
      if (!job.tw_in || tw_of(job.tw_in)->field != field)
        return set_error(ZNTT_ERR_INVALID_ARGUMENT, "coset extension job without an input table");
      if (tw_of(job.tw_in)->log_n > tw_of(job.tw)->log_n)
        return set_error(ZNTT_ERR_INVALID_ARGUMENT, "coset extension shrinks the vector");
      if (job.d_src == job.d_dst) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "coset extension in place");
    } else if (job.kind == ZNTT_JOB_POLY_MUL) {
      const uint64_t n = 1ull << tw_of(job.tw)->log_n;
      if (!job.d_src2) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "polynomial product without a second factor");
      if (job.len < 1 || job.len2 < 1 || job.len > n || job.len2 > n || job.len + job.len2 - 1 > n)
        return set_error(ZNTT_ERR_INVALID_ARGUMENT, "polynomial product does not fit the transform size");
      if (job.d_dst == job.d_src || job.d_dst == job.d_src2)
        return set_error(ZNTT_ERR_INVALID_ARGUMENT, "polynomial product into a factor");
    } else {
      return set_error(ZNTT_ERR_INVALID_ARGUMENT, "unknown job kind");
    }
  }
  zntt_batch* b = new zntt_batch();
  b->field = field;
  b->shape = shape >= 0 ? shape : kBatchShape;
  cudaStream_t st = c.stream;

  std::vector<JobPlan> plans(n_jobs);
  for (size_t j = 0; j < n_jobs; j++) {
    const zntt_job& job = jobs[j];
    const TwEntry* tw = tw_of(job.tw);
    const uint32_t L = tw->log_n;
    const uint4* src = reinterpret_cast<const uint4*>(job.d_src);
    uint4* dst = reinterpret_cast<uint4*>(job.d_dst);
    if (job.kind == ZNTT_JOB_NTT) {
      const Plan plan = batch_plan(field, L, b->shape);
      uint4* mid = dst;
      if (plan.np > 1 && (const void*)src == (const void*)dst) {
        void* s = nullptr;
        int rc = pool_get((size_t)32 << L, &s);
        if (rc) {
          free_batch(b);
          return rc;
        }
        b->scratch.push_back({s, (size_t)32 << L});
        mid = (uint4*)s;
      }
      uint64_t ninv[4];
      const bool inv = job.mode == ZNTT_INVERSE;
      if (inv) n_inverse(field, L, ninv);
      plan_transform(plans[j], tw, plan, L, src, mid, dst, inv, inv ? ninv : nullptr, nullptr, 1ull << L, 1ull << L);
    } else if (job.kind == ZNTT_JOB_POLY_MUL) {
      void* s1 = nullptr;
      void* s2 = nullptr;
      int rc = pool_get((size_t)32 << L, &s1);
      if (!rc) {
        b->scratch.push_back({s1, (size_t)32 << L});
        rc = pool_get((size_t)32 << L, &s2);
      }
      if (rc) {
        free_batch(b);
        return rc;
      }
      b->scratch.push_back({s2, (size_t)32 << L});
      plan_poly_mul(plans[j], tw, batch_plan(field, L, b->shape), src, job.len,
                    reinterpret_cast<const uint4*>(job.d_src2), job.len2, (uint4*)s1, (uint4*)s2, dst);
    } else {
      const TwEntry* twi = tw_of(job.tw_in);
      const uint32_t Li = twi->log_n;
      CosetTab* ct = nullptr;
      int rc = acquire_coset_tab(field, Li, job.shift, &ct, st);
      if (rc) {
        free_batch(b);
        return rc;
      }
      b->coset_tabs.push_back(ct);
      void* coef = nullptr;
      rc = pool_get((size_t)32 << Li, &coef);
      if (rc) {
        free_batch(b);
        return rc;
      }
      b->scratch.push_back({coef, (size_t)32 << Li});
      const Plan pin = batch_plan(field, Li, b->shape);
      const Plan pout = batch_plan(field, L, b->shape);
      plan_transform(plans[j], twi, pin, Li, src, (uint4*)coef, (uint4*)coef, true, nullptr, ct->d, 1ull << Li,
                     1ull << Li);
      plan_transform(plans[j], tw, pout, L, (const uint4*)coef, dst, dst, false, nullptr, nullptr, 1ull << Li,
                     1ull << L);
    }
  }

  // Passes in job order, then items level by level (biggest jobs first), so
  // that every prerequisite pass precedes its dependents in the queue.
  std::vector<uint32_t> first_pass(n_jobs);
  for (size_t j = 0; j < n_jobs; j++) {
    first_pass[j] = (uint32_t)b->passes.size();
    for (size_t p = 0; p < plans[j].passes.size(); p++) {
      BatchPass bp;
      bp.pp = plans[j].passes[p];
      bp.tiles = (uint32_t)plans[j].tiles[p];
      bp.dep = p == 0 ? kNoDep : (uint32_t)(b->passes.size() - 1);
      b->passes.push_back(bp);
    }
  }
  std::vector<size_t> order(n_jobs);
  for (size_t j = 0; j < n_jobs; j++) order[j] = j;
  std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t z) { return plans[a].work > plans[z].work; });
  size_t max_levels = 0;
  for (auto& jp : plans) max_levels = std::max(max_levels, jp.passes.size());
  for (size_t lvl = 0; lvl < max_levels; lvl++) {
    for (size_t j : order) {
      if (lvl >= plans[j].passes.size()) continue;
      const uint32_t pi = first_pass[j] + (uint32_t)lvl;
      for (uint32_t t = 0; t < b->passes[pi].tiles; t++) b->items.push_back({pi, t});
    }
  }
  b->ctl_words = 2 + b->passes.size();
  cudaError_t ce = cudaMalloc((void**)&b->d_passes, std::max<size_t>(1, b->passes.size()) * sizeof(BatchPass));
  if (ce == cudaSuccess)
    ce = cudaMalloc((void**)&b->d_items, std::max<size_t>(1, b->items.size()) * sizeof(BatchItem));
  if (ce == cudaSuccess) ce = cudaMalloc((void**)&b->d_ctl, b->ctl_words * 4);
  if (ce == cudaSuccess && !b->passes.empty())
    ce = cudaMemcpyAsync(b->d_passes, b->passes.data(), b->passes.size() * sizeof(BatchPass), cudaMemcpyHostToDevice,
                         st);
  if (ce == cudaSuccess && !b->items.empty())
    ce = cudaMemcpyAsync(b->d_items, b->items.data(), b->items.size() * sizeof(BatchItem), cudaMemcpyHostToDevice,
                         st);
  if (ce == cudaSuccess) ce = cudaMemsetAsync(b->d_ctl, 0, b->ctl_words * 4, st);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
  if (ce != cudaSuccess) {
    free_batch(b);
    return cuda_fail(ce, "batch set-up");
  }
  for (const BatchPass& bp : b->passes) b->ext = b->ext || pass_needs_ext(bp.pp);
  b->full = !b->passes.empty() && batch_all_full(b->shape, b->passes.data(), b->passes.size());
  b->grid = std::max(1, std::min<int>(batch_grid(field, b->shape, b->ext), (int)std::max<size_t>(1, b->items.size())));
  *out = b;
  return ZNTT_OK;
}

static int enqueue_batch(zntt_batch* b, cudaStream_t st) {
  cudaError_t ce = cudaMemsetAsync(b->d_ctl, 0, b->ctl_words * 4, st);
  if (ce != cudaSuccess) return cuda_fail(ce, "batch reset");
  if (b->items.empty()) return ZNTT_OK;
  ce = launch_batch(b->field, b->shape, b->ext, b->full, b->d_passes, b->d_items, (uint32_t)b->items.size(), b->d_ctl,
                    b->spin_limit, b->grid, st);
  if (ce != cudaSuccess) return cuda_fail(ce, "batch launch");
  return ZNTT_OK;
}

int zntt_batch_run(zntt_batch* b, void* stream) {
  clear_error();
  if (!b) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null batch");
  return enqueue_batch(b, stream ? (cudaStream_t)stream : ctx().stream);
}

int zntt_batch_run_graph(zntt_batch* b, void* stream) {
  clear_error();
  if (!b) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null batch");
  cudaStream_t st = stream ? (cudaStream_t)stream : ctx().stream;
  if (!b->graph_exec) {
    // Capture the queue reset and the persistent launch once; replays reuse it.
    cudaStream_t cap = nullptr;
    cudaError_t ce = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking);
    if (ce != cudaSuccess) return cuda_fail(ce, "capture stream");
    ce = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    int rc = ce == cudaSuccess ? enqueue_batch(b, cap) : ZNTT_OK;
    cudaError_t ce2 = ce == cudaSuccess ? cudaStreamEndCapture(cap, &b->graph) : ce;
    cudaStreamDestroy(cap);
    if (rc) return rc;
    if (ce2 != cudaSuccess) return cuda_fail(ce2, "graph capture");
    ce = cudaGraphInstantiate(&b->graph_exec, b->graph, 0);
    if (ce != cudaSuccess) return cuda_fail(ce, "graph instantiate");
  }
  cudaError_t ce = cudaGraphLaunch(b->graph_exec, st);
  if (ce != cudaSuccess) return cuda_fail(ce, "graph launch");
  return ZNTT_OK;
}

int zntt_batch_status(zntt_batch* b) {
  clear_error();
  if (!b) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null batch");
  uint32_t flag = 0;
  cudaError_t ce = cudaMemcpy(&flag, b->d_ctl + 1, 4, cudaMemcpyDeviceToHost);
  if (ce != cudaSuccess) return cuda_fail(ce, "batch status");
  if (flag) return set_error(ZNTT_ERR_TIMEOUT, "a batch item waited too long for its prerequisite pass");
  return ZNTT_OK;
}

int zntt_batch_set_spin_limit(zntt_batch* b, uint32_t spin_limit) {
  clear_error();
  if (!b) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null batch");
  Context& c = ctx();
  std::lock_guard<std::recursive_mutex> lock(c.mu);
  if (spin_limit == b->spin_limit) return ZNTT_OK;
  b->spin_limit = spin_limit;
  // The limit is a kernel argument: a captured graph holds the old value.
  // Replays may be in flight on any stream, so the device drains first.
  if (b->graph_exec || b->graph) {
    const cudaError_t ce = cudaDeviceSynchronize();
    if (ce != cudaSuccess) return cuda_fail(ce, "batch spin limit");
  }
  if (b->graph_exec) {
    cudaGraphExecDestroy(b->graph_exec);
    b->graph_exec = nullptr;
  }
  if (b->graph) {
    cudaGraphDestroy(b->graph);
    b->graph = nullptr;
  }
  return ZNTT_OK;
}

int zntt_batch_info(const zntt_batch* b, uint32_t* n_items, uint32_t* n_passes, int* grid, int* shape) {
  if (!b) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null batch");
  if (n_items) *n_items = (uint32_t)b->items.size();
  if (n_passes) *n_passes = (uint32_t)b->passes.size();
  if (grid) *grid = b->grid;
  if (shape) *shape = b->shape;
  return ZNTT_OK;
}

int zntt_batch_destroy(zntt_batch* b) {
  if (!b) return ZNTT_OK;
  Context& c = ctx();
  std::lock_guard<std::recursive_mutex> lock(c.mu);
  cudaStreamSynchronize(c.stream);
  free_batch(b);
  return ZNTT_OK;
}

int zntt_coset_lde_device(const zntt_twiddles* tw_in, const zntt_twiddles* tw_out, const uint64_t shift[4],
                          const uint64_t* d_evals, uint64_t* d_out, void* stream) {
  clear_error();
  if (!tw_in || !tw_out || !shift || !d_evals || !d_out) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null pointer");
  Context& c = ctx();
  if (c.device < 0) return set_error(ZNTT_ERR_NOT_INITIALIZED, "zntt_init has not been called");
  if (is_small_table(tw_in) != is_small_table(tw_out))
    return set_error(ZNTT_ERR_INVALID_ARGUMENT, "tables of different fields");
  if (is_small_table(tw_in)) return small_coset_lde(tw_in, tw_out, shift, d_evals, d_out, stream);
  const TwEntry* ti = tw_of(tw_in);
  const TwEntry* to = tw_of(tw_out);
  if (ti->field != to->field) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "tables of different fields");
  if (ti->log_n > to->log_n) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "coset extension shrinks the vector");
  if ((const void*)d_evals == (const void*)d_out) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "extension in place");
  std::lock_guard<std::recursive_mutex> lock(c.mu);
  cudaStream_t st = stream ? (cudaStream_t)stream : c.stream;
  CosetTab* ct = nullptr;
  int rc = acquire_coset_tab(ti->field, ti->log_n, shift, &ct, c.stream);
  if (rc) return rc;
  void* coef = nullptr;
  rc = pool_get((size_t)32 << ti->log_n, &coef);
  if (rc) {
    release_coset_tab(ct);
    return rc;
  }
  JobPlan jp;
  const Plan pin = tuned_plan(ti->field, ti->log_n);
  const Plan pout = tuned_plan(to->field, to->log_n);
  plan_transform(jp, ti, pin, ti->log_n, (const uint4*)d_evals, (uint4*)coef, (uint4*)coef, true, nullptr, ct->d,
                 1ull << ti->log_n, 1ull << ti->log_n);
  plan_transform(jp, to, pout, to->log_n, (const uint4*)coef, (uint4*)d_out, (uint4*)d_out, false, nullptr, nullptr,
                 1ull << ti->log_n, 1ull << to->log_n);
  cudaError_t ce = cudaSuccess;
  for (size_t p = 0; p < jp.passes.size() && ce == cudaSuccess; p++) {
    const int shape = p < pin.np ? pin.shape : pout.shape;
    ce = launch_ntt_pass(ti->field, shape, jp.passes[p], jp.tiles[p], st);
  }
  // The coefficient buffer and the table return to their owners only after
  // the stream is done with them.
  cudaError_t ce2 = cudaStreamSynchronize(st);
  pool_put(coef, (size_t)32 << ti->log_n);
  release_coset_tab(ct);
  if (ce != cudaSuccess) return cuda_fail(ce, "coset extension");
  if (ce2 != cudaSuccess) return cuda_fail(ce2, "coset extension");
  return ZNTT_OK;
}

int zntt_coset_lde_columns(const zntt_twiddles* tw_in, const zntt_twiddles* tw_out, const uint64_t shift[4],
                           const uint64_t* const* d_evals, uint64_t* const* d_out, uint32_t num_columns,
                           void* stream) {
  clear_error();
  if (!tw_in || !tw_out || !shift || !d_evals || !d_out) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null pointer");
  if (num_columns == 0) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "no columns");
  Context& c = ctx();
  if (c.device < 0) return set_error(ZNTT_ERR_NOT_INITIALIZED, "zntt_init has not been called");
  if (is_small_table(tw_in) != is_small_table(tw_out))
    return set_error(ZNTT_ERR_INVALID_ARGUMENT, "tables of different fields");
  if (is_small_table(tw_in)) return small_coset_lde_many(tw_in, tw_out, shift, d_evals, d_out, num_columns, stream);
  // The 256-bit fields: one extension per column (a batch of ZNTT_JOB_COSET_LDE jobs
  // runs them in one persistent launch instead).
  for (uint32_t k = 0; k < num_columns; k++) {
    const int rc = zntt_coset_lde_device(tw_in, tw_out, shift, d_evals[k], d_out[k], stream);
    if (rc) return rc;
  }
  return ZNTT_OK;
}

// ---- autotuner ---------------------------------------------------------------------

int zntt_autotune(int field, uint32_t log_n_min, uint32_t log_n_max) {
  clear_error();
  if (field != kBn254Fr && field != kBls12381Fr) return set_error(ZNTT_ERR_UNSUPPORTED_FIELD, "unsupported field");
  if (log_n_min < 1 || log_n_max > 28 || log_n_min > log_n_max)
    return set_error(ZNTT_ERR_INVALID_ARGUMENT, "autotune range must lie in 1..28");
  Context& c = ctx();
  if (c.device < 0) return set_error(ZNTT_ERR_NOT_INITIALIZED, "zntt_init has not been called");
  std::lock_guard<std::recursive_mutex> lock(c.mu);
  cudaStream_t st = c.stream;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int rc = ZNTT_OK;
  for (uint32_t L = log_n_min; L <= log_n_max && rc == ZNTT_OK; L++) {
    uint64_t root[4];
    rc = zntt_primitive_root(field, L, root);
    if (rc) break;
    TwEntry* tw = nullptr;
    rc = acquire_table(field, L, root, &tw);
    if (rc) break;
    void *x = nullptr, *y = nullptr;
    rc = pool_get((size_t)32 << L, &x);
    if (!rc) rc = pool_get((size_t)32 << L, &y);
    uint8_t seed[32] = {7};
    if (!rc) rc = zntt_random_elements(field, seed, (uint64_t*)x, (size_t)1 << L, nullptr);
    uint64_t ninv[4];
    n_inverse(field, L, ninv);
    for (int sh = 0; sh < kNumShapes && !rc; sh++) {
      const uint32_t lt = kShapes[sh].log_tile;
      TuneEntry best;
      best.us = 1e30;
      uint32_t last_np = 0, last_k0 = 0;
      for (uint32_t kmax = lt; kmax + 5 > lt && kmax >= 2 && !rc; kmax--) {
        const Plan plan = make_plan(L, sh, kmax);
        if (plan.np == last_np && plan.p[0].k == last_k0) continue;  // same plan as a larger kmax
        last_np = plan.np;
        last_k0 = plan.p[0].k;
        // Each repetition is a forward and an inverse transform (the inverse's
        // last pass also scales by 1/n): one plan serves both directions.
        auto both = [&]() {
          int r2 = run_plan(field, tw, plan, L, (const uint4*)x, (uint4*)y, nullptr, false, false, nullptr, st);
          if (!r2) r2 = run_plan(field, tw, plan, L, (const uint4*)x, (uint4*)y, nullptr, true, true, ninv, st);
          return r2;
        };
        for (int w = 0; w < 2 && !rc; w++) rc = both();
        const int reps = L >= 22 ? 5 : L >= 18 ? 20 : 50;
        cudaEventRecord(e0, st);
        for (int r = 0; r < reps && !rc; r++) rc = both();
        cudaEventRecord(e1, st);
        cudaError_t ce = cudaEventSynchronize(e1);
        if (ce != cudaSuccess) rc = cuda_fail(ce, "autotune");
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        const double us = 1e3 * ms / (2 * reps);  // per transform, both directions averaged
        if (!rc && us < best.us) {
          best.field = field;
          best.log_n = L;
          best.shape = sh;
          best.kmax = kmax;
          best.us = us;
        }
      }
      if (!rc) {
        c.tune.erase(std::remove_if(c.tune.begin(), c.tune.end(),
                                    [&](const TuneEntry& t) { return t.field == field && t.log_n == L && t.shape == sh; }),
                     c.tune.end());
        c.tune.push_back(best);
      }
    }
    cudaStreamSynchronize(st);
    if (x) pool_put(x, (size_t)32 << L);
    if (y) pool_put(y, (size_t)32 << L);
    release_table(tw);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc;
}

// One entry per line: {"gpu": "...", "field": F, "log_n": L, "shape": S, "kmax": K, "us": T}
int zntt_tune_save(const char* path) {
  clear_error();
  if (!path) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null path");
  Context& c = ctx();
  std::lock_guard<std::recursive_mutex> lock(c.mu);
  // Keep other GPUs' entries from an existing file.
  std::vector<std::string> keep;
  if (FILE* f = std::fopen(path, "r")) {
    char line[512];
    while (std::fgets(line, sizeof(line), f)) {
      const char* g = std::strstr(line, "\"gpu\": \"");
      if (!g) continue;
      std::string name(g + 8);
      name = name.substr(0, name.find('"'));
      if (name != c.gpu_name) keep.push_back(line);
    }
    std::fclose(f);
  }
  FILE* f = std::fopen(path, "w");
  if (!f) return set_error(ZNTT_ERR_INVALID_ARGUMENT, std::string("cannot write ") + path);
  std::fprintf(f, "[\n");
  bool firstl = true;
  for (const std::string& l : keep) {
    std::string t = l;
    while (!t.empty() && (t.back() == '\n' || t.back() == ',')) t.pop_back();
    std::fprintf(f, "%s%s", firstl ? "" : ",\n", t.c_str());
    firstl = false;
  }
  for (const TuneEntry& t : c.tune) {
    std::fprintf(f, "%s {\"gpu\": \"%s\", \"field\": %d, \"log_n\": %u, \"shape\": %d, \"kmax\": %u, \"us\": %.3f}",
                 firstl ? "" : ",\n", c.gpu_name.c_str(), t.field, t.log_n, t.shape, t.kmax, t.us);
    firstl = false;
  }
  std::fprintf(f, "\n]\n");
  std::fclose(f);
  return ZNTT_OK;
}

int zntt_tune_load(const char* path) {
  clear_error();
  if (!path) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null path");
  FILE* f = std::fopen(path, "r");
  if (!f) return set_error(ZNTT_ERR_INVALID_ARGUMENT, std::string("cannot read ") + path);
  Context& c = ctx();
  std::lock_guard<std::recursive_mutex> lock(c.mu);
  char line[512];
  int n = 0;
  while (std::fgets(line, sizeof(line), f)) {
    const char* g = std::strstr(line, "\"gpu\": \"");
    if (!g) continue;
    std::string name(g + 8);
    name = name.substr(0, name.find('"'));
    if (!c.gpu_name.empty() && name != c.gpu_name) continue;
    TuneEntry t;
    const char* q = std::strstr(line, "\"field\":");
    if (!q || std::sscanf(q, "\"field\": %d, \"log_n\": %u, \"shape\": %d, \"kmax\": %u, \"us\": %lf", &t.field,
                          &t.log_n, &t.shape, &t.kmax, &t.us) != 5)
      continue;
    if (t.shape < 0 || t.shape >= kNumShapes || t.kmax < 2 || t.kmax > (uint32_t)kShapes[t.shape].log_tile) continue;
    c.tune.erase(std::remove_if(c.tune.begin(), c.tune.end(),
                                [&](const TuneEntry& u) {
                                  return u.field == t.field && u.log_n == t.log_n && u.shape == t.shape;
                                }),
                 c.tune.end());
    c.tune.push_back(t);
    n++;
  }
  std::fclose(f);
  return n > 0 ? ZNTT_OK : set_error(ZNTT_ERR_INVALID_ARGUMENT, "no tuning entries for this GPU");
}

int zntt_tune_clear(void) {
  Context& c = ctx();
  std::lock_guard<std::recursive_mutex> lock(c.mu);
  c.tune.clear();
  return ZNTT_OK;
}

}  // extern "C"
