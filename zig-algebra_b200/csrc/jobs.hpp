// jobs.hpp -- job planning shared by batches (jobs.cu) and the server (serve.cu).
#pragma once

#include <cstdint>
#include <vector>

#include "runtime.hpp"

namespace zntt {

// n^-1 * g^i for i < 2^log_in, cached per (field, log_in, g) and reference counted.
struct CosetTab {
  int field = 0;
  uint32_t log_in = 0;
  uint64_t shift[4] = {0, 0, 0, 0};
  uint4* d = nullptr;
  size_t bytes = 0;
  int refs = 0;
};
int acquire_coset_tab(int field, uint32_t log_in, const uint64_t* shift, CosetTab** out, cudaStream_t st);
void release_coset_tab(CosetTab* t);
void free_coset_tabs();

// The passes of one job, in order, with the buffers they run between.
struct JobPlan {
  std::vector<PassParams> passes;  // tiles = 2^log_n >> (k + c)
  std::vector<uint64_t> tiles;
  size_t work = 0;                 // elements x stages, for ordering
};

// The tuned plan of a batch job; a length-1 vector gets one pass of no stage.
Plan batch_plan(int field, uint32_t log_n, int shape);

// Appends the passes of one transform src -> dst (mid: where passes after the
// first run in place); the last pass scales by scale_val or scale_tab when
// given and stores only the output positions below dst_len; the first pass
// reads zeros from input index src_len on.
void plan_transform(JobPlan& jp, const TwEntry* tw, const Plan& plan, uint32_t log_n, const uint4* src, uint4* mid,
                    uint4* dst, bool inverse, const uint64_t* scale_val, const uint4* scale_tab, uint64_t src_len,
                    uint64_t dst_len);

// The passes of one polynomial product (ZNTT_JOB_POLY_MUL) on 2^log_n points:
// forward(a) into s1, forward(b) into s2 with the last pass multiplying by s1,
// inverse of s2 (through s1) into dst, which receives len_a + len_b - 1
// coefficients.  s1 and s2 hold 2^log_n elements each.
void plan_poly_mul(JobPlan& jp, const TwEntry* tw, const Plan& plan, const uint4* a, uint64_t len_a, const uint4* b,
                   uint64_t len_b, uint4* s1, uint4* s2, uint4* dst);

}  // namespace zntt
