// small.hpp -- the SmallField (Goldilocks, BabyBear) path of the C ABI
// (small.cu), dispatched to by the entry points of runtime.cu when the field
// id or twiddle handle is a small field's.
#pragma once

#include <cstddef>
#include <cstdint>

#include "zntt.h"

namespace zntt {

bool is_small_field(int field);
// A twiddle handle made for a small field (its leading field id says so).
bool is_small_table(const void* handle);

int small_field_info(int field, uint64_t* modulus, uint32_t* two_adicity);
int small_primitive_root(int field, uint32_t log_n, uint64_t* root_out);
int small_bit_reverse(uint64_t* data, size_t len);
int small_ntt_root(int field, uint64_t* data, size_t len, size_t log_n, const uint64_t* root, bool inverse);
int small_precompute(int field, size_t log_n, const uint64_t* root, uint64_t* const* stage_out);
void small_free_twiddles(int field, const zntt_stage* stages, size_t num_stages);
int small_ntt_with_twiddles(int field, uint64_t* data, size_t len, size_t log_n, const zntt_stage* stages,
                            size_t num_stages, bool inverse);
int small_twiddles_acquire(int field, uint32_t log_n, const uint64_t* root, zntt_twiddles** out);
int small_twiddles_release(zntt_twiddles* tw);
int small_ntt_device(const zntt_twiddles* tw, const uint64_t* d_src, uint64_t* d_dst, uint64_t* d_scratch, int mode,
                     void* stream);
int small_domain_fill(int field, uint32_t log_n, uint64_t* d_out, void* stream);
int small_fri_fold(int field, const uint64_t* d_layer, uint32_t log_n, const uint64_t* alpha, uint64_t* d_out,
                   uint32_t log_table, void* stream);
int small_fold_params(int field, uint32_t log_table, const uint64_t* alpha, const uint64_t** tab_out,
                      uint64_t* half_inv_tw, uint64_t* alpha_tw);
// The 256-bit fields' fold constants (fri.cu): the resident table g^-j / 2 and 1/2
// (Montgomery limbs as eight 32-bit words).
int wide_fold_params(int field, uint32_t log_table, const void** tab_out, uint32_t half_inv[8]);
int small_poly_mul(int field, const uint64_t* a, size_t a_len, const uint64_t* b, size_t b_len, size_t max_degree,
                   uint64_t* out, int64_t* out_degree);
int small_ntt_columns(const zntt_twiddles* tw, const uint64_t* const* d_src, uint64_t* const* d_dst, uint32_t m,
                      int mode, void* stream);
int small_coset_lde_many(const zntt_twiddles* tw_in, const zntt_twiddles* tw_out, const uint64_t* shift,
                         const uint64_t* const* d_evals, uint64_t* const* d_out, uint32_t m, void* stream);
int small_coset_lde(const zntt_twiddles* tw_in, const zntt_twiddles* tw_out, const uint64_t* shift,
                    const uint64_t* d_evals, uint64_t* d_out, void* stream);
void small_shutdown();
// FRI fold tables of the 256-bit fields (fri.cu).
void fri_shutdown();

}  // namespace zntt
