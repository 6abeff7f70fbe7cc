// kernels.cuh -- launch interface between the host runtime and the sm_100a kernels.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace zntt {

// Field identifiers shared with the C ABI (include/zntt.h).
// 0 and 1: 256-bit Montgomery fields (32-byte elements, this file's kernels);
// 2 and 3: SmallField's Goldilocks and BabyBear (8-byte elements, small.cu).
enum FieldId : int { kBn254Fr = 0, kBls12381Fr = 1, kGoldilocksField = 2, kBabyBearField = 3 };

// One fused radix-2^k pass of the decimation-in-time network.
//
// The network is zig-ntt's (libs/ntt/src/root.zig:148-212): bit-reverse the
// input, then stages s = 1..log_n; stage s pairs positions q and q + 2^(s-1)
// inside blocks of 2^s and uses twiddle tw[s-1][q mod 2^(s-1)].  A pass runs
// stages S+1..S+k on tiles of 2^k positions that differ only in bits
// [S, S+k) of q, with 2^c neighbouring low-bit positions per tile so global
// rows are 2^c * 32 contiguous bytes.  The first pass (S == 0) gathers its
// tile from the natural-order input, which folds the bit reversal into the
// load: permuted block rev(col) holds input column col of the 2^k x 2^(L-k)
// row-major view, row r landing at tile row rev_k(r).
struct PassParams {
  const uint4* src;   // 2 uint4 per element
  uint4* dst;
  const uint4* tw;    // zig-ntt twiddle table, stage s at entry 2^s - 1
  uint32_t log_n;     // L
  uint32_t S;         // stages already applied
  uint32_t k;         // stages in this pass
  uint32_t c;         // log2 of contiguous positions per tile row
  uint32_t first;     // gather the input through the bit reversal
  uint32_t inverse;   // inttWithTwiddles mapping: w = 1 (j = 0) or -tw[s-1][2^(s-1) - j]
  uint32_t tw0_one;   // every stage's entry 0 is one (j = 0 needs no multiply)
  uint32_t scale;     // multiply each output by scale_val (or scale_tab[q]) after the last stage
  uint32_t scale_val[8];
  const uint4* scale_tab;  // when non-null, output position q is scaled by scale_tab[q]
  uint64_t src_len;   // first pass: natural input index >= src_len reads as zero (zero padding)
  uint64_t dst_len;   // output positions >= dst_len are not stored
};

// Pass kernel shapes.  Each shape is a compiled kernel: a tile of 2^log_tile
// elements (32 bytes each in shared memory), `threads` per CTA, `min_blocks`
// CTAs per SM for the register budget.  The autotuner picks a shape and a
// stage count per pass for each (field, log n).
struct PassShape {
  int log_tile, threads, min_blocks;
};
// 2^11 and 2^10 tiles in CTAs of 256 threads (3 per SM), and the same 24 warps
// per SM in smaller CTAs: 2^9 tiles in 128 threads (6 per SM) and 2^8 tiles in
// 64 threads (12 per SM), where each barrier waits on fewer warps (2^24
// BN254-Fr: 3.65 ms with 2^10 tiles, 3.49 ms with 2^9 or 2^8 tiles, B200).
// The last shape trades a 72-register budget (a few spilled words) for 28
// warps per SM: 2^22 and 2^24 BN254-Fr about 0.6% faster, BLS12-381-Fr slower.
constexpr int kNumShapes = 5;
constexpr PassShape kShapes[kNumShapes] = {{11, 256, 3}, {10, 256, 3}, {9, 128, 6}, {8, 64, 12}, {9, 128, 7}};
// The shape of persistent launches (batches and the server's slices): the
// 7-CTA 2^9 tile ran the mixed 520-transform batch 3.03 -> 2.94 ms and 64
// coset extensions 2^18 -> 2^20 16.95 -> 16.74 ms (BLS12-381-Fr) and 15.81 ->
// 15.45 ms (BN254-Fr) against the 6-CTA tile, and the 2^10 and 2^8 tiles
// slower still (B200).
constexpr int kBatchShape = 4;
constexpr int kLogTile = 11;  // the largest tile of any shape
constexpr int kDefaultShape = 0;

inline int shape_smem_bytes(int shape) { return (1 << kShapes[shape].log_tile) * 32; }

// A pass that pads its input with zeros, scales by a table or stores a prefix
// of its output runs the extension variant of the kernels.
inline bool pass_needs_ext(const PassParams& pp) {
  const uint64_t n = 1ull << pp.log_n;
  return (pp.first && pp.src_len < n) || (pp.scale && pp.scale_tab != nullptr) || pp.dst_len < n;
}

cudaError_t launch_ntt_pass(int field, int shape, const PassParams& pp, uint64_t num_tiles, cudaStream_t st);
cudaError_t configure_kernels();
cudaError_t configure_batch_kernels();

// ---- batched persistent launch ----------------------------------------------
// One pass of one job inside a batch, and one unit of work (a tile of a pass).
struct BatchPass {
  PassParams pp;
  uint32_t tiles;  // tiles in this pass
  uint32_t dep;    // pass that must finish first (kNoDep: none)
};
constexpr uint32_t kNoDep = 0xffffffffu;
struct BatchItem {
  uint32_t pass;
  uint32_t tile;
};
// ctl[0]: next item, ctl[1]: error flag, ctl[2 + p]: finished tiles of pass p.
// Every wait for a finished pass spins at most `spin_limit` rounds of ~1 us,
// then raises the error flag; every CTA stops at the next item once it is set.
// `full`: every pass has whole tiles (batch_all_full), so no bound checks.
cudaError_t launch_batch(int field, int shape, bool ext, bool full, const BatchPass* passes, const BatchItem* items,
                         uint32_t n_items, uint32_t* ctl, uint32_t spin_limit, int grid, cudaStream_t st);
// True when every pass's tile is the shape's whole tile (k + c == log_tile).
inline bool batch_all_full(int shape, const BatchPass* passes, size_t n) {
  for (size_t i = 0; i < n; i++)
    if (passes[i].pp.k + passes[i].pp.c != (uint32_t)kShapes[shape].log_tile) return false;
  return true;
}
int batch_grid(int field, int shape, bool ext);

// Flat zig-ntt twiddle table for one (field, log_n, root): entry 2^s - 1 + j
// of stage s is root^(j * 2^(log_n-1-s)).  The powers are assembled from three
// small host-made tables: pw[0][i] = root^i, pw[1][i] = root^(1024 i),
// pw[2][i] = root^(2^20 i), i < 1024 (each 1024 x 32 bytes, contiguous).
cudaError_t launch_twiddle_table(int field, const uint4* d_pw, uint4* d_table, uint32_t log_n,
                                 cudaStream_t st);

// out[i] = c * base^i for i < count (count <= 2^30), from the three power
// tables of `base` laid out as for launch_twiddle_table.
cudaError_t launch_powers(int field, const uint4* d_pw, const uint64_t* c, uint4* out, uint64_t count,
                          cudaStream_t st);

// dst[rev(i)] = src[i] for 2^log_n elements (out of place).
cudaError_t launch_bit_reverse(const uint4* src, uint4* dst, uint32_t log_n, cudaStream_t st);

// Elementwise device arithmetic for tests: op 0 mul, 1 add, 2 sub, 3 neg.
cudaError_t launch_elementwise(int field, int op, const uint4* a, const uint4* b, uint4* out,
                               uint64_t count, cudaStream_t st);

// Multiply-throughput probe: `iters` rounds of 8-long mad.lo/madc.hi carry
// chains per thread; returns through `sink` so nothing is optimised away.
cudaError_t launch_imad_probe(uint32_t* sink, uint32_t iters, int blocks, int threads, cudaStream_t st);
// Independent 32x32->64 multiply-adds per thread (8 per iteration).
cudaError_t launch_imad_wide_probe(unsigned long long* sink, uint32_t iters, int blocks, int threads,
                                   cudaStream_t st);
// Independent modular products per thread, to time the field multiply alone.
cudaError_t launch_modmul_probe(int field, uint4* sink, uint32_t iters, int blocks, int threads,
                                cudaStream_t st);

}  // namespace zntt
