// pass_tile.cuh -- one tile of one fused DIT pass, shared by the plain pass
// kernel and the batched persistent kernel.
//
// The network is zig-ntt's (libs/ntt/src/root.zig:148-212): stage s pairs
// DIT positions q and q + 2^(s-1) inside blocks of 2^s with twiddle
// tw[s-1][q mod 2^(s-1)].  A tile holds the 2^k positions that differ only in
// bits [S, S+k) of q, times 2^c neighbouring low-bit positions, in shared
// memory as two planes of 16-byte halves (half h of tile element e at
// sm[h * TILE + e]); stages run two at a time on four elements in registers.
#pragma once

#include "field.cuh"
#include "kernels.cuh"

namespace zntt {

__device__ __forceinline__ uint32_t rev_bits(uint32_t x, uint32_t bits) {
  return bits == 0 ? 0u : (__brev(x) >> (32 - bits));
}

template <uint32_t TILE>
__device__ __forceinline__ fe sm_load(const uint4* sm, uint32_t e) {
  uint4 lo = sm[e], hi = sm[TILE + e];
  fe r;
  r.v[0] = lo.x; r.v[1] = lo.y; r.v[2] = lo.z; r.v[3] = lo.w;
  r.v[4] = hi.x; r.v[5] = hi.y; r.v[6] = hi.z; r.v[7] = hi.w;
  return r;
}
template <uint32_t TILE>
__device__ __forceinline__ void sm_store(uint4* sm, uint32_t e, const fe& a) {
  sm[e] = make_uint4(a.v[0], a.v[1], a.v[2], a.v[3]);
  sm[TILE + e] = make_uint4(a.v[4], a.v[5], a.v[6], a.v[7]);
}

// Twiddle of global stage s (1-based) for butterfly index jg, with the
// forward (tw[s-1][jg]) or inttWithTwiddles (1 or -tw[s-1][2^(s-1) - jg])
// mapping.  `stw` points at tw[s-1]; returns false when the factor is one and
// the multiply can be skipped (unit0: entry 0 is one, always so for the inverse).  The inverse's factor is p - tw (fe_p_minus):
// the product equals the one by -tw mod p, also for a zero entry.
template <class F>
__device__ __forceinline__ bool twiddle(bool inverse, bool unit0, const uint4* stw, uint32_t half_g, uint32_t jg,
                                        fe& w) {
  if (jg == 0 && unit0) return false;
  if (!inverse) {
    w = fe_load_nc(stw + (jg << 1));
  } else {
    w = fe_p_minus<F>(fe_load_nc(stw + ((half_g - jg) << 1)));
  }
  return true;
}

// u, v -> u + w v, u - w v.  Lazy fields (4p < 2^256) keep u and v in
// [0, 2p) between stages; the last stage of a pass reduces them to [0, p), so
// every pass reads and writes canonical elements.
template <class F>
__device__ __forceinline__ void butterfly(fe& u, fe& v, bool mul, const fe& w) {
  if constexpr (F::kLazy) {
    const fe t = mul ? fe_mul<F, false>(w, v) : v;
    v = fe_sub2p<F>(u, t);
    u = fe_add2p<F>(u, t);
  } else {
    const fe t = mul ? fe_mul<F>(w, v) : v;
    v = fe_sub<F>(u, t);
    u = fe_add<F>(u, t);
  }
}

// [0, 2p) -> [0, p) after a pass's last stage (lazy fields only).
template <class F>
__device__ __forceinline__ void canonical(fe& x, bool last) {
  if constexpr (F::kLazy) {
    if (last) x = fe_reduce<F>(x);
  }
}

// Global loads of tile data: COHERENT reads through L2 only, for data other
// SMs wrote earlier in the same launch (the batched kernel).
template <bool COHERENT>
__device__ __forceinline__ uint4 load_data(const uint4* p) {
  if constexpr (COHERENT) return __ldcg(p);
  else return *p;
}

// EXT enables the extension features: zero padding of the first pass's input
// from index src_len, a per-position scale table, and storing only the output
// positions below dst_len.  Plain transforms compile without them (fewer live
// registers in the hot loop).  FULL: the tile is the shape's whole tile
// (k + c == LOG_TILE, every pass of a transform larger than one tile), so no
// thread needs a bound check; without the checks the pass runs about 5% faster
// (2^24 BN254-Fr, B200).  SCALE compiles the output scaling (the inverse's
// 1/n, the extension's factor table); a pass launched without it must not ask
// for scaling (pp.scale == 0).
template <class F, int LOG_TILE, int THREADS, bool COHERENT, bool EXT, bool FULL = false, bool SCALE = true>
__device__ __forceinline__ void ntt_tile(const PassParams& pp, uint64_t blk, uint4* sm) {
  constexpr uint32_t TILE_MAX = 1u << LOG_TILE;
  // The fields the stage loop reads, read once (for parameters held in
  // memory rather than in the kernel's parameter space, each later read would
  // be a load re-issued after every barrier).
  const uint32_t k = pp.k, c = pp.c, C = 1u << c, S = pp.S;
  const bool first = pp.first, inverse = pp.inverse, unit0 = pp.inverse | pp.tw0_one;
  const uint4* const tw = pp.tw;
  const uint32_t tile = FULL ? TILE_MAX : 1u << (k + c);
  const uint32_t tid = threadIdx.x;

  // Indices fit 32 bits: transforms and tables hold at most 2^31 elements, so
  // an element's 16-byte-half offset is below 2^32.
  const uint32_t b = (uint32_t)blk;
  uint32_t hi_base = 0, m0 = 0, col0 = 0;
  if (first) {
    col0 = b << c;
  } else {
    const uint32_t mlog = S - c;
    hi_base = (b >> mlog) << (S + k);
    m0 = (b & ((1u << mlog) - 1)) << c;
  }
  const uint32_t xcols_log = pp.log_n - k;
  const uint64_t src_len = pp.src_len;

  // ---- load: warp w stages the 128-element slices w, w + W, w + 2W, ... of
  // the tile (DIT order), column-fastest in 16-byte halves.  These are the
  // elements its radix-4 groups use while a group's span, 4 h C elements, stays
  // within 128: those stage pairs exchange data only inside the warp and
  // synchronise with __syncwarp instead of a CTA barrier (2^24: the load and
  // three of the four stage pairs of every pass). ----
  constexpr uint32_t W = THREADS / 32;
  static_assert(TILE_MAX / THREADS >= 4, "each warp stages whole 128-element slices");
  const uint32_t lane = tid & 31, warp = tid >> 5;
#pragma unroll
  for (uint32_t r = 0; r < 2 * TILE_MAX / THREADS; r++) {
    const uint32_t u = lane + 32 * (r & 7);
    const uint32_t e = (warp + (r >> 3) * W) * 128 + (u >> 1), h = u & 1;
    if (FULL || e < tile) {
      const uint32_t col = e & (C - 1), t = e >> c;
      uint32_t g;
      uint4 val;
      if (first) {
        g = (rev_bits(t, k) << xcols_log) + col0 + col;
        if (EXT && g >= src_len) val = make_uint4(0, 0, 0, 0);
        else val = load_data<COHERENT>(pp.src + ((g << 1) | h));
      } else {
        g = hi_base + (t << S) + m0 + col;
        val = load_data<COHERENT>(pp.src + ((g << 1) | h));
      }
      sm[h * TILE_MAX + e] = val;
    }
  }
  // A radix-4 pair whose h satisfies (h << (c + 2)) <= 128 is warp-local.
  if (k >= 2 && (C << 2) <= 128u) __syncwarp();
  else __syncthreads();

  // ---- radix-4 groups: stages i and i+1 on four elements in registers ----
  uint32_t i = 1;
  for (; i < k; i += 2) {
    const uint32_t h = 1u << (i - 1);
    const uint32_t half1 = 1u << (S + i - 1);  // stage S+i
    const uint32_t half2 = half1 << 1;         // stage S+i+1
    const uint4* stw1 = tw + ((half1 - 1) << 1);
    const uint4* stw2 = tw + ((half2 - 1) << 1);
#pragma unroll
    for (uint32_t q = 0; q < TILE_MAX / 4 / THREADS; q++) {
      const uint32_t ga = tid + q * THREADS;
      if (FULL || ga < tile / 4) {
        const uint32_t col = ga & (C - 1), g = ga >> c;
        const uint32_t j = g & (h - 1);
        const uint32_t t0 = ((g >> (i - 1)) << (i + 1)) | j;
        const uint32_t e0 = (t0 << c) | col, eh = h << c;
        uint32_t jg1, jg3;
        if (first) {
          jg1 = j;
          jg3 = j + h;
        } else {
          jg1 = (j << S) + m0 + col;
          jg3 = jg1 + (h << S);
        }
        fe w1, w2, w3;
        const bool m1 = twiddle<F>(inverse, unit0, stw1, half1, jg1, w1);
        const bool m2 = twiddle<F>(inverse, unit0, stw2, half2, jg1, w2);
        const bool m3 = twiddle<F>(inverse, unit0, stw2, half2, jg3, w3);
        fe x0 = sm_load<TILE_MAX>(sm, e0), x1 = sm_load<TILE_MAX>(sm, e0 + eh),
           x2 = sm_load<TILE_MAX>(sm, e0 + 2 * eh), x3 = sm_load<TILE_MAX>(sm, e0 + 3 * eh);
        butterfly<F>(x0, x1, m1, w1);
        butterfly<F>(x2, x3, m1, w1);
        butterfly<F>(x0, x2, m2, w2);
        butterfly<F>(x1, x3, m3, w3);
        const bool last = i + 2 > k;
        canonical<F>(x0, last);
        canonical<F>(x1, last);
        canonical<F>(x2, last);
        canonical<F>(x3, last);
        sm_store<TILE_MAX>(sm, e0, x0);
        sm_store<TILE_MAX>(sm, e0 + eh, x1);
        sm_store<TILE_MAX>(sm, e0 + 2 * eh, x2);
        sm_store<TILE_MAX>(sm, e0 + 3 * eh, x3);
      }
    }
    // The next pair (stages i+2, i+3) is warp-local when its h = 2^(i+1) is.
    if (i + 2 < k && ((2u << i) << (c + 2)) <= 128u) __syncwarp();
    else __syncthreads();
  }

  // ---- an odd stage count ends with one radix-2 stage (stage k of the pass).
  // Last rather than first: in a transform's first pass the first stage pair
  // then holds the factors that are one (stage 1, and stage 2's j = 0), so the
  // pass skips their products in whole warps (2^20 first pass 8% faster, B200).
  if (k & 1) {
    const uint32_t h = 1u << (k - 1);
    const uint32_t half_g = 1u << (S + k - 1);  // stage S+k
    const uint4* stw = tw + ((half_g - 1) << 1);
#pragma unroll
    for (uint32_t q = 0; q < TILE_MAX / 2 / THREADS; q++) {
      const uint32_t b = tid + q * THREADS;
      if (FULL || b < tile / 2) {
        const uint32_t col = b & (C - 1), g = b >> c;
        const uint32_t j = g & (h - 1);
        const uint32_t t0 = ((g >> (k - 1)) << k) | j;
        const uint32_t jg = first ? j : (j << S) + m0 + col;
        const uint32_t e0 = (t0 << c) | col, e1 = e0 + (h << c);
        fe u = sm_load<TILE_MAX>(sm, e0), v = sm_load<TILE_MAX>(sm, e1), w;
        const bool mul = twiddle<F>(inverse, unit0, stw, half_g, jg, w);
        butterfly<F>(u, v, mul, w);
        canonical<F>(u, true);
        canonical<F>(v, true);
        sm_store<TILE_MAX>(sm, e0, u);
        sm_store<TILE_MAX>(sm, e1, v);
      }
    }
    __syncthreads();
  }

  // ---- the inverse's 1/n (or a per-position factor table), then store ----
  if (SCALE && pp.scale) {
    fe sc;
#pragma unroll
    for (int q = 0; q < 8; q++) sc.v[q] = pp.scale_val[q];
#pragma unroll
    for (uint32_t q = 0; q < TILE_MAX / THREADS; q++) {
      const uint32_t e = tid + q * THREADS;
      if (FULL || e < tile) {
        const uint32_t col = e & (C - 1), row = e >> c;
        if (EXT && pp.scale_tab) {
          const uint32_t g = first ? (rev_bits(col0 + col, xcols_log) << k) + row : hi_base + (row << S) + m0 + col;
          sc = fe_load_nc(pp.scale_tab + (g << 1));
        }
        sm_store<TILE_MAX>(sm, e, fe_mul<F>(sm_load<TILE_MAX>(sm, e), sc));
      }
    }
    __syncthreads();
  }

#pragma unroll
  for (uint32_t q = 0; q < 2 * TILE_MAX / THREADS; q++) {
    const uint32_t idx = tid + q * THREADS;
    if (FULL || idx < 2 * tile) {
      const uint32_t h = idx & 1, e = idx >> 1, col = e & (C - 1), row = e >> c;
      uint32_t g;
      if (first) {
        g = (rev_bits(col0 + col, xcols_log) << k) + row;
      } else {
        g = hi_base + (row << S) + m0 + col;
      }
      if (!EXT || g < pp.dst_len) pp.dst[(g << 1) | h] = sm[h * TILE_MAX + ((row << c) | col)];
    }
  }
}

}  // namespace zntt
