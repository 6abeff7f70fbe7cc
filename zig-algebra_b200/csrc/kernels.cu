// kernels.cu -- sm_100a kernels of the NTT hot path.
//
// The transform is zig-ntt's radix-2 decimation-in-time network
// (libs/ntt/src/root.zig:148-212) executed as a few fused passes: each pass
// stages a tile of the vector in shared memory with coalesced 16-byte global
// loads, runs several butterfly stages on it, and writes it back.  All
// arithmetic is exact Montgomery arithmetic from field.cuh.
#include "field.cuh"
#include "kernels.cuh"

namespace zntt {

// Shared memory holds a tile as two planes of 16-byte halves: half h of tile
// element e is at sm[h * kTileMax + e], so a warp touching 32 consecutive
// elements reads 512 contiguous bytes per plane (no bank conflicts).
constexpr uint32_t kTileMax = 1u << kLogTile;

__device__ __forceinline__ fe sm_load(const uint4* sm, uint32_t e) {
  uint4 lo = sm[e], hi = sm[kTileMax + e];
  fe r;
  r.v[0] = lo.x; r.v[1] = lo.y; r.v[2] = lo.z; r.v[3] = lo.w;
  r.v[4] = hi.x; r.v[5] = hi.y; r.v[6] = hi.z; r.v[7] = hi.w;
  return r;
}
__device__ __forceinline__ void sm_store(uint4* sm, uint32_t e, const fe& a) {
  sm[e] = make_uint4(a.v[0], a.v[1], a.v[2], a.v[3]);
  sm[kTileMax + e] = make_uint4(a.v[4], a.v[5], a.v[6], a.v[7]);
}

__device__ __forceinline__ uint32_t rev_bits(uint32_t x, uint32_t bits) {
  return bits == 0 ? 0u : (__brev(x) >> (32 - bits));
}

// Twiddle of global stage s (1-based) for butterfly index jg, with the
// forward (tw[s-1][jg]) or inttWithTwiddles (1 or -tw[s-1][2^(s-1) - jg])
// mapping.  `stw` points at tw[s-1]; returns false when the factor is one
// and the multiply can be skipped.
template <class F>
__device__ __forceinline__ bool twiddle(const PassParams& pp, const uint4* stw, uint64_t half_g, uint64_t jg,
                                        fe& w) {
  if (jg == 0 && (pp.inverse | pp.tw0_one)) return false;
  if (!pp.inverse) {
    w = fe_load_nc(stw + (jg << 1));
  } else {
    w = fe_neg<F>(fe_load_nc(stw + ((half_g - jg) << 1)));
  }
  return true;
}

// u, v -> u + w v, u - w v
template <class F>
__device__ __forceinline__ void butterfly(fe& u, fe& v, bool mul, const fe& w) {
  const fe t = mul ? fe_mul<F>(w, v) : v;
  v = fe_sub<F>(u, t);
  u = fe_add<F>(u, t);
}

template <class F, int LOG_TILE, int THREADS, int MINB>
__global__ void __launch_bounds__(THREADS, MINB) ntt_pass_kernel(PassParams pp) {
  constexpr uint32_t TILE_MAX = 1u << LOG_TILE;
  extern __shared__ uint4 sm[];
  const uint32_t k = pp.k, c = pp.c, C = 1u << c;
  const uint32_t tile = 1u << (k + c);
  const uint32_t tid = threadIdx.x;
  const uint64_t blk = blockIdx.x;

  uint64_t hi_base = 0, m0 = 0, col0 = 0;
  if (pp.first) {
    col0 = blk << c;
  } else {
    const uint32_t mlog = pp.S - c;
    hi_base = (blk >> mlog) << (pp.S + k);
    m0 = (blk & ((1ull << mlog) - 1)) << c;
  }
  const uint32_t xcols_log = pp.log_n - k;

  // ---- load: column-fastest, 16-byte halves ----
#pragma unroll
  for (uint32_t q = 0; q < 2 * TILE_MAX / THREADS; q++) {
    const uint32_t idx = tid + q * THREADS;
    if (idx < 2 * tile) {
      const uint32_t h = idx & 1, e = idx >> 1, col = e & (C - 1), row = e >> c;
      uint64_t g;
      uint32_t t;
      if (pp.first) {
        g = ((uint64_t)row << xcols_log) + col0 + col;
        t = rev_bits(row, k);
      } else {
        g = hi_base + ((uint64_t)row << pp.S) + m0 + col;
        t = row;
      }
      sm[h * TILE_MAX + ((t << c) | col)] = pp.src[(g << 1) | h];
    }
  }
  __syncthreads();

  uint32_t i = 1;
  // ---- an odd stage count starts with one radix-2 stage ----
  if (k & 1) {
    const uint64_t half_g = 1ull << pp.S;  // stage S+1
    const uint4* stw = pp.tw + ((half_g - 1) << 1);
#pragma unroll
    for (uint32_t q = 0; q < TILE_MAX / 2 / THREADS; q++) {
      const uint32_t b = tid + q * THREADS;
      if (b < tile / 2) {
        const uint32_t col = b & (C - 1), t0 = (b >> c) << 1;  // half = 1: j = 0
        const uint64_t jg = pp.first ? 0 : m0 + col;
        const uint32_t e0 = (t0 << c) | col, e1 = e0 + C;
        fe u = sm_load(sm, e0), v = sm_load(sm, e1), w;
        const bool mul = twiddle<F>(pp, stw, half_g, jg, w);
        butterfly<F>(u, v, mul, w);
        sm_store(sm, e0, u);
        sm_store(sm, e1, v);
      }
    }
    __syncthreads();
    i = 2;
  }

  // ---- radix-4 groups: stages i and i+1 on four elements in registers ----
  for (; i < k; i += 2) {
    const uint32_t h = 1u << (i - 1);
    const uint64_t half1 = 1ull << (pp.S + i - 1);  // stage S+i
    const uint64_t half2 = half1 << 1;              // stage S+i+1
    const uint4* stw1 = pp.tw + ((half1 - 1) << 1);
    const uint4* stw2 = pp.tw + ((half2 - 1) << 1);
#pragma unroll
    for (uint32_t q = 0; q < TILE_MAX / 4 / THREADS; q++) {
      const uint32_t ga = tid + q * THREADS;
      if (ga < tile / 4) {
        const uint32_t col = ga & (C - 1), g = ga >> c;
        const uint32_t j = g & (h - 1);
        const uint32_t t0 = ((g >> (i - 1)) << (i + 1)) | j;
        const uint32_t e0 = (t0 << c) | col, eh = h << c;
        uint64_t jg1, jg3;
        if (pp.first) {
          jg1 = j;
          jg3 = j + h;
        } else {
          jg1 = ((uint64_t)j << pp.S) + m0 + col;
          jg3 = jg1 + ((uint64_t)h << pp.S);
        }
        fe w1, w2, w3;
        const bool m1 = twiddle<F>(pp, stw1, half1, jg1, w1);
        const bool m2 = twiddle<F>(pp, stw2, half2, jg1, w2);
        const bool m3 = twiddle<F>(pp, stw2, half2, jg3, w3);
        fe x0 = sm_load(sm, e0), x1 = sm_load(sm, e0 + eh), x2 = sm_load(sm, e0 + 2 * eh),
           x3 = sm_load(sm, e0 + 3 * eh);
        butterfly<F>(x0, x1, m1, w1);
        butterfly<F>(x2, x3, m1, w1);
        butterfly<F>(x0, x2, m2, w2);
        butterfly<F>(x1, x3, m3, w3);
        sm_store(sm, e0, x0);
        sm_store(sm, e0 + eh, x1);
        sm_store(sm, e0 + 2 * eh, x2);
        sm_store(sm, e0 + 3 * eh, x3);
      }
    }
    __syncthreads();
  }

  if (pp.scale) {
    fe sc;
#pragma unroll
    for (int q = 0; q < 8; q++) sc.v[q] = pp.scale_val[q];
#pragma unroll
    for (uint32_t q = 0; q < TILE_MAX / THREADS; q++) {
      const uint32_t e = tid + q * THREADS;
      if (e < tile) sm_store(sm, e, fe_mul<F>(sm_load(sm, e), sc));
    }
    __syncthreads();
  }

  // ---- store ----
#pragma unroll
  for (uint32_t q = 0; q < 2 * TILE_MAX / THREADS; q++) {
    const uint32_t idx = tid + q * THREADS;
    if (idx < 2 * tile) {
      const uint32_t h = idx & 1, e = idx >> 1, col = e & (C - 1), row = e >> c;
      uint64_t g;
      if (pp.first) {
        g = ((uint64_t)rev_bits((uint32_t)(col0 + col), xcols_log) << k) + row;
      } else {
        g = hi_base + ((uint64_t)row << pp.S) + m0 + col;
      }
      pp.dst[(g << 1) | h] = sm[h * TILE_MAX + ((row << c) | col)];
    }
  }
}

#define ZNTT_PASS(F) ntt_pass_kernel<F, kLogTile, kPassThreads, kPassMinBlocks>

cudaError_t configure_kernels() {
  cudaError_t e = cudaFuncSetAttribute(ZNTT_PASS(Bn254Fr), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       kPassSmemBytes);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(ZNTT_PASS(Bls12381Fr), cudaFuncAttributeMaxDynamicSharedMemorySize, kPassSmemBytes);
}

cudaError_t launch_ntt_pass(int field, const PassParams& pp, uint64_t num_tiles, cudaStream_t st) {
  dim3 grid((unsigned)num_tiles);
  if (field == kBn254Fr)
    ZNTT_PASS(Bn254Fr)<<<grid, kPassThreads, kPassSmemBytes, st>>>(pp);
  else
    ZNTT_PASS(Bls12381Fr)<<<grid, kPassThreads, kPassSmemBytes, st>>>(pp);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Twiddle table
// ---------------------------------------------------------------------------

template <class F>
__global__ void twiddle_table_kernel(const uint4* __restrict__ pw, uint4* __restrict__ table, uint32_t log_n) {
  const uint64_t total = (1ull << log_n) - 1;
  for (uint64_t f = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; f < total;
       f += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t s = 63 - __clzll(f + 1);           // stage: 2^s - 1 <= f < 2^(s+1) - 1
    const uint64_t j = f + 1 - (1ull << s);
    const uint64_t e = j << (log_n - 1 - s);           // exponent of root, < 2^(log_n-1)
    const uint32_t e0 = e & 1023, e1 = (e >> 10) & 1023, e2 = (uint32_t)(e >> 20);
    fe r = fe_mul<F>(fe_load_nc(pw + 2 * e0), fe_load_nc(pw + 2 * (1024 + e1)));
    r = fe_mul<F>(r, fe_load_nc(pw + 2 * (2048 + e2)));
    fe_store(table + 2 * f, r);
  }
}

cudaError_t launch_twiddle_table(int field, const uint4* d_pw, uint4* d_table, uint32_t log_n, cudaStream_t st) {
  if (log_n == 0) return cudaSuccess;
  const uint64_t total = (1ull << log_n) - 1;
  uint64_t blocks = (total + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  if (field == kBn254Fr)
    twiddle_table_kernel<Bn254Fr><<<(unsigned)blocks, 256, 0, st>>>(d_pw, d_table, log_n);
  else
    twiddle_table_kernel<Bls12381Fr><<<(unsigned)blocks, 256, 0, st>>>(d_pw, d_table, log_n);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Bit reversal (zig-ntt bitReverse, libs/ntt/src/root.zig:38-58), out of place
// ---------------------------------------------------------------------------

__global__ void bit_reverse_kernel(const uint4* __restrict__ src, uint4* __restrict__ dst, uint32_t log_n) {
  const uint64_t n2 = 2ull << log_n;  // uint4 count
  for (uint64_t idx = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; idx < n2;
       idx += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t i = idx >> 1;
    const uint64_t r = log_n == 0 ? 0 : (__brevll(i) >> (64 - log_n));
    dst[2 * r + (idx & 1)] = src[idx];
  }
}

cudaError_t launch_bit_reverse(const uint4* src, uint4* dst, uint32_t log_n, cudaStream_t st) {
  const uint64_t n2 = 2ull << log_n;
  uint64_t blocks = (n2 + 255) / 256;
  if (blocks > 148 * 32) blocks = 148 * 32;
  bit_reverse_kernel<<<(unsigned)blocks, 256, 0, st>>>(src, dst, log_n);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Elementwise arithmetic (device unit tests)
// ---------------------------------------------------------------------------

template <class F>
__global__ void elementwise_kernel(int op, const uint4* a, const uint4* b, uint4* out, uint64_t count) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count;
       i += (uint64_t)gridDim.x * blockDim.x) {
    fe x = fe_load(a + 2 * i);
    fe r;
    if (op == 3) {
      r = fe_neg<F>(x);
    } else {
      fe y = fe_load(b + 2 * i);
      r = op == 0 ? fe_mul<F>(x, y) : op == 1 ? fe_add<F>(x, y) : fe_sub<F>(x, y);
    }
    fe_store(out + 2 * i, r);
  }
}

cudaError_t launch_elementwise(int field, int op, const uint4* a, const uint4* b, uint4* out, uint64_t count,
                               cudaStream_t st) {
  uint64_t blocks = (count + 255) / 256;
  if (blocks > 148 * 8) blocks = 148 * 8;
  if (blocks == 0) return cudaSuccess;
  if (field == kBn254Fr)
    elementwise_kernel<Bn254Fr><<<(unsigned)blocks, 256, 0, st>>>(op, a, b, out, count);
  else
    elementwise_kernel<Bls12381Fr><<<(unsigned)blocks, 256, 0, st>>>(op, a, b, out, count);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Throughput probes for the roofline denominator
// ---------------------------------------------------------------------------

// 32-bit multiply-adds (mad.lo.u32), the multiply pipe's unit of issue: a
// full 32x32->64 product costs two of them (lo and hi), so one 8x32-bit CIOS
// field product (136 products) costs 272.  Each multiply takes the previous
// result as its multiplicand, so nothing can be hoisted; eight independent
// chains per thread.  Each iteration issues 8 multiply-adds.
__global__ void imad_probe_kernel(uint32_t* sink, uint32_t iters) {
  const uint32_t b = (blockIdx.x * 40503u + threadIdx.x * 2654435761u) | 1u;
  uint32_t acc[8];
#pragma unroll
  for (int q = 0; q < 8; q++) acc[q] = threadIdx.x * 977u + q * 131u + 1u;
  for (uint32_t it = 0; it < iters; it++) {
#pragma unroll
    for (int q = 0; q < 8; q++) asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(acc[q]) : "r"(b), "r"(q * 7u + 1u));
  }
  uint32_t x = 0;
#pragma unroll
  for (int q = 0; q < 8; q++) x ^= acc[q];
  if (x == 0x9e3779b9u) sink[0] = x;
}

cudaError_t launch_imad_probe(uint32_t* sink, uint32_t iters, int blocks, int threads, cudaStream_t st) {
  imad_probe_kernel<<<blocks, threads, 0, st>>>(sink, iters);
  return cudaGetLastError();
}

// Full 32x32->64 products (mad.wide.u32), the unit the field multiply needs
// 2N^2 + N = 136 of.  Each product's multiplicand is the low word of the
// previous result, so the product cannot be hoisted out of the loop; eight
// independent chains per thread keep the multiply pipe fed.  Each iteration
// issues 8 products.
__global__ void imad_wide_probe_kernel(unsigned long long* sink, uint32_t iters) {
  const uint32_t b = (blockIdx.x * 40503u + threadIdx.x * 2654435761u) | 1u;
  unsigned long long acc[8];
#pragma unroll
  for (int q = 0; q < 8; q++) acc[q] = (threadIdx.x * 977u + q * 131u) | 1u;
  for (uint32_t it = 0; it < iters; it++) {
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const uint32_t lo = (uint32_t)acc[q];
      asm volatile("mad.wide.u32 %0, %1, %2, %0;" : "+l"(acc[q]) : "r"(lo), "r"(b));
    }
  }
  unsigned long long x = 0;
#pragma unroll
  for (int q = 0; q < 8; q++) x ^= acc[q];
  if (x == 0x9e3779b97f4a7c15ull) sink[0] = x;
}

cudaError_t launch_imad_wide_probe(unsigned long long* sink, uint32_t iters, int blocks, int threads,
                                   cudaStream_t st) {
  imad_wide_probe_kernel<<<blocks, threads, 0, st>>>(sink, iters);
  return cudaGetLastError();
}

template <class F>
__global__ void modmul_probe_kernel(uint4* sink, uint32_t iters) {
  fe x0, x1, y;
#pragma unroll
  for (int q = 0; q < 8; q++) {
    x0.v[q] = (threadIdx.x * 2654435761u + q) & 0x0fffffff;
    x1.v[q] = (blockIdx.x * 40503u + q * 7) & 0x0fffffff;
    y.v[q] = (threadIdx.x * 0x01000193u + q * 3 + 5) & 0x0fffffff;
  }
  for (uint32_t it = 0; it < iters; it++) {
    x0 = fe_mul<F>(x0, y);
    x1 = fe_mul<F>(x1, y);
  }
  fe r = fe_add<F>(x0, x1);
  if (r.v[0] == 0x9e3779b9u) fe_store(sink, r);
}

cudaError_t launch_modmul_probe(int field, uint4* sink, uint32_t iters, int blocks, int threads, cudaStream_t st) {
  if (field == kBn254Fr)
    modmul_probe_kernel<Bn254Fr><<<blocks, threads, 0, st>>>(sink, iters);
  else
    modmul_probe_kernel<Bls12381Fr><<<blocks, threads, 0, st>>>(sink, iters);
  return cudaGetLastError();
}

}  // namespace zntt
