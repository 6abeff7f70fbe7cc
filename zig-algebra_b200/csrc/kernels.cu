// kernels.cu -- sm_100a kernels of the NTT hot path.
//
// The transform is zig-ntt's radix-2 decimation-in-time network
// (libs/ntt/src/root.zig:148-212) executed as a few fused passes: each pass
// stages a tile of the vector in shared memory with coalesced 16-byte global
// loads, runs several butterfly stages on it, and writes it back.  All
// arithmetic is exact Montgomery arithmetic from field.cuh.
#include <cstring>

#include "field.cuh"
#include "kernels.cuh"
#include "pass_tile.cuh"

namespace zntt {

// SCALE: the pass scales its outputs (the inverse's last pass, or an
// extension pass); the extension variants always include it.
template <class F, int LOG_TILE, int THREADS, int MINB, bool EXT, bool FULL, bool SCALE>
__global__ void __launch_bounds__(THREADS, MINB) ntt_pass_kernel(PassParams pp) {
  extern __shared__ uint4 sm[];
  ntt_tile<F, LOG_TILE, THREADS, false, EXT, FULL, SCALE>(pp, blockIdx.x, sm);
}

template <class F, int SH, bool EXT, bool FULL, bool SCALE>
static void* pass_ptr() {
  return (void*)ntt_pass_kernel<F, kShapes[SH].log_tile, kShapes[SH].threads, kShapes[SH].min_blocks, EXT, FULL,
                                SCALE>;
}

template <class F, int SH>
static cudaError_t set_shape_attrs() {
  void* fns[6] = {pass_ptr<F, SH, false, false, false>(), pass_ptr<F, SH, false, false, true>(),
                  pass_ptr<F, SH, false, true, false>(),  pass_ptr<F, SH, false, true, true>(),
                  pass_ptr<F, SH, true, false, true>(),   pass_ptr<F, SH, true, true, true>()};
  for (int i = 0; i < 6; i++) {
    cudaError_t e = cudaFuncSetAttribute(fns[i], cudaFuncAttributeMaxDynamicSharedMemorySize, shape_smem_bytes(SH));
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

template <class F>
static cudaError_t set_pass_attrs() {
  cudaError_t e = set_shape_attrs<F, 0>();
  if (e == cudaSuccess) e = set_shape_attrs<F, 1>();
  if (e == cudaSuccess) e = set_shape_attrs<F, 2>();
  if (e == cudaSuccess) e = set_shape_attrs<F, 3>();
  if (e == cudaSuccess) e = set_shape_attrs<F, 4>();
  return e;
}

cudaError_t configure_kernels() {
  cudaError_t e = set_pass_attrs<Bn254Fr>();
  if (e == cudaSuccess) e = set_pass_attrs<Bls12381Fr>();
  if (e != cudaSuccess) return e;
  return configure_batch_kernels();
}

template <class F, int SH, bool FULL>
static void launch_pass_full(bool ext, const PassParams& pp, dim3 grid, cudaStream_t st) {
  constexpr PassShape S = kShapes[SH];
  constexpr int T = S.threads;
  const int smem = shape_smem_bytes(SH);
  if (ext)
    ntt_pass_kernel<F, S.log_tile, T, S.min_blocks, true, FULL, true><<<grid, T, smem, st>>>(pp);
  else if (pp.scale || F::kScaleCompiled)
    ntt_pass_kernel<F, S.log_tile, T, S.min_blocks, false, FULL, true><<<grid, T, smem, st>>>(pp);
  else
    ntt_pass_kernel<F, S.log_tile, T, S.min_blocks, false, FULL, false><<<grid, T, smem, st>>>(pp);
}

template <class F, int SH>
static void launch_pass_shape(bool ext, const PassParams& pp, dim3 grid, cudaStream_t st) {
  // Passes whose tile is the shape's whole tile run the variant without bound checks.
  if (pp.k + pp.c == (uint32_t)kShapes[SH].log_tile) launch_pass_full<F, SH, true>(ext, pp, grid, st);
  else launch_pass_full<F, SH, false>(ext, pp, grid, st);
}

template <class F>
static void launch_pass_typed(int shape, bool ext, const PassParams& pp, dim3 grid, cudaStream_t st) {
  switch (shape) {
    case 0: launch_pass_shape<F, 0>(ext, pp, grid, st); break;
    case 1: launch_pass_shape<F, 1>(ext, pp, grid, st); break;
    case 2: launch_pass_shape<F, 2>(ext, pp, grid, st); break;
    case 3: launch_pass_shape<F, 3>(ext, pp, grid, st); break;
    default: launch_pass_shape<F, 4>(ext, pp, grid, st); break;
  }
}

cudaError_t launch_ntt_pass(int field, int shape, const PassParams& pp, uint64_t num_tiles, cudaStream_t st) {
  dim3 grid((unsigned)num_tiles);
  const bool ext = pass_needs_ext(pp);
  if (field == kBn254Fr)
    launch_pass_typed<Bn254Fr>(shape, ext, pp, grid, st);
  else
    launch_pass_typed<Bls12381Fr>(shape, ext, pp, grid, st);
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

// out[i] = c * base^i from three host-made power tables of the base
// (pw[0][i] = base^i, pw[1][i] = base^(1024 i), pw[2][i] = base^(2^20 i)).
template <class F>
__global__ void powers_kernel(const uint4* __restrict__ pw, fe c, uint4* __restrict__ out, uint64_t count) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t e0 = i & 1023, e1 = (i >> 10) & 1023, e2 = (uint32_t)(i >> 20);
    fe r = fe_mul<F>(fe_load_nc(pw + 2 * e0), fe_load_nc(pw + 2 * (1024 + e1)));
    r = fe_mul<F>(r, fe_load_nc(pw + 2 * (2048 + e2)));
    fe_store(out + 2 * i, fe_mul<F>(r, c));
  }
}

cudaError_t launch_powers(int field, const uint4* d_pw, const uint64_t* c, uint4* out, uint64_t count,
                          cudaStream_t st) {
  fe cv;
  std::memcpy(cv.v, c, 32);
  uint64_t blocks = (count + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  if (blocks == 0) return cudaSuccess;
  if (field == kBn254Fr)
    powers_kernel<Bn254Fr><<<(unsigned)blocks, 256, 0, st>>>(d_pw, cv, out, count);
  else
    powers_kernel<Bls12381Fr><<<(unsigned)blocks, 256, 0, st>>>(d_pw, cv, out, count);
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
