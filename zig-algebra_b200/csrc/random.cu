// random.cu -- seeded uniform field elements on the device.
//
// Reproduces, in parallel, the reference's sequential input generator:
// ChaCha20 keyed by a 32-byte seed, zero nonce, block counter from 0
// (libs/rng/src/chacha20.zig:36-110), consumed in order 32 bytes at a time by
// randomFieldElement (libs/rng/src/rng.zig:32-65), which reads the 32 bytes
// big-endian and rejects values >= p.  Chunk c of the stream is half c & 1 of
// block c >> 1, so every chunk can be produced independently: one kernel
// flags the accepted chunks, a prefix sum ranks them, and a second kernel
// writes accepted chunk number i to element i (converted to Montgomery form).
// The result is bit-identical to the sequential draw.
#include <cub/device/device_scan.cuh>

#include <cstring>
#include <vector>

#include "field.cuh"
#include "runtime.hpp"

namespace zntt {

struct ChaChaKey {
  uint32_t k[8];
};

__device__ __forceinline__ uint32_t rotl(uint32_t x, int r) { return __funnelshift_l(x, x, r); }

#define QR(a, b, c, d)              \
  a += b; d = rotl(d ^ a, 16);      \
  c += d; b = rotl(b ^ c, 12);      \
  a += b; d = rotl(d ^ a, 8);       \
  c += d; b = rotl(b ^ c, 7);

// One 64-byte block as 16 little-endian words.
__device__ __forceinline__ void chacha_block(const ChaChaKey& key, uint32_t counter, uint32_t out[16]) {
  const uint32_t s[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u, key.k[0], key.k[1],
                          key.k[2],    key.k[3],    key.k[4],    key.k[5],    key.k[6], key.k[7],
                          counter,     0u,          0u,          0u};
  uint32_t x0 = s[0], x1 = s[1], x2 = s[2], x3 = s[3], x4 = s[4], x5 = s[5], x6 = s[6], x7 = s[7];
  uint32_t x8 = s[8], x9 = s[9], x10 = s[10], x11 = s[11], x12 = s[12], x13 = s[13], x14 = s[14], x15 = s[15];
#pragma unroll 1
  for (int i = 0; i < 10; i++) {
    QR(x0, x4, x8, x12) QR(x1, x5, x9, x13) QR(x2, x6, x10, x14) QR(x3, x7, x11, x15)
    QR(x0, x5, x10, x15) QR(x1, x6, x11, x12) QR(x2, x7, x8, x13) QR(x3, x4, x9, x14)
  }
  out[0] = x0 + s[0]; out[1] = x1 + s[1]; out[2] = x2 + s[2]; out[3] = x3 + s[3];
  out[4] = x4 + s[4]; out[5] = x5 + s[5]; out[6] = x6 + s[6]; out[7] = x7 + s[7];
  out[8] = x8 + s[8]; out[9] = x9 + s[9]; out[10] = x10 + s[10]; out[11] = x11 + s[11];
  out[12] = x12 + s[12]; out[13] = x13 + s[13]; out[14] = x14 + s[14]; out[15] = x15 + s[15];
}

// The 32 bytes of one half-block read big-endian, as 8 little-endian u32 limbs:
// byte 0 of the chunk is the most significant byte.
__device__ __forceinline__ fe chunk_value(const uint32_t w[16], int half) {
  fe v;
#pragma unroll
  for (int q = 0; q < 8; q++) v.v[7 - q] = __byte_perm(w[8 * half + q], 0, 0x0123);
  return v;
}

template <class F>
__global__ void chacha_flag_kernel(ChaChaKey key, uint64_t block0, uint64_t nblocks, uint32_t* flags) {
  for (uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; b < nblocks;
       b += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t w[16];
    chacha_block(key, (uint32_t)(block0 + b), w);
    flags[2 * b] = fe_lt_p<F>(chunk_value(w, 0)) ? 1u : 0u;
    flags[2 * b + 1] = fe_lt_p<F>(chunk_value(w, 1)) ? 1u : 0u;
  }
}

template <class F>
__global__ void chacha_emit_kernel(ChaChaKey key, uint64_t block0, uint64_t nblocks, const uint32_t* flags,
                                   const uint32_t* rank, uint64_t out_base, uint64_t count, uint4* out) {
  for (uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; b < nblocks;
       b += (uint64_t)gridDim.x * blockDim.x) {
    if (!(flags[2 * b] | flags[2 * b + 1])) continue;
    uint32_t w[16];
    chacha_block(key, (uint32_t)(block0 + b), w);
#pragma unroll
    for (int h = 0; h < 2; h++) {
      if (!flags[2 * b + h]) continue;
      const uint64_t i = out_base + rank[2 * b + h];
      if (i < count) fe_store(out + 2 * i, fe_mul<F>(chunk_value(w, h), fe_r2<F>()));
    }
  }
}

}  // namespace zntt

using namespace zntt;

extern "C" int zntt_random_elements(int field, const uint8_t seed32[32], uint64_t* d_out, size_t count,
                                    void* stream) {
  clear_error();
  if (field != kBn254Fr && field != kBls12381Fr) return set_error(ZNTT_ERR_UNSUPPORTED_FIELD, "unsupported field");
  if (!seed32 || (!d_out && count)) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null pointer");
  if (ctx().device < 0) return set_error(ZNTT_ERR_NOT_INITIALIZED, "zntt_init has not been called");
  if (count == 0) return ZNTT_OK;
  Context& c = ctx();
  std::lock_guard<std::recursive_mutex> lock(c.mu);
  cudaStream_t st = stream ? (cudaStream_t)stream : c.stream;
  ChaChaKey key;
  for (int i = 0; i < 8; i++)
    key.k[i] = (uint32_t)seed32[4 * i] | ((uint32_t)seed32[4 * i + 1] << 8) | ((uint32_t)seed32[4 * i + 2] << 16) |
               ((uint32_t)seed32[4 * i + 3] << 24);
  // Acceptance is |p| / 2^256: 0.189 for BN254-Fr, 0.453 for BLS12-381-Fr.
  const double accept = field == kBn254Fr ? 0.1890 : 0.4530;
  uint64_t produced = 0, block = 0;
  while (produced < count) {
    const uint64_t want = count - produced;
    uint64_t nblocks = (uint64_t)((double)want / accept / 2.0 * 1.02) + 1024;
    if (nblocks > (1ull << 26)) nblocks = 1ull << 26;
    if (block + nblocks > (1ull << 32))
      return set_error(ZNTT_ERR_INVALID_ARGUMENT, "ChaCha20 block counter exhausted");
    const uint64_t nchunks = 2 * nblocks;
    void* flags = nullptr;
    void* rank = nullptr;
    void* tmp = nullptr;
    size_t tmp_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, (uint32_t*)nullptr, (uint32_t*)nullptr, (int)nchunks, st);
    cudaError_t e = c.pool.acquire(nchunks * 4, &flags);
    if (e == cudaSuccess) e = c.pool.acquire(nchunks * 4, &rank);
    if (e == cudaSuccess) e = c.pool.acquire(tmp_bytes, &tmp);
    auto cleanup = [&]() {
      if (flags) c.pool.release(flags, nchunks * 4);
      if (rank) c.pool.release(rank, nchunks * 4);
      if (tmp) c.pool.release(tmp, tmp_bytes);
    };
    if (e != cudaSuccess) {
      cleanup();
      return cuda_fail(e, "random buffers");
    }
    const int threads = 256;
    uint64_t grid = (nblocks + threads - 1) / threads;
    if (grid > 148 * 64) grid = 148 * 64;
    if (field == kBn254Fr)
      chacha_flag_kernel<Bn254Fr><<<(unsigned)grid, threads, 0, st>>>(key, block, nblocks, (uint32_t*)flags);
    else
      chacha_flag_kernel<Bls12381Fr><<<(unsigned)grid, threads, 0, st>>>(key, block, nblocks, (uint32_t*)flags);
    e = cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, (uint32_t*)flags, (uint32_t*)rank, (int)nchunks, st);
    if (e == cudaSuccess) {
      if (field == kBn254Fr)
        chacha_emit_kernel<Bn254Fr><<<(unsigned)grid, threads, 0, st>>>(
            key, block, nblocks, (uint32_t*)flags, (uint32_t*)rank, produced, count, (uint4*)d_out);
      else
        chacha_emit_kernel<Bls12381Fr><<<(unsigned)grid, threads, 0, st>>>(
            key, block, nblocks, (uint32_t*)flags, (uint32_t*)rank, produced, count, (uint4*)d_out);
      e = cudaGetLastError();
    }
    uint32_t last_rank = 0, last_flag = 0;
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(&last_rank, (uint32_t*)rank + nchunks - 1, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(&last_flag, (uint32_t*)flags + nchunks - 1, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cleanup();
    if (e != cudaSuccess) return cuda_fail(e, "random elements");
    produced += (uint64_t)last_rank + last_flag;
    block += nblocks;
  }
  return ZNTT_OK;
}
