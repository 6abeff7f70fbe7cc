// small.cu -- zig-ntt over zig-field's SmallField backend: Goldilocks and
// BabyBear (libs/field/src/field.zig:89-849), the fields of the reference's
// own known-answer transform tests (libs/ntt/src/root.zig:437-447).
//
// An element is SmallField's canonical u64 (8 bytes).  The transform is the
// same DIT network as the 256-bit path (root.zig:148-212; bit reversal folded
// into the first pass, tiles of 2^k positions x 2^c neighbouring columns,
// radix-4 register groups, 1/n fused into the last pass), on 8-byte elements
// with tiles of 2^12 in shared memory.  Twiddle tables live on the device in
// twiddle form (small_field.cuh); host tables handed across the C ABI are
// canonical, in zig-ntt's layout.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "runtime.hpp"
#include "small.hpp"
#include "small_field.cuh"

namespace zntt {

namespace {

// ---- host arithmetic ----------------------------------------------------------

struct SmallHost {
  int field;
  uint64_t p;
  uint32_t two_adicity;
  uint64_t r;  // R mod p: the twiddle-form factor (1 for Goldilocks, 2^32 for BabyBear)

  uint64_t mul(uint64_t a, uint64_t b) const { return (uint64_t)((unsigned __int128)a * b % p); }
  uint64_t pow(uint64_t a, uint64_t e) const {
    uint64_t r1 = 1 % p;
    while (e) {
      if (e & 1) r1 = mul(r1, a);
      a = mul(a, a);
      e >>= 1;
    }
    return r1;
  }
  uint64_t inv(uint64_t a) const { return pow(a, p - 2); }  // p prime; inv(0) = 0
  uint64_t to_tw(uint64_t w) const { return mul(w % p, r); }
};

const SmallHost kGoldilocksHost{kGoldilocksField, Goldilocks::P, 32, 1};
const SmallHost kBabyBearHost{kBabyBearField, BabyBear::P, 27, (uint64_t)(((unsigned __int128)1 << 32) % BabyBear::P)};

const SmallHost& small_host(int field) { return field == kGoldilocksField ? kGoldilocksHost : kBabyBearHost; }

// ---- kernels -------------------------------------------------------------------

constexpr int kSmallLogTile = 12;
constexpr int kSmallThreads = 256;
constexpr uint32_t kSmallKmax = 10;  // keeps 2^(12 - k) >= 4 columns (32-byte rows) per tile row
// Goldilocks transforms of 2^21 elements and more run on 2^11-element tiles in
// CTAs of 128 threads (10 per SM): the same warps per SM in smaller CTAs, whose
// barriers wait on fewer warps (2^24: 7.7% faster than 2^12 tiles in 256
// threads, B200).  BabyBear gains nothing from it and keeps the larger tile.
constexpr int kSmallLogTileB = 11;
constexpr int kSmallThreadsB = 128;
constexpr uint32_t kSmallKmaxB = 9;  // keeps 32-byte rows on 2^11-element tiles
bool small_use_b(int field, uint32_t log_n) { return field == kGoldilocksField && log_n >= 21; }

struct SmallPass {
  const uint64_t* src;
  uint64_t* dst;
  const uint64_t* tw;  // twiddle form, stage s at entry 2^s - 1
  uint32_t log_n, S, k, c, first, inverse, tw0_one, scale;
  uint64_t scale_val;  // twiddle form
  uint32_t src_len;    // column launches' first pass: natural index >= src_len reads as zero
};

__device__ __forceinline__ uint32_t rev_bits_small(uint32_t x, uint32_t bits) {
  return bits == 0 ? 0u : (__brev(x) >> (32 - bits));
}

// Twiddle of global stage s for butterfly jg: forward tw[s-1][jg], inverse 1
// (jg = 0) or -tw[s-1][2^(s-1) - jg] (root.zig:199); false when it is one.
// Indices are 32-bit: transforms are at most 2^31 elements.
template <class SF>
__device__ __forceinline__ bool small_twiddle(const SmallPass& pp, const uint64_t* stw, uint32_t half, uint32_t jg,
                                              uint64_t& w) {
  if (jg == 0 && (pp.inverse | pp.tw0_one)) return false;
  w = pp.inverse ? SF::neg(__ldg(stw + (half - jg))) : __ldg(stw + jg);
  return true;
}

template <class SF>
__device__ __forceinline__ void small_butterfly(uint64_t& u, uint64_t& v, bool mul, uint64_t w) {
  const uint64_t t = mul ? SF::mul(w, v) : v;
  v = SF::sub(u, t);
  u = SF::add(u, t);
}

// One tile of one pass.  PAD: the first pass reads natural indices at or
// beyond pp.src_len as zeros (a zero-padded input that is not stored).  FULL:
// the tile is the whole 2^LOG_TILE (k + c == LOG_TILE), so no bound checks
// (2^24 BabyBear about 10% faster without them on B200).
template <class SF, int LOG_TILE, int THREADS, bool PAD, bool FULL = false>
__device__ __forceinline__ void small_pass_body(const SmallPass& pp, uint32_t blk, uint64_t* sm) {
  constexpr uint32_t TILE_MAX = 1u << LOG_TILE;
  const uint32_t k = pp.k, c = pp.c, C = 1u << c;
  const uint32_t tile = FULL ? TILE_MAX : 1u << (k + c);
  const uint32_t tid = threadIdx.x;
  uint32_t hi_base = 0, m0 = 0, col0 = 0;
  if (pp.first) {
    col0 = blk << c;
  } else {
    const uint32_t mlog = pp.S - c;
    hi_base = (blk >> mlog) << (pp.S + k);
    m0 = (blk & ((1u << mlog) - 1)) << c;
  }
  const uint32_t xcols_log = pp.log_n - k;

#pragma unroll
  for (uint32_t q = 0; q < TILE_MAX / THREADS; q++) {
    const uint32_t e = tid + q * THREADS;
    if (FULL || e < tile) {
      const uint32_t col = e & (C - 1), row = e >> c;
      uint32_t g, t;
      if (pp.first) {
        g = (row << xcols_log) + col0 + col;
        t = rev_bits_small(row, k);
      } else {
        g = hi_base + (row << pp.S) + m0 + col;
        t = row;
      }
      sm[(t << c) | col] = (PAD && pp.first && g >= pp.src_len) ? 0 : pp.src[g];
    }
  }
  __syncthreads();

  uint32_t i = 1;
  if (k & 1) {
    const uint32_t half = 1u << pp.S;
    const uint64_t* stw = pp.tw + (half - 1);
#pragma unroll
    for (uint32_t q = 0; q < TILE_MAX / 2 / THREADS; q++) {
      const uint32_t b = tid + q * THREADS;
      if (FULL || b < tile / 2) {
        const uint32_t col = b & (C - 1), t0 = (b >> c) << 1;
        const uint32_t jg = pp.first ? 0 : m0 + col;
        const uint32_t e0 = (t0 << c) | col, e1 = e0 + C;
        uint64_t u = sm[e0], v = sm[e1], w = 0;
        const bool mul = small_twiddle<SF>(pp, stw, half, jg, w);
        small_butterfly<SF>(u, v, mul, w);
        sm[e0] = u;
        sm[e1] = v;
      }
    }
    __syncthreads();
    i = 2;
  }
  for (; i < k; i += 2) {
    const uint32_t h = 1u << (i - 1);
    const uint32_t half1 = 1u << (pp.S + i - 1), half2 = half1 << 1;
    const uint64_t* stw1 = pp.tw + (half1 - 1);
    const uint64_t* stw2 = pp.tw + (half2 - 1);
#pragma unroll
    for (uint32_t q = 0; q < TILE_MAX / 4 / THREADS; q++) {
      const uint32_t ga = tid + q * THREADS;
      if (FULL || ga < tile / 4) {
        const uint32_t col = ga & (C - 1), g = ga >> c;
        const uint32_t j = g & (h - 1);
        const uint32_t t0 = ((g >> (i - 1)) << (i + 1)) | j;
        const uint32_t e0 = (t0 << c) | col, eh = h << c;
        uint32_t jg1, jg3;
        if (pp.first) {
          jg1 = j;
          jg3 = j + h;
        } else {
          jg1 = (j << pp.S) + m0 + col;
          jg3 = jg1 + (h << pp.S);
        }
        uint64_t w1 = 0, w2 = 0, w3 = 0;
        const bool m1 = small_twiddle<SF>(pp, stw1, half1, jg1, w1);
        const bool m2 = small_twiddle<SF>(pp, stw2, half2, jg1, w2);
        const bool m3 = small_twiddle<SF>(pp, stw2, half2, jg3, w3);
        uint64_t x0 = sm[e0], x1 = sm[e0 + eh], x2 = sm[e0 + 2 * eh], x3 = sm[e0 + 3 * eh];
        small_butterfly<SF>(x0, x1, m1, w1);
        small_butterfly<SF>(x2, x3, m1, w1);
        small_butterfly<SF>(x0, x2, m2, w2);
        small_butterfly<SF>(x1, x3, m3, w3);
        sm[e0] = x0;
        sm[e0 + eh] = x1;
        sm[e0 + 2 * eh] = x2;
        sm[e0 + 3 * eh] = x3;
      }
    }
    __syncthreads();
  }

#pragma unroll
  for (uint32_t q = 0; q < TILE_MAX / THREADS; q++) {
    const uint32_t e = tid + q * THREADS;
    if (FULL || e < tile) {
      const uint32_t col = e & (C - 1), row = e >> c;
      const uint32_t g = pp.first ? (rev_bits_small(col0 + col, xcols_log) << k) + row
                                  : hi_base + (row << pp.S) + m0 + col;
      uint64_t x = sm[(row << c) | col];
      if (pp.scale) x = SF::mul(pp.scale_val, x);
      pp.dst[g] = x;
    }
  }
}

template <class SF, int LOG_TILE, int THREADS, bool FULL>
__global__ void __launch_bounds__(THREADS) small_pass_kernel(SmallPass pp) {
  __shared__ uint64_t sm[1u << LOG_TILE];
  small_pass_body<SF, LOG_TILE, THREADS, false, FULL>(pp, blockIdx.x, sm);
}

// The same pass over many columns of one size: column blockIdx.y reads
// srcs[y] and writes dsts[y] (device pointer tables).
template <class SF, int LOG_TILE, int THREADS, bool FULL>
__global__ void __launch_bounds__(THREADS) small_pass_cols_kernel(SmallPass pp, const uint64_t* const* srcs,
                                                                  uint64_t* const* dsts) {
  __shared__ uint64_t sm[1u << LOG_TILE];
  SmallPass q = pp;
  q.src = srcs[blockIdx.y];
  q.dst = dsts[blockIdx.y];
  small_pass_body<SF, LOG_TILE, THREADS, true, FULL>(q, blockIdx.x, sm);
}

// Flat table entry e = 2^s - 1 + j holds root^(j * 2^(log_n - 1 - s)), in
// twiddle form, from three power tables pw[t][i] = root^(i * 1024^t).
template <class SF>
__global__ void small_twiddle_kernel(const uint64_t* __restrict__ pw, uint64_t* __restrict__ out, uint32_t log_n) {
  const uint64_t total = (1ull << log_n) - 1;
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < total;
       e += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t s = 63 - __clzll(e + 1);
    const uint64_t j = e + 1 - (1ull << s);
    const uint64_t x = j << (log_n - 1 - s);
    uint64_t v = SF::mul(__ldg(pw + (x & 1023)), __ldg(pw + 1024 + ((x >> 10) & 1023)));
    out[e] = SF::mul(v, __ldg(pw + 2048 + (x >> 20)));
  }
}

// out[i] = in[i] * f (f chosen by the caller): converts between canonical and
// twiddle form (f = R^2 mod p, or the integer 1).  in and out may be the same
// array (each element is read, then written, by one thread), so the pointers
// are not restrict and the loads are coherent.
template <class SF>
__global__ void small_scale_kernel(const uint64_t* in, uint64_t* out, uint64_t count, uint64_t f) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = SF::mul(f, in[i]);
}

// out[i] = c * base^i for i < count (< 2^30), from power tables of base in
// twiddle form; c in twiddle form too.  mul(c_tw, v_tw) is the twiddle form of
// the product; with c = canonical one (not twiddle form) it is canonical.
template <class SF>
__global__ void small_powers_kernel(const uint64_t* __restrict__ pw, uint64_t c, uint64_t* __restrict__ out,
                                    uint64_t count) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t v = SF::mul(__ldg(pw + (i & 1023)), __ldg(pw + 1024 + ((i >> 10) & 1023)));
    out[i] = SF::mul(c, SF::mul(v, __ldg(pw + 2048 + (i >> 20))));
  }
}

// data[i] *= shift^i for i < count (< 2^30), the coset step of an extension,
// from power tables of the shift in twiddle form (so the product of three
// table entries is the twiddle form of shift^i, and its product with the
// canonical data[i] is canonical).
template <class SF>
__global__ void small_coset_scale_kernel(const uint64_t* __restrict__ pw, uint64_t* __restrict__ data,
                                         uint64_t count) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t v = SF::mul(__ldg(pw + (i & 1023)), __ldg(pw + 1024 + ((i >> 10) & 1023)));
    data[i] = SF::mul(SF::mul(v, __ldg(pw + 2048 + (i >> 20))), data[i]);
  }
}

// out[i] = a[i] * b[i] for canonical values: mul(a, R^2) is a in twiddle form
// (a R), whose product with the canonical b is canonical.
template <class SF>
__global__ void small_pointwise_kernel(const uint64_t* a, const uint64_t* __restrict__ b, uint64_t* out,
                                       uint64_t count, uint64_t r2) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = SF::mul(SF::mul(a[i], r2), b[i]);
}

// The coset step over m contiguous columns of 2^log_n values each: element
// i of every column times shift^i (i < 2^30, power tables as above).
template <class SF>
__global__ void small_coset_scale_cols_kernel(const uint64_t* __restrict__ pw, uint64_t* __restrict__ data,
                                              uint64_t total, uint32_t log_n) {
  const uint64_t mask = (1ull << log_n) - 1;
  for (uint64_t f = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; f < total; f += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t i = f & mask;
    const uint64_t v = SF::mul(__ldg(pw + (i & 1023)), __ldg(pw + 1024 + ((i >> 10) & 1023)));
    data[f] = SF::mul(SF::mul(v, __ldg(pw + 2048 + (i >> 20))), data[f]);
  }
}

// One FRI fold round (libs/fri/src/root.zig:396-403) on canonical values;
// half_inv, alpha and the table g^-j / 2 are in twiddle form.
template <class SF>
__global__ void small_fri_fold_kernel(const uint64_t* __restrict__ in, uint64_t* __restrict__ out,
                                      const uint64_t* __restrict__ tab, uint64_t half, uint32_t stride,
                                      uint64_t half_inv, uint64_t alpha) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < half; j += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t a = __ldg(in + j), b = __ldg(in + j + half);
    const uint64_t even = SF::mul(half_inv, SF::add(a, b));
    const uint64_t odd = SF::mul(__ldg(tab + (j << stride)), SF::sub(a, b));
    out[j] = SF::add(even, SF::mul(alpha, odd));
  }
}

__global__ void small_bit_reverse_kernel(const uint64_t* __restrict__ src, uint64_t* __restrict__ dst,
                                         uint32_t log_n) {
  const uint64_t n = 1ull << log_n;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    dst[__brevll(i) >> (64 - log_n)] = src[i];
}

int grid_for(uint64_t count) { return (int)std::min<uint64_t>((count + 255) / 256, 148 * 16); }

template <class SF, bool FULL>
static void launch_small_pass_t(const SmallPass& pp, uint64_t tiles, cudaStream_t st) {
  small_pass_kernel<SF, kSmallLogTile, kSmallThreads, FULL><<<(unsigned)tiles, kSmallThreads, 0, st>>>(pp);
}

cudaError_t launch_small_pass(int field, const SmallPass& pp, uint64_t tiles, cudaStream_t st) {
  const bool full = pp.k + pp.c == (uint32_t)kSmallLogTile;
  if (field == kGoldilocksField && pp.k + pp.c == (uint32_t)kSmallLogTileB) {
    // a whole 2^11-element tile: the smaller CTA
    small_pass_kernel<Goldilocks, kSmallLogTileB, kSmallThreadsB, true>
        <<<(unsigned)tiles, kSmallThreadsB, 0, st>>>(pp);
    return cudaGetLastError();
  }
  if (field == kGoldilocksField) {
    if (full) launch_small_pass_t<Goldilocks, true>(pp, tiles, st);
    else launch_small_pass_t<Goldilocks, false>(pp, tiles, st);
  } else {
    if (full) launch_small_pass_t<BabyBear, true>(pp, tiles, st);
    else launch_small_pass_t<BabyBear, false>(pp, tiles, st);
  }
  return cudaGetLastError();
}

cudaError_t launch_small_pass_cols(int field, const SmallPass& pp, uint64_t tiles, uint32_t m,
                                   const uint64_t* const* srcs, uint64_t* const* dsts, cudaStream_t st) {
  const dim3 grid((unsigned)tiles, m);
  const bool full = pp.k + pp.c == (uint32_t)kSmallLogTile;
  if (field == kGoldilocksField && pp.k + pp.c == (uint32_t)kSmallLogTileB) {
    small_pass_cols_kernel<Goldilocks, kSmallLogTileB, kSmallThreadsB, true>
        <<<grid, kSmallThreadsB, 0, st>>>(pp, srcs, dsts);
    return cudaGetLastError();
  }
  if (field == kGoldilocksField) {
    if (full)
      small_pass_cols_kernel<Goldilocks, kSmallLogTile, kSmallThreads, true><<<grid, kSmallThreads, 0, st>>>(pp, srcs, dsts);
    else
      small_pass_cols_kernel<Goldilocks, kSmallLogTile, kSmallThreads, false><<<grid, kSmallThreads, 0, st>>>(pp, srcs, dsts);
  } else {
    if (full)
      small_pass_cols_kernel<BabyBear, kSmallLogTile, kSmallThreads, true><<<grid, kSmallThreads, 0, st>>>(pp, srcs, dsts);
    else
      small_pass_cols_kernel<BabyBear, kSmallLogTile, kSmallThreads, false><<<grid, kSmallThreads, 0, st>>>(pp, srcs, dsts);
  }
  return cudaGetLastError();
}

cudaError_t launch_small_scale(int field, const uint64_t* in, uint64_t* out, uint64_t count, uint64_t f,
                               cudaStream_t st) {
  if (count == 0) return cudaSuccess;
  if (field == kGoldilocksField)
    small_scale_kernel<Goldilocks><<<grid_for(count), 256, 0, st>>>(in, out, count, f);
  else
    small_scale_kernel<BabyBear><<<grid_for(count), 256, 0, st>>>(in, out, count, f);
  return cudaGetLastError();
}

// ---- plans ---------------------------------------------------------------------

struct SmallPlanPass {
  uint32_t S, k, c;
};

std::vector<SmallPlanPass> small_plan(uint32_t log_n, int field) {
  std::vector<SmallPlanPass> plan;
  const bool b = small_use_b(field, log_n);
  const uint32_t lt = b ? kSmallLogTileB : kSmallLogTile;
  const uint32_t kmax = b ? kSmallKmaxB : kSmallKmax;
  if (log_n == 0) return plan;
  if (log_n <= lt) {
    plan.push_back({0, log_n, 0});
    return plan;
  }
  const uint32_t P = (log_n + kmax - 1) / kmax;
  uint32_t S = 0;
  for (uint32_t p = 0; p < P; p++) {
    const uint32_t k = log_n / P + (p < log_n % P ? 1 : 0);
    uint32_t c = lt - k;
    const uint32_t lim = p == 0 ? log_n - k : S;
    if (c > lim) c = lim;
    plan.push_back({S, k, c});
    S += k;
  }
  return plan;
}

// ---- tables ----------------------------------------------------------------------

// A device table.  The leading members match TwEntry's (field, log_n), so the
// 256-bit entry points recognise a small-field handle by its field and refuse it.
struct SmallTable {
  int field = 0;
  uint32_t log_n = 0;
  uint64_t root = 0;          // canonical; the key of root-derived tables
  uint64_t* d_table = nullptr;  // 2^log_n - 1 entries in twiddle form (one when log_n == 0)
  size_t bytes = 0;
  int refs = 0;
  bool tw0_one = true;
  bool foreign = false;
  uint64_t last_use = 0;
};

struct SmallRegistration {
  int field = 0;
  uint32_t log_n = 0;
  std::vector<const uint64_t*> stage_ptrs;
  std::vector<uint64_t> probe;  // entries 0 and 1 of each stage (when present)
  SmallTable* entry = nullptr;
};

struct SmallState {
  std::map<std::string, SmallTable*> by_key;
  std::vector<SmallTable*> all;
  std::vector<SmallRegistration> regs;
  uint64_t clock = 0;
  size_t idle_budget = (size_t)4 << 30;  // idle root-derived tables kept up to this
};

SmallState& small_state() {
  static SmallState s;
  return s;
}

std::string small_key(int field, uint32_t log_n, uint64_t root) {
  return std::to_string(field) + ":" + std::to_string(log_n) + ":" + std::to_string(root);
}

size_t small_entries(uint32_t log_n) { return log_n == 0 ? 1 : ((size_t)1 << log_n) - 1; }

void small_free_entry(SmallTable* e) {
  SmallState& s = small_state();
  if (e->d_table) cudaFree(e->d_table);
  s.all.erase(std::remove(s.all.begin(), s.all.end(), e), s.all.end());
  for (auto it = s.by_key.begin(); it != s.by_key.end(); ++it)
    if (it->second == e) {
      s.by_key.erase(it);
      break;
    }
  delete e;
}

// Frees idle root-derived tables, oldest first, until the idle ones (plus
// `need` bytes about to be allocated) fit the budget.
void small_evict(size_t need) {
  SmallState& s = small_state();
  for (;;) {
    size_t idle = 0;
    SmallTable* oldest = nullptr;
    for (SmallTable* e : s.all)
      if (e->refs == 0) {
        idle += e->bytes;
        if (!oldest || e->last_use < oldest->last_use) oldest = e;
      }
    if (!oldest || idle + need <= s.idle_budget) return;
    small_free_entry(oldest);
  }
}

// A caller's table is freed with its last user; a root-derived one stays
// cached while idle tables fit the budget.
void small_release(SmallTable* e) {
  if (!e) return;
  if (--e->refs <= 0) {
    e->refs = 0;
    if (e->foreign) small_free_entry(e);
    else small_evict(0);
  }
}

int small_acquire(int field, uint32_t log_n, uint64_t root, SmallTable** out) {
  Context& c = ctx();
  SmallState& s = small_state();
  const std::string key = small_key(field, log_n, root);
  auto it = s.by_key.find(key);
  if (it != s.by_key.end()) {
    it->second->refs++;
    it->second->last_use = ++s.clock;
    *out = it->second;
    return ZNTT_OK;
  }
  const SmallHost& H = small_host(field);
  SmallTable* e = new SmallTable();
  e->field = field;
  e->log_n = log_n;
  e->root = root;
  e->bytes = small_entries(log_n) * 8;
  small_evict(e->bytes);
  cudaError_t ce = cudaMalloc((void**)&e->d_table, e->bytes);
  if (ce != cudaSuccess) {
    delete e;
    return cuda_fail(ce, "twiddle table");
  }
  if (log_n > 0) {
    // pw[t][i] = root^(i * 1024^t), computed canonically, stored in twiddle form.
    std::vector<uint64_t> pw(3 * 1024);
    uint64_t step = root;
    for (int t = 0; t < 3; t++) {
      uint64_t cur = 1;
      for (int i = 0; i < 1024; i++) {
        pw[t * 1024 + i] = H.to_tw(cur);
        cur = H.mul(cur, step);
      }
      step = H.pow(step, 1024);
    }
    void* d_pw = nullptr;
    int rc = pool_get(pw.size() * 8, &d_pw);
    if (rc) {
      cudaFree(e->d_table);
      delete e;
      return rc;
    }
    ce = cudaMemcpyAsync(d_pw, pw.data(), pw.size() * 8, cudaMemcpyHostToDevice, c.stream);
    const uint64_t total = small_entries(log_n);
    if (ce == cudaSuccess) {
      if (field == kGoldilocksField)
        small_twiddle_kernel<Goldilocks><<<grid_for(total), 256, 0, c.stream>>>((const uint64_t*)d_pw, e->d_table,
                                                                                 log_n);
      else
        small_twiddle_kernel<BabyBear><<<grid_for(total), 256, 0, c.stream>>>((const uint64_t*)d_pw, e->d_table,
                                                                               log_n);
      ce = cudaGetLastError();
    }
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(c.stream);
    pool_put(d_pw, pw.size() * 8);
    if (ce != cudaSuccess) {
      cudaFree(e->d_table);
      delete e;
      return cuda_fail(ce, "twiddle table");
    }
  }
  e->refs = 1;
  e->last_use = ++s.clock;
  s.all.push_back(e);
  s.by_key[key] = e;
  *out = e;
  return ZNTT_OK;
}

// A caller's canonical host table, converted to twiddle form on the device.
int small_upload_foreign(int field, uint32_t log_n, const zntt_stage* stages, SmallTable** out) {
  Context& c = ctx();
  const SmallHost& H = small_host(field);
  SmallTable* e = new SmallTable();
  e->field = field;
  e->log_n = log_n;
  e->foreign = true;
  e->bytes = small_entries(log_n) * 8;
  cudaError_t ce = cudaMalloc((void**)&e->d_table, e->bytes);
  if (ce != cudaSuccess) {
    delete e;
    return cuda_fail(ce, "foreign twiddle table");
  }
  for (uint32_t s = 0; s < log_n && ce == cudaSuccess; s++) {
    if (stages[s].ptr[0] != 1) e->tw0_one = false;
    ce = cudaMemcpyAsync(e->d_table + (((size_t)1 << s) - 1), stages[s].ptr, ((size_t)1 << s) * 8,
                         cudaMemcpyHostToDevice, c.stream);
  }
  // Canonical -> twiddle form: mul(x, R^2) = x * R.  Entries at or above p are
  // reduced on the way (the reference's Fields are canonical already).
  if (ce == cudaSuccess)
    ce = launch_small_scale(field, e->d_table, e->d_table, small_entries(log_n) - (log_n == 0 ? 1 : 0),
                            H.mul(H.r, H.r), c.stream);
  if (ce != cudaSuccess) {
    cudaStreamSynchronize(c.stream);
    cudaFree(e->d_table);
    delete e;
    return cuda_fail(ce, "foreign twiddle upload");
  }
  e->refs = 1;
  small_state().all.push_back(e);
  *out = e;
  return ZNTT_OK;
}

SmallRegistration* small_find_registration(int field, uint32_t log_n, const zntt_stage* stages) {
  for (SmallRegistration& r : small_state().regs) {
    if (r.field != field || r.log_n != log_n) continue;
    bool same = true;
    for (uint32_t s = 0; s < log_n && same; s++) same = r.stage_ptrs[s] == stages[s].ptr;
    for (uint32_t s = 0; s < log_n && same; s++) {
      const size_t m = std::min<size_t>((size_t)1 << s, 2);
      same = std::memcmp(stages[s].ptr, &r.probe[2 * s], m * 8) == 0;
    }
    if (same) return &r;
  }
  return nullptr;
}

// ---- transforms ----------------------------------------------------------------

// src -> dst over 2^log_n device elements; scratch (2^log_n) is needed when
// src == dst and there are several passes.
// small_run over m columns at once: the first pass reads srcs[y] (zero beyond
// src_len) and writes dsts[y]; the later passes run in place on dsts[y], so no
// scratch is needed.  At least one pass (log_n >= 1).
int small_run_cols(const SmallTable* t, uint32_t m, const uint64_t* const* srcs, uint64_t* const* dsts,
                   uint32_t src_len, bool inverse, bool scale, uint64_t scale_tw, cudaStream_t st) {
  const std::vector<SmallPlanPass> plan = small_plan(t->log_n, t->field);
  for (size_t p = 0; p < plan.size(); p++) {
    SmallPass pp;
    std::memset(&pp, 0, sizeof(pp));
    pp.tw = t->d_table;
    pp.log_n = t->log_n;
    pp.S = plan[p].S;
    pp.k = plan[p].k;
    pp.c = plan[p].c;
    pp.first = p == 0;
    pp.inverse = inverse;
    pp.tw0_one = t->tw0_one;
    pp.scale = p + 1 == plan.size() && scale;
    pp.scale_val = scale_tw;
    pp.src_len = src_len;
    const uint64_t tiles = (1ull << t->log_n) >> (pp.k + pp.c);
    cudaError_t ce = launch_small_pass_cols(t->field, pp, tiles, m, p == 0 ? srcs : dsts, dsts, st);
    if (ce != cudaSuccess) return cuda_fail(ce, "small-field pass");
  }
  return ZNTT_OK;
}

int small_run(const SmallTable* t, const uint64_t* src, uint64_t* dst, uint64_t* scratch, bool inverse, bool scale,
              uint64_t scale_tw, cudaStream_t st) {
  const std::vector<SmallPlanPass> plan = small_plan(t->log_n, t->field);
  if (plan.empty()) {  // one element: a copy (the 1/n scale is by one)
    if (src != dst) {
      cudaError_t ce = cudaMemcpyAsync(dst, src, 8, cudaMemcpyDeviceToDevice, st);
      if (ce != cudaSuccess) return cuda_fail(ce, "copy");
    }
    return ZNTT_OK;
  }
  uint64_t* mid = (src == dst && plan.size() > 1) ? scratch : dst;
  for (size_t p = 0; p < plan.size(); p++) {
    const bool first = p == 0, last = p + 1 == plan.size();
    SmallPass pp;
    std::memset(&pp, 0, sizeof(pp));
    pp.src = first ? src : mid;
    pp.dst = last ? dst : mid;
    pp.tw = t->d_table;
    pp.log_n = t->log_n;
    pp.S = plan[p].S;
    pp.k = plan[p].k;
    pp.c = plan[p].c;
    pp.first = first;
    pp.inverse = inverse;
    pp.tw0_one = t->tw0_one;
    pp.scale = last && scale;
    pp.scale_val = scale_tw;
    const uint64_t tiles = (1ull << t->log_n) >> (pp.k + pp.c);
    cudaError_t ce = launch_small_pass(t->field, pp, tiles, st);
    if (ce != cudaSuccess) return cuda_fail(ce, "small-field pass");
  }
  return ZNTT_OK;
}

int small_transform_host(const SmallTable* t, uint64_t* data, bool inverse, bool scale, uint64_t scale_tw) {
  Context& c = ctx();
  const size_t bytes = ((size_t)8) << t->log_n;
  void* a = nullptr;
  void* b = nullptr;
  int rc = pool_get(bytes, &a);
  if (!rc) rc = pool_get(bytes, &b);
  cudaError_t ce = cudaSuccess;
  if (!rc) {
    ce = cudaMemcpyAsync(a, data, bytes, cudaMemcpyHostToDevice, c.stream);
    if (ce == cudaSuccess) rc = small_run(t, (const uint64_t*)a, (uint64_t*)b, nullptr, inverse, scale, scale_tw, c.stream);
    if (ce == cudaSuccess && !rc) ce = cudaMemcpyAsync(data, b, bytes, cudaMemcpyDeviceToHost, c.stream);
    cudaError_t ce2 = cudaStreamSynchronize(c.stream);
    if (ce == cudaSuccess) ce = ce2;
    if (ce != cudaSuccess && !rc) rc = cuda_fail(ce, "small-field transform");
  }
  if (a) pool_put(a, bytes);
  if (b) pool_put(b, bytes);
  return rc;
}

uint64_t n_inverse_tw(const SmallHost& H, uint32_t log_n) { return H.to_tw(H.inv(((uint64_t)1 << log_n) % H.p)); }

int check_small_shape(size_t len, size_t log_n) {
  if (log_n >= 64) return set_error(ZNTT_ERR_LOG_TOO_LARGE, "log_n >= 64");
  if (len != ((size_t)1 << log_n)) return set_error(ZNTT_ERR_LENGTH_MISMATCH, "data.len != 2^log_n");
  return ZNTT_OK;
}

int check_small_ready(size_t log_n) {
  if (log_n > 31) return set_error(ZNTT_ERR_OUT_OF_MEMORY, "transform larger than 2^31 elements");
  if (ctx().device < 0) return set_error(ZNTT_ERR_NOT_INITIALIZED, "zntt_init has not been called");
  return ZNTT_OK;
}

}  // namespace

bool is_small_field(int field) { return field == kGoldilocksField || field == kBabyBearField; }

bool is_small_table(const void* handle) {
  return handle && is_small_field(*static_cast<const int*>(handle));
}

int small_field_info(int field, uint64_t* modulus, uint32_t* two_adicity) {
  const SmallHost& H = small_host(field);
  if (modulus) {
    modulus[0] = H.p;
    modulus[1] = modulus[2] = modulus[3] = 0;
  }
  if (two_adicity) *two_adicity = H.two_adicity;
  return ZNTT_OK;
}

// roots.zig:22-30, 149-158: z = the first quadratic non-residue from 2, and
// the root of order 2^log_n is z^(odd_part << (two_adicity - log_n)) =
// z^((p - 1) >> log_n).
int small_primitive_root(int field, uint32_t log_n, uint64_t* root_out) {
  const SmallHost& H = small_host(field);
  if (log_n > H.two_adicity) return set_error(ZNTT_ERR_ORDER_TOO_LARGE, "log_n exceeds the two-adicity");
  uint64_t z = 2;
  while (H.pow(z, (H.p - 1) / 2) != H.p - 1) z++;
  root_out[0] = H.pow(z, (H.p - 1) >> log_n);
  root_out[1] = root_out[2] = root_out[3] = 0;
  return ZNTT_OK;
}

int small_bit_reverse(uint64_t* data, size_t len) {
  if (len == 0 || (len & (len - 1)) != 0) return set_error(ZNTT_ERR_INVALID_LENGTH, "length is 0 or not 2^k");
  if (!data) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null data");
  const uint32_t log_n = (uint32_t)__builtin_ctzll(len);
  int rc = check_small_ready(log_n);
  if (rc) return rc;
  if (len == 1) return ZNTT_OK;
  Context& c = ctx();
  std::lock_guard<std::recursive_mutex> lock(c.mu);
  void* a = nullptr;
  void* b = nullptr;
  rc = pool_get(len * 8, &a);
  if (!rc) rc = pool_get(len * 8, &b);
  cudaError_t ce = cudaSuccess;
  if (!rc) {
    ce = cudaMemcpyAsync(a, data, len * 8, cudaMemcpyHostToDevice, c.stream);
    if (ce == cudaSuccess) {
      small_bit_reverse_kernel<<<grid_for(len), 256, 0, c.stream>>>((const uint64_t*)a, (uint64_t*)b, log_n);
      ce = cudaGetLastError();
    }
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(data, b, len * 8, cudaMemcpyDeviceToHost, c.stream);
    cudaError_t ce2 = cudaStreamSynchronize(c.stream);
    if (ce == cudaSuccess) ce = ce2;
    if (ce != cudaSuccess) rc = cuda_fail(ce, "bit reverse");
  }
  if (a) pool_put(a, len * 8);
  if (b) pool_put(b, len * 8);
  return rc;
}

int small_ntt_root(int field, uint64_t* data, size_t len, size_t log_n, const uint64_t* root, bool inverse) {
  int rc = check_small_shape(len, log_n);
  if (rc) return rc;
  if (!data || !root) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null pointer");
  rc = check_small_ready(log_n);
  if (rc) return rc;
  if (log_n == 0) return ZNTT_OK;
  const SmallHost& H = small_host(field);
  Context& c = ctx();
  std::lock_guard<std::recursive_mutex> lock(c.mu);
  // intt(root) is ntt(root.inv()) followed by the 1/n scale (root.zig:100-106).
  const uint64_t r = inverse ? H.inv(root[0] % H.p) : root[0] % H.p;
  SmallTable* t = nullptr;
  rc = small_acquire(field, (uint32_t)log_n, r, &t);
  if (rc) return rc;
  rc = small_transform_host(t, data, false, inverse, n_inverse_tw(H, (uint32_t)log_n));
  small_release(t);
  return rc;
}

int small_precompute(int field, size_t log_n, const uint64_t* root, uint64_t* const* stage_out) {
  if (log_n >= 64) return set_error(ZNTT_ERR_LOG_TOO_LARGE, "log_n >= 64");
  if (log_n > 31) return set_error(ZNTT_ERR_OUT_OF_MEMORY, "transform larger than 2^31 elements");
  if (log_n == 0) return ZNTT_OK;
  if (!root || !stage_out) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null pointer");
  for (size_t s = 0; s < log_n; s++)
    if (!stage_out[s]) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null stage pointer");
  int rc = check_small_ready(log_n);
  if (rc) return rc;
  const SmallHost& H = small_host(field);
  Context& c = ctx();
  std::lock_guard<std::recursive_mutex> lock(c.mu);
  SmallTable* t = nullptr;
  rc = small_acquire(field, (uint32_t)log_n, root[0] % H.p, &t);
  if (rc) return rc;
  // Twiddle form -> canonical (mul by canonical one), then download by stage.
  const size_t entries = small_entries((uint32_t)log_n);
  void* canon = nullptr;
  rc = pool_get(entries * 8, &canon);
  if (rc) {
    small_release(t);
    return rc;
  }
  cudaError_t ce = launch_small_scale(field, t->d_table, (uint64_t*)canon, entries, 1, c.stream);
  for (size_t s = 0; s < log_n && ce == cudaSuccess; s++)
    ce = cudaMemcpyAsync(stage_out[s], (uint64_t*)canon + (((size_t)1 << s) - 1), ((size_t)1 << s) * 8,
                         cudaMemcpyDeviceToHost, c.stream);
  cudaError_t ce2 = cudaStreamSynchronize(c.stream);
  pool_put(canon, entries * 8);
  if (ce == cudaSuccess) ce = ce2;
  if (ce != cudaSuccess) {
    small_release(t);
    return cuda_fail(ce, "twiddle download");
  }
  SmallState& st = small_state();
  for (auto it = st.regs.begin(); it != st.regs.end();) {
    bool same = it->field == field && it->log_n == log_n;
    for (size_t s = 0; s < log_n && same; s++) same = it->stage_ptrs[s] == stage_out[s];
    if (same) {
      small_release(it->entry);
      it = st.regs.erase(it);
    } else {
      ++it;
    }
  }
  SmallRegistration r;
  r.field = field;
  r.log_n = (uint32_t)log_n;
  r.entry = t;
  r.probe.assign(2 * log_n, 0);
  for (size_t s = 0; s < log_n; s++) {
    r.stage_ptrs.push_back(stage_out[s]);
    const size_t m = std::min<size_t>((size_t)1 << s, 2);
    std::memcpy(&r.probe[2 * s], stage_out[s], m * 8);
  }
  st.regs.push_back(std::move(r));
  return ZNTT_OK;
}

void small_free_twiddles(int field, const zntt_stage* stages, size_t num_stages) {
  Context& c = ctx();
  std::lock_guard<std::recursive_mutex> lock(c.mu);
  if (!stages || num_stages == 0) return;
  SmallState& st = small_state();
  for (auto it = st.regs.begin(); it != st.regs.end(); ++it) {
    if (it->field != field || it->log_n != num_stages) continue;
    bool same = true;
    for (size_t s = 0; s < num_stages && same; s++) same = it->stage_ptrs[s] == stages[s].ptr;
    if (same) {
      small_release(it->entry);
      st.regs.erase(it);
      return;
    }
  }
}

int small_ntt_with_twiddles(int field, uint64_t* data, size_t len, size_t log_n, const zntt_stage* stages,
                            size_t num_stages, bool inverse) {
  int rc = check_small_shape(len, log_n);
  if (rc) return rc;
  if (num_stages != log_n) return set_error(ZNTT_ERR_INVALID_TWIDDLES, "twiddles.len != log_n");
  if (num_stages && !stages) return set_error(ZNTT_ERR_INVALID_TWIDDLES, "null twiddle table");
  for (size_t s = 0; s < num_stages; s++)
    if (stages[s].len != ((size_t)1 << s) || !stages[s].ptr)
      return set_error(ZNTT_ERR_INVALID_TWIDDLES, "twiddle stage " + std::to_string(s) + " has the wrong length");
  if (!data) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null data");
  rc = check_small_ready(log_n);
  if (rc) return rc;
  if (log_n == 0) return ZNTT_OK;
  const SmallHost& H = small_host(field);
  Context& c = ctx();
  std::lock_guard<std::recursive_mutex> lock(c.mu);
  SmallTable* t = nullptr;
  bool foreign = false;
  SmallRegistration* reg = small_find_registration(field, (uint32_t)log_n, stages);
  if (reg) {
    t = reg->entry;
  } else {
    rc = small_upload_foreign(field, (uint32_t)log_n, stages, &t);
    if (rc) return rc;
    foreign = true;
  }
  rc = small_transform_host(t, data, inverse, inverse, n_inverse_tw(H, (uint32_t)log_n));
  if (foreign) small_release(t);
  return rc;
}

int small_twiddles_acquire(int field, uint32_t log_n, const uint64_t* root, zntt_twiddles** out) {
  if (!root || !out) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null pointer");
  int rc = check_small_ready(log_n);
  if (rc) return rc;
  Context& c = ctx();
  std::lock_guard<std::recursive_mutex> lock(c.mu);
  SmallTable* t = nullptr;
  rc = small_acquire(field, log_n, root[0] % small_host(field).p, &t);
  if (rc) return rc;
  *out = reinterpret_cast<zntt_twiddles*>(t);
  return ZNTT_OK;
}

int small_twiddles_release(zntt_twiddles* tw) {
  Context& c = ctx();
  std::lock_guard<std::recursive_mutex> lock(c.mu);
  SmallTable* t = reinterpret_cast<SmallTable*>(tw);
  SmallState& s = small_state();
  if (std::find(s.all.begin(), s.all.end(), t) == s.all.end())
    return set_error(ZNTT_ERR_INVALID_ARGUMENT, "unknown twiddle handle");
  small_release(t);
  return ZNTT_OK;
}

int small_ntt_device(const zntt_twiddles* tw, const uint64_t* d_src, uint64_t* d_dst, uint64_t* d_scratch, int mode,
                     void* stream) {
  Context& c = ctx();
  std::lock_guard<std::recursive_mutex> lock(c.mu);
  const SmallTable* t = reinterpret_cast<const SmallTable*>(tw);
  const SmallHost& H = small_host(t->field);
  const bool inverse = mode == ZNTT_INVERSE;
  const uint64_t ninv = n_inverse_tw(H, t->log_n);
  cudaStream_t st = stream ? (cudaStream_t)stream : c.stream;
  const bool need_scratch = d_src == d_dst && small_plan(t->log_n, t->field).size() > 1;
  if (need_scratch && !d_scratch) {
    const size_t bytes = ((size_t)8) << t->log_n;
    void* s = nullptr;
    int rc = pool_get(bytes, &s);
    if (rc) return rc;
    rc = small_run(t, d_src, d_dst, (uint64_t*)s, inverse, inverse, ninv, st);
    cudaError_t ce = cudaStreamSynchronize(st);
    pool_put(s, bytes);
    if (rc) return rc;
    if (ce != cudaSuccess) return cuda_fail(ce, "transform");
    return ZNTT_OK;
  }
  return small_run(t, d_src, d_dst, d_scratch, inverse, inverse, ninv, st);
}

namespace {

std::map<std::pair<int, uint32_t>, uint64_t*>& small_fold_tables() {
  static std::map<std::pair<int, uint32_t>, uint64_t*> t;
  return t;
}

// c * base^i (i < count) on the device: in twiddle form when c is given in
// twiddle form, canonical when c is the plain integer 1.
int small_powers(int field, uint64_t base, uint64_t c, uint64_t* out, uint64_t count, cudaStream_t st) {
  const SmallHost& H = small_host(field);
  std::vector<uint64_t> pw(3 * 1024);
  uint64_t step = base % H.p;
  for (int t = 0; t < 3; t++) {
    uint64_t cur = 1;
    for (int i = 0; i < 1024; i++) {
      pw[t * 1024 + i] = H.to_tw(cur);
      cur = H.mul(cur, step);
    }
    step = H.pow(step, 1024);
  }
  void* d_pw = nullptr;
  int rc = pool_get(pw.size() * 8, &d_pw);
  if (rc) return rc;
  cudaError_t ce = cudaMemcpyAsync(d_pw, pw.data(), pw.size() * 8, cudaMemcpyHostToDevice, st);
  if (ce == cudaSuccess && count) {
    if (field == kGoldilocksField)
      small_powers_kernel<Goldilocks><<<grid_for(count), 256, 0, st>>>((const uint64_t*)d_pw, c, out, count);
    else
      small_powers_kernel<BabyBear><<<grid_for(count), 256, 0, st>>>((const uint64_t*)d_pw, c, out, count);
    ce = cudaGetLastError();
  }
  cudaError_t ce2 = cudaStreamSynchronize(st);  // the power tables return to the pool
  pool_put(d_pw, pw.size() * 8);
  if (ce == cudaSuccess) ce = ce2;
  if (ce != cudaSuccess) return cuda_fail(ce, "powers");
  return ZNTT_OK;
}

}  // namespace

int small_domain_fill(int field, uint32_t log_n, uint64_t* d_out, void* stream) {
  const SmallHost& H = small_host(field);
  if (log_n > H.two_adicity) return set_error(ZNTT_ERR_ORDER_TOO_LARGE, "domain larger than the two-adicity (Domain.init)");
  if (log_n > 30) return set_error(ZNTT_ERR_OUT_OF_MEMORY, "domain larger than 2^30 elements");
  Context& c = ctx();
  if (c.device < 0) return set_error(ZNTT_ERR_NOT_INITIALIZED, "zntt_init has not been called");
  std::lock_guard<std::recursive_mutex> lock(c.mu);
  uint64_t g[4];
  small_primitive_root(field, log_n, g);
  return small_powers(field, g[0], 1, d_out, 1ull << log_n, stream ? (cudaStream_t)stream : c.stream);
}

// The fold's constants for a small field: the resident table g^-j / 2 of the
// subgroup of order 2^log_table (made on first use), 1/2 and alpha, all three
// in twiddle form.
int small_fold_params(int field, uint32_t log_table, const uint64_t* alpha, const uint64_t** tab_out,
                      uint64_t* half_inv_tw, uint64_t* alpha_tw) {
  const SmallHost& H = small_host(field);
  Context& c = ctx();
  std::lock_guard<std::recursive_mutex> lock(c.mu);
  auto& tabs = small_fold_tables();
  const auto key = std::make_pair(field, log_table);
  const uint64_t half_inv = H.inv(2);
  auto it = tabs.find(key);
  if (it != tabs.end()) {
    *tab_out = it->second;
  } else {
    uint64_t g[4];
    small_primitive_root(field, log_table, g);
    const uint64_t count = 1ull << (log_table - 1);
    uint64_t* tab = nullptr;
    cudaError_t ce = cudaMalloc((void**)&tab, count * 8);
    if (ce != cudaSuccess) return cuda_fail(ce, "fold table");
    int rc = small_powers(field, H.inv(g[0]), H.to_tw(half_inv), tab, count, c.stream);
    if (rc) {
      cudaFree(tab);
      return rc;
    }
    tabs[key] = tab;
    *tab_out = tab;
  }
  *half_inv_tw = H.to_tw(half_inv);
  *alpha_tw = H.to_tw(alpha[0] % H.p);
  return ZNTT_OK;
}

int small_fri_fold(int field, const uint64_t* d_layer, uint32_t log_n, const uint64_t* alpha, uint64_t* d_out,
                   uint32_t log_table, void* stream) {
  const SmallHost& H = small_host(field);
  if (log_table == 0) log_table = log_n;
  if (log_n < 1 || log_n > log_table) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "a fold needs 1 <= log_n <= log_table");
  if (log_table > H.two_adicity) return set_error(ZNTT_ERR_ORDER_TOO_LARGE, "domain larger than the two-adicity");
  if (log_table > 31) return set_error(ZNTT_ERR_OUT_OF_MEMORY, "domain larger than 2^31 elements");
  const uint64_t n = 1ull << log_n, half = n / 2;
  const char* lo = reinterpret_cast<const char*>(d_layer);
  const char* oo = reinterpret_cast<const char*>(d_out);
  if (oo < lo + n * 8 && lo < oo + half * 8) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "fold output overlaps the layer");
  Context& c = ctx();
  if (c.device < 0) return set_error(ZNTT_ERR_NOT_INITIALIZED, "zntt_init has not been called");
  std::lock_guard<std::recursive_mutex> lock(c.mu);
  const uint64_t* tab = nullptr;
  uint64_t hv = 0, av = 0;
  int rc = small_fold_params(field, log_table, alpha, &tab, &hv, &av);
  if (rc) return rc;
  cudaStream_t st = stream ? (cudaStream_t)stream : c.stream;
  const uint32_t stride = log_table - log_n;
  if (field == kGoldilocksField)
    small_fri_fold_kernel<Goldilocks><<<grid_for(half), 256, 0, st>>>(d_layer, d_out, tab, half, stride, hv, av);
  else
    small_fri_fold_kernel<BabyBear><<<grid_for(half), 256, 0, st>>>(d_layer, d_out, tab, half, stride, hv, av);
  cudaError_t ce = cudaGetLastError();
  if (ce != cudaSuccess) return cuda_fail(ce, "fri fold");
  return ZNTT_OK;
}

void small_shutdown() {
  for (auto& kv : small_fold_tables())
    if (kv.second) cudaFree(kv.second);
  small_fold_tables().clear();
  SmallState& s = small_state();
  while (!s.all.empty()) small_free_entry(s.all.back());
  s.regs.clear();
}

}  // namespace zntt

extern "C" int zntt_bit_reverse_small(uint64_t* data, size_t len) {
  zntt::clear_error();
  return zntt::small_bit_reverse(data, len);
}

namespace zntt {

// The coset low-degree extension of m columns for a small field, the
// composition the 256-bit path runs in its fused passes, as device steps:
// the inverse transform of each column's 2^log_in evaluations (with 1/n),
// coefficient i times shift^i, and the forward transform of the coefficients
// zero-padded to 2^log_out.  Every launch covers all columns (below); inputs
// of one element, or more columns than a grid's second dimension, take the
// per-column path at the end.
int small_coset_lde_many(const zntt_twiddles* tw_in, const zntt_twiddles* tw_out, const uint64_t* shift,
                         const uint64_t* const* d_evals, uint64_t* const* d_out, uint32_t m, void* stream) {
  const SmallTable* ti = reinterpret_cast<const SmallTable*>(tw_in);
  const SmallTable* to = reinterpret_cast<const SmallTable*>(tw_out);
  if (ti->field != to->field) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "tables of different fields");
  if (ti->log_n > to->log_n) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "coset extension shrinks the vector");
  if (ti->log_n > 30) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "coset extension of more than 2^30 evaluations");
  const SmallHost& H = small_host(ti->field);
  if (shift[1] || shift[2] || shift[3] || shift[0] >= H.p || shift[0] == 0)
    return set_error(ZNTT_ERR_INVALID_ARGUMENT, "the shift must be a nonzero canonical element in word 0");
  const uint64_t n_in = 1ull << ti->log_n, n_out = 1ull << to->log_n;
  for (uint32_t k = 0; k < m; k++) {
    if (!d_evals[k] || !d_out[k]) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null column");
    const char* eo = reinterpret_cast<const char*>(d_evals[k]);
    const char* oo = reinterpret_cast<const char*>(d_out[k]);
    if (oo < eo + n_in * 8 && eo < oo + n_out * 8) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "extension in place");
  }
  Context& c = ctx();
  std::lock_guard<std::recursive_mutex> lock(c.mu);
  cudaStream_t st = stream ? (cudaStream_t)stream : c.stream;
  std::vector<uint64_t> pw(3 * 1024);
  uint64_t step = shift[0];
  for (int t = 0; t < 3; t++) {
    uint64_t cur = 1;
    for (int i = 0; i < 1024; i++) {
      pw[t * 1024 + i] = H.to_tw(cur);
      cur = H.mul(cur, step);
    }
    step = H.pow(step, 1024);
  }
  void* d_pw = nullptr;
  int rc = pool_get(pw.size() * 8, &d_pw);
  if (rc) return rc;
  if (ti->log_n >= 1 && m <= 65535) {
    // All columns per launch: the inverse transforms into a contiguous buffer of
    // m x 2^log_in coefficients, one coset-scaling launch over it, and the
    // forward transforms reading it zero-padded to 2^log_out, with the column
    // picked by blockIdx.y from device pointer tables.
    const size_t tmp_bytes = (size_t)m * n_in * 8, tab_bytes = (size_t)3 * m * 8;
    void* tmp = nullptr;
    void* tabs = nullptr;
    rc = pool_get(tmp_bytes, &tmp);
    if (!rc) rc = pool_get(tab_bytes, &tabs);
    if (rc) {
      if (tmp) pool_put(tmp, tmp_bytes);
      pool_put(d_pw, pw.size() * 8);
      return rc;
    }
    std::vector<const void*> h(3 * (size_t)m);
    for (uint32_t k = 0; k < m; k++) {
      h[k] = d_evals[k];
      h[m + k] = static_cast<uint64_t*>(tmp) + (size_t)k * n_in;
      h[2 * (size_t)m + k] = d_out[k];
    }
    const uint64_t* const* t_src = static_cast<const uint64_t* const*>(tabs);
    uint64_t* const* t_tmp = static_cast<uint64_t* const*>(tabs) + m;
    uint64_t* const* t_out = static_cast<uint64_t* const*>(tabs) + 2 * (size_t)m;
    cudaError_t ce = cudaMemcpyAsync(d_pw, pw.data(), pw.size() * 8, cudaMemcpyHostToDevice, st);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(tabs, h.data(), tab_bytes, cudaMemcpyHostToDevice, st);
    if (ce == cudaSuccess) {
      rc = small_run_cols(ti, m, t_src, t_tmp, (uint32_t)n_in, true, true, n_inverse_tw(H, ti->log_n), st);
      if (rc == ZNTT_OK) {
        if (ti->field == kGoldilocksField)
          small_coset_scale_cols_kernel<Goldilocks><<<grid_for((uint64_t)m * n_in), 256, 0, st>>>(
              (const uint64_t*)d_pw, static_cast<uint64_t*>(tmp), (uint64_t)m * n_in, ti->log_n);
        else
          small_coset_scale_cols_kernel<BabyBear><<<grid_for((uint64_t)m * n_in), 256, 0, st>>>(
              (const uint64_t*)d_pw, static_cast<uint64_t*>(tmp), (uint64_t)m * n_in, ti->log_n);
        ce = cudaGetLastError();
        if (ce == cudaSuccess) rc = small_run_cols(to, m, t_tmp, t_out, (uint32_t)n_in, false, false, 0, st);
      }
    }
    cudaError_t ce2 = cudaStreamSynchronize(st);  // the buffers return to the pool after the stream is done
    pool_put(d_pw, pw.size() * 8);
    pool_put(tmp, tmp_bytes);
    pool_put(tabs, tab_bytes);
    if (rc) return rc;
    if (ce == cudaSuccess) ce = ce2;
    if (ce != cudaSuccess) return cuda_fail(ce, "coset extension");
    return ZNTT_OK;
  }
  void* scratch = nullptr;
  const size_t sbytes = (size_t)8 << to->log_n;
  rc = pool_get(sbytes, &scratch);
  if (rc) {
    pool_put(d_pw, pw.size() * 8);
    return rc;
  }
  // One stream: the columns run one after another and share the power tables and
  // the forward transform's scratch (one-element inputs, or more columns than a
  // launch's second grid dimension holds).
  cudaError_t ce = cudaMemcpyAsync(d_pw, pw.data(), pw.size() * 8, cudaMemcpyHostToDevice, st);
  for (uint32_t k = 0; k < m && ce == cudaSuccess && rc == ZNTT_OK; k++) {
    uint64_t* out = d_out[k];
    rc = small_run(ti, d_evals[k], out, nullptr, true, true, n_inverse_tw(H, ti->log_n), st);  // out of place
    if (rc) break;
    if (ti->field == kGoldilocksField)
      small_coset_scale_kernel<Goldilocks><<<grid_for(n_in), 256, 0, st>>>((const uint64_t*)d_pw, out, n_in);
    else
      small_coset_scale_kernel<BabyBear><<<grid_for(n_in), 256, 0, st>>>((const uint64_t*)d_pw, out, n_in);
    ce = cudaGetLastError();
    if (ce == cudaSuccess && n_out > n_in) ce = cudaMemsetAsync(out + n_in, 0, (n_out - n_in) * 8, st);
    if (ce == cudaSuccess) rc = small_run(to, out, out, (uint64_t*)scratch, false, false, 0, st);
  }
  // The power tables and the scratch return to the pool after the stream is done.
  cudaError_t ce2 = cudaStreamSynchronize(st);
  pool_put(d_pw, pw.size() * 8);
  pool_put(scratch, sbytes);
  if (rc) return rc;
  if (ce == cudaSuccess) ce = ce2;
  if (ce != cudaSuccess) return cuda_fail(ce, "coset extension");
  return ZNTT_OK;
}

int small_coset_lde(const zntt_twiddles* tw_in, const zntt_twiddles* tw_out, const uint64_t* shift,
                    const uint64_t* d_evals, uint64_t* d_out, void* stream) {
  return small_coset_lde_many(tw_in, tw_out, shift, &d_evals, &d_out, 1, stream);
}

}  // namespace zntt

namespace zntt {

// Polynomial(F, max_degree).mul (libs/poly/src/poly.zig:197-212) for a small
// field, host coefficients one canonical u64 each: the same contract as the
// 256-bit path (fromCoeffs' length check, the zero polynomial, DegreeTooLarge,
// zero fill beyond the degree), computed as forward(a), forward(b), their
// pointwise product, and the inverse with 1/n over n = 2^L >= deg a + deg b + 1.
int small_poly_mul(int field, const uint64_t* a, size_t a_len, const uint64_t* b, size_t b_len, size_t max_degree,
                   uint64_t* out, int64_t* out_degree) {
  const SmallHost& H = small_host(field);
  if ((a_len && !a) || (b_len && !b) || !out || !out_degree) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null pointer");
  if (max_degree >= ((size_t)1 << 58)) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "max_degree out of range");
  if (a_len > max_degree + 1 || b_len > max_degree + 1)
    return set_error(ZNTT_ERR_DEGREE_TOO_LARGE, "a factor has more than max_degree + 1 coefficients");
  auto degree_of = [](const uint64_t* c, size_t len) {
    int64_t d = (int64_t)len - 1;
    while (d >= 0 && c[d] == 0) d--;
    return d;
  };
  for (size_t i = 0; i < a_len; i++)
    if (a[i] >= H.p) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "a coefficient is not canonical");
  for (size_t i = 0; i < b_len; i++)
    if (b[i] >= H.p) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "a coefficient is not canonical");
  const int64_t da = degree_of(a, a_len), db = degree_of(b, b_len);
  if (da < 0 || db < 0) {  // a zero factor: the zero polynomial (poly.zig:198)
    std::memset(out, 0, (max_degree + 1) * 8);
    *out_degree = -1;
    return ZNTT_OK;
  }
  const int64_t d = da + db;
  if ((uint64_t)d > max_degree)
    return set_error(ZNTT_ERR_DEGREE_TOO_LARGE, "the product's degree exceeds max_degree (Polynomial.mul)");
  uint32_t L = 0;
  while ((1ull << L) < (uint64_t)d + 1) L++;
  if (L > H.two_adicity) return set_error(ZNTT_ERR_ORDER_TOO_LARGE, "the product needs a transform beyond the two-adicity");
  Context& c = ctx();
  if (c.device < 0) return set_error(ZNTT_ERR_NOT_INITIALIZED, "zntt_init has not been called");
  std::lock_guard<std::recursive_mutex> lock(c.mu);
  uint64_t root[4];
  int rc = small_primitive_root(field, L, root);
  if (rc) return rc;
  zntt_twiddles* tw = nullptr;
  rc = small_twiddles_acquire(field, L, root, &tw);
  if (rc) return rc;
  const SmallTable* t = reinterpret_cast<const SmallTable*>(tw);
  const uint64_t n = 1ull << L;
  const size_t la = (size_t)da + 1, lb = (size_t)db + 1, lo = (size_t)d + 1;
  void* dev[3] = {nullptr, nullptr, nullptr};  // A, B (n each), scratch (n)
  for (int i = 0; i < 3 && !rc; i++) rc = pool_get(n * 8, &dev[i]);
  cudaStream_t st = c.stream;
  uint64_t* A = static_cast<uint64_t*>(dev[0]);
  uint64_t* B = static_cast<uint64_t*>(dev[1]);
  uint64_t* S = static_cast<uint64_t*>(dev[2]);
  cudaError_t ce = cudaSuccess;
  if (!rc) {
    ce = cudaMemcpyAsync(A, a, la * 8, cudaMemcpyHostToDevice, st);
    if (ce == cudaSuccess && n > la) ce = cudaMemsetAsync(A + la, 0, (n - la) * 8, st);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(B, b, lb * 8, cudaMemcpyHostToDevice, st);
    if (ce == cudaSuccess && n > lb) ce = cudaMemsetAsync(B + lb, 0, (n - lb) * 8, st);
    if (ce != cudaSuccess) rc = cuda_fail(ce, "polynomial upload");
  }
  if (!rc) rc = small_run(t, A, A, S, false, false, 0, st);
  if (!rc) rc = small_run(t, B, B, S, false, false, 0, st);
  if (!rc) {
    const uint64_t r2 = H.mul(H.r, H.r);
    if (field == kGoldilocksField)
      small_pointwise_kernel<Goldilocks><<<grid_for(n), 256, 0, st>>>(A, B, A, n, r2);
    else
      small_pointwise_kernel<BabyBear><<<grid_for(n), 256, 0, st>>>(A, B, A, n, r2);
    ce = cudaGetLastError();
    if (ce != cudaSuccess) rc = cuda_fail(ce, "pointwise product");
  }
  if (!rc) rc = small_run(t, A, B, S, true, true, n_inverse_tw(H, L), st);  // coefficients into B
  if (!rc) {
    ce = cudaMemcpyAsync(out, B, lo * 8, cudaMemcpyDeviceToHost, st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess) rc = cuda_fail(ce, "polynomial download");
  }
  if (rc) cudaStreamSynchronize(st);  // no copy or kernel may still use a pooled buffer
  for (int i = 0; i < 3; i++)
    if (dev[i]) pool_put(dev[i], n * 8);
  small_twiddles_release(tw);
  if (rc) return rc;
  std::memset(out + lo, 0, (max_degree + 1 - lo) * 8);
  *out_degree = degree_of(out, lo);
  return ZNTT_OK;
}

}  // namespace zntt

namespace zntt {

// Forward or inverse transforms of m columns of one size, out of place, every
// launch covering all columns (small_pass_cols_kernel).  Synchronous: the
// device pointer tables return to the pool when the stream is done.
int small_ntt_columns(const zntt_twiddles* tw, const uint64_t* const* d_src, uint64_t* const* d_dst, uint32_t m,
                      int mode, void* stream) {
  const SmallTable* t = reinterpret_cast<const SmallTable*>(tw);
  const SmallHost& H = small_host(t->field);
  const uint64_t n = 1ull << t->log_n;
  if (m > 65535) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "at most 65535 columns per call");
  for (uint32_t k = 0; k < m; k++) {
    if (!d_src[k] || !d_dst[k]) return set_error(ZNTT_ERR_INVALID_ARGUMENT, "null column");
    const char* a = reinterpret_cast<const char*>(d_src[k]);
    const char* b = reinterpret_cast<const char*>(d_dst[k]);
    if (a < b + n * 8 && b < a + n * 8)
      return set_error(ZNTT_ERR_INVALID_ARGUMENT, "a column's output overlaps its input (columns run out of place)");
  }
  Context& c = ctx();
  std::lock_guard<std::recursive_mutex> lock(c.mu);
  cudaStream_t st = stream ? (cudaStream_t)stream : c.stream;
  const bool inverse = mode == ZNTT_INVERSE;
  cudaError_t ce = cudaSuccess;
  if (t->log_n == 0) {  // one element per column: a copy (the 1/n scale is by one)
    for (uint32_t k = 0; k < m && ce == cudaSuccess; k++)
      ce = cudaMemcpyAsync(d_dst[k], d_src[k], 8, cudaMemcpyDeviceToDevice, st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess) return cuda_fail(ce, "copy");
    return ZNTT_OK;
  }
  const size_t tab_bytes = (size_t)2 * m * 8;
  void* tabs = nullptr;
  int rc = pool_get(tab_bytes, &tabs);
  if (rc) return rc;
  std::vector<const void*> h(2 * (size_t)m);
  for (uint32_t k = 0; k < m; k++) {
    h[k] = d_src[k];
    h[m + k] = d_dst[k];
  }
  ce = cudaMemcpyAsync(tabs, h.data(), tab_bytes, cudaMemcpyHostToDevice, st);
  if (ce == cudaSuccess)
    rc = small_run_cols(t, m, static_cast<const uint64_t* const*>(tabs), static_cast<uint64_t* const*>(tabs) + m,
                        (uint32_t)n, inverse, inverse, inverse ? n_inverse_tw(H, t->log_n) : 0, st);
  cudaError_t ce2 = cudaStreamSynchronize(st);
  pool_put(tabs, tab_bytes);
  if (rc) return rc;
  if (ce == cudaSuccess) ce = ce2;
  if (ce != cudaSuccess) return cuda_fail(ce, "column transforms");
  return ZNTT_OK;
}

}  // namespace zntt
