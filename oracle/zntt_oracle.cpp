// zntt_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A plain CPU restatement of zig-algebra's NTT hot path, used as the parity
// checker for the CUDA library and as the timed CPU baseline.  It is never
// linked into, loaded by, or called from the product library: only the test
// suite, the smoke check and the CPU-baseline leg of the benchmark load it.
//
// What it restates (paths are relative to the zig-algebra source tree):
//   libs/field/src/montgomery.zig:45-79    constants (R^2, -p^-1 mod 2^64, R mod p)
//   libs/field/src/montgomery.zig:197-245  add / sub / neg (conditional reduction)
//   libs/field/src/montgomery.zig:252-297  CIOS Montgomery multiplication
//   libs/field/src/montgomery.zig:328-405  halveMod, binary-GCD inverse, to/from Montgomery
//   libs/field/src/field.zig:870-878       two-adicity and odd part
//   libs/field/src/field.zig:911-921       fromInt
//   libs/field/src/field.zig:1265-1287     constant-time pow over BITS exponent bits
//   libs/field/src/roots.zig:22-30,149-171 Legendre symbol, QNR search, primitive root
//   libs/ntt/src/root.zig:33-212           sizeFromLog, bitReverse, ntt, intt,
//                                          precomputeTwiddles, nttWithTwiddles,
//                                          inttWithTwiddles (same error order,
//                                          same partial mutation on a bad stage)
//   libs/rng/src/chacha20.zig:36-160       ChaCha20 block function and keystream
//   libs/rng/src/rng.zig:32-65             randomFieldElement (big-endian rejection draw)
//   libs/poly/src/vector.zig:24-32,68-73   powers / hadamard (coset LDE composition)
//   libs/poly/src/poly.zig:76-107,197-224  fromCoeffs / normalize / mul (schoolbook) / eval
//   libs/fri/src/root.zig:133-166,396-403  Domain.init / at / fill and the proveOn fold round
//   libs/fri/src/root.zig:286-295, libs/merkle/src/merkle_tree.zig:146-180
//                                          hashPair and MerkleTree.initFromHashes (the layer
//                                          commitment), over BLAKE3 restated from its
//                                          published specification (single-chunk messages)
//   libs/parallel/src/root.zig:45-79       parallelFor fork-join semantics (harness only)
//
// The reference is Zig 0.16 and cannot be compiled in this environment; the
// restatement is pinned by the reference's own known-answer tests (the DFT
// vectors of libs/ntt/src/root.zig:438-449 over Goldilocks and BabyBear, run
// through the same generic code), the RFC 8439 vectors of
// libs/rng/src/root.zig:182-228, and an independent big-integer DFT.
//
// Every element crosses this C ABI as 4 little-endian u64 limbs; fields with a
// single limb use limb 0 and leave the rest zero.

#include <cstdint>
#include <cstring>
#include <cstdlib>
#include <vector>
#include <thread>
#include <algorithm>

typedef unsigned __int128 u128;

enum {
  ZO_OK = 0,
  ZO_LOG_TOO_LARGE = 1,
  ZO_LENGTH_MISMATCH = 2,
  ZO_INVALID_TWIDDLES = 3,
  ZO_INVALID_LENGTH = 4,
  ZO_OUT_OF_MEMORY = 5,
  ZO_ORDER_TOO_LARGE = 6,
  ZO_UNSUPPORTED_FIELD = 7,
  ZO_REJECTION_FAILED = 8,
  ZO_INVERSE_OF_ZERO = 9,
  ZO_DEGREE_TOO_LARGE = 13,  // libs/poly/src/poly.zig:77, 200 (same number as the product's code)
};

enum {
  ZO_BN254_FR = 0,
  ZO_BLS12_381_FR = 1,
  ZO_GOLDILOCKS = 2,
  ZO_BABYBEAR = 3,
  ZO_BN254_FP = 4,
};

// ---------------------------------------------------------------------------
// Montgomery arithmetic over N u64 limbs (montgomery.zig)
// ---------------------------------------------------------------------------

template <int N>
struct Elem {
  uint64_t l[N];
};

template <int N>
struct Mont {
  uint64_t P[N];
  uint64_t R2[N];
  uint64_t ONE[N];        // R mod p
  uint64_t HALF[N];       // (p + 1) / 2
  uint64_t M0INV;         // -p^-1 mod 2^64
  int BITS;
  int NUM_BYTES;
  int two_adicity;
  uint64_t odd_part[N];   // (p - 1) >> two_adicity

  static bool lt(const uint64_t* a, const uint64_t* b) {
    // montgomery.zig:143-150 -- borrow chain of a - b
    uint64_t borrow = 0;
    for (int i = 0; i < N; i++) {
      u128 z = (u128)a[i] - (u128)b[i] - (u128)borrow;
      borrow = (uint64_t)(z >> 64) != 0 ? 1 : 0;
    }
    return borrow != 0;
  }
  static bool is_zero(const uint64_t* a) {
    uint64_t acc = 0;
    for (int i = 0; i < N; i++) acc |= a[i];
    return acc == 0;
  }
  static void select(bool on, const uint64_t* a, const uint64_t* b, uint64_t* out) {
    uint64_t mask = (uint64_t)0 - (uint64_t)on;
    for (int i = 0; i < N; i++) out[i] = b[i] ^ (mask & (b[i] ^ a[i]));
  }
  static void shr1(uint64_t* a) {
    uint64_t carry = 0;
    for (int i = N - 1; i >= 0; i--) {
      uint64_t low = a[i] << 63;
      a[i] = (a[i] >> 1) | carry;
      carry = low;
    }
  }

  // montgomery.zig:197-217
  void add(const uint64_t* a, const uint64_t* b, uint64_t* r) const {
    uint64_t out[N];
    uint64_t carry = 0;
    for (int i = 0; i < N; i++) {
      u128 z = (u128)a[i] + b[i] + carry;
      out[i] = (uint64_t)z;
      carry = (uint64_t)(z >> 64);
    }
    bool out_lt_mod = lt(out, P);
    bool need_sub = (carry != 0) == out_lt_mod;
    uint64_t red[N];
    uint64_t borrow = 0;
    for (int i = 0; i < N; i++) {
      u128 z = (u128)out[i] - (u128)P[i] - (u128)borrow;
      red[i] = (uint64_t)z;
      borrow = (uint64_t)(z >> 64) != 0 ? 1 : 0;
    }
    select(need_sub, red, out, r);
  }

  // montgomery.zig:220-240
  void sub(const uint64_t* a, const uint64_t* b, uint64_t* r) const {
    uint64_t out[N];
    uint64_t borrow = 0;
    for (int i = 0; i < N; i++) {
      uint64_t ai = a[i], bi = b[i];
      uint64_t diff = ai - bi;
      uint64_t b1 = ai < bi ? 1 : 0;
      uint64_t b2 = diff < borrow ? 1 : 0;
      out[i] = diff - borrow;
      borrow = b1 | b2;
    }
    uint64_t red[N];
    uint64_t carry = 0;
    for (int i = 0; i < N; i++) {
      u128 z = (u128)out[i] + (u128)P[i] + carry;
      red[i] = (uint64_t)z;
      carry = (uint64_t)(z >> 64);
    }
    select(borrow != 0, red, out, r);
  }

  // montgomery.zig:243-245
  void neg(const uint64_t* a, uint64_t* r) const {
    uint64_t zero[N] = {0};
    sub(zero, a, r);
  }

  // montgomery.zig:252-297 -- CIOS with per-iteration shift
  void mul(const uint64_t* a, const uint64_t* b, uint64_t* r) const {
    uint64_t t[N + 2];
    for (int i = 0; i < N + 2; i++) t[i] = 0;
    for (int i = 0; i < N; i++) {
      uint64_t carry = 0;
      for (int j = 0; j < N; j++) {
        u128 z = (u128)t[j] + (u128)a[i] * (u128)b[j] + carry;
        t[j] = (uint64_t)z;
        carry = (uint64_t)(z >> 64);
      }
      u128 zc = (u128)t[N] + carry;
      t[N] = (uint64_t)zc;
      t[N + 1] = (uint64_t)(zc >> 64);

      uint64_t m = t[0] * M0INV;
      uint64_t c = 0;
      for (int j = 0; j < N; j++) {
        u128 z = (u128)t[j] + (u128)m * (u128)P[j] + c;
        t[j] = (uint64_t)z;
        c = (uint64_t)(z >> 64);
      }
      u128 zc2 = (u128)t[N] + c;
      t[N] = (uint64_t)zc2;
      t[N + 1] += (uint64_t)(zc2 >> 64);
      for (int j = 0; j < N + 1; j++) t[j] = t[j + 1];
      t[N + 1] = 0;
    }
    uint64_t out[N];
    for (int i = 0; i < N; i++) out[i] = t[i];
    uint64_t extra = t[N];
    bool need_sub = (extra != 0) | (!lt(out, P));
    uint64_t red[N];
    uint64_t borrow = 0;
    for (int i = 0; i < N; i++) {
      u128 z = (u128)out[i] - (u128)P[i] - (u128)borrow;
      red[i] = (uint64_t)z;
      borrow = (uint64_t)(z >> 64) != 0 ? 1 : 0;
    }
    select(need_sub, red, out, r);
  }

  void to_mont(const uint64_t* x, uint64_t* r) const { mul(x, R2, r); }
  void from_mont(const uint64_t* x, uint64_t* r) const {
    uint64_t one[N] = {0};
    one[0] = 1;
    mul(x, one, r);
  }

  // montgomery.zig:328-332 -- x/2 mod p by halving first
  void halve_mod(uint64_t* x) const {
    uint64_t odd = x[0] & 1;
    shr1(x);
    if (odd == 1) {
      uint64_t t[N];
      add(x, HALF, t);
      std::memcpy(x, t, sizeof(t));
    }
  }

  // montgomery.zig:347-375 -- binary extended GCD, canonical in/out
  bool binary_gcd_inverse(const uint64_t* a, uint64_t* out) const {
    if (is_zero(a)) return false;
    uint64_t u[N], v[N], x1[N], x2[N], tmp[N];
    std::memcpy(u, a, sizeof(u));
    std::memcpy(v, P, sizeof(v));
    for (int i = 0; i < N; i++) { x1[i] = 0; x2[i] = 0; }
    x1[0] = 1;
    while (!is_zero(v)) {
      if ((u[0] & 1) == 0) {
        shr1(u);
        halve_mod(x1);
      } else if ((v[0] & 1) == 0) {
        shr1(v);
        halve_mod(x2);
      } else if (lt(v, u)) {
        sub(u, v, tmp); std::memcpy(u, tmp, sizeof(u));
        shr1(u);
        sub(x1, x2, tmp); std::memcpy(x1, tmp, sizeof(x1));
        halve_mod(x1);
      } else {
        sub(v, u, tmp); std::memcpy(v, tmp, sizeof(v));
        shr1(v);
        sub(x2, x1, tmp); std::memcpy(x2, tmp, sizeof(x2));
        halve_mod(x2);
      }
    }
    std::memcpy(out, x1, sizeof(x1));
    return true;
  }

  // field.zig:1144-1152 (inv is total: inv(0) == 0) and montgomery.zig:386-395
  void inv(const uint64_t* x, uint64_t* r) const {
    uint64_t a[N], ia[N];
    from_mont(x, a);
    if (!binary_gcd_inverse(a, ia)) {
      for (int i = 0; i < N; i++) r[i] = 0;
      return;
    }
    to_mont(ia, r);
  }

  // field.zig:1265-1287 -- constant-time square-and-multiply over BITS bits.
  // The exponent is given as 8 little-endian u64 limbs (u512).
  void pow(const uint64_t* base_in, const uint64_t* exp8, uint64_t* r) const {
    uint64_t result[N], base[N], m[N], sq[N];
    std::memcpy(result, ONE, sizeof(result));
    std::memcpy(base, base_in, sizeof(base));
    for (int i = 0; i < BITS; i++) {
      bool bit = ((exp8[i / 64] >> (i % 64)) & 1) == 1;
      mul(result, base, m);
      select(bit, m, result, result);
      mul(base, base, sq);
      std::memcpy(base, sq, sizeof(base));
    }
    std::memcpy(r, result, sizeof(result));
  }
  void pow_u64(const uint64_t* base, uint64_t e, uint64_t* r) const {
    uint64_t exp8[8] = {e, 0, 0, 0, 0, 0, 0, 0};
    pow(base, exp8, r);
  }

  // field.zig:911-921 -- fromInt(x) = toMontgomery(x mod p); here x < 2^64
  void from_u64(uint64_t x, uint64_t* r) const {
    uint64_t v[N] = {0};
    v[0] = x;
    // reduce x mod p (only matters when p < 2^64)
    if (N == 1) v[0] = x % P[0];
    to_mont(v, r);
  }

  bool eq(const uint64_t* a, const uint64_t* b) const {
    for (int i = 0; i < N; i++)
      if (a[i] != b[i]) return false;
    return true;
  }

  // roots.zig:22-30 -- Euler's criterion: a^((p-1)/2)
  int legendre(const uint64_t* a) const {
    uint64_t half_exp[8] = {0};
    // odd_part << (two_adicity - 1)
    int sh = two_adicity - 1;
    for (int i = 0; i < N; i++) half_exp[i] = odd_part[i];
    for (int k = 0; k < sh; k++) {
      uint64_t carry = 0;
      for (int i = 0; i < 8; i++) {
        uint64_t nc = half_exp[i] >> 63;
        half_exp[i] = (half_exp[i] << 1) | carry;
        carry = nc;
      }
    }
    uint64_t rr[N];
    pow(a, half_exp, rr);
    uint64_t zero[N] = {0};
    if (eq(rr, zero)) return 0;
    if (eq(rr, ONE)) return 1;
    return -1;
  }

  // roots.zig:149-158 -- first QNR counting up from 2, raised to odd_part << shift
  int primitive_root(size_t log_size, uint64_t* r) const {
    if ((long)log_size > two_adicity) return ZO_ORDER_TOO_LARGE;
    uint64_t z[N], one[N], t[N];
    from_u64(2, z);
    std::memcpy(one, ONE, sizeof(one));
    while (legendre(z) != -1) {
      add(z, one, t);
      std::memcpy(z, t, sizeof(z));
    }
    uint64_t exp8[8] = {0};
    for (int i = 0; i < N; i++) exp8[i] = odd_part[i];
    int sh = two_adicity - (int)log_size;
    for (int k = 0; k < sh; k++) {
      uint64_t carry = 0;
      for (int i = 0; i < 8; i++) {
        uint64_t nc = exp8[i] >> 63;
        exp8[i] = (exp8[i] << 1) | carry;
        carry = nc;
      }
    }
    pow(z, exp8, r);
    return ZO_OK;
  }

  int qnr(uint64_t* r) const {
    uint64_t z[N], one[N], t[N];
    from_u64(2, z);
    std::memcpy(one, ONE, sizeof(one));
    while (legendre(z) != -1) {
      add(z, one, t);
      std::memcpy(z, t, sizeof(z));
    }
    std::memcpy(r, z, sizeof(z));
    return ZO_OK;
  }
};

// Build the constants of montgomery.zig:45-79 from the canonical modulus.
template <int N>
static Mont<N> make_mont(const uint64_t* p) {
  Mont<N> F;
  std::memset(&F, 0, sizeof(F));
  for (int i = 0; i < N; i++) F.P[i] = p[i];
  // bit length
  int bits = 0;
  for (int i = N - 1; i >= 0; i--) {
    if (p[i]) { bits = 64 * i + (64 - __builtin_clzll(p[i])); break; }
  }
  F.BITS = bits;
  F.NUM_BYTES = (bits + 7) / 8;
  // M0INV by Newton iteration (montgomery.zig:55-60)
  uint64_t p0 = p[0];
  uint64_t inv = 1;
  for (int k = 0; k < 6; k++) inv = inv * (2 - p0 * inv);
  F.M0INV = (uint64_t)0 - inv;
  // R mod p and R^2 mod p by modular doubling of 1 (each step x -> 2x mod p)
  uint64_t x[N] = {0};
  x[0] = 1;
  if (N == 1) x[0] = 1 % p[0];
  for (int k = 0; k < 64 * N; k++) { uint64_t t[N]; F.add(x, x, t); std::memcpy(x, t, sizeof(x)); }
  std::memcpy(F.ONE, x, sizeof(x));
  for (int k = 0; k < 64 * N; k++) { uint64_t t[N]; F.add(x, x, t); std::memcpy(x, t, sizeof(x)); }
  std::memcpy(F.R2, x, sizeof(x));
  // (p + 1) / 2
  {
    uint64_t h[N];
    std::memcpy(h, p, sizeof(h));
    Mont<N>::shr1(h);  // floor(p/2); p odd -> (p-1)/2
    // + 1
    for (int i = 0; i < N; i++) { h[i] += 1; if (h[i] != 0) break; }
    std::memcpy(F.HALF, h, sizeof(h));
  }
  // two-adicity and odd part of p - 1 (field.zig:870-878)
  uint64_t q[N];
  std::memcpy(q, p, sizeof(q));
  q[0] -= 1;  // p odd, no borrow
  int s = 0;
  while ((q[0] & 1) == 0) { Mont<N>::shr1(q); s++; }
  F.two_adicity = s;
  std::memcpy(F.odd_part, q, sizeof(q));
  return F;
}

static const uint64_t P_BN254_FR[4] = {0x43E1F593F0000001ULL, 0x2833E84879B97091ULL,
                                       0xB85045B68181585DULL, 0x30644E72E131A029ULL};
static const uint64_t P_BLS_FR[4] = {0xFFFFFFFF00000001ULL, 0x53BDA402FFFE5BFEULL,
                                     0x3339D80809A1D805ULL, 0x73EDA753299D7D48ULL};
static const uint64_t P_BN254_FP[4] = {0x3C208C16D87CFD47ULL, 0x97816A916871CA8DULL,
                                       0xB85045B68181585DULL, 0x30644E72E131A029ULL};
static const uint64_t P_GOLDILOCKS[1] = {0xFFFFFFFF00000001ULL};
static const uint64_t P_BABYBEAR[1] = {0x78000001ULL};

static const Mont<4>& bn254_fr() { static Mont<4> f = make_mont<4>(P_BN254_FR); return f; }
static const Mont<4>& bls_fr() { static Mont<4> f = make_mont<4>(P_BLS_FR); return f; }
static const Mont<4>& bn254_fp() { static Mont<4> f = make_mont<4>(P_BN254_FP); return f; }
static const Mont<1>& goldilocks() { static Mont<1> f = make_mont<1>(P_GOLDILOCKS); return f; }
static const Mont<1>& babybear() { static Mont<1> f = make_mont<1>(P_BABYBEAR); return f; }

// ---------------------------------------------------------------------------
// Element marshalling: the ABI always uses 4-u64 slots.
// ---------------------------------------------------------------------------

template <int N>
static void load(const uint64_t* slot, uint64_t* e) {
  for (int i = 0; i < N; i++) e[i] = slot[i];
}
template <int N>
static void store(uint64_t* slot, const uint64_t* e) {
  for (int i = 0; i < 4; i++) slot[i] = i < N ? e[i] : 0;
}

// ---------------------------------------------------------------------------
// zig-ntt restatement (libs/ntt/src/root.zig:33-212), generic over the field.
// Data is held as a vector of N-limb elements.
// ---------------------------------------------------------------------------

template <int N>
using Vec = std::vector<Elem<N>>;

// root.zig:33-36
static int size_from_log(size_t log_n, size_t* n) {
  if (log_n >= 64) return ZO_LOG_TOO_LARGE;
  *n = (size_t)1 << log_n;
  return ZO_OK;
}

// root.zig:38-58
template <int N>
static int bit_reverse(Elem<N>* data, size_t n) {
  if (n == 0 || (n & (n - 1)) != 0) return ZO_INVALID_LENGTH;
  int log_n = __builtin_ctzll(n);
  for (size_t i = 0; i < n; i++) {
    size_t j = 0;
    for (int k = 0; k < log_n; k++) j = (j << 1) | ((i >> k) & 1);
    if (j > i) std::swap(data[i], data[j]);
  }
  return ZO_OK;
}

// root.zig:65-90
template <int N>
static int ntt(const Mont<N>& F, Elem<N>* data, size_t len, size_t log_n, const uint64_t* root) {
  size_t n;
  int st = size_from_log(log_n, &n);
  if (st) return st;
  if (len != n) return ZO_LENGTH_MISMATCH;
  st = bit_reverse<N>(data, len);
  if (st) return st;
  for (size_t s = 1; s <= log_n; s++) {
    size_t m = (size_t)1 << s;
    size_t half_m = m >> 1;
    uint64_t wm[N];
    F.pow_u64(root, (uint64_t)1 << (log_n - s), wm);
    for (size_t k = 0; k < n; k += m) {
      uint64_t w[N];
      std::memcpy(w, F.ONE, sizeof(w));
      for (size_t j = 0; j < half_m; j++) {
        uint64_t t[N], u[N], w2[N];
        F.mul(w, data[k + j + half_m].l, t);
        std::memcpy(u, data[k + j].l, sizeof(u));
        F.add(u, t, data[k + j].l);
        F.sub(u, t, data[k + j + half_m].l);
        F.mul(w, wm, w2);
        std::memcpy(w, w2, sizeof(w));
      }
    }
  }
  return ZO_OK;
}

// root.zig:95-107
template <int N>
static int intt(const Mont<N>& F, Elem<N>* data, size_t len, size_t log_n, const uint64_t* root) {
  size_t n;
  int st = size_from_log(log_n, &n);
  if (st) return st;
  if (len != n) return ZO_LENGTH_MISMATCH;
  uint64_t root_inv[N];
  F.inv(root, root_inv);
  st = ntt<N>(F, data, len, log_n, root_inv);
  if (st) return st;
  uint64_t nf[N], n_inv[N];
  F.from_u64((uint64_t)n, nf);
  F.inv(nf, n_inv);
  for (size_t i = 0; i < n; i++) {
    uint64_t t[N];
    F.mul(data[i].l, n_inv, t);
    std::memcpy(data[i].l, t, sizeof(t));
  }
  return ZO_OK;
}

// root.zig:112-134 -- stage s stored at offset 2^s - 1 of one flat array
template <int N>
static int precompute_twiddles(const Mont<N>& F, size_t log_n, const uint64_t* root, Elem<N>* flat) {
  size_t n;
  int st = size_from_log(log_n, &n);
  if (st) return st;
  for (size_t s = 0; s < log_n; s++) {
    size_t half_m = (size_t)1 << s;
    Elem<N>* stage = flat + (half_m - 1);
    uint64_t wm[N], w[N];
    F.pow_u64(root, (uint64_t)1 << (log_n - s - 1), wm);
    std::memcpy(w, F.ONE, sizeof(w));
    for (size_t j = 0; j < half_m; j++) {
      std::memcpy(stage[j].l, w, sizeof(w));
      uint64_t w2[N];
      F.mul(w, wm, w2);
      std::memcpy(w, w2, sizeof(w));
    }
  }
  return ZO_OK;
}

// Fork-join over [0, count): libs/parallel/src/root.zig:45-79 semantics --
// at most `workers` threads (capped at 64), contiguous chunks, spawn and join
// per call, inline when there is one worker.  A harness construction: zig-ntt
// itself is single-threaded.
template <class Fn>
static void parallel_for(size_t count, int workers, Fn fn) {
  if (workers > 64) workers = 64;
  if (workers <= 1 || count < 2) {
    fn((size_t)0, count);
    return;
  }
  size_t nw = std::min((size_t)workers, count);
  size_t chunk = (count + nw - 1) / nw;
  std::vector<std::thread> th;
  th.reserve(nw);
  for (size_t w = 0; w < nw; w++) {
    size_t lo = w * chunk, hi = std::min(count, lo + chunk);
    if (lo >= hi) break;
    th.emplace_back([=]() { fn(lo, hi); });
  }
  for (auto& t : th) t.join();
}

// root.zig:148-212.  `stages[s]` points at 4-u64 slots; `lens[s]` its length.
// `workers` > 1 selects the fork-join harness over butterfly groups within a
// stage (same butterflies, same order per element, so the same result).
template <int N>
static int ntt_with_twiddles(const Mont<N>& F, Elem<N>* data, size_t len, size_t log_n,
                             const uint64_t* const* stages, const size_t* lens, size_t num_stages,
                             bool inverse, int workers) {
  size_t n;
  int st = size_from_log(log_n, &n);
  if (st) return st;
  if (len != n) return ZO_LENGTH_MISMATCH;
  if (num_stages != log_n) return ZO_INVALID_TWIDDLES;

  if (workers <= 1) {
    st = bit_reverse<N>(data, len);
    if (st) return st;
  } else {
    if (n == 0 || (n & (n - 1)) != 0) return ZO_INVALID_LENGTH;
    int lg = __builtin_ctzll(n);
    parallel_for(n, workers, [&](size_t lo, size_t hi) {
      for (size_t i = lo; i < hi; i++) {
        size_t j = 0;
        for (int k = 0; k < lg; k++) j = (j << 1) | ((i >> k) & 1);
        if (j > i) std::swap(data[i], data[j]);
      }
    });
  }

  for (size_t s = 1; s <= log_n; s++) {
    size_t m = (size_t)1 << s;
    size_t half_m = m >> 1;
    const uint64_t* stw = stages[s - 1];
    if (lens[s - 1] != half_m) return ZO_INVALID_TWIDDLES;  // after earlier stages mutated data
    // Load this stage's twiddles (forward: tw[j]; inverse: 1 or -tw[half_m - j]).
    std::vector<Elem<N>> w(half_m);
    for (size_t j = 0; j < half_m; j++) {
      if (!inverse) {
        load<N>(stw + 4 * j, w[j].l);
      } else if (j == 0) {
        std::memcpy(w[j].l, F.ONE, sizeof(w[j].l));
      } else {
        uint64_t t[N];
        load<N>(stw + 4 * (half_m - j), t);
        F.neg(t, w[j].l);
      }
    }
    auto body = [&](size_t lo, size_t hi) {
      // butterflies b in [lo, hi): block k = b / half_m, j = b % half_m
      for (size_t b = lo; b < hi; b++) {
        size_t k = (b / half_m) * m, j = b % half_m;
        uint64_t t[N], u[N];
        F.mul(w[j].l, data[k + j + half_m].l, t);
        std::memcpy(u, data[k + j].l, sizeof(u));
        F.add(u, t, data[k + j].l);
        F.sub(u, t, data[k + j + half_m].l);
      }
    };
    parallel_for(n / 2, workers, body);
  }

  if (inverse) {
    uint64_t nf[N], n_inv[N];
    F.from_u64((uint64_t)n, nf);
    F.inv(nf, n_inv);
    parallel_for(n, workers, [&](size_t lo, size_t hi) {
      for (size_t i = lo; i < hi; i++) {
        uint64_t t[N];
        F.mul(data[i].l, n_inv, t);
        std::memcpy(data[i].l, t, sizeof(t));
      }
    });
  }
  return ZO_OK;
}

// ---------------------------------------------------------------------------
// ChaCha20 keystream (libs/rng/src/chacha20.zig) and randomFieldElement
// (libs/rng/src/rng.zig:32-65)
// ---------------------------------------------------------------------------

static inline uint32_t rotl32(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }

static void chacha_quarter(uint32_t* x, int a, int b, int c, int d) {
  x[a] += x[b]; x[d] = rotl32(x[d] ^ x[a], 16);
  x[c] += x[d]; x[b] = rotl32(x[b] ^ x[c], 12);
  x[a] += x[b]; x[d] = rotl32(x[d] ^ x[a], 8);
  x[c] += x[d]; x[b] = rotl32(x[b] ^ x[c], 7);
}

static void chacha_block(const uint32_t* state, uint8_t* out) {
  uint32_t x[16];
  std::memcpy(x, state, sizeof(x));
  for (int i = 0; i < 10; i++) {
    chacha_quarter(x, 0, 4, 8, 12);
    chacha_quarter(x, 1, 5, 9, 13);
    chacha_quarter(x, 2, 6, 10, 14);
    chacha_quarter(x, 3, 7, 11, 15);
    chacha_quarter(x, 0, 5, 10, 15);
    chacha_quarter(x, 1, 6, 11, 12);
    chacha_quarter(x, 2, 7, 8, 13);
    chacha_quarter(x, 3, 4, 9, 14);
  }
  for (int j = 0; j < 16; j++) {
    uint32_t v = x[j] + state[j];
    out[4 * j + 0] = (uint8_t)v;
    out[4 * j + 1] = (uint8_t)(v >> 8);
    out[4 * j + 2] = (uint8_t)(v >> 16);
    out[4 * j + 3] = (uint8_t)(v >> 24);
  }
}

struct ChaCha {
  uint32_t state[16];
  uint8_t buffer[64];
  int available;
  bool exhausted;

  void init(const uint8_t* seed32, const uint8_t* nonce12) {
    state[0] = 0x61707865; state[1] = 0x3320646e; state[2] = 0x79622d32; state[3] = 0x6b206574;
    for (int i = 0; i < 8; i++)
      state[4 + i] = (uint32_t)seed32[4 * i] | ((uint32_t)seed32[4 * i + 1] << 8) |
                     ((uint32_t)seed32[4 * i + 2] << 16) | ((uint32_t)seed32[4 * i + 3] << 24);
    state[12] = 0;
    for (int i = 0; i < 3; i++)
      state[13 + i] = (uint32_t)nonce12[4 * i] | ((uint32_t)nonce12[4 * i + 1] << 8) |
                      ((uint32_t)nonce12[4 * i + 2] << 16) | ((uint32_t)nonce12[4 * i + 3] << 24);
    available = 0;
    exhausted = false;
  }
  bool refill() {
    if (exhausted) return false;
    chacha_block(state, buffer);
    available = 64;
    if (state[12] == 0xffffffffu) exhausted = true; else state[12] += 1;
    return true;
  }
  bool bytes(uint8_t* out, size_t len) {
    while (len > 0) {
      if (available == 0 && !refill()) return false;
      size_t take = std::min((size_t)available, len);
      size_t start = 64 - available;
      std::memcpy(out, buffer + start, take);
      out += take;
      len -= take;
      available -= (int)take;
    }
    return true;
  }
};

// rng.zig:32-65: NUM_BYTES bytes, assembled big-endian, rejected if >= p,
// at most 1024 attempts, then fromInt (into Montgomery form).
template <int N>
static int random_field_element(const Mont<N>& F, ChaCha& rng, uint64_t* out) {
  int nb = F.NUM_BYTES;
  uint8_t buf[64];
  for (int attempt = 0; attempt < 1024; attempt++) {
    if (!rng.bytes(buf, nb)) return ZO_REJECTION_FAILED;
    uint64_t v[8] = {0};
    for (int i = 0; i < nb; i++) {
      // v = (v << 8) | buf[i]
      uint64_t carry = buf[i];
      for (int k = 0; k < 8; k++) {
        uint64_t nc = v[k] >> 56;
        v[k] = (v[k] << 8) | carry;
        carry = nc;
      }
    }
    bool high_zero = true;
    for (int k = N; k < 8; k++) if (v[k]) high_zero = false;
    if (high_zero && Mont<N>::lt(v, F.P)) {
      F.to_mont(v, out);
      return ZO_OK;
    }
  }
  return ZO_REJECTION_FAILED;
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

template <class Body>
static int dispatch(int field, Body body) {
  switch (field) {
    case ZO_BN254_FR: return body(bn254_fr());
    case ZO_BLS12_381_FR: return body(bls_fr());
    case ZO_BN254_FP: return body(bn254_fp());
    case ZO_GOLDILOCKS: return body(goldilocks());
    case ZO_BABYBEAR: return body(babybear());
    default: return ZO_UNSUPPORTED_FIELD;
  }
}

template <int N>
static Vec<N> unpack(const uint64_t* slots, size_t n) {
  Vec<N> v(n);
  for (size_t i = 0; i < n; i++) load<N>(slots + 4 * i, v[i].l);
  return v;
}
template <int N>
static void pack(uint64_t* slots, const Vec<N>& v) {
  for (size_t i = 0; i < v.size(); i++) store<N>(slots + 4 * i, v[i].l);
}

extern "C" {

int zo_field_info(int field, uint64_t* modulus4, int* nlimbs, int* bits, int* two_adicity) {
  return dispatch(field, [&](const auto& F) -> int {
    constexpr int N = sizeof(F.P) / sizeof(uint64_t);
    for (int i = 0; i < 4; i++) modulus4[i] = i < N ? F.P[i] : 0;
    *nlimbs = N;
    *bits = F.BITS;
    *two_adicity = F.two_adicity;
    return ZO_OK;
  });
}

int zo_to_mont(int field, const uint64_t* canon, uint64_t* mont, size_t count) {
  return dispatch(field, [&](const auto& F) -> int {
    constexpr int N = sizeof(F.P) / sizeof(uint64_t);
    for (size_t i = 0; i < count; i++) {
      uint64_t a[N], r[N];
      load<N>(canon + 4 * i, a);
      F.to_mont(a, r);
      store<N>(mont + 4 * i, r);
    }
    return ZO_OK;
  });
}

int zo_from_mont(int field, const uint64_t* mont, uint64_t* canon, size_t count) {
  return dispatch(field, [&](const auto& F) -> int {
    constexpr int N = sizeof(F.P) / sizeof(uint64_t);
    for (size_t i = 0; i < count; i++) {
      uint64_t a[N], r[N];
      load<N>(mont + 4 * i, a);
      F.from_mont(a, r);
      store<N>(canon + 4 * i, r);
    }
    return ZO_OK;
  });
}

// op: 0 mul, 1 add, 2 sub, 3 neg (b unused), 4 inv (b unused)
int zo_elementwise(int field, int op, const uint64_t* a, const uint64_t* b, uint64_t* out, size_t count) {
  return dispatch(field, [&](const auto& F) -> int {
    constexpr int N = sizeof(F.P) / sizeof(uint64_t);
    for (size_t i = 0; i < count; i++) {
      uint64_t x[N], y[N] = {0}, r[N];
      load<N>(a + 4 * i, x);
      if (b) load<N>(b + 4 * i, y);
      switch (op) {
        case 0: F.mul(x, y, r); break;
        case 1: F.add(x, y, r); break;
        case 2: F.sub(x, y, r); break;
        case 3: F.neg(x, r); break;
        case 4: F.inv(x, r); break;
        default: return ZO_UNSUPPORTED_FIELD;
      }
      store<N>(out + 4 * i, r);
    }
    return ZO_OK;
  });
}

int zo_from_int(int field, uint64_t x, uint64_t* out) {
  return dispatch(field, [&](const auto& F) -> int {
    constexpr int N = sizeof(F.P) / sizeof(uint64_t);
    uint64_t r[N];
    F.from_u64(x, r);
    store<N>(out, r);
    return ZO_OK;
  });
}

int zo_pow(int field, const uint64_t* base, const uint64_t* exp8, uint64_t* out) {
  return dispatch(field, [&](const auto& F) -> int {
    constexpr int N = sizeof(F.P) / sizeof(uint64_t);
    uint64_t b[N], r[N];
    load<N>(base, b);
    F.pow(b, exp8, r);
    store<N>(out, r);
    return ZO_OK;
  });
}

int zo_primitive_root(int field, size_t log_n, uint64_t* out) {
  return dispatch(field, [&](const auto& F) -> int {
    constexpr int N = sizeof(F.P) / sizeof(uint64_t);
    uint64_t r[N];
    int st = F.primitive_root(log_n, r);
    if (st) return st;
    store<N>(out, r);
    return ZO_OK;
  });
}

int zo_qnr(int field, uint64_t* out) {
  return dispatch(field, [&](const auto& F) -> int {
    constexpr int N = sizeof(F.P) / sizeof(uint64_t);
    uint64_t r[N];
    F.qnr(r);
    store<N>(out, r);
    return ZO_OK;
  });
}

int zo_bit_reverse(int field, uint64_t* data, size_t len) {
  return dispatch(field, [&](const auto& F) -> int {
    constexpr int N = sizeof(F.P) / sizeof(uint64_t);
    (void)F;
    auto v = unpack<N>(data, len);
    int st = bit_reverse<N>(v.data(), len);
    if (st) return st;
    pack<N>(data, v);
    return ZO_OK;
  });
}

int zo_ntt(int field, uint64_t* data, size_t len, size_t log_n, const uint64_t* root, int inverse) {
  return dispatch(field, [&](const auto& F) -> int {
    constexpr int N = sizeof(F.P) / sizeof(uint64_t);
    auto v = unpack<N>(data, len);
    uint64_t r[N];
    load<N>(root, r);
    int st = inverse ? intt<N>(F, v.data(), len, log_n, r) : ntt<N>(F, v.data(), len, log_n, r);
    if (st) return st;
    pack<N>(data, v);
    return ZO_OK;
  });
}

// `flat` receives n - 1 slots: stage s at slot offset 2^s - 1.
int zo_precompute_twiddles(int field, size_t log_n, const uint64_t* root, uint64_t* flat) {
  return dispatch(field, [&](const auto& F) -> int {
    constexpr int N = sizeof(F.P) / sizeof(uint64_t);
    size_t n;
    int st = size_from_log(log_n, &n);
    if (st) return st;
    uint64_t r[N];
    load<N>(root, r);
    Vec<N> v(n > 0 ? n - 1 : 0);
    st = precompute_twiddles<N>(F, log_n, r, v.data());
    if (st) return st;
    pack<N>(flat, v);
    return ZO_OK;
  });
}

// Mirrors nttWithTwiddles/inttWithTwiddles including the reference's partial
// mutation of `data` when a later stage has the wrong length.
int zo_ntt_with_twiddles(int field, uint64_t* data, size_t len, size_t log_n,
                         const uint64_t* const* stages, const size_t* lens, size_t num_stages,
                         int inverse, int workers) {
  return dispatch(field, [&](const auto& F) -> int {
    constexpr int N = sizeof(F.P) / sizeof(uint64_t);
    auto v = unpack<N>(data, len);
    int st = ntt_with_twiddles<N>(F, v.data(), len, log_n, stages, lens, num_stages, inverse != 0, workers);
    // Always write back: on an early error `v` is unchanged, and on a bad
    // stage length it holds what the reference leaves in `data` (the bit
    // reversal and every stage before the bad one have run).
    pack<N>(data, v);
    return st;
  });
}

// In-place transform over 4-u64 slots without the unpack/pack copies: used by
// the timed CPU baseline (4-limb fields only, where the slot is the element).
int zo_ntt_with_twiddles_inplace4(int field, uint64_t* data, size_t len, size_t log_n,
                                  const uint64_t* const* stages, const size_t* lens,
                                  size_t num_stages, int inverse, int workers) {
  if (field != ZO_BN254_FR && field != ZO_BLS12_381_FR && field != ZO_BN254_FP) return ZO_UNSUPPORTED_FIELD;
  const Mont<4>& F = field == ZO_BN254_FR ? bn254_fr() : field == ZO_BLS12_381_FR ? bls_fr() : bn254_fp();
  return ntt_with_twiddles<4>(F, reinterpret_cast<Elem<4>*>(data), len, log_n, stages, lens, num_stages,
                              inverse != 0, workers);
}

// The same for the 64-bit fields (Goldilocks, BabyBear): `data` holds one
// u64 per element (Montgomery form); stages are 4-u64 slots as elsewhere.
int zo_ntt_with_twiddles_inplace1(int field, uint64_t* data, size_t len, size_t log_n,
                                  const uint64_t* const* stages, const size_t* lens,
                                  size_t num_stages, int inverse, int workers) {
  if (field != ZO_GOLDILOCKS && field != ZO_BABYBEAR) return ZO_UNSUPPORTED_FIELD;
  const Mont<1>& F = field == ZO_GOLDILOCKS ? goldilocks() : babybear();
  return ntt_with_twiddles<1>(F, reinterpret_cast<Elem<1>*>(data), len, log_n, stages, lens, num_stages,
                              inverse != 0, workers);
}

int zo_chacha20_stream(const uint8_t* seed32, const uint8_t* nonce12, uint8_t* out, size_t len) {
  ChaCha c;
  uint8_t zero_nonce[12] = {0};
  c.init(seed32, nonce12 ? nonce12 : zero_nonce);
  return c.bytes(out, len) ? ZO_OK : ZO_REJECTION_FAILED;
}

// Seeded uniform elements: ChaCha20 keyed by seed32, nonce 0, counter from 0,
// each element one randomFieldElement draw, output in Montgomery form.
int zo_random_elements(int field, const uint8_t* seed32, uint64_t* out, size_t count) {
  return dispatch(field, [&](const auto& F) -> int {
    constexpr int N = sizeof(F.P) / sizeof(uint64_t);
    ChaCha c;
    uint8_t zero_nonce[12] = {0};
    c.init(seed32, zero_nonce);
    for (size_t i = 0; i < count; i++) {
      uint64_t r[N];
      int st = random_field_element<N>(F, c, r);
      if (st) return st;
      store<N>(out + 4 * i, r);
    }
    return ZO_OK;
  });
}

// poly/src/vector.zig:24-32: [1, base, base^2, ...]
int zo_powers(int field, const uint64_t* base, uint64_t* out, size_t n) {
  return dispatch(field, [&](const auto& F) -> int {
    constexpr int N = sizeof(F.P) / sizeof(uint64_t);
    if (n == 0) return ZO_OK;
    uint64_t b[N], cur[N];
    load<N>(base, b);
    std::memcpy(cur, F.ONE, sizeof(cur));
    store<N>(out, cur);
    for (size_t i = 1; i < n; i++) {
      uint64_t t[N];
      F.mul(cur, b, t);
      std::memcpy(cur, t, sizeof(cur));
      store<N>(out + 4 * i, cur);
    }
    return ZO_OK;
  });
}

// Coset low-degree extension composed from the reference's pieces:
//   coeffs = inttWithTwiddles(evals) over 2^log_in with the primitive root,
//   zero-pad to 2^(log_in + log_blowup), multiply by powers(shift)
//   (poly/src/vector.zig hadamard), nttWithTwiddles over 2^log_out.
// `evals` has 2^log_in slots; `out` receives 2^log_out slots.
int zo_coset_lde(int field, const uint64_t* evals, size_t log_in, size_t log_blowup,
                 const uint64_t* shift, uint64_t* out, int workers) {
  return dispatch(field, [&](const auto& F) -> int {
    constexpr int N = sizeof(F.P) / sizeof(uint64_t);
    size_t log_out = log_in + log_blowup;
    size_t n_in = (size_t)1 << log_in, n_out = (size_t)1 << log_out;
    uint64_t root_in[N], root_out[N];
    int st = F.primitive_root(log_in, root_in);
    if (st) return st;
    st = F.primitive_root(log_out, root_out);
    if (st) return st;
    // twiddle tables
    Vec<N> tin(n_in > 1 ? n_in - 1 : 1), tout(n_out - 1);
    precompute_twiddles<N>(F, log_in, root_in, tin.data());
    precompute_twiddles<N>(F, log_out, root_out, tout.data());
    std::vector<uint64_t> tin4((n_in) * 4), tout4(n_out * 4);
    for (size_t i = 0; i + 1 < n_in; i++) store<N>(&tin4[4 * i], tin[i].l);
    for (size_t i = 0; i + 1 < n_out; i++) store<N>(&tout4[4 * i], tout[i].l);
    std::vector<const uint64_t*> sin(log_in), sout(log_out);
    std::vector<size_t> lin(log_in), lout(log_out);
    for (size_t s = 0; s < log_in; s++) { sin[s] = &tin4[4 * (((size_t)1 << s) - 1)]; lin[s] = (size_t)1 << s; }
    for (size_t s = 0; s < log_out; s++) { sout[s] = &tout4[4 * (((size_t)1 << s) - 1)]; lout[s] = (size_t)1 << s; }
    Vec<N> v = unpack<N>(evals, n_in);
    st = ntt_with_twiddles<N>(F, v.data(), n_in, log_in, sin.data(), lin.data(), log_in, true, workers);
    if (st) return st;
    Vec<N> w(n_out);
    uint64_t g[N], cur[N];
    load<N>(shift, g);
    std::memcpy(cur, F.ONE, sizeof(cur));
    for (size_t i = 0; i < n_out; i++) {
      if (i < n_in) {
        F.mul(v[i].l, cur, w[i].l);
      } else {
        for (int k = 0; k < N; k++) w[i].l[k] = 0;
      }
      uint64_t t[N];
      F.mul(cur, g, t);
      std::memcpy(cur, t, sizeof(cur));
    }
    st = ntt_with_twiddles<N>(F, w.data(), n_out, log_out, sout.data(), lout.data(), log_out, false, workers);
    if (st) return st;
    pack<N>(out, w);
    return ZO_OK;
  });
}

// X_k = sum_j x_j * root^(j*k) for selected k, by Horner evaluation of the
// polynomial x at z = root^k (the definition check of libs/ntt/src/main.zig:39-48,
// in O(n) per index).  `workers` threads split the requested indices.
int zo_dft_points(int field, const uint64_t* x, size_t n, const uint64_t* root, const uint64_t* ks,
                  size_t m, uint64_t* out, int workers) {
  return dispatch(field, [&](const auto& F) -> int {
    constexpr int N = sizeof(F.P) / sizeof(uint64_t);
    uint64_t w[N];
    load<N>(root, w);
    parallel_for(m, workers, [&](size_t lo, size_t hi) {
      for (size_t q = lo; q < hi; q++) {
        uint64_t z[N], acc[N] = {0}, t[N], xi[N];
        F.pow_u64(w, ks[q], z);
        for (size_t j = n; j-- > 0;) {
          F.mul(acc, z, t);
          load<N>(x + 4 * j, xi);
          F.add(t, xi, acc);
        }
        store<N>(out + 4 * q, acc);
      }
    });
    return ZO_OK;
  });
}

// Polynomial(F, max_degree) over coefficient arrays: fromCoeffs
// (libs/poly/src/poly.zig:76-84: more than max_degree + 1 coefficients is
// DegreeTooLarge, then normalize), normalize (:100-104: degree = index of the
// last non-zero coefficient, -1 for zero) and mul (:197-212: a zero factor
// gives zero; a product degree above max_degree is DegreeTooLarge; else
// r[i + j] += a_i * b_j for every pair, in the reference's order: i outer, j
// inner, then normalize).  out receives max_degree + 1 coefficients.  The
// harness splits the output coefficients over `workers` threads; each
// coefficient still accumulates its products in increasing i, as the
// reference's loops do for it.
int zo_poly_mul(int field, const uint64_t* a, size_t a_len, const uint64_t* b, size_t b_len, size_t max_degree,
                uint64_t* out, int64_t* out_degree, int workers) {
  return dispatch(field, [&](const auto& F) -> int {
    constexpr int N = sizeof(F.P) / sizeof(uint64_t);
    if (a_len > max_degree + 1 || b_len > max_degree + 1) return ZO_DEGREE_TOO_LARGE;
    auto degree = [&](const uint64_t* c, size_t len) -> int64_t {
      int64_t d = (int64_t)len - 1;
      while (d >= 0) {
        uint64_t x[N];
        load<N>(c + 4 * d, x);
        bool zero = true;
        for (int q = 0; q < N; q++) zero = zero && x[q] == 0;
        if (!zero) break;
        d--;
      }
      return d;
    };
    const int64_t da = degree(a, a_len), db = degree(b, b_len);
    std::memset(out, 0, (max_degree + 1) * 32);
    if (da < 0 || db < 0) {
      *out_degree = -1;
      return ZO_OK;
    }
    const int64_t d = da + db;
    if ((uint64_t)d > max_degree) return ZO_DEGREE_TOO_LARGE;
    Vec<N> va = unpack<N>(a, (size_t)da + 1), vb = unpack<N>(b, (size_t)db + 1);
    parallel_for((size_t)d + 1, workers, [&](size_t lo, size_t hi) {
      for (size_t k = lo; k < hi; k++) {
        uint64_t acc[N] = {0}, t[N];
        const size_t i0 = k > (size_t)db ? k - (size_t)db : 0, i1 = std::min(k, (size_t)da);
        for (size_t i = i0; i <= i1; i++) {
          F.mul(va[i].l, vb[k - i].l, t);
          F.add(acc, t, acc);
        }
        store<N>(out + 4 * k, acc);
      }
    });
    *out_degree = degree(out, (size_t)d + 1);
    return ZO_OK;
  });
}

// Horner evaluation of c (len coefficients) at each of m points
// (Polynomial.eval, libs/poly/src/poly.zig:214-224).
int zo_poly_eval(int field, const uint64_t* c, size_t len, const uint64_t* xs, size_t m, uint64_t* out, int workers) {
  return dispatch(field, [&](const auto& F) -> int {
    constexpr int N = sizeof(F.P) / sizeof(uint64_t);
    parallel_for(m, workers, [&](size_t lo, size_t hi) {
      for (size_t q = lo; q < hi; q++) {
        uint64_t z[N], acc[N] = {0}, t[N], ci[N];
        load<N>(xs + 4 * q, z);
        for (size_t j = len; j-- > 0;) {
          F.mul(acc, z, t);
          load<N>(c + 4 * j, ci);
          F.add(t, ci, acc);
        }
        store<N>(out + 4 * q, acc);
      }
    });
    return ZO_OK;
  });
}

}  // extern "C"

// Domain(F).init(log_n) (libs/fri/src/root.zig:133-138): omega =
// primitiveRootOfUnity(two_adicity), step_gen = omega^(2^(two_adicity - log_n)).
template <class FT, int N>
static int fri_step_gen(const FT& F, size_t log_n, uint64_t* step) {
  if ((long)log_n > F.two_adicity) return ZO_ORDER_TOO_LARGE;
  uint64_t omega[N];
  int st = F.primitive_root(F.two_adicity, omega);
  if (st) return st;
  std::memcpy(step, omega, sizeof(uint64_t) * N);
  for (size_t i = 0; i < (size_t)F.two_adicity - log_n; i++) F.mul(step, step, step);
  return ZO_OK;
}

extern "C" {

// Domain.fill (:155-166): x = one; each slot gets x, then x *= step_gen.
int zo_fri_domain_fill(int field, size_t log_n, uint64_t* out) {
  return dispatch(field, [&](const auto& F) -> int {
    constexpr int N = sizeof(F.P) / sizeof(uint64_t);
    uint64_t g[N], x[N];
    int st = fri_step_gen<std::decay_t<decltype(F)>, N>(F, log_n, g);
    if (st) return st;
    std::memcpy(x, F.ONE, sizeof(x));
    for (size_t i = 0; i < ((size_t)1 << log_n); i++) {
      store<N>(out + 4 * i, x);
      F.mul(x, g, x);
    }
    return ZO_OK;
  });
}

// One fold round of proveOn (:396-403): for j < n/2, x = dom.at(j) = step_gen^j,
// even = (f_j + f_{j+n/2}) * half_inv, odd = (f_j - f_{j+n/2}).div(x) * half_inv,
// next_j = even + alpha * odd, with half_inv = 1.div(2) and div = mul by inverse.
int zo_fri_fold(int field, const uint64_t* layer, size_t log_n, const uint64_t* alpha, uint64_t* out, int workers) {
  return dispatch(field, [&](const auto& F) -> int {
    constexpr int N = sizeof(F.P) / sizeof(uint64_t);
    if (log_n < 1) return ZO_LOG_TOO_LARGE;
    uint64_t g[N], two[N], half_inv[N], a[N];
    int st = fri_step_gen<std::decay_t<decltype(F)>, N>(F, log_n, g);
    if (st) return st;
    F.from_u64(2, two);
    F.inv(two, half_inv);
    load<N>(alpha, a);
    const size_t half = (size_t)1 << (log_n - 1);
    parallel_for(half, workers, [&](size_t lo, size_t hi) {
      uint64_t x[N];
      F.pow_u64(g, lo, x);
      for (size_t j = lo; j < hi; j++) {
        uint64_t fx[N], fn[N], s[N], d[N], xi[N], even[N], odd[N], t[N];
        load<N>(layer + 4 * j, fx);
        load<N>(layer + 4 * (j + half), fn);
        F.add(fx, fn, s);
        F.mul(s, half_inv, even);
        F.sub(fx, fn, d);
        F.inv(x, xi);
        F.mul(d, xi, t);
        F.mul(t, half_inv, odd);
        F.mul(a, odd, t);
        F.add(even, t, t);
        store<N>(out + 4 * j, t);
        F.mul(x, g, x);
      }
    });
    return ZO_OK;
  });
}

}  // extern "C"

// ---- BLAKE3 (single chunk) and the FRI layer commitment -------------------------

static const uint32_t kB3Iv[8] = {0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au,
                                  0x510E527Fu, 0x9B05688Cu, 0x1F83D9ABu, 0x5BE0CD19u};
static const uint8_t kB3Perm[16] = {2, 6, 3, 10, 7, 0, 4, 13, 1, 11, 12, 5, 9, 14, 15, 8};

static inline uint32_t rotr32(uint32_t x, int r) { return (x >> r) | (x << (32 - r)); }

static void b3_compress(const uint32_t cv[8], const uint32_t block[16], uint64_t counter, uint32_t len,
                        uint32_t flags, uint32_t out[8]) {
  uint32_t v[16], m[16];
  for (int i = 0; i < 8; i++) v[i] = cv[i];
  for (int i = 0; i < 4; i++) v[8 + i] = kB3Iv[i];
  v[12] = (uint32_t)counter;
  v[13] = (uint32_t)(counter >> 32);
  v[14] = len;
  v[15] = flags;
  for (int i = 0; i < 16; i++) m[i] = block[i];
  auto g = [&](int a, int b, int c, int d, uint32_t x, uint32_t y) {
    v[a] += v[b] + x;
    v[d] = rotr32(v[d] ^ v[a], 16);
    v[c] += v[d];
    v[b] = rotr32(v[b] ^ v[c], 12);
    v[a] += v[b] + y;
    v[d] = rotr32(v[d] ^ v[a], 8);
    v[c] += v[d];
    v[b] = rotr32(v[b] ^ v[c], 7);
  };
  for (int r = 0; r < 7; r++) {
    g(0, 4, 8, 12, m[0], m[1]);
    g(1, 5, 9, 13, m[2], m[3]);
    g(2, 6, 10, 14, m[4], m[5]);
    g(3, 7, 11, 15, m[6], m[7]);
    g(0, 5, 10, 15, m[8], m[9]);
    g(1, 6, 11, 12, m[10], m[11]);
    g(2, 7, 8, 13, m[12], m[13]);
    g(3, 4, 9, 14, m[14], m[15]);
    if (r < 6) {
      uint32_t t[16];
      for (int i = 0; i < 16; i++) t[i] = m[kB3Perm[i]];
      std::memcpy(m, t, sizeof(m));
    }
  }
  for (int i = 0; i < 8; i++) out[i] = v[i] ^ v[i + 8];
}

// BLAKE3-256 of a message of at most 1024 bytes (one chunk): blocks compressed
// in order from the IV, the first flagged CHUNK_START (1), the last CHUNK_END |
// ROOT (2 | 8).
static void b3_hash(const uint8_t* msg, size_t len, uint8_t out[32]) {
  uint32_t cv[8];
  std::memcpy(cv, kB3Iv, sizeof(cv));
  const size_t nblocks = len == 0 ? 1 : (len + 63) / 64;
  for (size_t b = 0; b < nblocks; b++) {
    uint8_t blk[64] = {0};
    const size_t bl = std::min<size_t>(64, len - b * 64);
    if (bl) std::memcpy(blk, msg + b * 64, bl);
    uint32_t words[16];
    for (int i = 0; i < 16; i++)
      words[i] = (uint32_t)blk[4 * i] | ((uint32_t)blk[4 * i + 1] << 8) | ((uint32_t)blk[4 * i + 2] << 16) |
                 ((uint32_t)blk[4 * i + 3] << 24);
    const uint32_t flags = (b == 0 ? 1u : 0u) | (b + 1 == nblocks ? 10u : 0u);
    b3_compress(cv, words, 0, (uint32_t)bl, flags, cv);
  }
  for (int i = 0; i < 8; i++)
    for (int k = 0; k < 4; k++) out[4 * i + k] = (uint8_t)(cv[i] >> (8 * k));
}

extern "C" {

int zo_blake3(const uint8_t* msg, size_t len, uint8_t* out) {
  if (len > 1024) return ZO_LENGTH_MISMATCH;
  b3_hash(msg, len, out);
  return ZO_OK;
}

// The commitment of one FRI layer (2^log_n slots): leaf j = BLAKE3(toBytes(f_j) ||
// toBytes(f_{j+n/2})) with toBytes the canonical value in NUM_BYTES little-endian
// bytes (libs/field/src/field.zig:244-252, 1002-1017), then the heap-ordered tree
// of initFromHashes: nodes[h + j] = leaf j, nodes[i] = BLAKE3(nodes[2i] ||
// nodes[2i+1]), h = n/2 (a power of two, so no padding).  `nodes` receives 2h
// digests, nodes[0] zero.
int zo_fri_commit_layer(int field, const uint64_t* layer, size_t log_n, uint8_t* nodes, int workers) {
  return dispatch(field, [&](const auto& F) -> int {
    constexpr int N = sizeof(F.P) / sizeof(uint64_t);
    if (log_n < 1) return ZO_LOG_TOO_LARGE;
    const size_t nb = (size_t)(F.BITS + 7) / 8, h = (size_t)1 << (log_n - 1);
    std::memset(nodes, 0, 32);
    auto bytes_of = [&](const uint64_t* slot, uint8_t* out) {
      uint64_t m[N], c[N];
      load<N>(slot, m);
      F.from_mont(m, c);
      for (size_t k = 0; k < nb; k++) out[k] = (uint8_t)(c[k / 8] >> (8 * (k % 8)));
    };
    parallel_for(h, workers, [&](size_t lo, size_t hi) {
      for (size_t j = lo; j < hi; j++) {
        uint8_t msg[64];
        bytes_of(layer + 4 * j, msg);
        bytes_of(layer + 4 * (j + h), msg + nb);
        b3_hash(msg, 2 * nb, nodes + 32 * (h + j));
      }
    });
    for (size_t w = h / 2; w >= 1; w /= 2) {
      parallel_for(w, w >= 4096 ? workers : 1, [&](size_t lo, size_t hi) {
        for (size_t i = w + lo; i < w + hi; i++) b3_hash(nodes + 32 * (2 * i), 64, nodes + 32 * i);
      });
    }
    return ZO_OK;
  });
}

// MerkleTree.init (libs/merkle/src/merkle_tree.zig:70-103) over rows of columns:
// leaf i = BLAKE3(toBytes(col_0[i]) || ... || toBytes(col_{m-1}[i])) -- the row
// serialized the way hashPair serializes a pair -- for 2^log_n rows (a power of
// two, so no padding leaves), then the same heap-ordered levels as above:
// nodes[n + i] = leaf i, nodes[1] the root, nodes[0] zero.  Rows of at most
// 1024 bytes (one BLAKE3 chunk).
int zo_merkle_commit_rows(int field, const uint64_t* const* cols, size_t num_cols, size_t log_n, uint8_t* nodes,
                          int workers) {
  return dispatch(field, [&](const auto& F) -> int {
    constexpr int N = sizeof(F.P) / sizeof(uint64_t);
    const size_t nb = (size_t)(F.BITS + 7) / 8, n = (size_t)1 << log_n;
    if (num_cols == 0 || num_cols * nb > 1024) return ZO_LENGTH_MISMATCH;
    std::memset(nodes, 0, 32);
    parallel_for(n, workers, [&](size_t lo, size_t hi) {
      std::vector<uint8_t> row(num_cols * nb);
      for (size_t i = lo; i < hi; i++) {
        for (size_t c = 0; c < num_cols; c++) {
          uint64_t m[N], v[N];
          load<N>(cols[c] + 4 * i, m);
          F.from_mont(m, v);
          for (size_t k = 0; k < nb; k++) row[c * nb + k] = (uint8_t)(v[k / 8] >> (8 * (k % 8)));
        }
        b3_hash(row.data(), row.size(), nodes + 32 * (n + i));
      }
    });
    for (size_t w = n / 2; w >= 1; w /= 2) {
      parallel_for(w, w >= 4096 ? workers : 1, [&](size_t lo, size_t hi) {
        for (size_t i = w + lo; i < w + hi; i++) b3_hash(nodes + 32 * (2 * i), 64, nodes + 32 * i);
      });
    }
    return ZO_OK;
  });
}

}  // extern "C"
