/* zntt.h -- C ABI of libzntt_cuda.so, the B200 (sm_100a) NTT library.
 *
 * The library replaces zig-algebra's NTT hot path, the Zig module `zig-ntt`
 * (libs/ntt/src/root.zig), for the two scalar fields it runs on in practice:
 * BN254-Fr (libs/curve/src/bn254.zig:67) and BLS12-381-Fr
 * (libs/curve/src/bls12_381.zig:66).  An element is the reference's
 * `BigField` value (libs/field/src/field.zig:884): four little-endian u64 limbs
 * in Montgomery form (x * 2^256 mod r), fully reduced.  Every function takes
 * plain pointers and sizes; arrays of elements are `4 * len` u64 words.
 *
 * Errors are integer status codes that map one to one onto zig-ntt's error
 * set (libs/ntt/src/root.zig:33-36, 43, 67-68, 150-152, 161) plus the device
 * failures a GPU adds.  Unlike zig-ntt, every argument is validated before
 * any data moves: on any error `data` is left untouched (zig-ntt leaves a
 * partially transformed buffer when a later twiddle stage has the wrong
 * length, libs/ntt/src/root.zig:161).
 *
 * Thread safety: calls may come from any thread; the library serialises them
 * on its own stream per device.  The plain entry points are synchronous, like
 * the reference.
 */
#ifndef ZNTT_H
#define ZNTT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
enum zntt_status {
  ZNTT_OK = 0,
  ZNTT_ERR_LOG_TOO_LARGE = 1,      /* error.LogTooLarge: log_n >= 64 (root.zig:33-36) */
  ZNTT_ERR_LENGTH_MISMATCH = 2,    /* error.LengthMismatch: len != 2^log_n (root.zig:68) */
  ZNTT_ERR_INVALID_TWIDDLES = 3,   /* error.InvalidTwiddles (root.zig:152, 161) */
  ZNTT_ERR_INVALID_LENGTH = 4,     /* error.InvalidLength: bitReverse len 0 / not 2^k (root.zig:43) */
  ZNTT_ERR_OUT_OF_MEMORY = 5,      /* error.OutOfMemory, or the vector does not fit on the device */
  ZNTT_ERR_ORDER_TOO_LARGE = 6,    /* error.OrderTooLarge: log_n > two-adicity (roots.zig:150) */
  ZNTT_ERR_UNSUPPORTED_FIELD = 7,  /* a field id other than the four below, or a small field
                                      where only the 256-bit ones are served */
  ZNTT_ERR_DEVICE = 8,             /* a CUDA call failed; see zntt_last_error() */
  ZNTT_ERR_TIMEOUT = 9,            /* a bounded device wait gave up */
  ZNTT_ERR_INVALID_ARGUMENT = 10,  /* null pointer, bad handle, unknown mode */
  ZNTT_ERR_NOT_INITIALIZED = 11,   /* zntt_init() has not run */
  ZNTT_ERR_REJECTED = 12,          /* admission refused (over the memory budget / queue full) */
  ZNTT_ERR_DEGREE_TOO_LARGE = 13   /* error.DegreeTooLarge: a polynomial beyond its capacity
                                      (libs/poly/src/poly.zig:77, 200) */
};

/* ---- fields ---------------------------------------------------------------- */
enum zntt_field {
  ZNTT_FIELD_BN254_FR = 0,      /* r = 0x30644e72...43e1f593f0000001, two-adicity 28 */
  ZNTT_FIELD_BLS12_381_FR = 1,  /* r = 0x73eda753...ffffffff00000001, two-adicity 32 */
  /* zig-field's SmallField backend (libs/field/src/field.zig:89-849), the fields of the
   * reference's own transform known-answer tests (libs/ntt/src/root.zig:437-447).  An element
   * is SmallField's canonical value, ONE uint64_t (8 bytes), not four Montgomery limbs; roots
   * and other scalars still pass as uint64_t[4] with the value in [0] and zeros after.  These
   * fields serve the seven zig-ntt entry points, zntt_field_info / zntt_primitive_root, the
   * device API (zntt_twiddles_acquire / _release, zntt_ntt_device), zntt_coset_lde_device, and
   * the FRI and Merkle entry points; bitReverse of 8-byte elements is zntt_bit_reverse_small.
   * zntt_poly_mul also serves them.  Batches, zntt_poly_mul_device, the server, the
   * pipelined host API and the allocation-free entry point take the 256-bit fields only and
   * reject a small-field table with ZNTT_ERR_UNSUPPORTED_FIELD. */
  ZNTT_FIELD_GOLDILOCKS = 2,    /* p = 2^64 - 2^32 + 1, two-adicity 32 */
  ZNTT_FIELD_BABYBEAR = 3       /* p = 15 * 2^27 + 1, two-adicity 27 */
};

/* One twiddle stage as zig-ntt hands it over: the layout of a Zig
 * `[]const F` slice (pointer, element count). */
typedef struct zntt_stage {
  const uint64_t* ptr;
  size_t len;
} zntt_stage;

/* ---- lifetime ------------------------------------------------------------- */
/* Selects the CUDA device and creates the library's stream and caches.
 * Idempotent for the same device. */
int zntt_init(int device);
/* Frees every device buffer, cache entry and stream. */
int zntt_shutdown(void);
/* Message of the last failure on the calling thread ("" when none). */
const char* zntt_last_error(void);
/* The library's device buffer pool: buffers taken from it (scratch and staging
 * of the transforms), cudaMalloc calls it made, and idle bytes it caches.  For
 * callers that watch device memory, and for tests that check an entry point
 * allocates nothing.  No counterpart in the reference. */
int zntt_pool_stats(uint64_t* acquires, uint64_t* device_mallocs, uint64_t* cached_bytes);
/* Modulus (canonical, 4 LE limbs) and two-adicity of a field. */
int zntt_field_info(int field, uint64_t modulus[4], uint32_t* two_adicity);
/* F.primitiveRootOfUnity(log_n) in Montgomery form: the first quadratic
 * non-residue counting up from 2 (5 for both fields) raised to
 * odd_part << (two_adicity - log_n) (libs/field/src/roots.zig:149-158). */
int zntt_primitive_root(int field, uint32_t log_n, uint64_t root_out[4]);

/* ---- zig-ntt drop-in: host data, synchronous -------------------------------
 * Each replaces the zig-ntt function named in its comment; `field` stands in
 * for the `comptime F` parameter. */

/* bitReverse(F, data)            libs/ntt/src/root.zig:38-58 */
int zntt_bit_reverse(uint64_t* data, size_t len);
/* bitReverse (root.zig:38-58) for 8-byte elements (ZNTT_FIELD_GOLDILOCKS / _BABYBEAR data). */
int zntt_bit_reverse_small(uint64_t* data, size_t len);
/* ntt(F, data, log_n, root)       libs/ntt/src/root.zig:65-90 */
int zntt_ntt(int field, uint64_t* data, size_t len, size_t log_n, const uint64_t root[4]);
/* intt(F, data, log_n, root)      libs/ntt/src/root.zig:95-107 */
int zntt_intt(int field, uint64_t* data, size_t len, size_t log_n, const uint64_t root[4]);
/* precomputeTwiddles(F, log_n, root, allocator)   libs/ntt/src/root.zig:112-134
 * The caller allocates the table as zig-ntt's allocator would (stage s:
 * 2^s elements) and passes the stage pointers; the library fills them from
 * the device and keeps the same table resident on the device, recognised
 * again by its stage addresses. */
int zntt_precompute_twiddles(int field, size_t log_n, const uint64_t root[4], uint64_t* const* stage_out);
/* freeTwiddles(F, twiddles, allocator)            libs/ntt/src/root.zig:136-141
 * Releases the device copy; the caller frees its own stage arrays. */
void zntt_free_twiddles(int field, const zntt_stage* stages, size_t num_stages);
/* nttWithTwiddles(F, data, log_n, twiddles)       libs/ntt/src/root.zig:148-175 */
int zntt_ntt_with_twiddles(int field, uint64_t* data, size_t len, size_t log_n, const zntt_stage* stages,
                           size_t num_stages);
/* inttWithTwiddles(F, data, log_n, twiddles)      libs/ntt/src/root.zig:180-212 */
int zntt_intt_with_twiddles(int field, uint64_t* data, size_t len, size_t log_n, const zntt_stage* stages,
                            size_t num_stages);

/* ---- device-resident API ------------------------------------------------------
 * For callers that keep vectors in HBM.  `stream` is a cudaStream_t (NULL: the
 * library's stream); calls are asynchronous on it. */
typedef struct zntt_twiddles zntt_twiddles;

/* Device twiddle table for (field, log_n, root), shared and reference counted:
 * the table precomputeTwiddles would build, kept on the device. */
int zntt_twiddles_acquire(int field, uint32_t log_n, const uint64_t root[4], zntt_twiddles** out);
int zntt_twiddles_release(zntt_twiddles* tw);

enum zntt_mode {
  ZNTT_FORWARD = 0,  /* nttWithTwiddles */
  ZNTT_INVERSE = 1   /* inttWithTwiddles (includes the 1/n scale) */
};

/* Transform 2^log_n device elements from d_src into d_dst (which may equal
 * d_src).  `d_scratch` (2^log_n elements, or NULL) is only used when
 * d_dst == d_src and the transform needs more than one pass; when NULL the
 * library borrows one from its pool. */
int zntt_ntt_device(const zntt_twiddles* tw, const uint64_t* d_src, uint64_t* d_dst, uint64_t* d_scratch,
                    int mode, void* stream);

/* Forward or inverse transforms of num_columns device columns of 2^log_n elements (the
 * table's size), column k from d_src[k] into d_dst[k], out of place.  For Goldilocks /
 * BabyBear every launch covers all columns (up to 65535) and the call waits for its stream;
 * for the 256-bit fields each column is one zntt_ntt_device call (stream-ordered). */
int zntt_ntt_device_columns(const zntt_twiddles* tw, const uint64_t* const* d_src, uint64_t* const* d_dst,
                            uint32_t num_columns, int mode, void* stream);

/* In-place transform of the 2^log_n device elements at d_data (log_n of the
 * twiddle handle, at most 18) that allocates no memory.  No counterpart in the
 * reference.  For callers that must not allocate device memory when they
 * transform: services that reserve all device memory up front under a fixed
 * budget, programs whose memory belongs to another allocator, and
 * latency-critical paths where cudaMalloc/cudaFree would block.  Its scratch
 * is an 8 MiB array inside the library, held by every device that loads the
 * library until the process exits.  The first call on a device looks up that
 * array's device address (make it before any stream capture).  All calls
 * share the array: calls that overlap on the GPU race.  Larger transforms are
 * rejected with ZNTT_ERR_INVALID_ARGUMENT. */
int zntt_ntt_device_inplace_noalloc(const zntt_twiddles* tw, uint64_t* d_data, int mode, void* stream);

/* ---- batches: many jobs in one persistent launch -----------------------------
 * A batch plans every job into passes and every pass into tiles, queues the
 * tiles level by level on the device, and runs them all in one persistent
 * launch that drains the queue (each tile waits, bounded, for its job's
 * previous pass).  Jobs of a batch share a field and may mix sizes and kinds. */
enum zntt_job_kind {
  ZNTT_JOB_NTT = 0,       /* nttWithTwiddles / inttWithTwiddles (libs/ntt/src/root.zig:148-212) */
  ZNTT_JOB_COSET_LDE = 1, /* intt of 2^log_in evaluations, zero-pad, c_i *= g^i, ntt of 2^log_n:
                             the composition of zig-ntt with libs/poly/src/vector.zig:24-32,68-73 */
  ZNTT_JOB_POLY_MUL = 2   /* product of two coefficient vectors (Polynomial.mul,
                             libs/poly/src/poly.zig:197-212) through transforms of 2^log_n points */
};
typedef struct zntt_job {
  int kind;                   /* zntt_job_kind */
  int mode;                   /* NTT jobs: ZNTT_FORWARD or ZNTT_INVERSE */
  const zntt_twiddles* tw;    /* the transform's table (coset extension: of the output size) */
  const zntt_twiddles* tw_in; /* coset extension: table of the input size (its inverse mapping is used) */
  const uint64_t* d_src;      /* 2^log_n device elements (coset extension: 2^log_in evaluations) */
  uint64_t* d_dst;            /* 2^log_n device elements; NTT jobs may transform in place */
  uint64_t shift[4];          /* coset extension: the shift g, Montgomery form */
  const uint64_t* d_src2;     /* polynomial product: the second factor's coefficients */
  uint64_t len, len2;         /* polynomial product: coefficient counts of d_src and d_src2, both at
                                 least 1 with len + len2 - 1 <= 2^log_n; d_dst receives the
                                 len + len2 - 1 product coefficients and must not overlap the
                                 factors; tw must be the table of the primitive 2^log_n-th root */
} zntt_job;
typedef struct zntt_batch zntt_batch;

/* Plans the jobs (shape: a pass shape index, or -1 for the library's batch
 * shape, 2^9-element tiles at 7 CTAs per SM) and
 * uploads the work queue; buffers stay owned by the caller and must outlive
 * the batch. */
int zntt_batch_create(int field, const zntt_job* jobs, size_t n_jobs, int shape, zntt_batch** out);
/* Resets the queue and launches the persistent kernel on `stream`. */
int zntt_batch_run(zntt_batch* b, void* stream);
/* The same, captured once into a CUDA graph and replayed on later calls. */
int zntt_batch_run_graph(zntt_batch* b, void* stream);
/* After the stream finished: ZNTT_OK, or ZNTT_ERR_TIMEOUT if a wait gave up. */
int zntt_batch_status(zntt_batch* b);
/* How many sleep rounds (about 0.25-1 us each) a tile waits for its job's
 * previous pass before it raises the batch's error flag (after which every CTA
 * stops at its next item and zntt_batch_status reports ZNTT_ERR_TIMEOUT).
 * Default ZNTT_BATCH_SPIN_LIMIT; 0 makes any wait give up at once, which is
 * how a test drives the timeout path without faulting anything.  Takes effect
 * at the next run (a captured graph is re-captured).  No counterpart in the
 * reference, which has no device waits. */
#define ZNTT_BATCH_SPIN_LIMIT 4194304u
int zntt_batch_set_spin_limit(zntt_batch* b, uint32_t spin_limit);
int zntt_batch_info(const zntt_batch* b, uint32_t* n_items, uint32_t* n_passes, int* grid, int* shape);
int zntt_batch_destroy(zntt_batch* b);

/* One coset low-degree extension with plain per-pass launches:
 * d_out = ntt_{2^log_n}((intt_{2^log_in}(d_evals) zero-padded) . g^i), where
 * log_in / log_n are those of tw_in / tw_out.  All four fields: with
 * Goldilocks / BabyBear tables the shift is a nonzero canonical value in word 0
 * and the call waits for its stream. */
int zntt_coset_lde_device(const zntt_twiddles* tw_in, const zntt_twiddles* tw_out, const uint64_t shift[4],
                          const uint64_t* d_evals, uint64_t* d_out, void* stream);
/* The same extension for num_columns columns (a prover's trace columns): column k from
 * d_evals[k] into d_out[k].  For Goldilocks / BabyBear every launch covers all columns (a
 * second grid dimension, up to 65535 columns; beyond that, or for one-element inputs, the
 * columns run one after another), with one wait at the end; for the 256-bit fields each
 * column is one zntt_coset_lde_device call. */
int zntt_coset_lde_columns(const zntt_twiddles* tw_in, const zntt_twiddles* tw_out, const uint64_t shift[4],
                           const uint64_t* const* d_evals, uint64_t* const* d_out, uint32_t num_columns,
                           void* stream);

/* ---- polynomial products -------------------------------------------------------
 * Polynomial(F, max_degree).mul (libs/poly/src/poly.zig:197-212) computes the
 * schoolbook product in O(deg^2).  These compute the same coefficients in
 * O(n log n) through three transforms of n = 2^log_n >= len_a + len_b - 1 points
 * (forward, forward with the pointwise product fused into its last pass,
 * inverse); exact field arithmetic makes every coefficient identical. */

/* d_out[0 .. len_a + len_b - 2] = the product of the coefficient vectors d_a
 * (len_a) and d_b (len_b), with plain per-pass launches on `stream`; tw is the
 * table of the primitive 2^log_n-th root with 2^log_n >= len_a + len_b - 1.
 * Coefficients are not normalized (leading zeros stay).  d_out must not
 * overlap the factors. */
int zntt_poly_mul_device(const zntt_twiddles* tw, const uint64_t* d_a, size_t len_a, const uint64_t* d_b,
                         size_t len_b, uint64_t* d_out, void* stream);

/* Polynomial(F, max_degree).mul with host coefficient arrays: a (a_len) and b
 * (b_len) are normalized like Polynomial.fromCoeffs (trailing zero
 * coefficients dropped; more than max_degree + 1 coefficients is
 * ZNTT_ERR_DEGREE_TOO_LARGE, poly.zig:76-77); a zero factor gives the zero
 * polynomial; a product degree above max_degree is ZNTT_ERR_DEGREE_TOO_LARGE
 * (poly.zig:198-200).  On success out[0 .. max_degree] holds the product's
 * coefficients followed by zeros (the reference's fixed coeffs array) and
 * *out_degree its degree, -1 for the zero polynomial.  Synchronous.  All four
 * fields: coefficients are four Montgomery limbs each for the 256-bit fields and one
 * canonical uint64_t each (below p, else ZNTT_ERR_INVALID_ARGUMENT) for Goldilocks and
 * BabyBear. */
int zntt_poly_mul(int field, const uint64_t* a, size_t a_len, const uint64_t* b, size_t b_len, size_t max_degree,
                  uint64_t* out, int64_t* out_degree);

/* ---- FRI on resident evaluations ------------------------------------------------
 * The data-parallel steps of zig-fri's prover (libs/fri/src/root.zig), so a coset
 * extension's output can be folded without leaving the device.  All four fields;
 * elements in the field's layout (four Montgomery limbs, or one canonical u64 for
 * Goldilocks / BabyBear); scalars as uint64_t[4]. */

/* Domain(F).fill (libs/fri/src/root.zig:155-166): d_out[i] = g^i for i < 2^log_n, g the
 * generator of the order-2^log_n subgroup (the field's primitiveRootOfUnity(log_n)).
 * ZNTT_ERR_ORDER_TOO_LARGE beyond the two-adicity (Domain.init's DomainTooLarge). */
int zntt_fri_domain_fill(int field, uint32_t log_n, uint64_t* d_out, void* stream);

/* One fold round of proveOn (libs/fri/src/root.zig:396-403) on a layer of 2^log_n
 * evaluations in natural order on the order-2^log_n subgroup:
 *   d_out[j] = (f[j] + f[j + n/2]) / 2 + alpha * (f[j] - f[j + n/2]) / (2 g^j),  j < n/2.
 * The factors 1/(2 g^j) come from a device table kept per (field, log_table), log_table
 * being the size of the largest layer folded with it (0: log_n); pass the first layer's
 * size for every round of one proof so that all rounds share one table.  Stream-ordered;
 * d_out must not overlap the layer. */
int zntt_fri_fold_device(int field, const uint64_t* d_layer, uint32_t log_n, const uint64_t alpha[4],
                         uint64_t* d_out, uint32_t log_table, void* stream);

/* The commitment of one FRI layer of 2^log_n evaluations (proveOn's commit step):
 * leaf j = BLAKE3(toBytes(f[j]) || toBytes(f[j + n/2])) (hashPair, libs/fri/src/root.zig:286-295;
 * toBytes = the canonical value in ceil(bits/8) little-endian bytes), and the heap-ordered
 * BLAKE3 Merkle tree of MerkleTree.initFromHashes (libs/merkle/src/merkle_tree.zig:146-180):
 * d_nodes (2^log_n digests of 32 bytes, 16-byte aligned) receives node 0 = zero, node 1 = the
 * root, node i = BLAKE3(node 2i || node 2i+1), node n/2 + j = leaf j.  When root_out is not
 * null the root is copied there and the call waits for the stream; otherwise it is
 * stream-ordered.  All four fields. */
int zntt_fri_commit_layer(int field, const uint64_t* d_layer, uint32_t log_n, uint8_t* d_nodes,
                          uint8_t* root_out, void* stream);

/* MerkleTree.init (libs/merkle/src/merkle_tree.zig:70-103) over the rows of num_columns
 * device columns of 2^log_n elements each (the commitment of a prover's extended trace
 * columns): leaf i = BLAKE3(toBytes(col_0[i]) || ... || toBytes(col_{m-1}[i])), the row
 * serialized in column order the way hashPair serializes a pair; d_nodes (2^(log_n+1)
 * digests of 32 bytes, 16-byte aligned) receives node 0 = zero, node 1 = the root,
 * node 2^log_n + i = leaf i.  Rows of at most 1024 bytes (32 columns of a 256-bit field,
 * 128 of Goldilocks, 256 of BabyBear); log_n <= 30.  root_out as in
 * zntt_fri_commit_layer. */
int zntt_merkle_commit_rows(int field, const uint64_t* const* d_columns, uint32_t num_columns, uint32_t log_n,
                            uint8_t* d_nodes, uint8_t* root_out, void* stream);

/* Openings of a row commitment (MerkleTree.prove, libs/merkle/src/merkle_tree.zig:206-233)
 * for num_queries rows i < 2^log_n of the columns committed by zntt_merkle_commit_rows
 * (d_nodes its node array): values_out + q * num_columns * NB receives row positions[q]'s
 * toBytes values in column order, paths_out + q * log_n * 32 its log_n sibling digests
 * from the leaf level up.  Host outputs; the call waits for them. */
int zntt_merkle_open_rows(int field, const uint64_t* const* d_columns, uint32_t num_columns, uint32_t log_n,
                          const uint8_t* d_nodes, const uint64_t* positions, size_t num_queries, uint8_t* values_out,
                          uint8_t* paths_out, void* stream);

/* One fold round followed by the commitment of the layer it makes, in one pass:
 * the same results as zntt_fri_fold_device(field, d_layer, log_n, alpha, d_out,
 * log_table) then zntt_fri_commit_layer(field, d_out, log_n - 1, d_nodes, root_out),
 * with the new layer's leaves hashed by the threads that fold their values (proveOn's
 * round r fold and round r + 1 commit, libs/fri/src/root.zig:372-403).  log_n >= 2;
 * alpha must be a field element; the layer, d_out and d_nodes must not overlap. */
int zntt_fri_fold_commit(int field, const uint64_t* d_layer, uint32_t log_n, const uint64_t alpha[4],
                         uint64_t* d_out, uint32_t log_table, uint8_t* d_nodes, uint8_t* root_out, void* stream);

/* The Fiat-Shamir challenge of FRI round `round`, computed by the caller's transcript
 * (proveOn's absorbBytes(root) then challengeFieldChecked, root.zig:386-388): writes alpha
 * in the field's scalar layout (Montgomery limbs below p; a small field's canonical value
 * in word 0, the other words zero) and returns 0, or nonzero to stop the phase.  It runs on
 * the thread that called zntt_fri_commit_phase while that call holds the library's lock:
 * it may call the library from that thread, but must not wait for another thread that
 * does. */
typedef int (*zntt_fri_challenge_fn)(void* user, uint32_t round, const uint8_t root[32], uint64_t alpha_out[4]);

/* The commit phase of proveOn (libs/fri/src/root.zig:372-403) on resident layers:
 * for r < rounds = log_domain - log_final, commit layer r (2^(log_domain - r)
 * evaluations in d_layers[r]) into d_nodes[r] as zntt_fri_commit_layer does, copy its
 * root to roots_out + 32 r, ask `challenge` for alpha_r, and fold layer r into
 * d_layers[r + 1] with one shared 1/(2x) table.  d_layers holds rounds + 1 device
 * vectors (d_layers[0] the evaluations), d_nodes rounds node arrays of
 * 2^(log_domain - r) x 32 bytes.  Checks Config.rounds' size rules (root.zig:188-195:
 * log_final < log_domain, log_final <= 12) and log_domain <= the two-adicity
 * (ZNTT_ERR_ORDER_TOO_LARGE); a callback error or an alpha that is not a field element is
 * ZNTT_ERR_INVALID_ARGUMENT.  Returns after the last fold has finished.  All four fields. */
int zntt_fri_commit_phase(int field, uint32_t log_domain, uint32_t log_final, uint64_t* const* d_layers,
                          uint8_t* const* d_nodes, uint8_t* roots_out, zntt_fri_challenge_fn challenge, void* user,
                          void* stream);

/* The openings of buildQueries (libs/fri/src/root.zig:551-571) from the commit phase's
 * resident layers and trees, for num_queries positions e0 < 2^log_domain (the caller's
 * challengeU64() % 2^log_domain): per query q and round r < rounds, with
 * j = e0 mod 2^(log_domain - r - 1),
 *   values_out + (q rounds + r) 2 NB: toBytes(f_r[j]) || toBytes(f_r[j + half])
 *     (serializePair; NB = 32, 8 or 4 bytes),
 *   paths_out: the siblings of leaf j in tree r from the leaf level up
 *     (MerkleTree.prove, libs/merkle/src/merkle_tree.zig:206-233), log_domain - r - 1
 *     digests of 32 bytes, queries one after another and rounds in order within one.
 * Host outputs; the call waits for them. */
int zntt_fri_query_extract(int field, uint32_t log_domain, uint32_t rounds, const uint64_t* const* d_layers,
                           const uint8_t* const* d_nodes, const uint64_t* positions, size_t num_queries,
                           uint8_t* values_out, uint8_t* paths_out, void* stream);

/* ---- serving: a continuously batching request server ---------------------------
 * Requests carry pinned host buffers.  A worker thread admits them in FIFO
 * order while their device buffers fit the HBM budget, turns whatever is
 * admitted into one batch (one persistent launch) whenever one of `slots`
 * streams is free -- so new arrivals overlap on the device with batches
 * already running -- and posts completions with CLOCK_MONOTONIC timestamps.
 * Twiddle tables of every size served stay resident.  The server reserves
 * min(hbm_budget_bytes, 8 GiB) of device memory when it is created and carves
 * request buffers from it, reusing freed ones by size, so steady serving makes
 * no cudaMalloc (one issued while batches run can stall the worker for
 * hundreds of milliseconds); past that reserve, buffers come from the
 * library's pool.  `serial` runs one request at a time with plain per-pass
 * launches (the baseline batching is measured against). */
typedef struct zntt_server_config {
  int field;
  size_t hbm_budget_bytes;  /* device bytes for request buffers (inputs, outputs, scratch) */
  int slots;                /* batches in flight at once (streams) */
  int max_batch_jobs;       /* requests per batch */
  uint32_t max_items;       /* tiles per batch queue */
  int serial;               /* 1: one request at a time, plain launches */
  size_t max_batch_bytes;   /* a batch stops growing past this many input+output bytes
                               (0: 64 MiB); a larger request runs alone */
} zntt_server_config;
typedef struct zntt_request {
  int kind;                 /* ZNTT_JOB_NTT or ZNTT_JOB_COSET_LDE */
  int mode;                 /* NTT: ZNTT_FORWARD or ZNTT_INVERSE */
  uint32_t log_n;           /* transform size; coset extension: output size */
  uint32_t log_in;          /* coset extension: input size */
  const uint64_t* h_in;     /* pinned host input (2^log_n, or 2^log_in evaluations) */
  uint64_t* h_out;          /* pinned host output, 2^log_n elements */
  uint64_t shift[4];        /* coset extension: g, Montgomery form */
  uint64_t user_tag;
  uint64_t arrival_ns;      /* CLOCK_MONOTONIC arrival time, for latency */
} zntt_request;
typedef struct zntt_completion {
  uint64_t user_tag;
  int status;               /* ZNTT_OK or the failure */
  uint64_t arrival_ns, admit_ns, done_ns;
} zntt_completion;
typedef struct zntt_server_stats {
  uint64_t submitted, completed, rejected, batches, max_batch_jobs, max_inflight_jobs, peak_bytes, pending;
  uint64_t max_launch_ns;   /* longest host time spent forming and enqueueing one batch */
  uint64_t max_batch_ns;    /* longest enqueue-to-completion time of one batch */
} zntt_server_stats;
typedef struct zntt_server zntt_server;

int zntt_server_create(const zntt_server_config* cfg, zntt_server** out);
/* Queues a request (any thread, non-blocking); ZNTT_ERR_REJECTED if it can
 * never fit the budget. */
int zntt_server_submit(zntt_server* s, const zntt_request* r);
/* Moves up to `cap` completions to `out`, waiting up to wait_ms for one. */
int zntt_server_poll(zntt_server* s, zntt_completion* out, size_t cap, size_t* n, int wait_ms);
int zntt_server_stats_get(zntt_server* s, zntt_server_stats* st);
/* Finishes every queued request, then frees the server. */
int zntt_server_destroy(zntt_server* s);
/* CLOCK_MONOTONIC in nanoseconds (the clock of arrival_ns / done_ns). */
uint64_t zntt_now_ns(void);

/* ---- autotuner ------------------------------------------------------------------
 * Times every pass shape and stage count per pass for each log n in
 * [log_n_min, log_n_max] on this GPU, a forward and an inverse transform
 * each (one plan serves both directions), and keeps the fastest; plans use the
 * table from then on.  The table persists as JSON lines keyed by GPU name;
 * zntt_init loads the file named by ZNTT_TUNE_FILE when it exists. */
int zntt_autotune(int field, uint32_t log_n_min, uint32_t log_n_max);
int zntt_tune_save(const char* path);
int zntt_tune_load(const char* path);
int zntt_tune_clear(void);

/* Transforms `count` host vectors of 2^log_n elements (log_n of the table) in
 * place, nttWithTwiddles / inttWithTwiddles semantics, overlapping each
 * vector's host<->device copies with its neighbours' transforms (three
 * streams, both copy engines).  Synchronous; pinned host memory gives full
 * PCIe bandwidth. */
int zntt_ntt_host_many(const zntt_twiddles* tw, uint64_t* const* h_data, size_t count, int mode);

/* Seeded uniform elements on the device: element i is the i-th
 * randomFieldElement draw (libs/rng/src/rng.zig:32-65) from the ChaCha20
 * stream keyed by seed32 with a zero nonce and counter from 0
 * (libs/rng/src/chacha20.zig:81-110), in Montgomery form. */
int zntt_random_elements(int field, const uint8_t seed32[32], uint64_t* d_out, size_t count, void* stream);

/* Elementwise device arithmetic (op 0 mul, 1 add, 2 sub, 3 neg) over `count`
 * device elements; exposed for the arithmetic parity tests. */
int zntt_elementwise_device(int field, int op, const uint64_t* d_a, const uint64_t* d_b, uint64_t* d_out,
                            size_t count, void* stream);

/* ---- roofline probes ---------------------------------------------------------
 * Throughput of the multiply pipe and of the field product on this device,
 * measured with CUDA events.  zntt_probe_imad counts dependent 32-bit
 * multiply-adds (mad.lo.u32), the multiply pipe's unit of issue; a full
 * 32x32->64 product takes two, so an 8x32-bit CIOS product (136 products)
 * takes 272 and imad_per_second / 272 is the modmul roofline. */
int zntt_probe_imad(double* imad_per_second);
/* 32x32->64 multiply-adds (mad.wide.u32) per second: one 8x32-bit CIOS
 * product needs 2*8*8 + 8 = 136 of them, so this / 136 is the modmul ceiling. */
int zntt_probe_mul_wide(double* products_per_second);
/* Single-block BLAKE3 compressions per second, chained in registers with the
 * instruction mix of the commitment's node levels and no memory traffic: the
 * roofline of zntt_fri_commit_layer, which makes n - 1 compressions. */
int zntt_probe_blake3(double* compressions_per_second);
int zntt_probe_modmul(int field, double* modmul_per_second);

#ifdef __cplusplus
}
#endif

#endif /* ZNTT_H */
