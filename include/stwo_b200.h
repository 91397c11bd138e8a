/*
 * stwo_b200 — B200-native (sm_100a) backend for stwo's Circle-STARK commit +
 * FRI path.  Flat C ABI: plain pointers and sizes, no torch types.
 *
 * Conventions
 *  - Every entry point returns 0 on success or a negative STWO_B200_E* code,
 *    and writes a NUL-terminated message into (err, err_len) when err != NULL.
 *    No entry point aborts the process.
 *  - Pointers named d_* are device pointers on the context's device.  Arrays
 *    of device pointers (e.g. `uint32_t* const* d_cols`) are HOST arrays whose
 *    elements are device pointers.
 *  - `stream` is a cudaStream_t passed as void* (NULL = legacy default
 *    stream).  Work is enqueued; nothing synchronises unless documented.
 *  - Field elements are u32 words: M31 in [0, 2^31-1); QM31 columns are four
 *    M31 coordinate columns (SecureColumnByCoords layout).
 *  - Columns are evaluations in bit-reversed circle-domain order, or
 *    coefficients in natural order (CpuBackend order), exactly as stwo's
 *    CircleEvaluation<_, _, BitReversedOrder> / CircleCoefficients.
 *  - Twiddle trees use CpuBackend's layout with canonical values (SimdBackend
 *    stores the same values doubled): 2^R words for a root coset of log size
 *    R.  Every domain used with a tree must be a doubling of its root coset.
 *
 * Reference interfaces replaced (paths relative to the vendored stwo crate
 * vendor/stwo-upstream-dev-62b228e/crates/stwo/src/ of teddyjfpender/stwo-metal,
 * and to crates/stwo-metal-sys/src/raw.rs for the reference's CUDA ABI):
 */
#ifndef STWO_B200_H
#define STWO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  STWO_B200_OK = 0,
  STWO_B200_EARG = -1,     /* invalid argument (size, alignment, null) */
  STWO_B200_ECUDA = -2,    /* CUDA runtime error */
  STWO_B200_ENOMEM = -3,   /* device allocation failed */
  STWO_B200_ETIMEOUT = -4, /* a bounded device wait gave up */
  STWO_B200_ESTATE = -5    /* call not valid in the current state */
};

/* ------------------------------------------------------------ runtime --- */
/* Library version string. */
const char* stwo_b200_version(void);

/* Number of kernels launched by this library since load (all threads). */
uint64_t stwo_b200_launch_count(void);

/* Selects `device`, checks it is sm_100 and prepares the stream-ordered
 * memory pool.  Replaces the reference's global runtime probe
 * (crates/stwo-metal-sys/src/metal.rs:4424-4448 metal_runtime_support). */
int stwo_b200_init(int device, char* err, size_t err_len);

/* Device memory from the stream-ordered pool (cudaMallocAsync).  Replaces
 * cuda_malloc_uint32_t / cuda_free_memory (raw.rs:57,71). */
int stwo_b200_alloc(size_t bytes, void** d_out, void* stream, char* err, size_t err_len);
int stwo_b200_free(void* d_ptr, void* stream, char* err, size_t err_len);
/* Async copies; host buffers should be pinned for overlap.  Replace
 * copy_uint32_t_vec_from_{host_to_device,device_to_host} (raw.rs:43-50). */
int stwo_b200_memcpy_h2d(void* d_dst, const void* h_src, size_t bytes, void* stream, char* err, size_t err_len);
int stwo_b200_memcpy_d2h(void* h_dst, const void* d_src, size_t bytes, void* stream, char* err, size_t err_len);
int stwo_b200_memcpy_d2d(void* d_dst, const void* d_src, size_t bytes, void* stream, char* err, size_t err_len);
int stwo_b200_memset(void* d_dst, int value, size_t bytes, void* stream, char* err, size_t err_len);
int stwo_b200_stream_create(void** stream_out, char* err, size_t err_len);
int stwo_b200_stream_destroy(void* stream, char* err, size_t err_len);
int stwo_b200_stream_sync(void* stream, char* err, size_t err_len);
/* Pinned host memory for the e2e copies. */
int stwo_b200_host_alloc(size_t bytes, void** h_out, char* err, size_t err_len);
int stwo_b200_host_free(void* h_ptr, char* err, size_t err_len);

/* ------------------------------------------------------------ ColumnOps -- */
/* ColumnOps<BaseField>::bit_reverse_column (prover/backend/mod.rs:37-39;
 * SimdBackend prover/backend/simd/bit_reverse.rs:22-33), in place.  Replaces
 * bit_reverse_base_field (raw.rs:77). */
int stwo_b200_bit_reverse_column(uint32_t* d_col, uint32_t log_size, void* stream, char* err, size_t err_len);
/* bit_reverse_column over many columns in one launch per run of equal sizes
 * (the loop over columns that callers of prover/backend/mod.rs:37-39 write):
 * out of place (d_dst[i] <- bit-reversed d_src[i]) or in place where
 * d_dst[i] == d_src[i].  Columns of one run must not overlap. */
int stwo_b200_bit_reverse_columns(const uint32_t* const* d_src, uint32_t* const* d_dst, const uint32_t* log_sizes,
                                  uint32_t n_cols, void* stream, char* err, size_t err_len);

/* -------------------------------------------------------------- PolyOps -- */
/* PolyOps::precompute_twiddles (prover/poly/circle/ops.rs:144; SimdBackend
 * prover/backend/simd/circle.rs:449-486) for the coset
 * (initial_index, log_size): writes 2^log_size twiddles and their inverses.
 * Replaces precompute_twiddles (raw.rs:84-88). */
int stwo_b200_precompute_twiddles(uint64_t initial_index, uint32_t log_size, uint32_t* d_twiddles,
                                  uint32_t* d_itwiddles, void* stream, char* err, size_t err_len);

/* PolyOps::interpolate_columns (prover/poly/circle/ops.rs:29-40 ->
 * PolyOps::interpolate ops.rs:24, simd/circle.rs:138-166): in place, evaluation ->
 * coefficients, for n_cols columns of sizes 2^log_sizes[i] on canonic
 * circle domains.  `half_initial_indices` may be NULL (canonic domains) or
 * give each domain's half-coset initial index (only read for log size <= 2).
 * Replaces ntt_b2n_column (raw.rs:472-479). */
int stwo_b200_interpolate_columns(uint32_t* const* d_cols, const uint32_t* log_sizes,
                                  const uint64_t* half_initial_indices, uint32_t n_cols, const uint32_t* d_itwiddles,
                                  uint32_t tree_log_size, void* stream, char* err, size_t err_len);

/* Out-of-place form of stwo_b200_interpolate_columns: reads d_evals[i],
 * writes d_coeffs[i] (stwo's interpolate consumes its evaluation; this form
 * leaves it intact at no extra traffic). */
int stwo_b200_interpolate_columns_into(const uint32_t* const* d_evals, uint32_t* const* d_coeffs,
                                       const uint32_t* log_sizes, const uint64_t* half_initial_indices,
                                       uint32_t n_cols, const uint32_t* d_itwiddles, uint32_t tree_log_size,
                                       void* stream, char* err, size_t err_len);

/* Interpolation of natural-order evaluations: the pair
 * CircleEvaluation<_, _, NaturalOrder>::bit_reverse (core/poly/circle/
 * evaluation.rs:61-64, i.e. ColumnOps::bit_reverse_column) + PolyOps::interpolate
 * in one call.  Reads d_natural[i] (natural order), writes d_coeffs[i].  Where
 * every column of a size is out of place (d_natural[i] != d_coeffs[i]) and the
 * size is >= 3, the bit reversal is done by the loads of the first FFT pass;
 * otherwise by one batched bit-reversal launch into d_coeffs first.  In place
 * (d_natural[i] == d_coeffs[i]) is allowed. */
int stwo_b200_interpolate_columns_natural(const uint32_t* const* d_natural, uint32_t* const* d_coeffs,
                                          const uint32_t* log_sizes, const uint64_t* half_initial_indices,
                                          uint32_t n_cols, const uint32_t* d_itwiddles, uint32_t tree_log_size,
                                          void* stream, char* err, size_t err_len);

/* PolyOps::evaluate_polynomials (prover/poly/circle/ops.rs:110-211 ->
 * evaluate_into, simd/circle.rs:388-443): coefficients (2^log_sizes[i]) ->
 * evaluations on CanonicCoset(log_sizes[i] + log_blowup), bit-reversed.
 * Replaces evaluate_columns (raw.rs:90-97). */
int stwo_b200_evaluate_polynomials(const uint32_t* const* d_coeffs, const uint32_t* log_sizes, uint32_t n_cols,
                                   uint32_t log_blowup, uint32_t* const* d_evals, const uint32_t* d_twiddles,
                                   uint32_t tree_log_size, void* stream, char* err, size_t err_len);

/* stwo_b200_interpolate_columns followed by stwo_b200_evaluate_polynomials
 * for n_cols columns of one log size, as CommitmentTreeProver::new runs them
 * for a trace (crates/stwo/src/prover/pcs/mod.rs:707-781): reads d_src[i]
 * (bit-reversed evaluations on CanonicCoset(log_size); d_src NULL: d_coeffs
 * holds them and is transformed in place), writes the coefficients to
 * d_coeffs[i] and their evaluations on CanonicCoset(log_size + log_blowup)
 * to d_evals[i].  Same words as the two calls; the interpolation's last pass
 * and the evaluation's first run as one kernel where the pass plan allows
 * (a last pass of 10 layers starting at layer 10, 11 or 12: log sizes 20
 * and 21 by default; blowup 1 or 2).  No single reference
 * counterpart: the reference runs ntt_b2n_column then evaluate_columns
 * (raw.rs:472-479, 90-97). */
int stwo_b200_interpolate_evaluate_columns(const uint32_t* const* d_src, uint32_t* const* d_coeffs,
                                           uint32_t* const* d_evals, uint32_t n_cols, uint32_t log_size,
                                           uint32_t log_blowup, const uint32_t* d_itwiddles, const uint32_t* d_twiddles,
                                           uint32_t tree_log_size, void* stream, char* err, size_t err_len);

/* ------------------------------------------------------ MerkleOpsLifted -- */
/* MerkleOpsLifted<Blake2sMerkleHasherGeneric<m31_output>>::build_leaves
 * (prover/vcs_lifted/ops.rs:14-15; spec prover/backend/cpu/merkle_lifted.rs:
 * 44-78).  Columns must already be sorted by non-decreasing log size.
 * Writes 2^lifting_log_size 32-byte leaves (1 leaf when n_cols == 0).
 * Columns of more than one size hash in stages, as SimdBackend does
 * (backend/simd/blake2s_lifted.rs:42-160); the chaining values between
 * stages take a stream-ordered temporary of 32 * 2^lifting_log_size bytes
 * (build_leaves_layers below takes the tree's layers instead), and one more
 * of that size when more than 1024 columns hash at the lifting size.
 * Replaces commit_on_first_layer_lifted (raw.rs:176-183). */
int stwo_b200_merkle_build_leaves(const uint32_t* const* d_cols, const uint32_t* log_sizes, uint32_t n_cols,
                                  uint32_t lifting_log_size, int m31_output, uint8_t* d_leaves, void* stream,
                                  char* err, size_t err_len);

/* MerkleOpsLifted::build_next_layer (prover/vcs_lifted/ops.rs:19;
 * cpu/merkle_lifted.rs:80-85): 2^prev_log_size hashes -> half as many. */
int stwo_b200_merkle_build_next_layer(const uint8_t* d_prev, uint32_t prev_log_size, int m31_output,
                                      uint8_t* d_out, void* stream, char* err, size_t err_len);

/* MerkleOpsLifted::build_merkle_layers (prover/vcs_lifted/ops.rs:29-45):
 * stable-sorts the columns by length, builds leaves and all node layers.
 * d_layers[k] (k = 0..lifting_log_size, root first) receives 2^k hashes. */
int stwo_b200_merkle_build_layers(const uint32_t* const* d_cols, const uint32_t* log_sizes, uint32_t n_cols,
                                  uint32_t lifting_log_size, int m31_output, uint8_t* const* d_layers,
                                  void* stream, char* err, size_t err_len);

/* Node layers of a lifted tree whose leaves are already in
 * d_layers[lifting_log_size]: fills d_layers[lifting_log_size-1 .. 0]
 * (the second half of build_merkle_layers, prover/vcs_lifted/ops.rs:39-43). */
int stwo_b200_merkle_build_nodes(uint8_t* const* d_layers, uint32_t lifting_log_size, int m31_output,
                                 void* stream, char* err, size_t err_len);

/* The first half of build_merkle_layers (prover/vcs_lifted/ops.rs:37-38):
 * build_leaves of columns already sorted by non-decreasing log size into
 * d_layers[lifting_log_size], with d_layers[k] (k < lifting_log_size, 2^k
 * hashes each) as the chaining values between the hashing stages, so that
 * nothing is allocated unless more than 1024 columns hash at the lifting
 * size.  build_nodes overwrites d_layers[k < lifting_log_size] afterwards. */
int stwo_b200_merkle_build_leaves_layers(const uint32_t* const* d_cols, const uint32_t* log_sizes, uint32_t n_cols,
                                         uint32_t lifting_log_size, int m31_output, uint8_t* const* d_layers,
                                         void* stream, char* err, size_t err_len);

/* Throughput probe (no reference counterpart): `blocks` x 256 threads each
 * chain `iters` Blake2s compressions in registers.  compressions / elapsed
 * time is the integer-pipe ceiling the leaf kernel is measured against. */
int stwo_b200_blake2s_probe(uint32_t blocks, uint32_t iters, uint32_t* d_out, void* stream, char* err,
                            size_t err_len);

/* Throughput probe (no reference counterpart): `blocks` x 256 threads each
 * apply `iters` rounds of 80 M31 butterflies (the FFT passes' arithmetic) to
 * 32 register-held values.  80 * iters * threads / elapsed time is the
 * integer-issue ceiling the FFT passes are measured against. */
int stwo_b200_butterfly_probe(uint32_t blocks, uint32_t iters, uint32_t* d_out, void* stream, char* err,
                              size_t err_len);

/* ------------------------------------------------------------ MerkleOps -- */
/* MerkleOps<Blake2sMerkleHasherGeneric<m31_output>>::commit_on_layer
 * (prover/vcs/ops.rs:24-28; cpu/blake2s.rs:13-26): node i = Blake2s(
 * prev[2i] || prev[2i+1] (when d_prev != NULL) || LE32(col[i]) for cols).
 * Replaces commit_on_layer_with_previous / commit_on_first_layer
 * (raw.rs:169-190). */
int stwo_b200_commit_on_layer(uint32_t log_size, const uint8_t* d_prev, const uint32_t* const* d_cols,
                              uint32_t n_cols, int m31_output, uint8_t* d_out, void* stream, char* err,
                              size_t err_len);

/* -------------------------------------------------------------- FriOps --- */
/* FriOps::fold_line (prover/fri.rs:39-50; simd/fri.rs:32-122): 4 coordinate
 * columns of a line evaluation of size 2^log_size on a domain in the tree's
 * tower -> 2^(log_size - fold_step).  alpha = 4 M31 words.
 * Replaces fold_line (raw.rs:142-149). */
int stwo_b200_fold_line(const uint32_t* const* d_in4, uint32_t log_size, const uint32_t* alpha,
                        uint32_t fold_step, const uint32_t* d_itwiddles, uint32_t tree_log_size,
                        uint32_t* const* d_out4, void* stream, char* err, size_t err_len);

/* FriOps::fold_circle_into_line (prover/fri.rs:61-69; simd/fri.rs:124-172):
 * dst (2^(log_size-1)) <- dst * alpha^2 + fold(src (2^log_size)).
 * `half_initial_index` is the source circle domain's half-coset initial
 * index (read only for log_size <= 4).  Replaces fold_circle_into_line
 * (raw.rs:151-158). */
int stwo_b200_fold_circle_into_line(uint32_t* const* d_dst4, const uint32_t* const* d_src4, uint32_t log_size,
                                    uint64_t half_initial_index, const uint32_t* alpha,
                                    const uint32_t* d_itwiddles, uint32_t tree_log_size, void* stream, char* err,
                                    size_t err_len);

/* FriOps::decompose (prover/fri.rs:92-104; simd/fri.rs:174-195,265-296):
 * g = f -/+ lambda; lambda (4 words) is written to host memory (the call
 * synchronises `stream`). */
int stwo_b200_decompose(const uint32_t* const* d_in4, uint32_t log_size, uint32_t* const* d_out4,
                        uint32_t* lambda_out, void* stream, char* err, size_t err_len);

/* FriOps::decompose without device allocation.  No counterpart in the
 * reference: for callers that cannot let the library allocate device memory
 * mid-run (a prover service whose admission controller has already divided
 * HBM between requests, or a host runtime that owns every device
 * allocation).  Same results as stwo_b200_decompose; the reduction scratch
 * (18,960 bytes) is a fixed device array that every GPU loading the library
 * keeps until exit.  Inputs up to 2^30 elements per coordinate; larger sizes
 * are rejected.  The first call on a device looks up the array's device
 * address and caches it per device (a cudaDeviceReset between calls is not
 * supported).  Calls share the array: calls that overlap on the GPU race.
 * Like stwo_b200_decompose, the call synchronises `stream` before it
 * returns, to hand lambda to the host. */
int stwo_b200_decompose_noalloc(const uint32_t* const* d_in4, uint32_t log_size, uint32_t* const* d_out4,
                                uint32_t* lambda_out, void* stream, char* err, size_t err_len);

/* --------------------------------------------- QuotientOps (PCS quotients) */
/* One term of a sample batch: column d_cols[column_index] sampled to
 * sample_value (QM31) with random coefficient random_coeff (QM31): the
 * NumeratorData of core/pcs/quotients.rs:63-71. */
typedef struct stwo_b200_numerator_term {
  uint32_t column_index;
  uint32_t sample_value[4];
  uint32_t random_coeff[4];
} stwo_b200_numerator_term;
/* ColumnSampleBatch (core/pcs/quotients.rs:55-61): the point
 * CirclePoint<SecureField> as 8 words (x then y, 4 each) and its terms (host). */
typedef struct stwo_b200_sample_batch {
  uint32_t point[8];
  const stwo_b200_numerator_term* terms;
  uint32_t n_terms;
} stwo_b200_sample_batch;

/* QuotientOps::accumulate_numerators (prover/pcs/quotient_ops.rs:22-33;
 * SimdBackend prover/backend/simd/quotients.rs:34-71, 124-134) for n_cols
 * device columns of 2^log_size words (bit-reversed evaluations): for batch b,
 * d_out[4b .. 4b+3] (the 4 coordinate columns of its partial numerator, 2^log_size
 * words each) receive sum_i (c_i * col_i[p] - b_i) at every row p, and
 * first_linear_term_out[4b .. 4b+3] (host) receives sum_i a_i, where
 * (a_i, b_i, c_i) are the complex-conjugate line coefficients of the term
 * times its random coefficient (core/constraints.rs:119-134).  No reference
 * CUDA-ABI counterpart (the reference computed quotients on the host). */
int stwo_b200_accumulate_numerators(const uint32_t* const* d_cols, uint32_t n_cols, uint32_t log_size,
                                    const stwo_b200_sample_batch* batches, uint32_t n_batches, uint32_t* const* d_out,
                                    uint32_t* first_linear_term_out, void* stream, char* err, size_t err_len);

/* AccumulatedNumerators (prover/pcs/quotient_ops.rs:48-74) of one sample point:
 * the partial numerator's 4 device coordinate columns of 2^log_size words and
 * the first linear term. */
typedef struct stwo_b200_accumulated_numerators {
  uint32_t sample_point[8];
  const uint32_t* d_partial[4];
  uint32_t log_size;
  uint32_t first_linear_term[4];
} stwo_b200_accumulated_numerators;

/* QuotientOps::compute_quotients_and_combine (quotient_ops.rs:35-45;
 * simd/quotients.rs:73-164): on the bit-reversed CanonicCoset(lifting_log_size)
 * domain, d_out4 (4 coordinate columns of 2^lifting_log_size words) receives
 * sum_z (lift(num_z) - A_z * p.y) / den_z(p), each partial numerator lifted
 * to the lifting size (l(i, r) = ((i >> (r + 1)) << 1) + (i & 1)). */
int stwo_b200_compute_quotients_and_combine(const stwo_b200_accumulated_numerators* accs, uint32_t n_accs,
                                            uint32_t lifting_log_size, uint32_t* const* d_out4, void* stream,
                                            char* err, size_t err_len);

/* ----------------------------------------------------- AccumulationOps -- */
/* AccumulationOps::accumulate (prover/air/accumulation.rs:127-130;
 * simd/accumulation.rs:13-18): column += other, coordinate-wise, `len`
 * elements (4 coordinate columns each). */
int stwo_b200_accumulate(uint32_t* const* d_col4, const uint32_t* const* d_other4, uint64_t len, void* stream,
                         char* err, size_t err_len);
/* AccumulationOps::generate_secure_powers (accumulation.rs:132-133;
 * simd/accumulation.rs:20-39): d_out (device, 16-byte aligned) receives
 * felt^0 .. felt^(n_powers-1), 4 words each. */
int stwo_b200_generate_secure_powers(const uint32_t* felt, uint32_t n_powers, uint32_t* d_out, void* stream,
                                     char* err, size_t err_len);
/* AccumulationOps::lift_and_accumulate (accumulation.rs:135-145;
 * simd/accumulation.rs:45-80): n_cols secure columns (d_cols4[4k .. 4k+3],
 * 2^log_sizes[k] words each, log sizes strictly increasing) -> d_out4 (the
 * size of the last; may be the last column itself) = the coordinate-wise sum
 * of every column lifted to that size.  Columns of fewer than 16 elements
 * take part in the sum as the trait defines it (SimdBackend's packed loop
 * would leave such a column out). */
int stwo_b200_lift_and_accumulate(const uint32_t* const* d_cols4, const uint32_t* log_sizes, uint32_t n_cols,
                                  uint32_t* const* d_out4, void* stream, char* err, size_t err_len);

/* ------------------------------------------------- PolyOps::eval_at_point */
/* PolyOps::batch_eval_at_point (prover/poly/circle/ops.rs:44-63;
 * simd/circle.rs:168-230): n_polys polynomials of 2^log_size natural-order
 * coefficients (device) at the point (8 words: x, y) -> values_out (host,
 * 4 words per polynomial).  Synchronises `stream`.  Replaces the reference's
 * Metal eval_at_point kernels (crates/stwo-metal-sys/metal/eval_at_point.metal). */
int stwo_b200_batch_eval_at_point(const uint32_t* const* d_coeffs, uint32_t n_polys, uint32_t log_size,
                                  const uint32_t* point, uint32_t* values_out, void* stream, char* err,
                                  size_t err_len);
/* PolyOps::eval_at_point (ops.rs:44-48) of one polynomial. */
int stwo_b200_eval_at_point(const uint32_t* d_coeffs, uint32_t log_size, const uint32_t* point, uint32_t* value_out,
                            void* stream, char* err, size_t err_len);

/* ---------------------------------------------------------- GrindOps ----- */
/* GrindOps<Blake2sChannel(Generic)>::grind (prover/backend/simd/grind.rs:25-96)
 * from the channel's 32-byte digest: the smallest nonce (hi << 32) | low,
 * low < 2^20, whose Blake2s hash after the proof-of-work prefix has at least
 * pow_bits (<= 32) trailing zeros.  m31_channel selects
 * Blake2sM31Channel.  Synchronises `stream`. */
int stwo_b200_grind(const uint8_t* digest, uint32_t pow_bits, int m31_channel, uint64_t* nonce_out, void* stream,
                    char* err, size_t err_len);

/* ------------------------------------------------ ColumnOps<SecureField> */
/* ColumnOps<SecureField>::bit_reverse_column (prover/backend/mod.rs:37-39) of
 * a secure column stored as 4 coordinate columns (SecureColumnByCoords), in
 * place. */
int stwo_b200_bit_reverse_secure_column(uint32_t* const* d_coords4, uint32_t log_size, void* stream, char* err,
                                        size_t err_len);
/* The same for QM31 values stored 4 words each (16-byte aligned), in place.
 * Replaces bit_reverse_secure_field (raw.rs:86). */
int stwo_b200_bit_reverse_secure_field(uint32_t* d_values, uint32_t log_size, void* stream, char* err,
                                       size_t err_len);

/* --------------------------------------------------------- FFT pass plans */
/* Pass plan of every n-layer circle FFT: n_passes (1-4) layer counts of 1-12,
 * low layers first, summing to n; the first at least 3 when there are several
 * (the later passes are strided).  n_passes = 0 restores the default split.
 * Process-wide; results do not depend on the plan.  No reference counterpart:
 * the SIMD backend's radix-8 loop structure is fixed (simd/fft/ifft.rs:33-57);
 * these are the autotuner's knobs. */
int stwo_b200_fft_set_plan(uint32_t log_size, const uint32_t* pass_layers, uint32_t n_passes, char* err,
                           size_t err_len);
int stwo_b200_fft_get_plan(uint32_t log_size, uint32_t* pass_layers, uint32_t cap, uint32_t* n_passes, char* err,
                           size_t err_len);

/* --------------------------------------------------------- trace commit -- */
/* CommitmentTreeProver::new for one column set (crates/stwo/src/prover/pcs/
 * mod.rs:707-781): interpolate_columns (prover/poly/circle/ops.rs:29-40) from
 * bit-reversed canonic-coset evaluations, evaluate_polynomials on the
 * log_blowup domain (ops.rs:110-211), then the lifted Blake2s tree of the
 * evaluations (prover/vcs_lifted/prover.rs:33-42) with lifting log size
 * max(log_sizes) + log_blowup.  flags: */
#define STWO_B200_COMMIT_PER_COLUMN 1u /* launches per column (the plain form) */
#define STWO_B200_COMMIT_GRAPH 2u      /* capture once per buffer set, replay */
typedef struct stwo_b200_committer stwo_b200_committer;
int stwo_b200_committer_create(const uint32_t* log_sizes, uint32_t n_cols, uint32_t log_blowup, int m31_output,
                               const uint32_t* d_twiddles, const uint32_t* d_itwiddles, uint32_t tree_log_size,
                               uint32_t flags, stwo_b200_committer** out, char* err, size_t err_len);
int stwo_b200_committer_destroy(stwo_b200_committer* committer, char* err, size_t err_len);
int stwo_b200_committer_lifting_log_size(const stwo_b200_committer* committer, uint32_t* out, char* err,
                                         size_t err_len);
/* d_evals[i]: column i (2^log_sizes[i] words, read only); d_coeffs[i] and
 * d_ldes[i] (2^(log_sizes[i]+log_blowup) words) receive its coefficients and
 * evaluations; d_layers[k] (2^k hashes of 32 bytes, k = 0..lifting log size)
 * the tree, root first.  Ordered after the work already on `stream`, and the
 * work on `stream` after it. */
int stwo_b200_committer_commit(stwo_b200_committer* committer, const uint32_t* const* d_evals,
                               uint32_t* const* d_coeffs, uint32_t* const* d_ldes, uint8_t* const* d_layers,
                               void* stream, char* err, size_t err_len);
/* committer_commit with the columns in host memory (h_evals[i], 2^log_sizes[i]
 * words; pinned memory for asynchronous copies): copies them into d_evals one
 * log-size group at a time, largest first, on the committer's copy stream, and
 * transforms each group as soon as its copies land, so the transforms overlap
 * the remaining copies.  The same outputs as committer_commit on the same
 * columns.  Ordered after the work already on `stream`, and the work on
 * `stream` after it. */
int stwo_b200_committer_commit_from_host(stwo_b200_committer* committer, const uint32_t* const* h_evals,
                                         uint32_t* const* d_evals, uint32_t* const* d_coeffs, uint32_t* const* d_ldes,
                                         uint8_t* const* d_layers, void* stream, char* err, size_t err_len);
/* Times every candidate pass plan of each (log_size, column count) group of
 * the committer on these buffers (reps timed runs each) and keeps the fastest
 * as the process-wide plan; cache_path (optional) is read first and written
 * with the choices ("log_size n_columns T1,T2,..." per line).  Clobbers
 * d_coeffs and d_ldes.  No reference counterpart. */
int stwo_b200_committer_autotune(stwo_b200_committer* committer, const uint32_t* const* d_evals,
                                 uint32_t* const* d_coeffs, uint32_t* const* d_ldes, const char* cache_path,
                                 uint32_t reps, char* err, size_t err_len);

/* ----------------------------------------------------- Wide-Fibonacci prove */
/* PcsConfig + FriConfig fields of crates/stwo/src/core/pcs/mod.rs:31-80 and
 * core/fri.rs:31-80 (defaults: pow_bits 10, log_blowup 1, n_queries 3,
 * log_last_layer_degree_bound 0, line_fold_step 1), plus the AIR shape
 * (examples/src/wide_fibonacci/mod.rs:80-101) and the channel flavour
 * (0 = Blake2sMerkleChannel, 1 = Blake2sM31MerkleChannel). */
typedef struct stwo_b200_wide_fib_config {
  uint32_t log_n_rows;
  uint32_t n_cols;
  uint32_t log_blowup;
  uint32_t pow_bits;
  uint32_t n_queries;
  uint32_t log_last_layer_degree_bound;
  uint32_t line_fold_step;
  int32_t m31_channel;
} stwo_b200_wide_fib_config;

/* A prover owns every device buffer of one proof shape (twiddles, trace,
 * trees, FRI layers) and reuses them across proofs on `stream`. */
typedef struct stwo_b200_prover stwo_b200_prover;
int stwo_b200_prover_create(const stwo_b200_wide_fib_config* cfg, stwo_b200_prover** out, void* stream, char* err,
                            size_t err_len);
int stwo_b200_prover_destroy(stwo_b200_prover* prover, char* err, size_t err_len);

/* stwo::prover::prove::<B200Backend, Blake2sMerkleChannel> of the
 * Wide-Fibonacci component (crates/stwo/src/prover/mod.rs:32-138, driven as in
 * the reference harness fixtures/standalone-benchmarks/src/bin/
 * wide_fibonacci_simd_prove.rs:117-150: empty preprocessed tree, trace tree,
 * prove).  d_a / d_b: the first two trace columns (2^log_n_rows words each,
 * device memory).  Writes the canonical proof bytes to proof_out (host) when
 * non-NULL and its length to *proof_len.  Synchronises the prover's stream. */
int stwo_b200_prove_wide_fib(stwo_b200_prover* prover, const uint32_t* d_a, const uint32_t* d_b,
                             uint8_t* proof_out, size_t proof_cap, size_t* proof_len, char* err, size_t err_len);

/* stwo_b200_prove_wide_fib with the two input columns in HOST memory (the
 * same bytes out).  The prover copies them in 4 row chunks on its own copy
 * stream and generates each chunk's trace rows as soon as the chunk lands, so
 * with pinned (page-locked) inputs the host-to-device copy overlaps the trace
 * generation; pageable inputs are copied synchronously.  The first call
 * allocates a 2 x 2^log_n_rows-word input buffer and the copy stream. */
int stwo_b200_prove_wide_fib_host(stwo_b200_prover* prover, const uint32_t* h_a, const uint32_t* h_b,
                                  uint8_t* proof_out, size_t proof_cap, size_t* proof_len, char* err, size_t err_len);

/* The same proof with n_cols (3..the prover's n_cols) trace columns: the
 * buffers are sized for the prover's n_cols and any narrower trace of the
 * same log_n_rows reuses them.  No reference counterpart (a resident prover
 * of the serving loop). */
int stwo_b200_prove_wide_fib_cols(stwo_b200_prover* prover, uint32_t n_cols, const uint32_t* d_a,
                                  const uint32_t* d_b, uint8_t* proof_out, size_t proof_cap, size_t* proof_len,
                                  char* err, size_t err_len);
/* Device bytes a prover of this configuration allocates (computed, nothing is
 * allocated; host-only, needs no GPU).  For HBM admission. */
int stwo_b200_prover_footprint(const stwo_b200_wide_fib_config* cfg, size_t* device_bytes, char* err,
                               size_t err_len);

/* Per-phase device time (CUDA events on the prover's stream), accumulated over
 * the proofs made since timing was enabled.  Phases, in order: 0 trace
 * generation, 1 trace interpolate, 2 trace evaluate, 3 trace Merkle,
 * 4 composition, 5 composition interpolate, 6 composition evaluate,
 * 7 composition Merkle, 8 OODS sampling, 9 FRI quotients, 10 FRI Merkle,
 * 11 FRI folds, 12 grind, 13 decommit (each phase spans to the next one,
 * host channel work included).  No reference counterpart (the reference's
 * env-gated timers STWO_METAL_PROFILE_* play this role). */
int stwo_b200_prover_set_timing(stwo_b200_prover* prover, int enable, char* err, size_t err_len);
int stwo_b200_prover_phase_times(stwo_b200_prover* prover, double* ms_out, uint32_t n, uint32_t* proofs, char* err,
                                 size_t err_len);

/* Wait bound of the prover's column-streaming kernels (composition,
 * quotients): a consumer warp polls a stage's mbarrier at most `polls` times
 * before it gives up, sets the prover's error flag and leaves; the prove then
 * returns STWO_B200_ETIMEOUT.  0 gives up at the first wait (every such
 * prove fails); STWO_B200_STREAM_SPIN_DEFAULT restores the default.  The
 * producer's own waits, including its wait for copies still in flight before
 * its block exits, keep the default bound.  No reference counterpart: this
 * exercises the failure path of the bounded device waits. */
#define STWO_B200_STREAM_SPIN_DEFAULT (1u << 22)
int stwo_b200_prover_set_stream_spin(stwo_b200_prover* prover, uint32_t polls, char* err, size_t err_len);

/* ---------------------------------------------------------- serving ------ */
/* Continuous batching of Wide-Fibonacci prove requests on the current GPU
 * (no reference counterpart: the reference proves one request at a time).
 * `slots` requests run at once, each on its own resident prover and stream;
 * provers (buffers, twiddles, captured FRI graph) stay resident per (log_n,
 * width class = n_cols rounded up to a multiple of 64, PCS config) and are
 * evicted least recently used when a new one must fit hbm_budget_bytes.  A
 * request waits until a slot is free and its prover is idle or fits; the
 * queue is scanned in arrival order.  A proof is the same as when the request
 * is proved alone. */
typedef struct stwo_b200_server stwo_b200_server;
typedef struct stwo_b200_server_stats {
  uint64_t completed, provers_created, provers_reused, provers_evicted;
  uint64_t resident_bytes;
  uint32_t residents, max_running, queued, pad;
} stwo_b200_server_stats;
int stwo_b200_server_create(size_t hbm_budget_bytes, uint32_t slots, stwo_b200_server** out, char* err,
                            size_t err_len);
/* Finishes every submitted request, then frees the resident provers. */
int stwo_b200_server_destroy(stwo_b200_server* server, char* err, size_t err_len);
/* Copies the two input columns (host, 2^log_n_rows words each) and queues the
 * request; fails at once when its prover could never fit the budget. */
int stwo_b200_server_submit(stwo_b200_server* server, const stwo_b200_wide_fib_config* cfg, const uint32_t* a,
                            const uint32_t* b, uint64_t* ticket, char* err, size_t err_len);
/* Blocks until the request is done; writes its proof and, when times_ms is
 * non-NULL, [queued, on a prover, latency] in milliseconds.  Returns the
 * request's own status. */
int stwo_b200_server_wait(stwo_b200_server* server, uint64_t ticket, uint8_t* proof_out, size_t proof_cap,
                          size_t* proof_len, double* times_ms, char* err, size_t err_len);
int stwo_b200_server_get_stats(stwo_b200_server* server, stwo_b200_server_stats* out, char* err, size_t err_len);

/* ------------------------------------------------ FRI commit + decommit -- */
/* FriProver::commit + decommit (crates/stwo/src/prover/fri.rs:133-350) of one
 * secure column on CanonicCoset(log_size), with the folding alphas supplied
 * instead of drawn from a channel: a lifted Blake2s tree of the circle layer,
 * the circle-to-line fold (FriOps::fold_circle_into_line), then per line layer
 * its tree and a fold by 2 (FriOps::fold_line) down to a single value; then
 * the decommitment of the query positions.  d_itwiddles: an inverse twiddle
 * tree covering log_size - 1 (e.g. of CanonicCoset(log_size + 1).half_coset).
 * Buffers for every layer and tree are allocated at create. */
typedef struct stwo_b200_fri_prover stwo_b200_fri_prover;
int stwo_b200_fri_prover_create(uint32_t log_size, int m31_output, const uint32_t* d_itwiddles,
                                uint32_t tree_log_size, void* stream, stwo_b200_fri_prover** out, char* err,
                                size_t err_len);
int stwo_b200_fri_prover_destroy(stwo_b200_fri_prover* prover, char* err, size_t err_len);
/* d_coords4: the column's 4 coordinate columns (device, 2^log_size words each,
 * bit-reversed circle-domain order); alphas: log_size QM31 values (host, 4
 * words each; alpha 0 folds the circle layer); queries: sorted distinct
 * positions in [0, 2^log_size).  Writes the FriProof bytes (first layer,
 * inner layers, last-layer value; the proof's canonical layout) to proof_out
 * when non-NULL and their length to *proof_len.  Synchronises its stream. */
int stwo_b200_fri_prove_seeded(stwo_b200_fri_prover* prover, const uint32_t* const* d_coords4,
                               const uint32_t* alphas, const uint64_t* queries, uint32_t n_queries,
                               uint8_t* proof_out, size_t proof_cap, size_t* proof_len, char* err, size_t err_len);

#ifdef __cplusplus
}
#endif
#endif /* STWO_B200_H */
