/*
 * algebra_linear_gpu — B200 (sm_100a) LU solver behind the API of the
 * cpmech/algebra_linear 4.0.0 crate's dense and sparse LU path.
 *
 * C ABI: plain pointers and sizes, column-major storage (a[i + j*n]),
 * 0-based indices. Every entry point returns an int status (ALG_OK = 0).
 * The host-pointer entry points are drop-ins for the Rust functions they cite:
 * they copy the caller's arrays to the GPU, compute there, and copy results
 * back into the same arrays. There is no CPU fallback: without a usable CUDA
 * device every compute entry point returns ALG_NO_DEVICE.
 *
 * Threading: the host-pointer drop-ins share one library context per device,
 * guarded by a mutex (calls serialise). An alg_ctx is owned by one thread at a
 * time, like a `&mut` borrow in the reference.
 */
#ifndef ALGEBRA_LINEAR_GPU_H
#define ALGEBRA_LINEAR_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------
 * 1..4 mirror lapack::LapackError (src/lapack/mod.rs:76-96).
 * 100..108 mirror sparse::faer::Error in declaration order
 * (src/sparse/faer/error.rs:5-24).
 * 200.. are conditions only a GPU implementation has. */
#define ALG_OK 0
#define ALG_SINGULAR 1
#define ALG_BAD_SHAPE 2
#define ALG_CONVERGENCE 3
#define ALG_NOT_IMPLEMENTED 4

#define ALG_SP_BAD_SHAPE 100
#define ALG_SP_INVALID_STRUCTURE 101
#define ALG_SP_UNSORTED_ROWS 102
#define ALG_SP_DUPLICATE_ENTRY 103
#define ALG_SP_SINGULAR 104
#define ALG_SP_INDEX_OVERFLOW 105
#define ALG_SP_STRUCTURE_MISMATCH 106
#define ALG_SP_NOT_FINITE 107
#define ALG_SP_NOT_FACTORIZED 108

#define ALG_CUDA_ERROR 200
#define ALG_OUT_OF_DEVICE_MEMORY 201
#define ALG_TIMEOUT 202
#define ALG_INVALID_ARGUMENT 203
#define ALG_NO_DEVICE 204

/* Message for a status code (static storage). The sparse messages are the
 * reference's Display strings (src/sparse/faer/error.rs:27-41). */
const char* alg_status_string(int status);

/* Library version string. */
const char* alg_version(void);

/* Number of CUDA kernels this library has launched in this process (all
 * contexts). Lets a caller count the device work inside a timed region. */
unsigned long long alg_kernel_launch_count(void);

/* ---- dense drop-ins (host pointers) -------------------------------------- */

/* Arithmetic of the trailing updates in the FP64 form.
 * ALG_UPDATE_EXACT: every entry is updated as the reference's scalar loop does
 *   (rounded product, rounded difference, in pivot order), so the factors,
 *   pivots and determinant are bit-identical to lapack::dgetrf.
 * ALG_UPDATE_FMA: fused multiply-adds (twice the FP64 rate); pivots agree with
 *   the reference unless two candidates tie to within rounding. */
#define ALG_UPDATE_EXACT 0
#define ALG_UPDATE_FMA 1

/* Replaces `pub fn dgetrf(a: &mut [f64], n: usize)
 *   -> Result<(Vec<usize>, f64), LapackError>` (src/lapack/mod.rs:181-185).
 * a: n*n column-major, overwritten with packed unit-lower L and U.
 * ipiv: n entries, 0-based sequential row interchanges. det: ±prod(u_kk).
 * n = 0: *det = 1, ALG_OK. On ALG_SINGULAR the contents of a and ipiv are
 * unspecified (the reference leaves a partly factored). */
int alg_dgetrf(double* a, size_t n, size_t* ipiv, double* det);

/* Replaces `pub fn dgetrf_rect(a: &mut [f64], nrows: usize, ncols: usize,
 *   ipiv: &mut [usize]) -> Result<(), LapackError>` (src/lapack/mod.rs:202-238).
 * ALG_BAD_SHAPE if nrows < ncols; ncols = 0 is ALG_OK. */
int alg_dgetrf_rect(double* a, size_t nrows, size_t ncols, size_t* ipiv);

/* Replaces `pub fn dgesv(a: &mut [f64], b: &mut [f64])
 *   -> Result<(), LapackError>` (src/lapack/mod.rs:309-323), n = b.len().
 * a is destroyed (holds the LU factors); b becomes x. */
int alg_dgesv(double* a, double* b, size_t n);

/* Replaces `pub fn dgetri(lu: &mut [f64], n: usize, ipiv: &[usize])
 *   -> Result<(), LapackError>` (src/lapack/mod.rs:249-298): lu (n*n, the
 * factors from alg_dgetrf) becomes the inverse, computed column by column
 * with the reference's interchange, row-dot and division order (bit-identical
 * results). ALG_SINGULAR, with lu unchanged, when some u_ii is zero;
 * ALG_BAD_SHAPE when an ipiv entry is out of range. */
int alg_dgetri(double* lu, size_t n, const size_t* ipiv);

/* ---- complex twins (src/lapack/complex.rs) ------------------------------
 * A complex entry is an interleaved (re, im) pair of doubles, the layout of
 * the reference's Complex64 (num_complex::Complex<f64>), of C99 double
 * complex and of numpy complex128; matrices are column-major, so an n x n
 * matrix is 2 n^2 doubles. Results are bit-identical to the reference: the
 * same |Re| + |Im| pivots and the num-complex 0.4 operator formulas with every
 * product, sum and quotient rounded on its own. */

/* Replaces `pub fn zgetrf(a: &mut [Complex64], n: usize)
 *   -> Result<Vec<usize>, LapackError>` (src/lapack/complex.rs:67-124): a is
 * factored in place (unit-lower L below the diagonal, U on and above it);
 * ipiv (n entries, 0-based: rows k and ipiv[k] swapped at step k). On
 * ALG_SINGULAR, a holds the reference's partial state and ipiv is not
 * written. */
int alg_zgetrf(double* a, size_t n, size_t* ipiv);

/* Replaces `pub fn zgetrf_rect(a: &mut [Complex64], nrows: usize, ncols:
 *   usize, ipiv: &mut [usize]) -> Result<(), LapackError>`
 * (src/lapack/complex.rs:169-208): the nrows x ncols panel (nrows >= ncols,
 * else ALG_BAD_SHAPE) factored in place, ipiv ncols entries. */
int alg_zgetrf_rect(double* a, size_t nrows, size_t ncols, size_t* ipiv);

/* Replaces `pub fn zgesv(a: &mut [Complex64], b: &mut [Complex64])
 *   -> Result<(), LapackError>` (src/lapack/complex.rs:279-312): a (2 n^2
 * doubles) is left holding its LU factors, b (2 n doubles) holds x. */
int alg_zgesv(double* a, double* b, size_t n);

/* Replaces `pub fn zgetri(lu: &mut [Complex64], n: usize, ipiv: &[usize])
 *   -> Result<(), LapackError>` (src/lapack/complex.rs:217-271): lu (the
 * factors and pivots from alg_zgetrf) becomes the inverse (U inverted in
 * place, inv(A) L = inv(U) solved from the last column down, the
 * interchanges undone as column swaps). ALG_SINGULAR on a zero u_jj, with the
 * columns before j already inverted as the reference leaves them;
 * ALG_BAD_SHAPE when an ipiv entry is out of range. */
int alg_zgetri(double* lu, size_t n, const size_t* ipiv);

/* dgesv with nrhs right-hand sides, b n x nrhs column-major: the reference's
 * dgetrf followed by its dgetrs (src/lapack/mod.rs:330-354) per column. */
int alg_dgesv_nrhs(double* a, double* b, size_t n, size_t nrhs);

/* alg_dgesv_nrhs with a chosen update arithmetic (ALG_UPDATE_*); ipiv may be
 * NULL, else receives the n interchanges. */
int alg_dgesv_ex(int update, double* a, double* b, size_t n, size_t nrhs, size_t* ipiv);

/* ---- device-resident API -------------------------------------------------
 * An alg_ctx holds a CUDA stream (the caller's, or its own) and the device
 * workspace; device pointers are the caller's. Calls are stream-ordered and
 * return once the status is known (they synchronise the stream). */
typedef struct alg_ctx alg_ctx;

/* Context on the current CUDA device; stream = NULL means the context makes
 * and owns a non-blocking stream. */
int alg_ctx_create(void* cuda_stream, alg_ctx** out);
void alg_ctx_destroy(alg_ctx* ctx);
/* Rebinds the stream (e.g. to the caller framework's current stream). */
int alg_ctx_set_stream(alg_ctx* ctx, void* cuda_stream);
/* Every device-side wait of the triangular solves (the dataflow sweeps of
 * alg_dgetrs_dev, alg_dgesv_dev, the host drop-ins and the mixed form's
 * refinement) gives up after limit_ns nanoseconds (0: the default, 2 s):
 * the kernel raises an abort flag, every CTA returns, and the call reports
 * ALG_TIMEOUT; the context stays usable. No counterpart in the reference. */
int alg_ctx_set_wait_limit(alg_ctx* ctx, unsigned long long limit_ns);
/* Failure injection for tests of that path (no counterpart in the
 * reference): the next `count` triangular sweeps on this context start with
 * a wait on a flag that nothing sets, so the wait runs out after the limit
 * and the call reports ALG_TIMEOUT; nothing faults or hangs. */
int alg_ctx_inject_stuck_wait(alg_ctx* ctx, int count);

/* In-place LU of the n x n device matrix d_a (leading dimension lda >= n).
 * d_ipiv: n int32, LAPACK-style sequential interchanges (0-based).
 * d_perm: n int32, the net row permutation (row i of P*A is row perm[i] of A);
 * either may be NULL. */
int alg_dgetrf_dev(alg_ctx* ctx, int update, double* d_a, int n, int lda,
                   int32_t* d_ipiv, int32_t* d_perm);

/* Panel LU of the nrows x ncols device matrix (nrows >= ncols), the device
 * form of dgetrf_rect (src/lapack/mod.rs:202-238): interchanges stay within the
 * ncols columns; d_ipiv receives ncols entries. */
int alg_dgetrf_rect_dev(alg_ctx* ctx, int update, double* d_a, int nrows, int ncols, int lda,
                        int32_t* d_ipiv);

/* Solves with factors from alg_dgetrf_dev: d_b is n x nrhs (leading dim ldb),
 * overwritten with x. */
int alg_dgetrs_dev(alg_ctx* ctx, const double* d_lu, int n, int lda,
                   const int32_t* d_perm, double* d_b, int nrhs, int ldb);

/* The device form of alg_dgetri: d_lu (factors from alg_dgetrf_dev, leading
 * dimension lda) becomes the inverse; d_perm is the net permutation that
 * alg_dgetrf_dev returned. */
int alg_dgetri_dev(alg_ctx* ctx, double* d_lu, int n, int lda, const int32_t* d_perm);

/* Per-kernel-class timing of a context's launches with CUDA events, for
 * roofline reporting. Classes: 0 panel, 1 row interchange, 2 trsm,
 * 3 CUDA-core update, 4 tensor-core update, 5 triangular solve, 6 FP64
 * residual, 7 precision cast, 8 batched systems (and the sparse small fronts),
 * 9 sparse factorization (whole), 10 other.
 * flops/bytes are the algorithmic counts of the timed launches. */
int alg_ctx_set_profiling(alg_ctx* ctx, int on);
int alg_ctx_profile_reset(alg_ctx* ctx);
int alg_ctx_profile_get(alg_ctx* ctx, int kernel_class, unsigned long long* launches,
                        double* total_ms, double* flops, double* bytes);

/* The reference's DLARNV stream (src/lapack/families.rs:166-249, `larnv`)
 * generated on the device: n values into d_x (dist 1 = Uniform(0,1),
 * 2 = Symmetric(-1,1)), bit-identical to the CPU stream for the same seed
 * (four 12-bit words, last odd); seed_out (may be NULL) receives the seed the
 * reference would hold after the call. Stream-ordered, no sync. */
int alg_larnv_dev(alg_ctx* ctx, int dist, const uint32_t seed[4], size_t n, double* d_x,
                  uint32_t seed_out[4]);

/* alg_dgetrf_dev + alg_dgetrs_dev; d_ipiv may be NULL. */
int alg_dgesv_dev(alg_ctx* ctx, int update, double* d_a, int n, int lda,
                  double* d_b, int nrhs, int ldb, int32_t* d_ipiv);

/* ---- mixed precision: low-precision LU + FP64 iterative refinement -------
 * The dsgesv contract: A is factorized in low precision (FP32 working copy;
 * trailing updates in FP32, TF32 or BF16 with FP32 accumulation), x is
 * refined in FP64 until the normwise backward error
 * ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf) is within tol
 * (default 10 n 2^-53, the FP64 level), falling back to GMRES-IR and then to
 * a full FP64 factorization. A is unchanged unless the FP64 fallback ran, in
 * which case it holds the FP64 LU factors as after dgesv. */
#define ALG_PREC_FP32 0
#define ALG_PREC_TF32 1
#define ALG_PREC_BF16 2
/* TF32x3: each FP32 operand split into TF32 high and low parts and three
 * TF32 products (hi hi + hi lo + lo hi) accumulated in FP32 on the tensor
 * cores, FP32-level accuracy (Ootomo and Yokota, IJHPCA 2022). */
#define ALG_PREC_TF32X3 3

/* Stabilisation of the low-precision LU: partial pivoting (the reference's
 * strategy, column-serial panel); tournament pivoting (CALU's TSLU, Grigori,
 * Demmel and Xiang, SIMAX 2011: each leaf panel's pivot rows are chosen by a
 * reduction tree of partial-pivoting LUs over row blocks, so the column-serial
 * chain runs on 256-row blocks instead of the whole panel); or a random
 * butterfly transformation of A followed by LU without pivoting (Baboulin,
 * Dongarra, Herrmann, Tomov, ACM TOMS 2013; needs n divisible by 4; falls back
 * to pivoting on a zero pivot). AUTO: tournament pivoting for n >= 2048,
 * partial pivoting below; LU without pivoting keeps a large growth factor on
 * matrices that are random to begin with, butterflies or not. */
#define ALG_PIVOT_AUTO 0
#define ALG_PIVOT_PARTIAL 1
#define ALG_PIVOT_RBT 2
#define ALG_PIVOT_TOURNAMENT 3

#define ALG_MIXED_PATH_IR 1
#define ALG_MIXED_PATH_GMRES 2
#define ALG_MIXED_PATH_FP64 3

typedef struct {
  int precision;    /* ALG_PREC_* of the trailing updates */
  double tol;       /* backward-error target; <= 0 means 10 n 2^-53 */
  int max_ir;       /* refinement steps before the fallback (<= 0: 30) */
  int no_fallback;  /* nonzero: return ALG_CONVERGENCE instead of refactorizing in FP64 */
  int no_gmres;     /* nonzero: skip GMRES-IR when plain refinement stalls */
  int gmres_restart;/* Krylov dimension of GMRES-IR (<= 0: 30) */
  int pivoting;     /* ALG_PIVOT_*: how the low-precision LU is kept stable */
  int reserved;
} alg_mixed_opts;

typedef struct {
  int path;            /* ALG_MIXED_PATH_* that produced x */
  int precision;
  int ir_iterations;
  int gmres_iterations;
  double backward_error;  /* worst over the right-hand sides; -1 on the FP64 path */
  double reserved[4];     /* [0]: 1 when the butterfly form ran; [1]: 1 when tournament pivoting ran */
} alg_mixed_report;

void alg_mixed_opts_default(alg_mixed_opts* opts);

/* Host drop-in: a n x n, b n x nrhs (column-major); b becomes x. */
int alg_dgesv_mixed(const alg_mixed_opts* opts, double* a, double* b, size_t n, size_t nrhs,
                    alg_mixed_report* report);

/* Device form: d_a is read (and only overwritten on the FP64 fallback). */
int alg_dgesv_mixed_dev(alg_ctx* ctx, const alg_mixed_opts* opts, double* d_a, int n, int lda,
                        double* d_b, int nrhs, int ldb, alg_mixed_report* report);

/* ---- batched dgesv: many independent systems of uneven order ------------
 * Each system is the reference's dgesv (src/lapack/mod.rs:309-354) on its own
 * n_i x n_i matrix (1 <= n_i <= 512). Matrices and right-hand sides live
 * packed in two device buffers at the offsets alg_batch_offsets reports
 * (column-major, leading dimension n_i). A plan sorts the systems into size
 * buckets (largest first) and issues one persistent launch per bucket.
 * mixed = 0: FP64 LU with partial pivoting (A becomes its LU, b becomes x).
 * mixed = 1: FP32 LU + FP64 refinement to the backward error 10 n 2^-53
 * (A is left unchanged; b becomes x; alg_batch_eta reports each system's
 * backward error). d_info: per system 0, 1 + the first zero pivot's column,
 * or -(iterations + 1) when refinement did not reach the target. */
typedef struct alg_batch alg_batch;
int alg_batch_create(alg_ctx* ctx, int count, const int* n_host, int mixed, alg_batch** out);
int alg_batch_offsets(const alg_batch* batch, int64_t* a_off, int64_t* b_off);
/* Stream-ordered; no synchronisation. */
int alg_batch_solve(alg_batch* batch, double* d_a, double* d_b, int* d_info);
/* The same launch sequence captured once in a CUDA graph (per buffer set) and
 * replayed; the capturing call solves the batch too. */
int alg_batch_solve_graph(alg_batch* batch, double* d_a, double* d_b, int* d_info);
/* Autotuner: for every size bucket, times each launch shape on this batch
 * (restoring the inputs from d_a_src/d_b_src before each trial): 128, 256 or
 * 512 threads per CTA (the trailing update's register micro-tile 4 x 8, 4 x 4
 * or 4 x 2 per thread) times a 16- or 32-column panel, and keeps the fastest;
 * threads_out (may be NULL) receives one value per bucket, alg_batch_panels
 * the panel widths. Shapes from an earlier run can be set directly with
 * alg_batch_set_config (host-side; not inside a stream capture). */
int alg_batch_autotune(alg_batch* batch, double* d_a, double* d_b, int* d_info, const double* d_a_src,
                       const double* d_b_src, int* threads_out);
int alg_batch_info(const alg_batch* batch, int* n_buckets, int* caps, int* threads, int* counts,
                   double* flops);
int alg_batch_panels(const alg_batch* batch, int* panels);
int alg_batch_set_config(alg_batch* batch, int bucket, int threads, int panel);
int alg_batch_eta(const alg_batch* batch, double* eta_host);
/* Copies the pivots of the last solve (0-based pivot rows of each system's
 * LU, FP64 or FP32, at the b offsets) to ipiv_host (sum of the orders ints). */
int alg_batch_ipiv(const alg_batch* batch, int* ipiv_host);
void alg_batch_destroy(alg_batch* batch);

/* The tensor-core trailing update of the low-precision LU on device buffers:
 * C (FP32, M x N) -= A (M x K) * B (K x N), all column-major, operands
 * rounded to prec (ALG_PREC_TF32 or ALG_PREC_BF16; ALG_PREC_TF32X3 splits
 * them into TF32 pairs), FP32 accumulation. K must be a multiple of 64 (BF16)
 * or 32 (TF32, TF32x3). Synchronises. Exposed for
 * tests and benchmarks of the kernel on its own. */
int alg_gemm_tc_sub_dev(alg_ctx* ctx, int prec, int M, int N, int K, const float* A, int lda,
                        const float* B, int ldb, float* C, int ldc);

/* FP64 C (M x N) -= A (M x K) * B (K x N) on the FP64 tensor cores (the
 * update of the fused FP64 forms); column-major, synchronises. Exposed for
 * tests and benchmarks of the kernel on its own. */
int alg_gemm_dmma_sub_dev(alg_ctx* ctx, int M, int N, int K, const double* A, int lda, const double* B, int ldb,
                          double* C, int ldc);

/* ---- sparse LU (sparse::faer::SparseLu, src/sparse/faer/sparse_lu.rs) -----
 * The handle owns the symbolic analysis (host) and the numeric factors (GPU).
 * CSC arrays are borrowed per call and never retained: col_ptr (n + 1),
 * row_idx (nnz, strictly increasing within a column), values (nnz). All
 * indices 0-based. Status codes are ALG_SP_* (error.rs:5-24) plus the GPU
 * codes 200..204. */
#define ALG_SPLU_SIMPLICIAL 0 /* LuMethod::Simplicial (solver.rs:71-82) */
#define ALG_SPLU_SUPERNODAL 1 /* LuMethod::Supernodal */
#define ALG_SPLU_AUTO 2       /* LuMethod::Auto { flop_ratio_threshold } */

typedef struct alg_splu alg_splu;

/* SparseLuStats (src/sparse/faer/stats.rs:13-35); times in seconds. */
typedef struct {
  size_t n, nnz_a, nnz_l, nnz_u;
  double fill_ratio;
  size_t flops_estimate;
  int method;          /* ALG_SPLU_SIMPLICIAL / ALG_SPLU_SUPERNODAL */
  int has_flop_ratio;  /* Option<f64> */
  double flop_ratio;
  double ordering_time;
  double factorization_time;
} alg_splu_stats;

/* SparseLu::analyze (sparse_lu.rs:64-78): n = col_ptr_len - 1; a row index
 * >= n is ALG_SP_BAD_SHAPE, then the CSC validation of csc.rs:39-76; COLAMD,
 * the supernodal symbolic analysis and the GPU front plan run on the host
 * (no GPU needed). flop_ratio_threshold is used by ALG_SPLU_AUTO (the
 * reference's default is 40.0). The numeric factorization runs on the GPU
 * for every method: the reference's simplicial numeric path has no GPU
 * counterpart here, so a handle whose effective method is Simplicial is
 * factored by the supernodal GPU path (same pivots, values to rounding). */
int alg_splu_analyze(const size_t* col_ptr, size_t col_ptr_len, const size_t* row_idx, size_t row_idx_len,
                     int method, double flop_ratio_threshold, alg_splu** out);
/* SparseLu::factorize (sparse_lu.rs:91-121): CSC view errors, then
 * ALG_SP_STRUCTURE_MISMATCH (order, nnz and FNV-1a fingerprint),
 * ALG_SP_NOT_FINITE, ALG_SP_SINGULAR. Synchronises. On failure the previous
 * factors and statistics stay in place. The first factorization places the
 * handle's factors on the device current at that call (or on the device of
 * the context given to alg_splu_set_ctx); later calls on the handle are made
 * with that device current. */
int alg_splu_factorize(alg_splu* lu, const size_t* col_ptr, size_t col_ptr_len, const size_t* row_idx,
                       size_t row_idx_len, const double* values, size_t values_len);
/* SparseLu::solve (sparse_lu.rs:125-130): ALG_SP_NOT_FACTORIZED before a
 * successful factorization, ALG_SP_BAD_SHAPE if b_len != n. b becomes x. */
int alg_splu_solve(const alg_splu* lu, double* b, size_t b_len);
/* effective_method (sparse_lu.rs:137-140): ALG_SPLU_SIMPLICIAL / _SUPERNODAL. */
int alg_splu_effective_method(const alg_splu* lu);
/* flop_ratio (sparse_lu.rs:146-149): returns 1 and sets *ratio when the
 * supernodal symbolic analysis ran (method Supernodal or Auto), else 0. */
int alg_splu_flop_ratio(const alg_splu* lu, double* ratio);
/* stats (sparse_lu.rs:152-155): ALG_SP_NOT_FACTORIZED until a factorization
 * has succeeded (the reference's None). */
int alg_splu_get_stats(const alg_splu* lu, alg_splu_stats* out);
void alg_splu_free(alg_splu* lu);

/* SparseLu<Complex64> (the handle is generic over SparseScalar, lu.rs:20-82;
 * analyze is shared, the pattern alone): factorize and solve with complex
 * values, values_len entries / b_len entries as interleaved (re, im)
 * doubles. Pivots by the modulus, multipliers by Complex::inv, in FP64
 * (the mixed-precision setting applies to real factorizations only). The
 * first factorization fixes a handle's scalar: a real call on a complex
 * handle, or the reverse, is ALG_INVALID_ARGUMENT. Same errors otherwise as
 * the real calls; ALG_SP_NOT_FINITE when either part is not finite. */
int alg_zsplu_factorize(alg_splu* lu, const size_t* col_ptr, size_t col_ptr_len, const size_t* row_idx,
                        size_t row_idx_len, const double* values, size_t values_len);
int alg_zsplu_solve(const alg_splu* lu, double* b, size_t b_len);

/* Inspection (no reference counterpart; for tests and tools): the symbolic
 * analysis (any pointer may be NULL; supernode_ptr holds n_supernodes + 1)
 * and the row permutation of the current factors (position -> row). */
int alg_splu_symbolic(const alg_splu* lu, size_t* col_perm, size_t* col_perm_inv, size_t* col_counts,
                      size_t* supernode_ptr, size_t* n_supernodes);
int alg_splu_row_perm(const alg_splu* lu, size_t* row_perm);
typedef struct {
  size_t n_fronts, n_small_fronts, small_levels, solve_levels, max_front_rows, max_front_cols;
  size_t factor_bytes, work_bytes;
  double plan_flops;
  int structurally_singular;
  int n_lanes;            /* concurrent lanes of large fronts (independent subtrees) */
  size_t top_fronts;      /* large fronts factored after the lanes */
} alg_splu_plan;
int alg_splu_plan_info(const alg_splu* lu, alg_splu_plan* out);

/* Device-resident use: bind a context (its stream) before the first
 * factorization; d_values (nnz, CSC order of the analyzed pattern) and d_b
 * (n) are device pointers. factorize_dev synchronises (it reports the
 * outcome); solve_dev is stream-ordered. */
int alg_splu_set_ctx(alg_splu* lu, alg_ctx* ctx);
int alg_splu_factorize_dev(alg_splu* lu, const double* d_values);
int alg_splu_solve_dev(alg_splu* lu, double* d_b);

/* A handle sharing src's symbolic analysis and GPU plan (no new ordering),
 * with its own numeric state: for several streams factoring the same
 * pattern concurrently. */
int alg_splu_clone(const alg_splu* src, alg_splu** out);
/* factorize for the analyzed pattern itself: only the nnz values (host) are
 * passed; ALG_SP_NOT_FINITE, ALG_SP_SINGULAR as alg_splu_factorize. */
int alg_splu_factorize_values(alg_splu* lu, const double* values);

/* Mixed precision (no counterpart in the reference, whose sparse LU is FP64
 * only): the precision of the next factorizations. ALG_SPLU_FP64 (the
 * default) is the reference's arithmetic. ALG_PREC_FP32 / ALG_PREC_TF32 /
 * ALG_PREC_TF32X3 / ALG_PREC_BF16 factor the fronts in FP32 (the large
 * fronts' trailing updates in FP32, or on the tensor cores with TF32, split
 * TF32x3 or BF16 operands and FP32 accumulation) and refine every solve in FP64 against A's values until the
 * normwise backward error ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf)
 * is at most tol (<= 0: 10 n 2^-53); when max_ir steps (<= 0: 10) do not get
 * there, or refinement stalls, the factor set is recomputed in FP64 from the
 * same values and the solve is direct (an FP32 zero pivot at factorization
 * time does the same). A mixed-form solve synchronises once per refinement
 * step, solve_dev included. */
#define ALG_SPLU_FP64 (-1)
int alg_splu_set_precision(alg_splu* lu, int precision, double tol, int max_ir);
typedef struct {
  int precision;          /* ALG_SPLU_FP64 or ALG_PREC_* of the factors the last solve used */
  int iterations;         /* refinement steps of the last solve (0 on the FP64 form) */
  int fell_back;          /* 1: the last solve recomputed the factors in FP64 */
  int factor_precision;   /* precision of the current factors */
  double backward_error;  /* the last refined solve's backward error; -1 when not measured */
} alg_splu_refine_report;
int alg_splu_last_solve(const alg_splu* lu, alg_splu_refine_report* out);

/* ---- serving loop (no counterpart in the reference) -----------------------
 * A device-resident request loop: requests are queued in arrival order and
 * taken by worker threads (each with its own CUDA stream and workspace) as
 * soon as a worker is idle and the request's device bytes fit in the HBM
 * budget, so arriving requests are admitted while others run and their work
 * overlaps on the GPU. Dense requests: dgesv of order n (A is not modified;
 * x receives the solution; precision ALG_REQ_FP64 = FP64 LU with fused
 * updates, ALG_REQ_MIXED = FP32 LU + FP64 refinement). Sparse requests:
 * refactorize `pattern` (an analyzed handle, shared read-only) with `values`
 * and solve; each worker keeps its own factors of each pattern on the
 * device. A request's result depends only on its inputs (deterministic
 * kernels, private workspaces), so it is the same alone and in a mix.
 * Timestamps are steady-clock nanoseconds (alg_server_now_ns). */
#define ALG_REQ_DENSE 0
#define ALG_REQ_SPARSE 1
#define ALG_REQ_FP64 0
#define ALG_REQ_MIXED 1
typedef struct {
  int kind;
  int precision;
  size_t n;
  const double* a;          /* dense: n x n column-major, host */
  const double* values;     /* sparse: nnz values in the pattern's CSC order, host */
  const alg_splu* pattern;  /* sparse: analyzed handle */
  const double* b;          /* n, host */
  double* x;                /* n, host: the solution */
  /* filled by the server */
  int status;
  int worker;
  double backward_error;    /* dense mixed: the refinement's final backward error; else -1 */
  int64_t t_submit_ns, t_start_ns, t_done_ns;
  volatile int done;
} alg_request;
typedef struct alg_server alg_server;
/* max_dense_n: largest dense order (workspaces are sized and kernels set up
 * at creation, before the workers start). */
int alg_server_create(int n_workers, size_t hbm_budget_bytes, size_t max_dense_n, alg_server** out);
/* Queues a request (it must stay alive until done); returns at once. */
int alg_server_submit(alg_server* server, alg_request* request);
/* Blocks until the request is done; returns its status. */
int alg_server_wait(alg_server* server, alg_request* request);
/* Blocks until the queue is empty and no request is running. */
int alg_server_drain(alg_server* server);
unsigned long long alg_server_completed(const alg_server* server);
int64_t alg_server_now_ns(void);
void alg_server_destroy(alg_server* server);

/* ---- allocation-free solve of one small system ---------------------------
 * No counterpart in the reference crate. For callers that cannot call
 * cudaMalloc: code that runs inside another library's memory pool which owns
 * the device's free memory, serving loops where the device-wide
 * synchronisation of cudaMalloc/cudaFree would stall other streams, and
 * callers that must not meet out-of-memory after start-up. This entry point
 * allocates nothing, and needs no alg_ctx (creating one allocates).
 *
 * Solves A x = b for ONE system of order 1 <= n <= ALG_NOALLOC_MAX_N with the
 * mixed form of the batched kernel (FP32 LU with partial pivoting, FP64
 * refinement to the backward error 10 n 2^-53, at most 10 steps): the same
 * kernel, CTA size and arithmetic as a one-system alg_batch plan with
 * mixed = 1. d_a (n x n, column-major, leading dimension n) is only read;
 * d_b (n) becomes x; *d_info receives 0, 1 + the first zero pivot's column,
 * or -(iterations + 1) when refinement missed the target. d_ipiv (n ints,
 * the FP32 LU's 0-based pivot rows) and d_eta (the backward error) may be
 * NULL. When *d_info > 0 (a zero pivot) neither d_b nor *d_eta is written.
 * All pointers are device pointers; the work is queued on `stream` (a
 * cudaStream_t of the current context; NULL is the default stream) and the
 * call returns without synchronising.
 *
 * Set-up: a call with n = 0 (the pointers are then ignored and may be NULL)
 * queues nothing and only does the host-side set-up for the current device
 * and CUDA context: it loads the library's device code for this entry point,
 * looks up the static array's device address and sets the kernel's
 * shared-memory limit. It returns ALG_OK, or ALG_NO_DEVICE without a GPU.
 * The first call with n > 0 does the same set-up if no call has done it yet
 * in the current context. Make the set-up call at start-up, before any
 * stream capture: it is the only call that can meet out-of-memory.
 *
 * Working memory: one static device array of ALG_NOALLOC_SCRATCH_BYTES (the
 * FP32 copy of A, a residual vector, pivots, a work counter). It comes into
 * being on a device when the library's device code is loaded there: at the
 * set-up call under CUDA's default lazy module loading, or when the context
 * is created under CUDA_MODULE_LOADING=EAGER. From then on that GPU holds it
 * until the context is destroyed (process exit or cudaDeviceReset); after a
 * reset, or in another context, the next call repeats the set-up. Do not
 * pass a stream of one context while another is current.
 * n > ALG_NOALLOC_MAX_N (or n < 0) returns ALG_BAD_SHAPE and queues nothing.
 * The array keeps the previous call's contents; the work counter must be 0
 * when the kernel starts, and each call resets it itself, in stream order,
 * so the caller clears nothing. All calls on one device share the array:
 * calls that overlap on the GPU (on different streams, or from different
 * host threads without ordering) race on it and give wrong results; calls
 * queued on one stream are safe. */
#define ALG_NOALLOC_MAX_N 512
#define ALG_NOALLOC_SCRATCH_BYTES 1054976
int alg_dgesv_mixed_noalloc(void* stream, const double* d_a, double* d_b, int n, int* d_ipiv, int* d_info,
                            double* d_eta);

#ifdef __cplusplus
}
#endif

#endif /* ALGEBRA_LINEAR_GPU_H */
