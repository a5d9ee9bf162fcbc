// Raw declarations of the C ABI of libalgebra_linear_gpu, written by
// gen_ffi.py from include/algebra_linear_gpu.h; do not edit by hand.
// The meaning of every constant, field and function is documented in the header.
#![allow(non_camel_case_types, non_snake_case, dead_code)]

use core::ffi::{c_char, c_int, c_ulonglong, c_void};

pub const ALG_OK: c_int = 0;
pub const ALG_SINGULAR: c_int = 1;
pub const ALG_BAD_SHAPE: c_int = 2;
pub const ALG_CONVERGENCE: c_int = 3;
pub const ALG_NOT_IMPLEMENTED: c_int = 4;
pub const ALG_SP_BAD_SHAPE: c_int = 100;
pub const ALG_SP_INVALID_STRUCTURE: c_int = 101;
pub const ALG_SP_UNSORTED_ROWS: c_int = 102;
pub const ALG_SP_DUPLICATE_ENTRY: c_int = 103;
pub const ALG_SP_SINGULAR: c_int = 104;
pub const ALG_SP_INDEX_OVERFLOW: c_int = 105;
pub const ALG_SP_STRUCTURE_MISMATCH: c_int = 106;
pub const ALG_SP_NOT_FINITE: c_int = 107;
pub const ALG_SP_NOT_FACTORIZED: c_int = 108;
pub const ALG_CUDA_ERROR: c_int = 200;
pub const ALG_OUT_OF_DEVICE_MEMORY: c_int = 201;
pub const ALG_TIMEOUT: c_int = 202;
pub const ALG_INVALID_ARGUMENT: c_int = 203;
pub const ALG_NO_DEVICE: c_int = 204;
pub const ALG_UPDATE_EXACT: c_int = 0;
pub const ALG_UPDATE_FMA: c_int = 1;
pub const ALG_PREC_FP32: c_int = 0;
pub const ALG_PREC_TF32: c_int = 1;
pub const ALG_PREC_BF16: c_int = 2;
pub const ALG_PREC_TF32X3: c_int = 3;
pub const ALG_PIVOT_AUTO: c_int = 0;
pub const ALG_PIVOT_PARTIAL: c_int = 1;
pub const ALG_PIVOT_RBT: c_int = 2;
pub const ALG_PIVOT_TOURNAMENT: c_int = 3;
pub const ALG_MIXED_PATH_IR: c_int = 1;
pub const ALG_MIXED_PATH_GMRES: c_int = 2;
pub const ALG_MIXED_PATH_FP64: c_int = 3;
pub const ALG_SPLU_SIMPLICIAL: c_int = 0;
pub const ALG_SPLU_SUPERNODAL: c_int = 1;
pub const ALG_SPLU_AUTO: c_int = 2;
pub const ALG_SPLU_FP64: c_int = -1;
pub const ALG_REQ_DENSE: c_int = 0;
pub const ALG_REQ_SPARSE: c_int = 1;
pub const ALG_REQ_FP64: c_int = 0;
pub const ALG_REQ_MIXED: c_int = 1;
pub const ALG_NOALLOC_MAX_N: c_int = 512;
pub const ALG_NOALLOC_SCRATCH_BYTES: c_int = 1054976;

#[repr(C)]
pub struct alg_ctx {
    _private: [u8; 0],
}

#[repr(C)]
pub struct alg_batch {
    _private: [u8; 0],
}

#[repr(C)]
pub struct alg_splu {
    _private: [u8; 0],
}

#[repr(C)]
pub struct alg_server {
    _private: [u8; 0],
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct alg_mixed_opts {
    pub precision: c_int,
    pub tol: f64,
    pub max_ir: c_int,
    pub no_fallback: c_int,
    pub no_gmres: c_int,
    pub gmres_restart: c_int,
    pub pivoting: c_int,
    pub reserved: c_int,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct alg_mixed_report {
    pub path: c_int,
    pub precision: c_int,
    pub ir_iterations: c_int,
    pub gmres_iterations: c_int,
    pub backward_error: f64,
    pub reserved: [f64; 4],
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct alg_splu_stats {
    pub n: usize,
    pub nnz_a: usize,
    pub nnz_l: usize,
    pub nnz_u: usize,
    pub fill_ratio: f64,
    pub flops_estimate: usize,
    pub method: c_int,
    pub has_flop_ratio: c_int,
    pub flop_ratio: f64,
    pub ordering_time: f64,
    pub factorization_time: f64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct alg_splu_plan {
    pub n_fronts: usize,
    pub n_small_fronts: usize,
    pub small_levels: usize,
    pub solve_levels: usize,
    pub max_front_rows: usize,
    pub max_front_cols: usize,
    pub factor_bytes: usize,
    pub work_bytes: usize,
    pub plan_flops: f64,
    pub structurally_singular: c_int,
    pub n_lanes: c_int,
    pub top_fronts: usize,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct alg_splu_refine_report {
    pub precision: c_int,
    pub iterations: c_int,
    pub fell_back: c_int,
    pub factor_precision: c_int,
    pub backward_error: f64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct alg_request {
    pub kind: c_int,
    pub precision: c_int,
    pub n: usize,
    pub a: *const f64,
    pub values: *const f64,
    pub pattern: *const alg_splu,
    pub b: *const f64,
    pub x: *mut f64,
    pub status: c_int,
    pub worker: c_int,
    pub backward_error: f64,
    pub t_submit_ns: i64,
    pub t_start_ns: i64,
    pub t_done_ns: i64,
    pub done: c_int,
}

#[link(name = "algebra_linear_gpu")]
unsafe extern "C" {
    pub fn alg_status_string(status: c_int) -> *const c_char;
    pub fn alg_version() -> *const c_char;
    pub fn alg_kernel_launch_count() -> c_ulonglong;
    pub fn alg_dgetrf(a: *mut f64, n: usize, ipiv: *mut usize, det: *mut f64) -> c_int;
    pub fn alg_dgetrf_rect(a: *mut f64, nrows: usize, ncols: usize, ipiv: *mut usize) -> c_int;
    pub fn alg_dgesv(a: *mut f64, b: *mut f64, n: usize) -> c_int;
    pub fn alg_dgetri(lu: *mut f64, n: usize, ipiv: *const usize) -> c_int;
    pub fn alg_zgetrf(a: *mut f64, n: usize, ipiv: *mut usize) -> c_int;
    pub fn alg_zgetrf_rect(a: *mut f64, nrows: usize, ncols: usize, ipiv: *mut usize) -> c_int;
    pub fn alg_zgesv(a: *mut f64, b: *mut f64, n: usize) -> c_int;
    pub fn alg_zgetri(lu: *mut f64, n: usize, ipiv: *const usize) -> c_int;
    pub fn alg_dgesv_nrhs(a: *mut f64, b: *mut f64, n: usize, nrhs: usize) -> c_int;
    pub fn alg_dgesv_ex(update: c_int, a: *mut f64, b: *mut f64, n: usize, nrhs: usize, ipiv: *mut usize) -> c_int;
    pub fn alg_ctx_create(cuda_stream: *mut c_void, out: *mut *mut alg_ctx) -> c_int;
    pub fn alg_ctx_destroy(ctx: *mut alg_ctx);
    pub fn alg_ctx_set_stream(ctx: *mut alg_ctx, cuda_stream: *mut c_void) -> c_int;
    pub fn alg_ctx_set_wait_limit(ctx: *mut alg_ctx, limit_ns: c_ulonglong) -> c_int;
    pub fn alg_ctx_inject_stuck_wait(ctx: *mut alg_ctx, count: c_int) -> c_int;
    pub fn alg_dgetrf_dev(ctx: *mut alg_ctx, update: c_int, d_a: *mut f64, n: c_int, lda: c_int, d_ipiv: *mut i32, d_perm: *mut i32) -> c_int;
    pub fn alg_dgetrf_rect_dev(ctx: *mut alg_ctx, update: c_int, d_a: *mut f64, nrows: c_int, ncols: c_int, lda: c_int, d_ipiv: *mut i32) -> c_int;
    pub fn alg_dgetrs_dev(ctx: *mut alg_ctx, d_lu: *const f64, n: c_int, lda: c_int, d_perm: *const i32, d_b: *mut f64, nrhs: c_int, ldb: c_int) -> c_int;
    pub fn alg_dgetri_dev(ctx: *mut alg_ctx, d_lu: *mut f64, n: c_int, lda: c_int, d_perm: *const i32) -> c_int;
    pub fn alg_ctx_set_profiling(ctx: *mut alg_ctx, on: c_int) -> c_int;
    pub fn alg_ctx_profile_reset(ctx: *mut alg_ctx) -> c_int;
    pub fn alg_ctx_profile_get(ctx: *mut alg_ctx, kernel_class: c_int, launches: *mut c_ulonglong, total_ms: *mut f64, flops: *mut f64, bytes: *mut f64) -> c_int;
    pub fn alg_larnv_dev(ctx: *mut alg_ctx, dist: c_int, seed: *const u32, n: usize, d_x: *mut f64, seed_out: *mut u32) -> c_int;
    pub fn alg_dgesv_dev(ctx: *mut alg_ctx, update: c_int, d_a: *mut f64, n: c_int, lda: c_int, d_b: *mut f64, nrhs: c_int, ldb: c_int, d_ipiv: *mut i32) -> c_int;
    pub fn alg_mixed_opts_default(opts: *mut alg_mixed_opts);
    pub fn alg_dgesv_mixed(opts: *const alg_mixed_opts, a: *mut f64, b: *mut f64, n: usize, nrhs: usize, report: *mut alg_mixed_report) -> c_int;
    pub fn alg_dgesv_mixed_dev(ctx: *mut alg_ctx, opts: *const alg_mixed_opts, d_a: *mut f64, n: c_int, lda: c_int, d_b: *mut f64, nrhs: c_int, ldb: c_int, report: *mut alg_mixed_report) -> c_int;
    pub fn alg_batch_create(ctx: *mut alg_ctx, count: c_int, n_host: *const c_int, mixed: c_int, out: *mut *mut alg_batch) -> c_int;
    pub fn alg_batch_offsets(batch: *const alg_batch, a_off: *mut i64, b_off: *mut i64) -> c_int;
    pub fn alg_batch_solve(batch: *mut alg_batch, d_a: *mut f64, d_b: *mut f64, d_info: *mut c_int) -> c_int;
    pub fn alg_batch_solve_graph(batch: *mut alg_batch, d_a: *mut f64, d_b: *mut f64, d_info: *mut c_int) -> c_int;
    pub fn alg_batch_autotune(batch: *mut alg_batch, d_a: *mut f64, d_b: *mut f64, d_info: *mut c_int, d_a_src: *const f64, d_b_src: *const f64, threads_out: *mut c_int) -> c_int;
    pub fn alg_batch_info(batch: *const alg_batch, n_buckets: *mut c_int, caps: *mut c_int, threads: *mut c_int, counts: *mut c_int, flops: *mut f64) -> c_int;
    pub fn alg_batch_panels(batch: *const alg_batch, panels: *mut c_int) -> c_int;
    pub fn alg_batch_set_config(batch: *mut alg_batch, bucket: c_int, threads: c_int, panel: c_int) -> c_int;
    pub fn alg_batch_eta(batch: *const alg_batch, eta_host: *mut f64) -> c_int;
    pub fn alg_batch_ipiv(batch: *const alg_batch, ipiv_host: *mut c_int) -> c_int;
    pub fn alg_batch_destroy(batch: *mut alg_batch);
    pub fn alg_gemm_tc_sub_dev(ctx: *mut alg_ctx, prec: c_int, M: c_int, N: c_int, K: c_int, A: *const f32, lda: c_int, B: *const f32, ldb: c_int, C: *mut f32, ldc: c_int) -> c_int;
    pub fn alg_gemm_dmma_sub_dev(ctx: *mut alg_ctx, M: c_int, N: c_int, K: c_int, A: *const f64, lda: c_int, B: *const f64, ldb: c_int, C: *mut f64, ldc: c_int) -> c_int;
    pub fn alg_splu_analyze(col_ptr: *const usize, col_ptr_len: usize, row_idx: *const usize, row_idx_len: usize, method: c_int, flop_ratio_threshold: f64, out: *mut *mut alg_splu) -> c_int;
    pub fn alg_splu_factorize(lu: *mut alg_splu, col_ptr: *const usize, col_ptr_len: usize, row_idx: *const usize, row_idx_len: usize, values: *const f64, values_len: usize) -> c_int;
    pub fn alg_splu_solve(lu: *const alg_splu, b: *mut f64, b_len: usize) -> c_int;
    pub fn alg_splu_effective_method(lu: *const alg_splu) -> c_int;
    pub fn alg_splu_flop_ratio(lu: *const alg_splu, ratio: *mut f64) -> c_int;
    pub fn alg_splu_get_stats(lu: *const alg_splu, out: *mut alg_splu_stats) -> c_int;
    pub fn alg_splu_free(lu: *mut alg_splu);
    pub fn alg_zsplu_factorize(lu: *mut alg_splu, col_ptr: *const usize, col_ptr_len: usize, row_idx: *const usize, row_idx_len: usize, values: *const f64, values_len: usize) -> c_int;
    pub fn alg_zsplu_solve(lu: *const alg_splu, b: *mut f64, b_len: usize) -> c_int;
    pub fn alg_splu_symbolic(lu: *const alg_splu, col_perm: *mut usize, col_perm_inv: *mut usize, col_counts: *mut usize, supernode_ptr: *mut usize, n_supernodes: *mut usize) -> c_int;
    pub fn alg_splu_row_perm(lu: *const alg_splu, row_perm: *mut usize) -> c_int;
    pub fn alg_splu_plan_info(lu: *const alg_splu, out: *mut alg_splu_plan) -> c_int;
    pub fn alg_splu_set_ctx(lu: *mut alg_splu, ctx: *mut alg_ctx) -> c_int;
    pub fn alg_splu_factorize_dev(lu: *mut alg_splu, d_values: *const f64) -> c_int;
    pub fn alg_splu_solve_dev(lu: *mut alg_splu, d_b: *mut f64) -> c_int;
    pub fn alg_splu_clone(src: *const alg_splu, out: *mut *mut alg_splu) -> c_int;
    pub fn alg_splu_factorize_values(lu: *mut alg_splu, values: *const f64) -> c_int;
    pub fn alg_splu_set_precision(lu: *mut alg_splu, precision: c_int, tol: f64, max_ir: c_int) -> c_int;
    pub fn alg_splu_last_solve(lu: *const alg_splu, out: *mut alg_splu_refine_report) -> c_int;
    pub fn alg_server_create(n_workers: c_int, hbm_budget_bytes: usize, max_dense_n: usize, out: *mut *mut alg_server) -> c_int;
    pub fn alg_server_submit(server: *mut alg_server, request: *mut alg_request) -> c_int;
    pub fn alg_server_wait(server: *mut alg_server, request: *mut alg_request) -> c_int;
    pub fn alg_server_drain(server: *mut alg_server) -> c_int;
    pub fn alg_server_completed(server: *const alg_server) -> c_ulonglong;
    pub fn alg_server_now_ns() -> i64;
    pub fn alg_server_destroy(server: *mut alg_server);
    pub fn alg_dgesv_mixed_noalloc(stream: *mut c_void, d_a: *const f64, d_b: *mut f64, n: c_int, d_ipiv: *mut c_int, d_info: *mut c_int, d_eta: *mut f64) -> c_int;
}
