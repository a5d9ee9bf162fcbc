// C entry points of the sparse LU (SparseLu, src/sparse/faer/sparse_lu.rs).
//
// analyze runs on the host (validation, COLAMD, supernodal symbolic analysis
// and the static front plan) and needs no GPU, as in the reference, where it
// runs once per pattern. factorize uploads the plan on first use, factors on
// the GPU into the spare of two factor sets and, on success, makes it the
// current one: a failed factorization leaves the previous factors and
// statistics in place (sparse_lu.rs:82-83, 114-115).
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>

#include "sparse_numeric.cuh"

using alg::sp::idx;

struct alg_splu {
  size_t n = 0, nnz = 0;
  uint64_t fingerprint = 0;
  int effective = ALG_SPLU_SIMPLICIAL;
  int has_ratio = 0;
  double flop_ratio = 0.0;
  double ordering_time = 0.0;
  alg::sp::Supernodal sym;
  alg::sp::FrontPlan plan;
  alg_ctx* ctx = nullptr;
  bool own_ctx = false;
  alg::sp::DeviceLu dev;
  bool dev_ready = false;
  int cur = -1;  // factor set of the last successful factorization
  int prec = -1;       // precision of the next factorization (-1: FP64)
  double tol = 0.0;    // the mixed form's refinement target and step limit
  int max_ir = 0;
  int has_stats = 0;
  alg_splu_stats stats{};
};

namespace {

constexpr int kSmallFrontRows = 256;
constexpr double kChainTolerance = 0.05;
constexpr int kLanes = 2;

// CscView::new for an n x n matrix (csc.rs:39-76, 178-189).
int check_view(const alg_splu* lu, const size_t* col_ptr, size_t col_ptr_len, const size_t* row_idx,
               size_t row_idx_len, size_t values_len) {
  if (col_ptr_len != lu->n + 1 || col_ptr == nullptr || (row_idx_len > 0 && row_idx == nullptr))
    return ALG_SP_BAD_SHAPE;
  const int rc = alg::sp::validate_csc(lu->n, lu->n, col_ptr, col_ptr_len, row_idx, row_idx_len);
  if (rc != ALG_OK) return rc;
  if (values_len != col_ptr[lu->n]) return ALG_SP_BAD_SHAPE;
  return ALG_OK;
}

// Uploads the plan and allocates the arenas on first use; the first
// factorization fixes the handle's scalar (words = 1 real, 2 complex) and a
// later call with the other scalar is rejected (ALG_INVALID_ARGUMENT).
int ensure_device(alg_splu* lu, int words = 1) {
  if (lu->dev_ready) return lu->dev.words == words ? ALG_OK : ALG_INVALID_ARGUMENT;
  if (lu->ctx == nullptr) {
    const int rc = alg_ctx_create(nullptr, &lu->ctx);
    if (rc != ALG_OK) return rc;
    lu->own_ctx = true;
  }
  const int rc = lu->dev.init(lu->ctx, &lu->plan, words);
  if (rc != ALG_OK) {
    lu->dev.release();
    return rc;
  }
  lu->dev_ready = true;
  return ALG_OK;
}

// Numeric factorization of the values already in dev.d_values.
int factor_loaded(alg_splu* lu) {
  const auto t0 = std::chrono::steady_clock::now();
  if (lu->plan.structurally_singular) return ALG_SP_SINGULAR;
  const int set = lu->cur < 0 ? 0 : 1 - lu->cur;
  lu->dev.prec = lu->prec;
  lu->dev.tol = lu->tol;
  lu->dev.max_ir = lu->max_ir;
  ALG_TRY(lu->dev.factor(set));
  alg::sp::Stats st;
  const int rc = lu->dev.finish(set, &st);
  if (rc != ALG_OK) return rc;
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  lu->cur = set;
  alg_splu_stats& s = lu->stats;
  s.n = lu->n;
  s.nnz_a = lu->nnz;
  s.nnz_l = st.nnz_l;
  s.nnz_u = st.nnz_u;
  s.fill_ratio = lu->nnz == 0 ? 0.0 : (double)(st.nnz_l + st.nnz_u) / (double)lu->nnz;
  s.flops_estimate = st.flops_estimate;
  s.method = lu->effective;
  s.has_flop_ratio = lu->has_ratio;
  s.flop_ratio = lu->flop_ratio;
  s.ordering_time = lu->ordering_time;
  s.factorization_time = secs;
  lu->has_stats = 1;
  return ALG_OK;
}

__global__ void nonfinite_kernel(const double* v, size_t n, int* flag) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    if (!isfinite(v[i])) atomicExch(flag, 1);
}

}  // namespace

extern "C" {

int alg_splu_analyze(const size_t* col_ptr, size_t col_ptr_len, const size_t* row_idx, size_t row_idx_len,
                     int method, double flop_ratio_threshold, alg_splu** out) {
  if (out == nullptr) return ALG_INVALID_ARGUMENT;
  *out = nullptr;
  if (col_ptr_len == 0 || col_ptr == nullptr) return ALG_SP_BAD_SHAPE;
  if (method != ALG_SPLU_SIMPLICIAL && method != ALG_SPLU_SUPERNODAL && method != ALG_SPLU_AUTO)
    return ALG_INVALID_ARGUMENT;
  const size_t n = col_ptr_len - 1;
  if (row_idx_len > 0 && row_idx == nullptr) return ALG_SP_BAD_SHAPE;
  for (size_t q = 0; q < row_idx_len; ++q)
    if (row_idx[q] >= n) return ALG_SP_BAD_SHAPE;  // more rows than columns
  int rc = alg::sp::validate_csc(n, n, col_ptr, col_ptr_len, row_idx, row_idx_len);
  if (rc != ALG_OK) return rc;
  if (n > (size_t)INT32_MAX / 2 || row_idx_len > (size_t)INT64_MAX / 4) return ALG_SP_INDEX_OVERFLOW;
  auto lu = std::make_unique<alg_splu>();
  lu->n = n;
  lu->nnz = row_idx_len;
  alg::sp::Pattern p;
  p.n = (idx)n;
  p.col_ptr = col_ptr;
  p.row_idx = row_idx;
  lu->fingerprint = alg::sp::fingerprint(p);
  std::vector<idx> perm, perm_inv;
  const auto t0 = std::chrono::steady_clock::now();
  rc = alg::sp::colamd_order(p, 0.5, 0.5, true, &perm, &perm_inv);
  lu->ordering_time = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (rc != ALG_OK) return rc;
  // the supernodal structure (relaxation 4 / 0.1, solver.rs:37-42,134-141)
  rc = alg::sp::supernodal_analyze(p, perm, perm_inv, 4, 0.1, &lu->sym);
  if (rc != ALG_OK) return rc;
  if (method != ALG_SPLU_SIMPLICIAL) {
    double squares = 0.0;
    for (idx c : lu->sym.col_counts) squares += (double)c * (double)c;
    lu->flop_ratio = row_idx_len == 0 ? 0.0 : squares / (double)row_idx_len;
    lu->has_ratio = 1;
  }
  if (method == ALG_SPLU_SUPERNODAL)
    lu->effective = ALG_SPLU_SUPERNODAL;
  else if (method == ALG_SPLU_AUTO)
    lu->effective = lu->flop_ratio > flop_ratio_threshold ? ALG_SPLU_SUPERNODAL : ALG_SPLU_SIMPLICIAL;
  else
    lu->effective = ALG_SPLU_SIMPLICIAL;
  // GPU plan: the reference's partition with chains of children merged;
  // large fronts in kLanes concurrent lanes (ALG_SPLU_LANES overrides)
  {
    int lanes = kLanes;
    if (const char* e = std::getenv("ALG_SPLU_LANES")) lanes = std::max(1, std::min(8, std::atoi(e)));
    // the reference's partition cut at its etree breaks (ALG_SPLU_KEEP_GLUED=1:
    // measurement switch that keeps it whole)
    alg::sp::Supernodal chains;
    if (std::getenv("ALG_SPLU_KEEP_GLUED"))
      chains = lu->sym;
    else
      alg::sp::split_at_etree_breaks(lu->sym, &chains);
    alg::sp::FrontPlan first;
    rc = alg::sp::build_front_plan(p, chains, kSmallFrontRows, lanes, &first);
    if (rc != ALG_OK) return rc;
    std::vector<idx> ptr;
    // the merge rules' tolerance and traffic weight (ALG_SPLU_CHAIN_TOL,
    // ALG_SPLU_MERGE_TRAFFIC: measurement switches)
    double tol = kChainTolerance, traffic = 1.0;
    if (const char* e = std::getenv("ALG_SPLU_CHAIN_TOL")) tol = std::max(0.0, std::atof(e));
    if (const char* e = std::getenv("ALG_SPLU_MERGE_TRAFFIC")) traffic = std::max(0.0, std::atof(e));
    alg::sp::amalgamate_chains(first, chains, tol, traffic, &ptr);
    if (ptr.size() == chains.supernode_ptr.size()) {
      lu->plan = std::move(first);
    } else {
      alg::sp::Supernodal coarse;
      alg::sp::repartition(chains, ptr, &coarse);
      rc = alg::sp::build_front_plan(p, coarse, kSmallFrontRows, lanes, &lu->plan);
      if (rc != ALG_OK) return rc;
    }
  }
  *out = lu.release();
  return ALG_OK;
}

int alg_splu_factorize(alg_splu* lu, const size_t* col_ptr, size_t col_ptr_len, const size_t* row_idx,
                       size_t row_idx_len, const double* values, size_t values_len) {
  if (lu == nullptr) return ALG_INVALID_ARGUMENT;
  int rc = check_view(lu, col_ptr, col_ptr_len, row_idx, row_idx_len, values_len);
  if (rc != ALG_OK) return rc;
  alg::sp::Pattern p;
  p.n = (idx)lu->n;
  p.col_ptr = col_ptr;
  p.row_idx = row_idx;
  if (row_idx_len != lu->nnz || alg::sp::fingerprint(p) != lu->fingerprint) return ALG_SP_STRUCTURE_MISMATCH;
  for (size_t q = 0; q < values_len; ++q)
    if (!std::isfinite(values[q])) return ALG_SP_NOT_FINITE;
  if (lu->n == 0) {
    lu->cur = 0;
    lu->stats = alg_splu_stats{};
    lu->stats.method = lu->effective;
    lu->stats.has_flop_ratio = lu->has_ratio;
    lu->stats.flop_ratio = lu->flop_ratio;
    lu->stats.ordering_time = lu->ordering_time;
    lu->has_stats = 1;
    return ALG_OK;
  }
  if (lu->plan.structurally_singular) return ALG_SP_SINGULAR;
  ALG_TRY(ensure_device(lu));
  ALG_CUDA_TRY(cudaMemcpyAsync(lu->dev.d_values, values, sizeof(double) * values_len, cudaMemcpyHostToDevice,
                               lu->ctx->stream));
  return factor_loaded(lu);
}

}  // extern "C"

namespace {

// solve with b of n values of `words` doubles each, from and to the host
int solve_host(alg_splu* lu, double* b, size_t b_len, int words) {
  if (lu->cur < 0) return ALG_SP_NOT_FACTORIZED;
  if (b_len != lu->n || (b_len > 0 && b == nullptr)) return ALG_SP_BAD_SHAPE;
  if (lu->n == 0) return ALG_OK;
  if (lu->dev.words != words) return ALG_INVALID_ARGUMENT;
  cudaStream_t st = lu->ctx->stream;
  const size_t bytes = sizeof(double) * words * lu->n;
  ALG_CUDA_TRY(cudaMemcpyAsync(lu->dev.d_rhs, b, bytes, cudaMemcpyHostToDevice, st));
  ALG_TRY(alg::status_reset(lu->ctx));
  ALG_TRY(lu->dev.solve(lu->cur));
  ALG_CUDA_TRY(cudaMemcpyAsync(b, lu->dev.d_rhs, bytes, cudaMemcpyDeviceToHost, st));
  ALG_TRY(alg::status_fetch(lu->ctx));  // synchronises
  if (lu->ctx->h_status->timeout) return ALG_TIMEOUT;
  return ALG_OK;
}

}  // namespace

extern "C" {

int alg_splu_solve(const alg_splu* lu, double* b, size_t b_len) {
  if (lu == nullptr) return ALG_INVALID_ARGUMENT;
  return solve_host(const_cast<alg_splu*>(lu), b, b_len, 1);
}

// SparseLu<Complex64>::factorize (sparse_lu.rs:91-121 with T = Complex64):
// values holds values_len complex entries as interleaved (re, im) doubles.
int alg_zsplu_factorize(alg_splu* lu, const size_t* col_ptr, size_t col_ptr_len, const size_t* row_idx,
                        size_t row_idx_len, const double* values, size_t values_len) {
  if (lu == nullptr) return ALG_INVALID_ARGUMENT;
  int rc = check_view(lu, col_ptr, col_ptr_len, row_idx, row_idx_len, values_len);
  if (rc != ALG_OK) return rc;
  if (values_len > 0 && values == nullptr) return ALG_SP_BAD_SHAPE;
  alg::sp::Pattern p;
  p.n = (idx)lu->n;
  p.col_ptr = col_ptr;
  p.row_idx = row_idx;
  if (row_idx_len != lu->nnz || alg::sp::fingerprint(p) != lu->fingerprint) return ALG_SP_STRUCTURE_MISMATCH;
  for (size_t q = 0; q < 2 * values_len; ++q)
    if (!std::isfinite(values[q])) return ALG_SP_NOT_FINITE;  // either part (lu.rs:79-81)
  if (lu->dev_ready && lu->dev.words != 2) return ALG_INVALID_ARGUMENT;
  if (lu->n == 0) {
    lu->cur = 0;
    lu->stats = alg_splu_stats{};
    lu->stats.method = lu->effective;
    lu->stats.has_flop_ratio = lu->has_ratio;
    lu->stats.flop_ratio = lu->flop_ratio;
    lu->stats.ordering_time = lu->ordering_time;
    lu->has_stats = 1;
    return ALG_OK;
  }
  if (lu->plan.structurally_singular) return ALG_SP_SINGULAR;
  ALG_TRY(ensure_device(lu, 2));
  ALG_CUDA_TRY(cudaMemcpyAsync(lu->dev.d_values, values, sizeof(double) * 2 * values_len, cudaMemcpyHostToDevice,
                               lu->ctx->stream));
  return factor_loaded(lu);
}

// SparseLu<Complex64>::solve (sparse_lu.rs:125-130): b holds n complex
// entries as interleaved (re, im) doubles and becomes x.
int alg_zsplu_solve(const alg_splu* lu, double* b, size_t b_len) {
  if (lu == nullptr) return ALG_INVALID_ARGUMENT;
  return solve_host(const_cast<alg_splu*>(lu), b, b_len, 2);
}

int alg_splu_effective_method(const alg_splu* lu) { return lu ? lu->effective : ALG_INVALID_ARGUMENT; }

int alg_splu_flop_ratio(const alg_splu* lu, double* ratio) {
  if (lu == nullptr || ratio == nullptr) return -1;
  *ratio = lu->flop_ratio;
  return lu->has_ratio;
}

int alg_splu_get_stats(const alg_splu* lu, alg_splu_stats* out) {
  if (lu == nullptr || out == nullptr) return ALG_INVALID_ARGUMENT;
  if (!lu->has_stats) return ALG_SP_NOT_FACTORIZED;
  *out = lu->stats;
  return ALG_OK;
}

int alg_splu_symbolic(const alg_splu* lu, size_t* col_perm, size_t* col_perm_inv, size_t* col_counts,
                      size_t* supernode_ptr, size_t* n_supernodes) {
  if (lu == nullptr) return ALG_INVALID_ARGUMENT;
  const auto& S = lu->sym;
  for (size_t i = 0; i < lu->n; ++i) {
    if (col_perm) col_perm[i] = (size_t)S.col_perm[i];
    if (col_perm_inv) col_perm_inv[i] = (size_t)S.col_perm_inv[i];
    if (col_counts) col_counts[i] = (size_t)S.col_counts[i];
  }
  if (n_supernodes) *n_supernodes = (size_t)S.n_supernodes();
  if (supernode_ptr)
    for (size_t s = 0; s < S.supernode_ptr.size(); ++s) supernode_ptr[s] = (size_t)S.supernode_ptr[s];
  return ALG_OK;
}

int alg_splu_row_perm(const alg_splu* lu, size_t* row_perm) {
  if (lu == nullptr || row_perm == nullptr) return ALG_INVALID_ARGUMENT;
  if (lu->cur < 0) return ALG_SP_NOT_FACTORIZED;
  if (lu->n == 0) return ALG_OK;
  std::vector<int32_t> h(lu->n);
  ALG_CUDA_TRY(cudaMemcpy(h.data(), lu->dev.fac[lu->cur].row_perm, sizeof(int32_t) * lu->n, cudaMemcpyDeviceToHost));
  for (size_t i = 0; i < lu->n; ++i) row_perm[i] = (size_t)h[i];
  return ALG_OK;
}

int alg_splu_plan_info(const alg_splu* lu, alg_splu_plan* out) {
  if (lu == nullptr || out == nullptr) return ALG_INVALID_ARGUMENT;
  const auto& F = lu->plan;
  out->n_fronts = (size_t)F.ns;
  size_t nsmall = 0, maxr = 0, maxc = 0;
  for (const auto& d : F.fronts) {
    nsmall += d.small ? 1 : 0;
    maxr = std::max<size_t>(maxr, (size_t)d.rows);
    maxc = std::max<size_t>(maxc, (size_t)(d.size + d.ncb));
  }
  out->n_small_fronts = nsmall;
  out->small_levels = F.small_level_ptr.empty() ? 0 : F.small_level_ptr.size() - 1;
  out->solve_levels = F.solve_level_ptr.empty() ? 0 : F.solve_level_ptr.size() - 1;
  out->max_front_rows = maxr;
  out->max_front_cols = maxc;
  out->factor_bytes = 8 * (size_t)(F.l_total + F.u_total);
  out->work_bytes = 8 * (size_t)(F.block_total + F.stack_total + F.front_buf);
  out->plan_flops = F.flops;
  out->structurally_singular = F.structurally_singular ? 1 : 0;
  out->n_lanes = F.n_lanes;
  out->top_fronts = F.top_fronts.size();
  return ALG_OK;
}

int alg_splu_set_ctx(alg_splu* lu, alg_ctx* ctx) {
  if (lu == nullptr || ctx == nullptr || lu->dev_ready) return ALG_INVALID_ARGUMENT;
  lu->ctx = ctx;
  lu->own_ctx = false;
  return ALG_OK;
}

int alg_splu_factorize_dev(alg_splu* lu, const double* d_values) {
  if (lu == nullptr || (lu->nnz > 0 && d_values == nullptr)) return ALG_INVALID_ARGUMENT;
  if (lu->n == 0) {
    lu->cur = 0;
    return ALG_OK;
  }
  if (lu->plan.structurally_singular) return ALG_SP_SINGULAR;
  ALG_TRY(ensure_device(lu));
  cudaStream_t st = lu->ctx->stream;
  if (lu->nnz > 0) {
    ALG_CUDA_TRY(cudaMemcpyAsync(lu->dev.d_values, d_values, sizeof(double) * lu->nnz, cudaMemcpyDeviceToDevice, st));
    ALG_CUDA_TRY(cudaMemsetAsync(lu->dev.d_flag + 1, 0, sizeof(int), st));
    nonfinite_kernel<<<std::max(1, std::min(4 * lu->ctx->sm_count, (int)((lu->nnz + 255) / 256))), 256, 0, st>>>(
        lu->dev.d_values, lu->nnz, lu->dev.d_flag + 1);
    alg::count_launches();
    int bad = 0;
    ALG_CUDA_TRY(cudaMemcpyAsync(&bad, lu->dev.d_flag + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    ALG_CUDA_TRY(cudaStreamSynchronize(st));
    if (bad) return ALG_SP_NOT_FINITE;
  }
  return factor_loaded(lu);
}

int alg_splu_solve_dev(alg_splu* lu, double* d_b) {
  if (lu == nullptr) return ALG_INVALID_ARGUMENT;
  if (lu->cur < 0) return ALG_SP_NOT_FACTORIZED;
  if (lu->n == 0) return ALG_OK;
  if (d_b == nullptr || lu->dev.words != 1) return ALG_INVALID_ARGUMENT;
  cudaStream_t st = lu->ctx->stream;
  ALG_CUDA_TRY(cudaMemcpyAsync(lu->dev.d_rhs, d_b, sizeof(double) * lu->n, cudaMemcpyDeviceToDevice, st));
  ALG_TRY(lu->dev.solve(lu->cur));
  ALG_CUDA_TRY(cudaMemcpyAsync(d_b, lu->dev.d_rhs, sizeof(double) * lu->n, cudaMemcpyDeviceToDevice, st));
  return ALG_OK;
}

int alg_splu_clone(const alg_splu* src, alg_splu** out) {
  if (src == nullptr || out == nullptr) return ALG_INVALID_ARGUMENT;
  auto lu = std::make_unique<alg_splu>();
  lu->n = src->n;
  lu->nnz = src->nnz;
  lu->fingerprint = src->fingerprint;
  lu->effective = src->effective;
  lu->has_ratio = src->has_ratio;
  lu->flop_ratio = src->flop_ratio;
  lu->ordering_time = src->ordering_time;
  lu->sym = src->sym;
  lu->plan = src->plan;
  lu->prec = src->prec;
  lu->tol = src->tol;
  lu->max_ir = src->max_ir;
  *out = lu.release();
  return ALG_OK;
}

int alg_splu_factorize_values(alg_splu* lu, const double* values) {
  if (lu == nullptr || (lu->nnz > 0 && values == nullptr)) return ALG_INVALID_ARGUMENT;
  for (size_t q = 0; q < lu->nnz; ++q)
    if (!std::isfinite(values[q])) return ALG_SP_NOT_FINITE;
  if (lu->n == 0) {
    lu->cur = 0;
    return ALG_OK;
  }
  if (lu->plan.structurally_singular) return ALG_SP_SINGULAR;
  ALG_TRY(ensure_device(lu));
  ALG_CUDA_TRY(cudaMemcpyAsync(lu->dev.d_values, values, sizeof(double) * lu->nnz, cudaMemcpyHostToDevice,
                               lu->ctx->stream));
  return factor_loaded(lu);
}

int alg_splu_set_precision(alg_splu* lu, int precision, double tol, int max_ir) {
  if (lu == nullptr) return ALG_INVALID_ARGUMENT;
  if (precision != ALG_SPLU_FP64 && precision != ALG_PREC_FP32 && precision != ALG_PREC_TF32 &&
      precision != ALG_PREC_BF16 && precision != ALG_PREC_TF32X3)
    return ALG_INVALID_ARGUMENT;
  if (!(tol == tol)) return ALG_INVALID_ARGUMENT;
  lu->prec = precision;
  lu->tol = tol;
  lu->max_ir = max_ir;
  return ALG_OK;
}

int alg_splu_last_solve(const alg_splu* lu, alg_splu_refine_report* out) {
  if (lu == nullptr || out == nullptr) return ALG_INVALID_ARGUMENT;
  if (lu->cur < 0) return ALG_SP_NOT_FACTORIZED;
  out->precision = lu->dev.last.precision;
  out->iterations = lu->dev.last.iterations;
  out->fell_back = lu->dev.last.fell_back;
  out->factor_precision = lu->dev_ready ? lu->dev.fac[lu->cur].prec : ALG_SPLU_FP64;
  out->backward_error = lu->dev.last.backward_error;
  return ALG_OK;
}

void alg_splu_free(alg_splu* lu) {
  if (lu == nullptr) return;
  if (lu->dev_ready) {
    cudaStreamSynchronize(lu->ctx->stream);
    lu->dev.release();
  }
  if (lu->own_ctx) alg_ctx_destroy(lu->ctx);
  delete lu;
}

}  // extern "C"
