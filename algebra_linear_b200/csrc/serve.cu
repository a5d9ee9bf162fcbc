// A device-resident request loop for mixed dense and sparse solves.
//
// Requests (dense dgesv of any order, or refactorize+solve of an analyzed
// sparse pattern with fresh values) are queued in arrival order. Worker
// threads, each with its own CUDA stream and workspace, take the oldest
// request as soon as they are idle and the request's device bytes fit in the
// remaining HBM budget, so requests that arrive while others run are admitted
// as slots and memory free up and their work overlaps on the device. Every
// worker keeps its own numeric copy of each sparse pattern (one shared
// symbolic analysis), so the factors of the last refactorization stay on the
// device. A request's result depends only on its inputs: each runs the same
// deterministic kernels alone or in the mix.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "context.cuh"

namespace {

int64_t now_ns() {
  return std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

size_t dense_bytes(const alg_request& r) {
  const size_t n = r.n;
  size_t b = 8 * n * n + 64 * n;
  if (r.precision == ALG_REQ_MIXED) b += 4 * n * n + 8 * n * 40;  // FP32 copy, refinement and Krylov vectors
  return b;
}

}  // namespace

struct alg_server {
  struct Worker {
    std::thread th;
    alg_ctx* ctx = nullptr;
    std::map<const alg_splu*, alg_splu*> clones;  // pattern -> this worker's numeric copy
    double* d_a = nullptr;
    double* d_b = nullptr;
    size_t cap_n = 0;
  };
  std::vector<Worker> workers;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<alg_request*> queue;
  size_t budget = 0, in_use = 0;
  int active = 0;  // requests taken by a worker and not finished
  bool stop = false;
  std::atomic<unsigned long long> completed{0};
  int device = 0;
};

namespace {

int ensure_dense(alg_server::Worker& w, size_t n) {
  if (n <= w.cap_n) return ALG_OK;
  if (w.d_a) cudaFree(w.d_a);
  if (w.d_b) cudaFree(w.d_b);
  w.d_a = w.d_b = nullptr;
  w.cap_n = 0;
  ALG_CUDA_TRY(cudaMalloc(&w.d_a, sizeof(double) * n * n));
  ALG_CUDA_TRY(cudaMalloc(&w.d_b, sizeof(double) * n));
  w.cap_n = n;
  return ALG_OK;
}

int run_dense(alg_server::Worker& w, alg_request* r) {
  const size_t n = r->n;
  if (n == 0) return ALG_OK;
  if (n > (size_t)w.cap_n) return ALG_BAD_SHAPE;
  cudaStream_t st = w.ctx->stream;
  ALG_CUDA_TRY(cudaMemcpyAsync(w.d_a, r->a, sizeof(double) * n * n, cudaMemcpyHostToDevice, st));
  ALG_CUDA_TRY(cudaMemcpyAsync(w.d_b, r->b, sizeof(double) * n, cudaMemcpyHostToDevice, st));
  int rc;
  if (r->precision == ALG_REQ_MIXED) {
    alg_mixed_opts o;
    alg_mixed_opts_default(&o);
    // requests share the GPU with the other workers' kernels: the
    // tournament's single-launch form is a cooperative launch that waits for
    // enough idle SMs, while partial pivoting is nearly as fast at the
    // orders served here
    o.pivoting = ALG_PIVOT_PARTIAL;
    alg_mixed_report rep;
    rc = alg_dgesv_mixed_dev(w.ctx, &o, w.d_a, (int)n, (int)n, w.d_b, 1, (int)n, &rep);
    r->backward_error = rep.backward_error;
  } else {
    rc = alg_dgesv_dev(w.ctx, ALG_UPDATE_FMA, w.d_a, (int)n, (int)n, w.d_b, 1, (int)n, nullptr);
    r->backward_error = -1.0;
  }
  if (rc != ALG_OK) return rc;
  ALG_CUDA_TRY(cudaMemcpyAsync(r->x, w.d_b, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
  ALG_CUDA_TRY(cudaStreamSynchronize(st));
  return ALG_OK;
}

int run_sparse(alg_server::Worker& w, alg_request* r) {
  alg_splu*& lu = w.clones[r->pattern];
  if (lu == nullptr) {
    ALG_TRY(alg_splu_clone(r->pattern, &lu));
    ALG_TRY(alg_splu_set_ctx(lu, w.ctx));
  }
  const size_t n = r->n;
  ALG_TRY(alg_splu_factorize_values(lu, r->values));
  std::copy(r->b, r->b + n, r->x);
  ALG_TRY(alg_splu_solve(lu, r->x, n));
  r->backward_error = -1.0;
  return ALG_OK;
}

void worker_loop(alg_server* S, int id) {
  alg_server::Worker& w = S->workers[id];
  cudaSetDevice(S->device);
  for (;;) {
    alg_request* r = nullptr;
    size_t bytes = 0;
    {
      std::unique_lock<std::mutex> lk(S->mu);
      for (;;) {
        if (S->stop && S->queue.empty()) return;
        if (!S->queue.empty()) {
          alg_request* head = S->queue.front();
          bytes = head->kind == ALG_REQ_DENSE ? dense_bytes(*head) : 0;
          if (S->in_use + bytes <= S->budget || S->in_use == 0) {
            r = head;
            S->queue.pop_front();
            S->in_use += bytes;
            S->active += 1;
            break;
          }
        }
        S->cv_work.wait(lk);
      }
    }
    r->t_start_ns = now_ns();
    r->worker = id;
    int rc = ALG_INVALID_ARGUMENT;
    if (r->kind == ALG_REQ_DENSE)
      rc = run_dense(w, r);
    else if (r->kind == ALG_REQ_SPARSE && r->pattern)
      rc = run_sparse(w, r);
    r->status = rc;
    r->t_done_ns = now_ns();
    {
      std::lock_guard<std::mutex> lk(S->mu);
      S->in_use -= bytes;
      S->active -= 1;
      r->done = 1;
      S->completed.fetch_add(1);
    }
    S->cv_done.notify_all();
    S->cv_work.notify_all();
  }
}

}  // namespace

extern "C" {

int alg_server_create(int n_workers, size_t hbm_budget_bytes, size_t max_dense_n, alg_server** out) {
  if (out == nullptr || n_workers < 1 || n_workers > 64) return ALG_INVALID_ARGUMENT;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    return ALG_NO_DEVICE;
  }
  auto* S = new alg_server();
  ALG_CUDA_TRY(cudaGetDevice(&S->device));
  S->budget = hbm_budget_bytes;
  S->workers.resize(n_workers);
  int rc = ALG_OK;
  for (auto& w : S->workers) {
    rc = alg_ctx_create(nullptr, &w.ctx);
    if (rc == ALG_OK) rc = ensure_dense(w, std::max<size_t>(max_dense_n, 1));
    if (rc != ALG_OK) break;
  }
  if (rc == ALG_OK && max_dense_n > 0) {
    // one small solve per worker before the threads start: kernel attributes
    // and workspaces are set up here, outside the concurrent phase
    const size_t n = std::min<size_t>(max_dense_n, 64);
    std::vector<double> a(n * n, 0.0), b(n, 1.0), x(n);
    for (size_t i = 0; i < n; ++i) a[i + i * n] = 2.0;
    for (auto& w : S->workers) {
      for (int prec : {ALG_REQ_FP64, ALG_REQ_MIXED}) {
        alg_request r{};
        r.kind = ALG_REQ_DENSE;
        r.precision = prec;
        r.n = n;
        r.a = a.data();
        r.b = b.data();
        r.x = x.data();
        rc = run_dense(w, &r);
        if (rc != ALG_OK) break;
      }
      if (rc != ALG_OK) break;
    }
  }
  if (rc != ALG_OK) {
    for (auto& w : S->workers) {
      if (w.d_a) cudaFree(w.d_a);
      if (w.d_b) cudaFree(w.d_b);
      if (w.ctx) alg_ctx_destroy(w.ctx);
    }
    delete S;
    return rc;
  }
  for (int i = 0; i < n_workers; ++i) S->workers[i].th = std::thread(worker_loop, S, i);
  *out = S;
  return ALG_OK;
}

int alg_server_submit(alg_server* S, alg_request* r) {
  if (S == nullptr || r == nullptr) return ALG_INVALID_ARGUMENT;
  if (r->kind == ALG_REQ_DENSE && (r->n > S->workers[0].cap_n || (r->n > 0 && (!r->a || !r->b || !r->x))))
    return r->n > S->workers[0].cap_n ? ALG_BAD_SHAPE : ALG_INVALID_ARGUMENT;
  if (r->kind == ALG_REQ_SPARSE && (r->pattern == nullptr || !r->b || !r->x)) return ALG_INVALID_ARGUMENT;
  if (r->kind != ALG_REQ_DENSE && r->kind != ALG_REQ_SPARSE) return ALG_INVALID_ARGUMENT;
  r->done = 0;
  r->status = -1;
  r->t_submit_ns = now_ns();
  {
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->stop) return ALG_INVALID_ARGUMENT;
    S->queue.push_back(r);
  }
  S->cv_work.notify_one();
  return ALG_OK;
}

int alg_server_wait(alg_server* S, alg_request* r) {
  if (S == nullptr || r == nullptr) return ALG_INVALID_ARGUMENT;
  std::unique_lock<std::mutex> lk(S->mu);
  S->cv_done.wait(lk, [&] { return r->done != 0; });
  return r->status;
}

int alg_server_drain(alg_server* S) {
  if (S == nullptr) return ALG_INVALID_ARGUMENT;
  std::unique_lock<std::mutex> lk(S->mu);
  S->cv_done.wait(lk, [&] { return S->queue.empty() && S->active == 0; });
  return ALG_OK;
}

unsigned long long alg_server_completed(const alg_server* S) { return S ? S->completed.load() : 0; }

int64_t alg_server_now_ns(void) { return now_ns(); }

void alg_server_destroy(alg_server* S) {
  if (S == nullptr) return;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
  }
  S->cv_work.notify_all();
  for (auto& w : S->workers)
    if (w.th.joinable()) w.th.join();
  for (auto& w : S->workers) {
    for (auto& kv : w.clones) alg_splu_free(kv.second);
    if (w.d_a) cudaFree(w.d_a);
    if (w.d_b) cudaFree(w.d_b);
    if (w.ctx) alg_ctx_destroy(w.ctx);
  }
  delete S;
}

}  // extern "C"
