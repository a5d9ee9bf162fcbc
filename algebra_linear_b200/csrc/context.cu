// Context, workspace arena, status block and status strings.
#include <atomic>
#include <climits>
#include <cstring>
#include <map>
#include <memory>

#include "context.cuh"

namespace alg {

static thread_local char g_last_error[512];
static std::atomic<unsigned long long> g_launches{0};

void count_launches(unsigned long long k) { g_launches.fetch_add(k, std::memory_order_relaxed); }

void record_cuda_error(cudaError_t e, const char* what, const char* file, int line) {
  std::snprintf(g_last_error, sizeof(g_last_error), "%s: %s (%s:%d)", cudaGetErrorString(e), what,
                file, line);
  if (std::getenv("ALG_VERBOSE") != nullptr) std::fprintf(stderr, "[algebra_linear_gpu] %s\n", g_last_error);
}

__global__ void status_reset_kernel(DevStatus* s) {
  if (threadIdx.x == 0) {
    s->singular_col = INT_MAX;
    s->timeout = 0;
    s->bad_input = 0;
  }
}

int ctx_init(alg_ctx* ctx, cudaStream_t stream) {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    return ALG_NO_DEVICE;
  }
  ALG_CUDA_TRY(cudaGetDevice(&ctx->device));
  ALG_CUDA_TRY(cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, ctx->device));
  if (stream == nullptr) {
    ALG_CUDA_TRY(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    ctx->own_stream = true;
  } else {
    ctx->stream = stream;
    ctx->own_stream = false;
  }
  ALG_CUDA_TRY(cudaMalloc(&ctx->d_status, sizeof(DevStatus)));
  ALG_CUDA_TRY(cudaMallocHost(&ctx->h_status, sizeof(DevStatus)));
  ctx->bufs.assign(WS_COUNT, alg_ctx::Buf{});
  return ALG_OK;
}

static cudaEvent_t prof_event(alg_ctx* ctx) {
  if (!ctx->prof_pool.empty()) {
    cudaEvent_t e = ctx->prof_pool.back();
    ctx->prof_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

int prof_begin(alg_ctx* ctx, int cls) {
  alg_ctx* pc = ctx->prof_parent ? ctx->prof_parent : ctx;
  if (!pc->prof_on) return -1;
  alg_ctx::ProfPending pp;
  pp.cls = cls;
  pp.e0 = prof_event(pc);
  pp.e1 = prof_event(pc);
  pp.flops = pp.bytes = 0;
  cudaEventRecord(pp.e0, ctx->stream);
  pc->prof_pending.push_back(pp);
  return (int)pc->prof_pending.size() - 1;
}

void prof_end(alg_ctx* ctx, int token, double flops, double bytes) {
  alg_ctx* pc = ctx->prof_parent ? ctx->prof_parent : ctx;
  if (token < 0 || !pc->prof_on) return;
  auto& pp = pc->prof_pending[token];
  pp.flops = flops;
  pp.bytes = bytes;
  cudaEventRecord(pp.e1, ctx->stream);
}

void prof_collect(alg_ctx* ctx) {
  if (ctx->prof_pending.empty()) return;
  cudaStreamSynchronize(ctx->stream);
  for (auto& pp : ctx->prof_pending) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, pp.e0, pp.e1) == cudaSuccess) {
      auto& t = ctx->prof[pp.cls];
      t.launches += 1;
      t.ms += ms;
      t.flops += pp.flops;
      t.bytes += pp.bytes;
    }
    ctx->prof_pool.push_back(pp.e0);
    ctx->prof_pool.push_back(pp.e1);
  }
  cudaGetLastError();
  ctx->prof_pending.clear();
}

int ctx_lookahead_streams(alg_ctx* ctx) {
  if (ctx->la_stream[0]) return ALG_OK;
  int least = 0, greatest = 0;
  ALG_CUDA_TRY(cudaDeviceGetStreamPriorityRange(&least, &greatest));
  ALG_CUDA_TRY(cudaStreamCreateWithPriority(&ctx->la_stream[0], cudaStreamNonBlocking, greatest));
  ALG_CUDA_TRY(cudaStreamCreateWithPriority(&ctx->la_stream[1], cudaStreamNonBlocking, least));
  for (auto& e : ctx->la_event) ALG_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  return ALG_OK;
}

void ctx_release(alg_ctx* ctx) {
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (auto& s : ctx->la_stream)
    if (s) {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
      s = nullptr;
    }
  for (auto& e : ctx->la_event)
    if (e) {
      cudaEventDestroy(e);
      e = nullptr;
    }
  prof_collect(ctx);
  for (auto e : ctx->prof_pool) cudaEventDestroy(e);
  ctx->prof_pool.clear();
  for (auto& b : ctx->bufs) {
    if (b.ptr) cudaFree(b.ptr);
    b = alg_ctx::Buf{};
  }
  if (ctx->d_status) cudaFree(ctx->d_status);
  if (ctx->h_status) cudaFreeHost(ctx->h_status);
  if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
  ctx->d_status = nullptr;
  ctx->h_status = nullptr;
  ctx->stream = nullptr;
}

int ws_get(alg_ctx* ctx, int slot, size_t bytes, void** out) {
  auto& b = ctx->bufs[slot];
  if (bytes == 0) bytes = 256;
  if (b.bytes < bytes) {
    if (b.ptr) {
      ALG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
      ALG_CUDA_TRY(cudaFree(b.ptr));
      b = alg_ctx::Buf{};
    }
    const size_t want = (bytes + 4095) & ~size_t(4095);
    ALG_CUDA_TRY(cudaMalloc(&b.ptr, want));
    b.bytes = want;
  }
  *out = b.ptr;
  return ALG_OK;
}

int default_ctx(alg_ctx** out) {
  static std::mutex registry_mu;
  static std::map<int, std::unique_ptr<alg_ctx>> registry;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    return ALG_NO_DEVICE;
  }
  int dev = 0;
  ALG_CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> g(registry_mu);
  auto it = registry.find(dev);
  if (it == registry.end()) {
    auto ctx = std::make_unique<alg_ctx>();
    ALG_TRY(ctx_init(ctx.get(), nullptr));
    it = registry.emplace(dev, std::move(ctx)).first;
  }
  *out = it->second.get();
  return ALG_OK;
}

int status_reset(alg_ctx* ctx) {
  status_reset_kernel<<<1, 32, 0, ctx->stream>>>(ctx->d_status);
  count_launches();
  ALG_CUDA_TRY(cudaGetLastError());
  return ALG_OK;
}

int status_fetch(alg_ctx* ctx) {
  ALG_CUDA_TRY(cudaMemcpyAsync(ctx->h_status, ctx->d_status, sizeof(DevStatus),
                               cudaMemcpyDeviceToHost, ctx->stream));
  ALG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  prof_collect(ctx);
  if (ctx->h_status->timeout) return ALG_TIMEOUT;
  if (ctx->h_status->bad_input) return ALG_INVALID_ARGUMENT;
  return ALG_OK;
}

}  // namespace alg

extern "C" {

const char* alg_status_string(int status) {
  switch (status) {
    case ALG_OK: return "ok";
    case ALG_SINGULAR: return "the matrix is singular";
    case ALG_BAD_SHAPE: return "inconsistent shape or length";
    case ALG_CONVERGENCE: return "iterative refinement did not converge";
    case ALG_NOT_IMPLEMENTED: return "not implemented";
    case ALG_SP_BAD_SHAPE: return "inconsistent shape or length";
    case ALG_SP_INVALID_STRUCTURE: return "invalid CSC structure";
    case ALG_SP_UNSORTED_ROWS: return "row indices must be strictly increasing within a column";
    case ALG_SP_DUPLICATE_ENTRY: return "duplicate entry in a column";
    case ALG_SP_SINGULAR: return "the matrix is singular";
    case ALG_SP_INDEX_OVERFLOW: return "index or workspace size overflow";
    case ALG_SP_STRUCTURE_MISMATCH: return "the matrix pattern differs from the symbolic analysis";
    case ALG_SP_NOT_FINITE: return "the matrix has a NaN or infinite entry";
    case ALG_SP_NOT_FACTORIZED: return "the matrix has not been factorized";
    case ALG_CUDA_ERROR: return "CUDA error";
    case ALG_OUT_OF_DEVICE_MEMORY: return "out of device memory";
    case ALG_TIMEOUT: return "a device-side wait ran out of time";
    case ALG_INVALID_ARGUMENT: return "invalid argument";
    case ALG_NO_DEVICE: return "no CUDA device";
    default: return "unknown status";
  }
}

unsigned long long alg_kernel_launch_count(void) {
  return alg::g_launches.load(std::memory_order_relaxed);
}

const char* alg_version(void) { return "algebra_linear_gpu 0.1.0 (sm_100a)"; }

int alg_ctx_create(void* cuda_stream, alg_ctx** out) {
  if (out == nullptr) return ALG_INVALID_ARGUMENT;
  auto* ctx = new alg_ctx();
  const int rc = alg::ctx_init(ctx, static_cast<cudaStream_t>(cuda_stream));
  if (rc != ALG_OK) {
    alg::ctx_release(ctx);
    delete ctx;
    *out = nullptr;
    return rc;
  }
  *out = ctx;
  return ALG_OK;
}

void alg_ctx_destroy(alg_ctx* ctx) {
  if (ctx == nullptr) return;
  alg::ctx_release(ctx);
  delete ctx;
}

int alg_ctx_set_wait_limit(alg_ctx* ctx, unsigned long long limit_ns) {
  if (ctx == nullptr) return ALG_INVALID_ARGUMENT;
  ctx->wait_limit_ns = limit_ns;
  return ALG_OK;
}

int alg_ctx_inject_stuck_wait(alg_ctx* ctx, int count) {
  if (ctx == nullptr || count < 0) return ALG_INVALID_ARGUMENT;
  ctx->stuck_waits = count;
  return ALG_OK;
}

int alg_ctx_set_stream(alg_ctx* ctx, void* cuda_stream) {
  if (ctx == nullptr) return ALG_INVALID_ARGUMENT;
  if (ctx->own_stream && ctx->stream) {
    cudaStreamSynchronize(ctx->stream);
    cudaStreamDestroy(ctx->stream);
  }
  ctx->own_stream = false;
  ctx->stream = static_cast<cudaStream_t>(cuda_stream);
  if (ctx->stream == nullptr) {
    ALG_CUDA_TRY(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    ctx->own_stream = true;
  }
  return ALG_OK;
}

int alg_ctx_set_profiling(alg_ctx* ctx, int on) {
  if (ctx == nullptr) return ALG_INVALID_ARGUMENT;
  alg::prof_collect(ctx);
  ctx->prof_on = on != 0;
  return ALG_OK;
}

int alg_ctx_profile_reset(alg_ctx* ctx) {
  if (ctx == nullptr) return ALG_INVALID_ARGUMENT;
  alg::prof_collect(ctx);
  for (auto& t : ctx->prof) t = alg_ctx::ProfTotal{};
  return ALG_OK;
}

int alg_ctx_profile_get(alg_ctx* ctx, int kernel_class, unsigned long long* launches,
                        double* total_ms, double* flops, double* bytes) {
  if (ctx == nullptr || kernel_class < 0 || kernel_class >= ALG_K_COUNT) return ALG_INVALID_ARGUMENT;
  alg::prof_collect(ctx);
  const auto& t = ctx->prof[kernel_class];
  if (launches) *launches = t.launches;
  if (total_ms) *total_ms = t.ms;
  if (flops) *flops = t.flops;
  if (bytes) *bytes = t.bytes;
  return ALG_OK;
}

}  // extern "C"
