// The library context: device, stream, status block and a growable
// workspace arena. One context is used by one thread at a time.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <mutex>
#include <vector>

#include "common.cuh"

// Kernel classes timed by the context's profiler (alg_ctx_set_profiling).
enum AlgKernelClass : int {
  ALG_K_PANEL = 0,   // leaf panel LU (cluster)
  ALG_K_LASWP,       // deferred row interchanges
  ALG_K_TRSM,        // U12 = L11^-1 A12
  ALG_K_GEMM,        // trailing update on the CUDA cores
  ALG_K_GEMM_TC,     // trailing update on the tensor cores (tcgen05)
  ALG_K_SOLVE,       // triangular solves
  ALG_K_RESID,       // FP64 residual / norms
  ALG_K_CAST,        // precision conversion
  ALG_K_BATCH,       // batched small systems
  ALG_K_SPARSE,      // sparse factorization / solve
  ALG_K_MISC,
  ALG_K_COUNT
};

struct alg_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int sm_count = 0;
  alg::DevStatus* d_status = nullptr;   // device status block
  alg::DevStatus* h_status = nullptr;   // pinned host mirror
  // Arena of named device buffers, grown on demand and reused across calls.
  struct Buf {
    void* ptr = nullptr;
    size_t bytes = 0;
  };
  std::vector<Buf> bufs;
  std::mutex mu;  // serialises the shared per-device contexts of the drop-ins
  // profiler: event pairs around launches of the timed classes; a context
  // with a parent records its launches (on its own stream) in the parent's
  // profile (the lanes of a sparse factorization)
  alg_ctx* prof_parent = nullptr;
  bool prof_on = false;
  struct ProfPending {
    int cls;
    cudaEvent_t e0, e1;
    double flops, bytes;
  };
  std::vector<ProfPending> prof_pending;
  std::vector<cudaEvent_t> prof_pool;
  struct ProfTotal {
    unsigned long long launches = 0;
    double ms = 0, flops = 0, bytes = 0;
  };
  ProfTotal prof[ALG_K_COUNT];
  // look-ahead LU: a high-priority stream for the panel chain and a
  // low-priority one for the rest of each trailing update (created on use)
  cudaStream_t la_stream[2] = {nullptr, nullptr};
  cudaEvent_t la_event[4] = {nullptr, nullptr, nullptr, nullptr};
  // bounded device waits of the dataflow solves: the limit (alg_ctx_set_wait_limit)
  // and the number of coming solves whose first block waits on a flag that
  // nothing sets (alg_ctx_inject_stuck_wait: tests of the timeout path)
  unsigned long long wait_limit_ns = 0;  // 0: the library default (2 s)
  int stuck_waits = 0;
};

namespace alg {

// Named workspace slots of the arena.
enum WsSlot : int {
  WS_A = 0,       // matrix copy (host drop-ins)
  WS_B,           // right-hand sides (host drop-ins)
  WS_X,           // solve scratch
  WS_IPIV,
  WS_PERM,
  WS_LAB,
  WS_PERM_TMP,
  WS_A32,         // low-precision working matrix (mixed form)
  WS_R,           // residual (mixed form)
  WS_KRYLOV,      // GMRES basis (mixed form)
  WS_PARTIAL,     // reduction partials
  WS_MISC,
  WS_GMRES,       // GMRES basis and work vectors (mixed form)
  WS_PRECOND,     // preconditioner scratch (mixed form)
  WS_RBT,         // butterfly coefficients (mixed form)
  WS_IDENT,       // identity permutation
  WS_BATCH,       // batched-solve queues
  WS_TSLU,        // tournament-pivoting panel scratch
  WS_TC_CHAIN,    // tensor-core operands of the look-ahead chain's narrow update
  WS_COUNT
};

// Returns a device buffer of at least `bytes` for `slot`, growing it if needed.
int ws_get(alg_ctx* ctx, int slot, size_t bytes, void** out);

// Shared per-device context used by the host-pointer drop-ins (created on first
// use; lives until process exit). Locks ctx->mu; the caller unlocks via guard.
int default_ctx(alg_ctx** out);

// Clears the status block (singular_col = INT_MAX, flags = 0) on the stream.
int status_reset(alg_ctx* ctx);
// Copies the status block to the host mirror and synchronises the stream.
int status_fetch(alg_ctx* ctx);

int ctx_init(alg_ctx* ctx, cudaStream_t stream);

// Profiler hooks: prof_begin records a start event (if profiling is on) and
// returns a token; prof_end records the stop event with the launch's
// algorithmic flops/bytes. prof_collect (called after a stream sync) folds
// finished pairs into the per-class totals.
int prof_begin(alg_ctx* ctx, int cls);
void prof_end(alg_ctx* ctx, int token, double flops, double bytes);
void prof_collect(alg_ctx* ctx);
void ctx_release(alg_ctx* ctx);
// The look-ahead streams and events of ctx (created on first use).
int ctx_lookahead_streams(alg_ctx* ctx);

}  // namespace alg
