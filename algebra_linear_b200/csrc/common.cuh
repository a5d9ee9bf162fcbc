// Shared helpers of the B200 LU kernels: status words, error plumbing,
// exact/fused arithmetic selectors and bounded waits.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <climits>

#include "algebra_linear_gpu.h"

namespace alg {

// Device status block, one per context. Kernels only ever lower
// singular_col (atomicMin) or raise the flags; the host clears it per call.
struct DevStatus {
  int singular_col;   // first column whose pivot was exactly zero, INT_MAX if none
  int timeout;        // a bounded wait ran out (kernel returned early)
  int bad_input;      // a kernel met an argument it rejects
  int pad[5];
};

// Arithmetic of one multiply-subtract `acc - l * u`.
//  EXACT = true : rounded product, then rounded difference (two roundings),
//                 the operation order of the reference's scalar loop
//                 (src/lapack/mod.rs:156-158), reproduced bit for bit.
//  EXACT = false: one fused multiply-add (one rounding), twice the FP64 rate.
template <bool EXACT>
__device__ __forceinline__ double msub(double acc, double l, double u) {
  if constexpr (EXACT) {
    return __dsub_rn(acc, __dmul_rn(l, u));
  } else {
    return __fma_rn(-l, u, acc);
  }
}
template <bool EXACT>
__device__ __forceinline__ float msub(float acc, float l, float u) {
  if constexpr (EXACT) {
    return __fsub_rn(acc, __fmul_rn(l, u));
  } else {
    return __fmaf_rn(-l, u, acc);
  }
}

__device__ __forceinline__ double div_rn(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }

__device__ __forceinline__ uint64_t global_timer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Every spin-wait in this library gives up after this long, raises the
// timeout flag of its status block and lets its kernel return.
constexpr uint64_t kWaitLimitNs = 2000000000ull;  // 2 s

}  // namespace alg

#define ALG_CUDA_TRY(expr)                                              \
  do {                                                                  \
    cudaError_t _e = (expr);                                            \
    if (_e != cudaSuccess) {                                            \
      alg::record_cuda_error(_e, #expr, __FILE__, __LINE__);            \
      return _e == cudaErrorMemoryAllocation ? ALG_OUT_OF_DEVICE_MEMORY \
                                             : ALG_CUDA_ERROR;          \
    }                                                                   \
  } while (0)

#define ALG_TRY(expr)            \
  do {                           \
    int _rc = (expr);            \
    if (_rc != ALG_OK) return _rc; \
  } while (0)

namespace alg {
void record_cuda_error(cudaError_t e, const char* what, const char* file, int line);
// Process-wide count of kernels this library has launched (relaxed atomic).
void count_launches(unsigned long long k = 1);
}
