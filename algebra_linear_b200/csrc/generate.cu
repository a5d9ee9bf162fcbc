// Device generator of the LAPACK DLARNV stream the reference's tests use
// (src/lapack/families.rs:166-249), for building the dense workloads on the
// GPU with the same values the CPU reference would draw.
//
// DLARUV keeps a 48-bit state x and returns x * a^i mod 2^48 (i = 1..n) for
// a batch of n <= 128 values, the new state being the last product; DLARNV
// draws batches of 64. Value v of the stream is therefore s * a^(v+1) mod 2^48
// for the starting state s, whatever the batching. Its conversion to (0,1),
// R*(w1 + R*(w2 + R*(w3 + R*w4))) with R = 2^-12 over the four 12-bit words,
// is exact in double precision (48 significant bits), so the value is exactly
// x / 2^48 and never rounds to 1.0 (the reference's retry branch cannot fire
// in double precision).
#include <cstdint>

#include "context.cuh"

namespace alg {
namespace {

constexpr uint64_t kMult = 33952834046453ULL;
constexpr uint64_t kMask48 = (1ULL << 48) - 1;

__host__ __device__ inline uint64_t mulmod48(uint64_t a, uint64_t b) { return (a * b) & kMask48; }

__host__ __device__ inline uint64_t powmod48(uint64_t base, uint64_t e) {
  uint64_t r = 1;
  while (e) {
    if (e & 1) r = mulmod48(r, base);
    base = mulmod48(base, base);
    e >>= 1;
  }
  return r;
}

constexpr int kGenThreads = 256;
constexpr int kGenPerThread = 64;

__global__ void larnv_kernel(int dist, uint64_t s, size_t n, double* x) {
  const size_t first = ((size_t)blockIdx.x * kGenThreads + threadIdx.x) * kGenPerThread;
  if (first >= n) return;
  uint64_t v = mulmod48(s, powmod48(kMult, first + 1));
  const size_t last = first + kGenPerThread < n ? first + kGenPerThread : n;
  for (size_t i = first; i < last; ++i) {
    const double u = __dmul_rn((double)v, 0x1p-48);  // exact: x / 2^48
    x[i] = dist == 1 ? u : __dsub_rn(__dmul_rn(2.0, u), 1.0);
    v = mulmod48(v, kMult);
  }
}

}  // namespace
}  // namespace alg

extern "C" int alg_larnv_dev(alg_ctx* ctx, int dist, const uint32_t seed[4], size_t n, double* d_x,
                             uint32_t seed_out[4]) {
  if (ctx == nullptr || seed == nullptr) return ALG_INVALID_ARGUMENT;
  if (dist != 1 && dist != 2) return ALG_INVALID_ARGUMENT;
  for (int i = 0; i < 4; ++i)
    if (seed[i] > 4095) return ALG_INVALID_ARGUMENT;
  const uint64_t s = ((uint64_t)seed[0] << 36) | ((uint64_t)seed[1] << 24) | ((uint64_t)seed[2] << 12) | seed[3];
  if (n > 0) {
    if (d_x == nullptr) return ALG_INVALID_ARGUMENT;
    const size_t per_block = (size_t)alg::kGenThreads * alg::kGenPerThread;
    const size_t blocks = (n + per_block - 1) / per_block;
    alg::larnv_kernel<<<(unsigned)blocks, alg::kGenThreads, 0, ctx->stream>>>(dist, s, n, d_x);
    alg::count_launches();
    ALG_CUDA_TRY(cudaGetLastError());
  }
  if (seed_out) {
    const uint64_t t = alg::mulmod48(s, alg::powmod48(alg::kMult, n));
    seed_out[0] = (uint32_t)((t >> 36) & 4095);
    seed_out[1] = (uint32_t)((t >> 24) & 4095);
    seed_out[2] = (uint32_t)((t >> 12) & 4095);
    seed_out[3] = (uint32_t)(t & 4095);
  }
  return ALG_OK;
}
