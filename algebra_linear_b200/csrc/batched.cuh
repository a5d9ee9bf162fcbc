// Batched dense dgesv (many uneven systems, one persistent launch per bucket).
#pragma once

#include "context.cuh"

namespace alg {

struct BatchSpec {
  int count = 0;
  const int* d_n = nullptr;
  const long long* d_a_off = nullptr;
  const long long* d_b_off = nullptr;
  double* d_a = nullptr;
  double* d_b = nullptr;
  float* d_a32 = nullptr;
  int* d_ipiv = nullptr;
  double* d_work = nullptr;
  int* d_info = nullptr;
  double* d_eta = nullptr;
  int mixed = 0;
  int max_ir = 10;
  double tol_scale = 10.0;
  double flops = 0.0;
};

struct BucketLaunch {
  int count = 0;
  int cap = 0;          // largest order in the bucket
  int threads = 256;    // CTA size chosen by the autotuner
  int panel = 32;       // panel width (16 or 32) chosen by the autotuner
  int grid = 1;         // persistent CTAs (resident on the device at once)
  const int* d_order = nullptr;
  int* d_queue = nullptr;
};

int batch_launch_bucket(alg_ctx* ctx, const BatchSpec& sp, const BucketLaunch& bl);
// Kernel attributes and the persistent grid of a bucket (host side; call
// outside any stream capture).
int batch_configure_bucket(alg_ctx* ctx, bool mixed, BucketLaunch* bl);
int batch_max_order();

}  // namespace alg
