// Trailing update on the tensor cores (tcgen05): placeholder until the
// kernel lands; callers get ALG_NOT_IMPLEMENTED, never a silent substitute.
#include "dense.cuh"

namespace alg {
int gemm_tc_sub_dev(alg_ctx*, int, int, int, int, const float*, int, const float*, int, float*, int) {
  return ALG_NOT_IMPLEMENTED;
}
}  // namespace alg
