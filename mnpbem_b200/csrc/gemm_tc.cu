// tcgen05 tensor-core complex64 GEMM (placeholder until the kernel lands).
#include "dense.cuh"

namespace bem200 {
size_t gemm_tc_workspace(int, int, int, GemmEngine) { return 0; }
int gemm_tc_c64(const LaContext&, int, int, int, float2, const float2*, long long, const float2*, long long, float2,
                float2*, long long) {
  set_error("gemm_tc_c64: tensor-core engine not built");
  return BEM200_ERR_UNSUPPORTED;
}
}  // namespace bem200
