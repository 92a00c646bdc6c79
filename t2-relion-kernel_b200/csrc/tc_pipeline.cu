// tc_pipeline.cu -- tensor-core coarse pass (placeholder until the tcgen05
// kernels land).
#include <cuda_runtime.h>

#include "common.cuh"

namespace b200d2 {
size_t tc_workspace_bytes(const b200d2_view&, const b200d2_batch&, int) { return 0; }
int tc_run(const b200d2_view&, const b200d2_batch&, int, void*, size_t, cudaStream_t) {
  return B200D2_ERR_UNSUPPORTED;
}
}  // namespace b200d2
namespace b200d2 {
const char* tc_stage_name(int, int) { return nullptr; }
int tc_run_stage(const b200d2_view&, const b200d2_batch&, int, int, void*, size_t, cudaStream_t) {
  return B200D2_ERR_UNSUPPORTED;
}
}  // namespace b200d2
