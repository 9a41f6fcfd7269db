// Instantiates the FP32 split-TF32 sweep shapes with 4 angle tile(s) of 8.
#include "sweep_tc.cuh"

namespace snapb200 {
cudaError_t sweep_tc32_dispatch_nt4(int kt, int op, const SweepParams *p, int grid,
                                     cudaStream_t st, int *blocks, size_t *smem) {
  return tc::dispatch_nt<4>(kt, op, p, grid, st, blocks, smem);
}
}  // namespace snapb200
