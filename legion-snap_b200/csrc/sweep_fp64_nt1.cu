// Instantiates the FP64 sweep shapes with 1 angle tile(s) of 8 (one file per
// angle-tile count so the shapes compile in parallel).
#include "sweep_fp64.cuh"

namespace snapb200 {
cudaError_t sweep_fp64_dispatch_nt1(int mk, int ty, int op, const SweepParams *p, int grid,
                                    cudaStream_t st, int *blocks, size_t *smem) {
  return fp64::dispatch_nt<1>(mk, ty, op, p, grid, st, blocks, smem);
}
}  // namespace snapb200
