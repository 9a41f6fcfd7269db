// Instantiates the fp64 sweep shapes with 7 angle tile(s) of 8 (one file per
// precision and angle-tile count, so the shapes compile in parallel).
#include "sweep.cuh"

namespace snapb200 {
cudaError_t sweep_fp64_dispatch_nt7(int mk, int ty, int op, const SweepParams *p, int grid,
                                    cudaStream_t st, int *blocks, size_t *smem) {
  return sw::dispatch_nt<double, 7>(mk, ty, op, p, grid, st, blocks, smem);
}
}  // namespace snapb200
