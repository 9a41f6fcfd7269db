// Instantiates the fp64 adjoint sweep shapes for angle-tile counts 5 6 7 8.
#include "adjoint.cuh"

namespace snapb200 {
cudaError_t adjoint_fp64_dispatch_nt5(int mk, int op, const SweepParams *p, int grid, cudaStream_t st,
                                    int *blocks, size_t *smem) {
  return adj::dispatch_nt<double, 5>(mk, op, p, grid, st, blocks, smem);
}
cudaError_t adjoint_fp64_dispatch_nt6(int mk, int op, const SweepParams *p, int grid, cudaStream_t st,
                                    int *blocks, size_t *smem) {
  return adj::dispatch_nt<double, 6>(mk, op, p, grid, st, blocks, smem);
}
cudaError_t adjoint_fp64_dispatch_nt7(int mk, int op, const SweepParams *p, int grid, cudaStream_t st,
                                    int *blocks, size_t *smem) {
  return adj::dispatch_nt<double, 7>(mk, op, p, grid, st, blocks, smem);
}
cudaError_t adjoint_fp64_dispatch_nt8(int mk, int op, const SweepParams *p, int grid, cudaStream_t st,
                                    int *blocks, size_t *smem) {
  return adj::dispatch_nt<double, 8>(mk, op, p, grid, st, blocks, smem);
}
}  // namespace snapb200
