// Instantiates the fp32 adjoint sweep shapes for angle-tile counts 1 2 3 4.
#include "adjoint.cuh"

namespace snapb200 {
cudaError_t adjoint_fp32_dispatch_nt1(int mk, int op, const SweepParams *p, int grid, cudaStream_t st,
                                    int *blocks, size_t *smem) {
  return adj::dispatch_nt<float, 1>(mk, op, p, grid, st, blocks, smem);
}
cudaError_t adjoint_fp32_dispatch_nt2(int mk, int op, const SweepParams *p, int grid, cudaStream_t st,
                                    int *blocks, size_t *smem) {
  return adj::dispatch_nt<float, 2>(mk, op, p, grid, st, blocks, smem);
}
cudaError_t adjoint_fp32_dispatch_nt3(int mk, int op, const SweepParams *p, int grid, cudaStream_t st,
                                    int *blocks, size_t *smem) {
  return adj::dispatch_nt<float, 3>(mk, op, p, grid, st, blocks, smem);
}
cudaError_t adjoint_fp32_dispatch_nt4(int mk, int op, const SweepParams *p, int grid, cudaStream_t st,
                                    int *blocks, size_t *smem) {
  return adj::dispatch_nt<float, 4>(mk, op, p, grid, st, blocks, smem);
}
}  // namespace snapb200
