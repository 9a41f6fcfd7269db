// Shape dispatch of the adjoint sweep kernels (adjoint.cuh).
#include "internal.h"

namespace snapb200 {

#define SNAP_ADJ_DECL(P, N)                                                                    \
  cudaError_t adjoint_##P##_dispatch_nt##N(int, int, const SweepParams *, int, cudaStream_t, int *, \
                                           size_t *);
SNAP_ADJ_DECL(fp64, 1) SNAP_ADJ_DECL(fp64, 2) SNAP_ADJ_DECL(fp64, 3) SNAP_ADJ_DECL(fp64, 4)
SNAP_ADJ_DECL(fp64, 5) SNAP_ADJ_DECL(fp64, 6) SNAP_ADJ_DECL(fp64, 7) SNAP_ADJ_DECL(fp64, 8)
SNAP_ADJ_DECL(fp32, 1) SNAP_ADJ_DECL(fp32, 2) SNAP_ADJ_DECL(fp32, 3) SNAP_ADJ_DECL(fp32, 4)
SNAP_ADJ_DECL(fp32, 5) SNAP_ADJ_DECL(fp32, 6) SNAP_ADJ_DECL(fp32, 7) SNAP_ADJ_DECL(fp32, 8)
#undef SNAP_ADJ_DECL

namespace {
using Fn = cudaError_t (*)(int, int, const SweepParams *, int, cudaStream_t, int *, size_t *);
const Fn kFp64[9] = {nullptr, adjoint_fp64_dispatch_nt1, adjoint_fp64_dispatch_nt2,
                     adjoint_fp64_dispatch_nt3, adjoint_fp64_dispatch_nt4,
                     adjoint_fp64_dispatch_nt5, adjoint_fp64_dispatch_nt6,
                     adjoint_fp64_dispatch_nt7, adjoint_fp64_dispatch_nt8};
const Fn kFp32[9] = {nullptr, adjoint_fp32_dispatch_nt1, adjoint_fp32_dispatch_nt2,
                     adjoint_fp32_dispatch_nt3, adjoint_fp32_dispatch_nt4,
                     adjoint_fp32_dispatch_nt5, adjoint_fp32_dispatch_nt6,
                     adjoint_fp32_dispatch_nt7, adjoint_fp32_dispatch_nt8};
}  // namespace

bool adjoint_supported(const SweepShape &sh) {
  return sh.TY == 4 && sh.NT >= 1 && sh.NT <= 8 && sh.MK >= 0 && sh.MK <= 4;
}

cudaError_t adjoint_dispatch(int fp32, const SweepShape &sh, int op, const SweepParams *p, int grid,
                             cudaStream_t st, int *blocks, size_t *smem) {
  if (!adjoint_supported(sh)) return cudaErrorInvalidValue;
  return (fp32 ? kFp32 : kFp64)[sh.NT](sh.MK, op, p, grid, st, blocks, smem);
}

}  // namespace snapb200
