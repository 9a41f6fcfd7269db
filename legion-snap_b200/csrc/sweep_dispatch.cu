// Entry points of the sweep kernels: shape dispatch over the per-precision,
// per-angle-tile translation units (the kernel itself is in sweep.cuh).
#include "snap_b200.h"
#include "sweep.cuh"
#include "sweep_tc.cuh"

#include <algorithm>
#include <string>

namespace snapb200 {
namespace {

using DispatchFn = cudaError_t (*)(int, int, int, const SweepParams *, int, cudaStream_t, int *,
                                   size_t *);
const DispatchFn kFp64[9] = {nullptr,
                             sweep_fp64_dispatch_nt1, sweep_fp64_dispatch_nt2,
                             sweep_fp64_dispatch_nt3, sweep_fp64_dispatch_nt4,
                             sweep_fp64_dispatch_nt5, sweep_fp64_dispatch_nt6,
                             sweep_fp64_dispatch_nt7, sweep_fp64_dispatch_nt8};
const DispatchFn kFp32[9] = {nullptr,
                             sweep_fp32_dispatch_nt1, sweep_fp32_dispatch_nt2,
                             sweep_fp32_dispatch_nt3, sweep_fp32_dispatch_nt4,
                             sweep_fp32_dispatch_nt5, sweep_fp32_dispatch_nt6,
                             sweep_fp32_dispatch_nt7, sweep_fp32_dispatch_nt8};

using TcFn = cudaError_t (*)(int, int, const SweepParams *, int, cudaStream_t, int *, size_t *);
const TcFn kTc32[9] = {nullptr,
                       sweep_tc32_dispatch_nt1, sweep_tc32_dispatch_nt2, sweep_tc32_dispatch_nt3,
                       sweep_tc32_dispatch_nt4, sweep_tc32_dispatch_nt5, sweep_tc32_dispatch_nt6,
                       sweep_tc32_dispatch_nt7, sweep_tc32_dispatch_nt8};

bool supported(const SweepShape &sh) {
  return (sh.TY == 8 || sh.TY == 4) && sh.NT >= 1 && sh.NT <= 8 && sh.MK >= 0 && sh.MK <= 4;
}

cudaError_t dispatch(const DispatchFn *table, const SweepShape &sh, int op, const SweepParams *p,
                     int grid, cudaStream_t st, int *blocks, size_t *smem) {
  if (!supported(sh)) return cudaErrorInvalidValue;
  return table[sh.NT](sh.MK, sh.TY, op, p, grid, st, blocks, smem);
}

}  // namespace

bool sweep_fp64_supported(const SweepShape &sh) { return supported(sh); }
bool sweep_fp32_supported(const SweepShape &sh) { return supported(sh); }

cudaError_t launch_sweep_fp64(const SweepShape &sh, const SweepParams &p, int grid,
                              cudaStream_t st) {
  return dispatch(kFp64, sh, 0, &p, grid, st, nullptr, nullptr);
}
cudaError_t launch_sweep_fp64_td(const SweepShape &sh, const SweepParams &p, int grid,
                                 cudaStream_t st) {
  if (!supported(sh) || sh.MK != 0) return cudaErrorInvalidValue;
  return kFp64[sh.NT](-1, sh.TY, 0, &p, grid, st, nullptr, nullptr);
}
cudaError_t sweep_fp64_td_occupancy(const SweepShape &sh, int *blocks_per_sm, size_t *smem) {
  if (!supported(sh) || sh.MK != 0) return cudaErrorInvalidValue;
  return kFp64[sh.NT](-1, sh.TY, 1, nullptr, 0, nullptr, blocks_per_sm, smem);
}
cudaError_t launch_sweep_fp32(const SweepShape &sh, const SweepParams &p, int grid,
                              cudaStream_t st) {
  return dispatch(kFp32, sh, 0, &p, grid, st, nullptr, nullptr);
}

bool sweep_tc32_supported(const SweepShape &sh) {
  return sh.TY == 4 && sh.NT >= 1 && sh.NT <= 8 && sh.KT >= 0 && sh.KT <= 2;
}
cudaError_t launch_sweep_tc32(const SweepShape &sh, const SweepParams &p, int grid,
                              cudaStream_t st) {
  if (!sweep_tc32_supported(sh)) return cudaErrorInvalidValue;
  return kTc32[sh.NT](sh.KT, 0, &p, grid, st, nullptr, nullptr);
}
cudaError_t sweep_tc32_occupancy(const SweepShape &sh, int *blocks_per_sm, size_t *smem) {
  if (!sweep_tc32_supported(sh)) return cudaErrorInvalidValue;
  return kTc32[sh.NT](sh.KT, 1, nullptr, 0, nullptr, blocks_per_sm, smem);
}

cudaError_t sweep_fp64_occupancy(const SweepShape &sh, int *blocks_per_sm, size_t *smem) {
  return dispatch(kFp64, sh, 1, nullptr, 0, nullptr, blocks_per_sm, smem);
}
cudaError_t sweep_fp32_occupancy(const SweepShape &sh, int *blocks_per_sm, size_t *smem) {
  return dispatch(kFp32, sh, 1, nullptr, 0, nullptr, blocks_per_sm, smem);
}

size_t sweep_fp64_smem(const SweepShape &sh) {
  size_t smem = 0;
  dispatch(kFp64, sh, 2, nullptr, 0, nullptr, nullptr, &smem);
  return smem;
}
size_t sweep_fp32_smem(const SweepShape &sh) {
  size_t smem = 0;
  dispatch(kFp32, sh, 2, nullptr, 0, nullptr, nullptr, &smem);
  return smem;
}

}  // namespace snapb200

namespace {

template <typename T>
__global__ void division_selftest_kernel(const T *a, const T *b, long long n, T *out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    out[4 * i] = snapb200::sw::recip(b[i]);
    out[4 * i + 1] = snapb200::sw::recip_rn(b[i]);
    out[4 * i + 2] = snapb200::sw::divide(a[i], b[i]);
    out[4 * i + 3] = snapb200::sw::div_rn(a[i], b[i]);
  }
}

}  // namespace

extern "C" int snap_selftest_division(int precision, const void *a, const void *b, long long n,
                                      void *out, void *stream) {
  if (!a || !b || !out || n < 0 || (precision != SNAP_FP64 && precision != SNAP_FP32))
    return snapb200::set_last_error(SNAP_ERR_BAD_ARG, "snap_selftest_division: bad argument");
  if (n == 0) return SNAP_OK;
  const int grid = (int)std::min<long long>((n + 255) / 256, 4096);
  cudaStream_t st = (cudaStream_t)stream;
  if (precision == SNAP_FP64)
    division_selftest_kernel<double><<<grid, 256, 0, st>>>((const double *)a, (const double *)b,
                                                           n, (double *)out);
  else
    division_selftest_kernel<float><<<grid, 256, 0, st>>>((const float *)a, (const float *)b, n,
                                                          (float *)out);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return snapb200::set_last_error(SNAP_ERR_CUDA, std::string("snap_selftest_division: ") +
                                                       cudaGetErrorString(e));
  return SNAP_OK;
}
