// FP32 sweep (placeholder until the mixed-precision form lands): reports no
// compiled shapes, so FP32 contexts are refused with SNAP_ERR_UNSUPPORTED.
#include "internal.h"

namespace snapb200 {
bool sweep_fp32_supported(const SweepShape &) { return false; }
cudaError_t launch_sweep_fp32(const SweepShape &, const SweepParams &, int, cudaStream_t) {
  return cudaErrorNotSupported;
}
cudaError_t sweep_fp32_occupancy(const SweepShape &, int *, size_t *) {
  return cudaErrorNotSupported;
}
size_t sweep_fp32_smem(const SweepShape &) { return 0; }
}  // namespace snapb200
