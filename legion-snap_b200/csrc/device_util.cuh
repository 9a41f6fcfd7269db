// Device helpers: FP64 tensor-core MMA, device-scope flags, bounded waits.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace snapb200 {

// D(8x8) += A(8x4, row) * B(4x8, col) in FP64 on the tensor cores.
// Lane l holds A[l/4][l%4], B[l%4][l/4] and D[l/4][2(l%4)+{0,1}].
// Not volatile: the MMA has no side effects, so the compiler may interleave
// independent accumulator chains instead of issuing them in source order.
__device__ __forceinline__ void dmma_8x8x4(double &c0, double &c1, double a, double b) {
  asm(
      "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(c0), "+d"(c1)
      : "d"(a), "d"(b));
}

__device__ __forceinline__ long long global_timer_ns() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ int ld_acquire_gpu(const int *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_release_gpu(int *p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ int ld_volatile(const int *p) {
  return *(const volatile int *)p;
}

// Waits until *flag >= need.  Gives up (returning false) when the device
// error word is set by someone else, or after timeout_ns of device time /
// a hard iteration cap, in which case it records a timeout in the error word.
// Every call ends.
__device__ __forceinline__ bool bounded_wait_geq(const int *flag, int need, int *err,
                                                 long long timeout_ns, int timeout_code) {
  if (ld_acquire_gpu(flag) >= need) return true;
  const long long t0 = global_timer_ns();
  for (unsigned spins = 0;; ++spins) {
    if (ld_acquire_gpu(flag) >= need) return true;
    if (ld_volatile(err) != 0) return false;
    if (spins > 32) __nanosleep(spins < 1024 ? 64 : 256);
    if (global_timer_ns() - t0 > timeout_ns || spins > (1u << 26)) {
      atomicCAS(err, 0, timeout_code);
      return false;
    }
  }
}

// Waits until *flag >= need and returns the last value it read with acquire
// semantics (>= need on success, so a caller can keep it and skip later waits
// for smaller needs).  Returns a smaller value when the device error word is
// set by someone else, or after timeout_ns of device time / a hard iteration
// cap, in which case it records a timeout in the error word.  Every call ends.
__device__ __forceinline__ int wait_value_geq(const int *flag, int need, int *err,
                                              long long timeout_ns, int timeout_code) {
  int v = ld_acquire_gpu(flag);
  if (v >= need) return v;
  const long long t0 = global_timer_ns();
  for (unsigned spins = 0;; ++spins) {
    v = ld_acquire_gpu(flag);
    if (v >= need) return v;
    if (ld_volatile(err) != 0) return v;
    if (spins > 32) __nanosleep(spins < 1024 ? 64 : 256);
    if (global_timer_ns() - t0 > timeout_ns || spins > (1u << 26)) {
      atomicCAS(err, 0, timeout_code);
      return v;
    }
  }
}

}  // namespace snapb200
