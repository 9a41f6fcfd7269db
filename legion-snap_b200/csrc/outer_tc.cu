// Outer source with the group-to-group scattering contraction on the BF16
// tensor cores (the precision form's fast outer source).
//
// Same result as outer_source_kernel (kernels.cu; reference: CalcOuterSource,
// outer.cc:107-217, gpu_outer.cu:76-441):
//   q2[g][c][k] = qi[g][c] [k = 0] + sum_{g' != g} slgg[g][mat(c)][g'][l(k)] phi[g'][c][k]
// For a fixed moment k (hence band l) and material, this is a GEMM of the
// G x G scattering block with the G x cells flux block; it runs on
// mma.m16n8k16 with the output groups as rows, the input groups as k and 8
// cells as columns.  BF16 keeps 8 mantissa bits, so both operands are split
// x = hi + lo (hi the BF16 rounding of x, lo that of the remainder) and the
// product is accumulated as lo*hi + hi*lo + hi*hi in FP32: relative error of
// order 2^-16.  That is not the FP64 source: the solve driver uses this only
// while the outer iteration is still far from converged and switches to the
// FP64 source for the final outer iterations (a mixed-precision refinement:
// the converged fixed point is the one of the FP64 source).
//
// A CTA takes 32 cells (4 warps x 8) and walks the moment bands: for band l
// it stages the split scattering blocks of every material (MMA fragment
// layout, built once per call by tc_tables_kernel) and the split flux of the
// band's moments (input group fastest) in shared memory, then each warp forms
// its 8 cells x all output groups for each moment of the band.  A cell tile
// holding several materials computes each present material and selects per
// column.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "internal.h"

namespace snapb200 {
namespace {

constexpr int TCELLS = 32;   // cells per CTA (4 warps x 8)


// two BF16 values packed low (first) / high (second)
__device__ __forceinline__ uint32_t pack_bf16(__nv_bfloat16 lo_half, __nv_bfloat16 hi_half) {
  return (uint32_t)__bfloat16_as_ushort(lo_half) | ((uint32_t)__bfloat16_as_ushort(hi_half) << 16);
}
// split x = hi + lo, both BF16 rounded to nearest
__device__ __forceinline__ void split_bf16(double x, __nv_bfloat16 &hi, __nv_bfloat16 &lo) {
  hi = __double2bfloat16(x);
  lo = __double2bfloat16(x - (double)__bfloat162float(hi));
}

// Scattering blocks in the A-fragment layout of mma.m16n8k16 (row-major
// A[row = output group][col = input group]); lane l = 4r + t holds
// reg 0 = A[r][2t, 2t+1], reg 1 = A[r+8][2t, 2t+1], reg 2 = A[r][2t+8, 2t+9],
// reg 3 = A[r+8][2t+8, 2t+9].  Table [l][mat][mt][kt][lane][8]: regs 0-3 hi,
// 4-7 lo.  The diagonal (in-group scattering, handled by the inner source)
// and the padding beyond G are zero.
__global__ void tc_tables_kernel(const double *__restrict__ slgg, int G, int nmat, int nmom,
                                 int GT, uint32_t *__restrict__ tab) {
  const long long n = (long long)nmom * nmat * GT * GT * 32 * 4;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int reg = (int)(i % 4), lane = (int)((i / 4) % 32);
    long long rest = i / 128;
    const int kt = (int)(rest % GT);
    rest /= GT;
    const int mt = (int)(rest % GT);
    rest /= GT;
    const int m = (int)(rest % nmat);
    const int l = (int)(rest / nmat);
    const int r = lane >> 2, t = lane & 3;
    const int row = 16 * mt + r + ((reg & 1) ? 8 : 0);
    const int col = 16 * kt + 2 * t + ((reg & 2) ? 8 : 0);
    __nv_bfloat16 h[2], lo[2];
    for (int e = 0; e < 2; ++e) {
      const int c = col + e;
      const double v = (row < G && c < G && row != c)
                           ? slgg[(((size_t)row * nmat + m) * G + c) * nmom + l]
                           : 0.0;
      split_bf16(v, h[e], lo[e]);
    }
    uint32_t *dst = tab + (i / 4) * 8;
    dst[reg] = pack_bf16(h[0], h[1]);
    dst[4 + reg] = pack_bf16(lo[0], lo[1]);
  }
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], uint4 a, uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a.x), "r"(a.y), "r"(a.z), "r"(a.w), "r"(b0), "r"(b1));
}

// Dynamic shared memory: fragments [nmat][GT][GT][32] x 2 uint4 (hi, lo),
// then the band's split flux, hi and lo, each [2*nmom-1][TCELLS][PG] BF16
// with PG = 16*GT + 8 (the pad spreads the 8 cells of a fragment load over
// all banks).
__global__ void __launch_bounds__(128)
    outer_source_tc_kernel(const double *__restrict__ qi, const uint32_t *__restrict__ tab,
                           const int32_t *__restrict__ mat, const double *__restrict__ flux,
                           double *__restrict__ q2grp, int G, int nmat, int nmom, int M,
                           long long C, int GT) {
  extern __shared__ __align__(16) uint4 smem_u4[];
  const int PG = 16 * GT + 8;
  const int KMAX = 2 * nmom - 1;
  uint4 *sA = smem_u4;                                        // [nmat][GT][GT][32][2]
  __nv_bfloat16 *sPh = (__nv_bfloat16 *)(sA + (size_t)nmat * GT * GT * 64);
  __nv_bfloat16 *sPl = sPh + (size_t)KMAX * TCELLS * PG;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int r = lane >> 2, t = lane & 3;
  const long long ntiles = (C + TCELLS - 1) / TCELLS;

  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long c0 = tile * TCELLS;
    // this lane's output columns: cells 8w + 2t, 8w + 2t + 1 of the tile
    const long long ca = c0 + 8 * w + 2 * t, cb = ca + 1;
    const int mata = ca < C ? mat[ca] - 1 : -1, matb = cb < C ? mat[cb] - 1 : -1;
    // materials present in the warp's 8 cells (lanes 0-7 look at one cell each)
    const long long cm = c0 + 8 * w + (lane & 7);
    const unsigned present = __reduce_or_sync(0xffffffffu, (lane < 8 && cm < C) ? 1u << (mat[cm] - 1) : 0u);
    for (int l = 0; l < nmom; ++l) {
      const int k0 = l * l, nk = 2 * l + 1;
      __syncthreads();
      // stage the scattering fragments of band l and the band's split flux
      const uint4 *src = (const uint4 *)(tab + (size_t)l * nmat * GT * GT * 32 * 8);
      for (int i = tid; i < nmat * GT * GT * 64; i += blockDim.x) sA[i] = src[i];
      // (moment fastest, then cell: neighbouring threads read neighbouring words)
      for (int i = tid; i < nk * TCELLS * 16 * GT; i += blockDim.x) {
        const int kk = i % nk, cc = (i / nk) % TCELLS, g = i / (nk * TCELLS);
        const long long c = c0 + cc;
        const double v = (g < G && c < C) ? flux[((size_t)g * C + c) * M + k0 + kk] : 0.0;
        __nv_bfloat16 h, lo;
        split_bf16(v, h, lo);
        const size_t at = ((size_t)kk * TCELLS + cc) * PG + g;
        sPh[at] = h;
        sPl[at] = lo;
      }
      __syncthreads();
      for (int kk = 0; kk < nk; ++kk) {
        const int k = k0 + kk;
        // B fragments: rows = input groups 16kt + 2t (+1, +8, +9), column = cell 8w + r
        const __nv_bfloat16 *bh = sPh + ((size_t)kk * TCELLS + 8 * w + r) * PG + 2 * t;
        const __nv_bfloat16 *bl = sPl + ((size_t)kk * TCELLS + 8 * w + r) * PG + 2 * t;
        for (int mt = 0; mt < GT; ++mt) {
          float out[4] = {0.0f, 0.0f, 0.0f, 0.0f};
          for (int m = 0; m < nmat; ++m) {
            if (!((present >> m) & 1u)) continue;
            float d[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            for (int kt = 0; kt < GT; ++kt) {
              const uint4 *a = sA + ((((size_t)m * GT + mt) * GT + kt) * 32 + lane) * 2;
              const uint4 ah = a[0], al = a[1];
              const uint32_t bh0 = *(const uint32_t *)(bh + 16 * kt);
              const uint32_t bh1 = *(const uint32_t *)(bh + 16 * kt + 8);
              const uint32_t bl0 = *(const uint32_t *)(bl + 16 * kt);
              const uint32_t bl1 = *(const uint32_t *)(bl + 16 * kt + 8);
              mma_bf16(d, al, bh0, bh1);
              mma_bf16(d, ah, bl0, bl1);
              mma_bf16(d, ah, bh0, bh1);
            }
            if (mata == m) { out[0] = d[0]; out[2] = d[2]; }
            if (matb == m) { out[1] = d[1]; out[3] = d[3]; }
          }
          // rows 16mt + r and 16mt + r + 8 (output groups), columns ca, cb
          const int g_a = 16 * mt + r, g_b = g_a + 8;
          auto put = [&](int g, long long c, float v) {
            if (g >= G || c >= C) return;
            double q = (double)v;
            if (k == 0) q += qi[(size_t)g * C + c];
            q2grp[((size_t)g * C + c) * M + k] = q;
          };
          put(g_a, ca, out[0]);
          put(g_a, cb, out[1]);
          put(g_b, ca, out[2]);
          put(g_b, cb, out[3]);
        }
      }
    }
  }
}

}  // namespace

size_t outer_tc_table_words(int G, int nmat, int nmom) {
  const int GT = (G + 15) / 16;
  return (size_t)nmom * nmat * GT * GT * 32 * 8;
}

size_t outer_tc_smem_bytes(int G, int nmat, int nmom) {
  const int GT = (G + 15) / 16, PG = 16 * GT + 8;
  return sizeof(uint4) * (size_t)nmat * GT * GT * 64 +
         2 * sizeof(__nv_bfloat16) * (size_t)(2 * nmom - 1) * TCELLS * PG;
}

cudaError_t k_outer_source_tc(const double *qi, const double *slgg, const int32_t *mat,
                              const double *flux, double *q2grp, uint32_t *tab, int G, int nmat,
                              int nmom, int M, long long C, cudaStream_t st) {
  const int GT = (G + 15) / 16;
  const size_t smem = outer_tc_smem_bytes(G, nmat, nmom);
  if (smem > 200 * 1024 || nmat > 32) return cudaErrorInvalidValue;
  tc_tables_kernel<<<64, 256, 0, st>>>(slgg, G, nmat, nmom, GT, tab);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(outer_source_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 0, blocks = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, outer_source_tc_kernel, 128, smem);
  const long long tiles = (C + TCELLS - 1) / TCELLS;
  const int grid = (int)std::min<long long>(tiles, (long long)std::max(blocks, 1) * sms);
  outer_source_tc_kernel<<<grid, 128, smem, st>>>(qi, tab, mat, flux, q2grp, G, nmat, nmom, M, C,
                                                  GT);
  return cudaGetLastError();
}

}  // namespace snapb200
