// Outer source with the group-to-group scattering contraction on the
// fifth-generation tensor cores (tcgen05.mma, kind::f16: BF16 operands, FP32
// accumulation in tensor memory) -- the precision form's fast outer source.
//
// Same result as the FP64 outer source (kernels.cu; reference:
// CalcOuterSource, outer.cc:107-217, gpu_outer.cu:76-441):
//   q2[g][c][k] = qi[g][c] [k = 0] + sum_{g' != g} slgg[g][mat(c)][g'][l(k)] phi[g'][c][k]
// For one moment k (hence band l) and 128 cells this is a GEMM
//   D[c][g] = sum_{g'} A[c][g'] B[g][g'],   A = phi[.][c][k], B = S_l,mat
// with the cells as the MMA's M = 128 rows (tensor-memory lanes), the output
// groups as N and the input groups as K.  BF16 keeps 8 mantissa bits, so
// both operands are split x = hi + lo (hi the BF16 rounding of x, lo that of
// the remainder) and the product is accumulated as hi*hi + hi*lo + lo*hi:
// relative error of order 2^-16.  That is not the FP64 source: the solve
// driver uses this only while the outer iteration is still far from
// converged and switches to the FP64 source for the final outer iterations
// (a mixed-precision refinement: the converged fixed point is the one of the
// FP64 source).  Cells of different materials: the A operand is staged once
// per material with the rows of other materials zeroed, and the materials'
// products accumulate into the same tensor-memory tile.
//
// Operands live in shared memory in the K-major layout without swizzle:
// 8-row x 16-byte core matrices, the two core matrices of one 16-element K
// step 128 bytes apart (leading byte offset), consecutive 8-row groups 256
// bytes apart (stride byte offset), K steps one after another.  The
// scattering operands of every band and material (built per call by
// tcb_table_kernel in that layout) are copied into shared memory once per
// CTA with one bulk copy (cp.async.bulk, completion on an mbarrier).  Per
// moment the 128 threads convert their cell's flux to the split operands,
// one elected thread issues the MMAs and commits them to an mbarrier, and
// every MC moments the four warps read their 32 lanes of the accumulators
// back (tcgen05.ld) and store the MC consecutive moments of each (group,
// cell) as one 32-byte run.  Every wait is bounded and records a timeout in
// the device error word.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "device_util.cuh"
#include "internal.h"

namespace snapb200 {
namespace {

constexpr int TCR = 128;   // cells per tile = MMA rows; 4 warps, warp w owns lanes 32w..32w+31
constexpr int MCMAX = 4;   // moments per accumulator batch

__host__ __device__ inline int pad16(int x) { return (x + 15) / 16 * 16; }

// Byte offset of element (row r, k) of a K-major BF16 operand tile of R rows.
__host__ __device__ inline uint32_t kmajor_offset(int R, int r, int k) {
  return (uint32_t)((k >> 4) * (R / 8) * 256 + (r >> 3) * 256 + ((k >> 3) & 1) * 128 +
                    (r & 7) * 16 + (k & 7) * 2);
}

// Shared-memory matrix descriptor: start address, leading byte offset 128,
// stride byte offset 256, descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128 >> 4) << 16) |
         ((uint64_t)(256 >> 4) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, N columns, M = 128 rows.
__host__ __device__ inline uint32_t idesc_bf16(int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(TCR >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

// Waits until the phase with parity `parity` of the mbarrier has completed.
// Gives up after timeout_ns of device time or an iteration cap (recording a
// timeout), or when the device error word is set.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int *err,
                                          long long timeout_ns) {
  const long long t0 = global_timer_ns();
  for (unsigned spins = 0;; ++spins) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if ((spins & 63u) == 63u) {
      if (ld_volatile(err) != 0) return false;
      if (global_timer_ns() - t0 > timeout_ns || spins > (1u << 24)) {
        atomicCAS(err, 0, DEV_ERR_TIMEOUT);
        return false;
      }
    }
  }
}

__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// D[tmem] (+)= A * B^T, M = 128, K = 16, one elected thread.
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}

// Arrives on the mbarrier once every MMA this thread issued so far is done.
__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

// 16 consecutive FP32 accumulator columns of this thread's lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void split_bf16(double x, __nv_bfloat16 &hi, __nv_bfloat16 &lo) {
  hi = __double2bfloat16(x);
  lo = __double2bfloat16(x - (double)__bfloat162float(hi));
}

// Scattering operands B[g][g'] = S_l,mat[g][g'] (diagonal and padding zero),
// split into BF16 hi and lo, each an N x KP tile in the K-major layout;
// order [l][mat][part].
__global__ void tcb_table_kernel(const double *__restrict__ slgg, int G, int nmat, int nmom, int N,
                                 int KP, __nv_bfloat16 *__restrict__ tab) {
  const long long per = (long long)N * KP;
  const long long n = (long long)nmom * nmat * per;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(i % KP), row = (int)((i / KP) % N);
    const long long lm = i / per;
    const int m = (int)(lm % nmat), l = (int)(lm / nmat);
    const double v = (row < G && k < G && row != k)
                         ? slgg[(((size_t)row * nmat + m) * G + k) * nmom + l]
                         : 0.0;
    __nv_bfloat16 h, lo;
    split_bf16(v, h, lo);
    __nv_bfloat16 *tile = tab + (size_t)lm * 2 * per;
    const uint32_t off = kmajor_offset(N, row, k) / 2;
    tile[off] = h;
    tile[per + off] = lo;
  }
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// Warp roles: warps 0-3 convert the flux (thread = cell row of the tile),
// warps 4-7 drain the accumulators (warp w owns tensor-memory lanes
// 32(w-4)..32(w-4)+31), one thread of warp 8 issues the MMAs.  A batch is
// (tile of 128 cells, MC consecutive moments); its operands and
// accumulators are double-buffered (buffer = batch parity), with mbarriers
//   full[buf]: the converted operands are in shared memory (128 arrivals),
//   mma[buf]:  the batch's MMAs are done (tcgen05.commit): the operands may
//              be overwritten and the accumulators read,
//   free[buf]: the accumulators have been read (128 arrivals),
// so the conversion of batch b+1 and the drain of batch b-1 overlap the
// MMAs of batch b.
constexpr int TC_THREADS = 9 * 32;

__global__ void __launch_bounds__(TC_THREADS)
    outer_source_tc_kernel(const double *__restrict__ qi, const __nv_bfloat16 *__restrict__ tab,
                           const int32_t *__restrict__ mat, const double *__restrict__ flux,
                           double *__restrict__ q2grp, int G, int N, int KP, int nmat, int nmom,
                           int M, int MC, long long C, int tmem_cols, int *err,
                           long long timeout_ns) {
  extern __shared__ __align__(1024) unsigned char tc_smem[];
  const size_t b_tile = (size_t)N * KP * 2, a_tile = (size_t)TCR * KP * 2;
  const size_t b_bytes = (size_t)nmom * nmat * 2 * b_tile, a_buf = (size_t)MC * 2 * a_tile;
  unsigned char *sB = tc_smem;            // [l][mat][hi, lo] N x KP
  unsigned char *sA = tc_smem + b_bytes;  // [buf][moment of the batch][hi, lo] 128 x KP
  __shared__ __align__(8) uint64_t s_bar[7];   // tab, full[2], mma[2], free[2]
  __shared__ uint32_t s_tmem;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t bar_tab = smem_u32(&s_bar[0]);
  auto bar_full = [&](int b) { return smem_u32(&s_bar[1 + b]); };
  auto bar_mma = [&](int b) { return smem_u32(&s_bar[3 + b]); };
  auto bar_free = [&](int b) { return smem_u32(&s_bar[5 + b]); };
  const int tcols = MC * nmat * N;   // accumulator columns of one buffer

  if (tid == 0) {
    mbar_init(bar_tab, 1);
    for (int b = 0; b < 2; ++b) {
      mbar_init(bar_full(b), TCR);
      mbar_init(bar_mma(b), 1);
      mbar_init(bar_free(b), TCR);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&s_tmem)),
                 "r"(tmem_cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = s_tmem;

  const int nbt = (M + MC - 1) / MC;   // batches per tile
  const long long ntiles = (C + TCR - 1) / TCR;
  const long long my_tiles = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const long long nb = my_tiles * nbt;
  auto batch_tile = [&](long long b) { return blockIdx.x + (b / nbt) * (long long)gridDim.x; };
  const bool runs4 = (M & 3) == 0;   // a batch of 4 moments is one aligned 32-byte run

  if (warp < 4) {
    // ---- conversion: cell row tid of each batch's operands
    for (long long b = 0; b < nb; ++b) {
      const int buf = (int)(b & 1);
      const uint32_t use = (uint32_t)(b >> 1);
      if (use > 0 && !mbar_wait(bar_mma(buf), (use - 1) & 1u, err, timeout_ns)) break;
      const long long c = batch_tile(b) * TCR + tid;
      const bool valid = c < C;
      const int m0 = (int)(b % nbt) * MC, mc = min(MC, M - m0);
      unsigned char *A = sA + (size_t)buf * a_buf;
      for (int k8 = 0; k8 < KP; k8 += 8) {
        double x[8][MCMAX];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const int gi = k8 + e;
          const double *src = flux + ((size_t)gi * C + c) * M + m0;
          if (valid && gi < G && mc == 4 && runs4) {
            const double2 v0 = __ldg((const double2 *)src), v1 = __ldg((const double2 *)src + 1);
            x[e][0] = v0.x;
            x[e][1] = v0.y;
            x[e][2] = v1.x;
            x[e][3] = v1.y;
          } else {
#pragma unroll
            for (int mm = 0; mm < MCMAX; ++mm)
              x[e][mm] = (valid && gi < G && mm < mc) ? __ldg(src + mm) : 0.0;
          }
        }
        const uint32_t off = kmajor_offset(TCR, tid, k8);
#pragma unroll
        for (int mm = 0; mm < MCMAX; ++mm) {
          if (mm >= mc) break;
          __align__(16) __nv_bfloat16 h[8], lo[8];
#pragma unroll
          for (int e = 0; e < 8; ++e) split_bf16(x[e][mm], h[e], lo[e]);
          unsigned char *t = A + (size_t)mm * 2 * a_tile;
          *(uint4 *)(t + off) = *(const uint4 *)h;
          *(uint4 *)(t + a_tile + off) = *(const uint4 *)lo;
        }
      }
      // visible to the tensor cores, then count this row in
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive(bar_full(buf));
    }
  } else if (warp < 8) {
    // ---- drain: lane row 32(warp-4) + lane of each batch's accumulators
    const int row = (warp - 4) * 32 + lane;
    const uint32_t lane_addr = tmem + ((uint32_t)((warp - 4) * 32) << 16);
    for (long long b = 0; b < nb; ++b) {
      const int buf = (int)(b & 1);
      const uint32_t use = (uint32_t)(b >> 1);
      if (!mbar_wait(bar_mma(buf), use & 1u, err, timeout_ns)) break;
      fence_after_sync();
      const long long c = batch_tile(b) * TCR + row;
      const bool valid = c < C;
      const int matr = valid ? mat[c] - 1 : -1;
      const int m0 = (int)(b % nbt) * MC, mc = min(MC, M - m0);
      const uint32_t tb = lane_addr + (uint32_t)(buf * tcols);
      for (int gb = 0; gb < N; gb += 16) {
        float v[MCMAX][16];
#pragma unroll
        for (int mm = 0; mm < MCMAX; ++mm) {
          if (mm >= mc) break;
          for (int mi = 0; mi < nmat; ++mi) {
            float t[16];
            tmem_ld16(tb + (uint32_t)((mm * nmat + mi) * N + gb), t);
            tmem_wait_ld();
            if (mi == matr) {
#pragma unroll
              for (int j = 0; j < 16; ++j) v[mm][j] = t[j];
            }
          }
        }
        if (!valid) continue;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int g = gb + j;
          if (g >= G) break;
          double o[MCMAX];
#pragma unroll
          for (int mm = 0; mm < MCMAX; ++mm) o[mm] = mm < mc ? (double)v[mm][j] : 0.0;
          if (m0 == 0) o[0] += qi[(size_t)g * C + c];
          double *dst = q2grp + ((size_t)g * C + c) * M + m0;
          if (mc == 4 && runs4) {
            *(double2 *)dst = make_double2(o[0], o[1]);
            *(double2 *)(dst + 2) = make_double2(o[2], o[3]);
          } else {
#pragma unroll
            for (int mm = 0; mm < MCMAX; ++mm)
              if (mm < mc) dst[mm] = o[mm];
          }
        }
      }
      fence_before_sync();
      mbar_arrive(bar_free(buf));
    }
  } else if (lane == 0) {
    // ---- MMA issue: moment mm, material mi -> columns buf * tcols + (mm * nmat + mi) * N
    const uint32_t idesc = idesc_bf16(N);
    if (nb > 0) {
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_tab),
                   "r"((uint32_t)b_bytes)
                   : "memory");
      for (size_t off = 0; off < b_bytes; off += 16384) {
        const uint32_t len = (uint32_t)(b_bytes - off < 16384 ? b_bytes - off : 16384);
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                smem_u32(sB + off)),
            "l"((const unsigned char *)tab + off), "r"(len), "r"(bar_tab)
            : "memory");
      }
    }
    bool ok = nb == 0 || mbar_wait(bar_tab, 0, err, timeout_ns);
    for (long long b = 0; ok && b < nb; ++b) {
      const int buf = (int)(b & 1);
      const uint32_t use = (uint32_t)(b >> 1);
      if (!mbar_wait(bar_full(buf), use & 1u, err, timeout_ns)) break;
      if (use > 0 && !mbar_wait(bar_free(buf), (use - 1) & 1u, err, timeout_ns)) break;
      fence_after_sync();
      const int m0 = (int)(b % nbt) * MC, mc = min(MC, M - m0);
      const unsigned char *A = sA + (size_t)buf * a_buf;
      for (int mm = 0; mm < mc; ++mm) {
        const int k = m0 + mm;
        int l = 0;
        while ((l + 1) * (l + 1) <= k) ++l;
        const uint32_t a_hi = smem_u32(A + (size_t)mm * 2 * a_tile), a_lo = a_hi + (uint32_t)a_tile;
        for (int mi = 0; mi < nmat; ++mi) {
          const uint32_t d = tmem + (uint32_t)(buf * tcols + (mm * nmat + mi) * N);
          const uint32_t b_hi = smem_u32(sB + ((size_t)l * nmat + mi) * 2 * b_tile),
                         b_lo = b_hi + (uint32_t)b_tile;
          for (int s = 0; s < KP / 16; ++s) {
            const uint32_t ao = (uint32_t)s * (TCR / 8) * 256, bo = (uint32_t)s * (N / 8) * 256;
            mma_bf16(d, smem_desc(a_hi + ao), smem_desc(b_hi + bo), idesc, s > 0);
            mma_bf16(d, smem_desc(a_hi + ao), smem_desc(b_lo + bo), idesc, 1);
            mma_bf16(d, smem_desc(a_lo + ao), smem_desc(b_hi + bo), idesc, 1);
          }
        }
      }
      mma_commit(bar_mma(buf));
    }
  }
  // every role has finished (or given up); the drain waited for the last MMAs
  fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    fence_after_sync();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tmem_cols)
                 : "memory");
  }
}

// Launch plan: moments per batch MC (the largest of 4, 2, 1 whose
// accumulators, MC * nmat tiles of N columns, fit the 512 tensor-memory
// columns and whose operands fit 200 KB of shared memory), the tensor-memory
// columns to allocate (a power of two >= 32) and the shared-memory bytes.
struct TcPlan {
  int N, KP, MC, cols;
  size_t smem;
};

bool tc_plan(int G, int nmat, int nmom, TcPlan *pl) {
  pl->N = pad16(G);
  pl->KP = pad16(G);
  const size_t b_bytes = (size_t)nmom * nmat * 2 * pl->N * pl->KP * 2;
  for (int mc = MCMAX; mc >= 1; mc /= 2) {
    const size_t smem = b_bytes + 2 * (size_t)mc * 2 * TCR * pl->KP * 2;   // two operand buffers
    if (2LL * mc * nmat * pl->N <= 512 && smem <= 220 * 1024) {            // two accumulator buffers
      pl->MC = mc;
      pl->smem = smem;
      pl->cols = 32;
      while (pl->cols < 2 * mc * nmat * pl->N) pl->cols <<= 1;
      return true;
    }
  }
  return false;
}

}  // namespace

size_t outer_tc_table_words(int G, int nmat, int nmom) {
  // BF16 words, counted in 32-bit units
  return (size_t)nmom * nmat * 2 * pad16(G) * pad16(G) / 2;
}

bool outer_tc_supported(int G, int nmat, int nmom) {
  TcPlan pl;
  return tc_plan(G, nmat, nmom, &pl);
}

bool outer_tc_preferred(int G, int nmat, int nmom) {
  TcPlan pl;
  return tc_plan(G, nmat, nmom, &pl) && pl.MC == MCMAX;
}

cudaError_t k_outer_source_tc(const double *qi, const double *slgg, const int32_t *mat,
                              const double *flux, double *q2grp, uint32_t *tab, int G, int nmat,
                              int nmom, int M, long long C, int *err, long long timeout_ns,
                              cudaStream_t st) {
  TcPlan pl;
  if (!tc_plan(G, nmat, nmom, &pl)) return cudaErrorInvalidValue;
  tcb_table_kernel<<<64, 256, 0, st>>>(slgg, G, nmat, nmom, pl.N, pl.KP, (__nv_bfloat16 *)tab);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(outer_source_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)pl.smem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(outer_source_tc_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                           (int)cudaSharedmemCarveoutMaxShared);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 0, smem_sm = 0;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev)) !=
      cudaSuccess)
    return e;
  cudaFuncAttributes fa;
  if ((e = cudaFuncGetAttributes(&fa, outer_source_tc_kernel)) != cudaSuccess) return e;
  // resident CTAs: by shared memory (with the static part and the per-CTA
  // reserve), by the 512 tensor-memory columns, by registers
  const int by_smem = (int)((size_t)smem_sm / (pl.smem + 2048));
  const int by_regs = 65536 / (((fa.numRegs + 7) / 8 * 8) * TC_THREADS);
  const int blocks = std::max(1, std::min(std::min(by_smem, 512 / pl.cols), by_regs));
  const long long tiles = (C + TCR - 1) / TCR;
  const int grid = (int)std::min<long long>(tiles, (long long)blocks * sms);
  outer_source_tc_kernel<<<grid, TC_THREADS, pl.smem, st>>>(qi, (const __nv_bfloat16 *)tab, mat, flux,
                                                     q2grp, G, pl.N, pl.KP, nmat, nmom, M, pl.MC,
                                                     C, pl.cols, err, timeout_ns);
  return cudaGetLastError();
}

}  // namespace snapb200
