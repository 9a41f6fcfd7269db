// Outer source with the group-to-group scattering contraction on the
// fifth-generation tensor cores (tcgen05.mma, kind::f16: BF16 operands, FP32
// accumulation in tensor memory) -- the precision form's fast outer source.
//
// Same result as the FP64 outer source (kernels.cu; reference:
// CalcOuterSource, outer.cc:107-217, gpu_outer.cu:76-441):
//   q2[g][c][k] = qi[g][c] [k = 0] + sum_{g' != g} slgg[g][mat(c)][g'][l(k)] phi[g'][c][k]
// For 128 (cell, moment) rows this is a GEMM per band l and material
//   D[(c,k)][g] = sum_{g'} A[(c,k)][g'] B[g][g'],   A = phi[g'][c][k], B = S_l,mat
// with the rows as the MMA's M = 128 (tensor-memory lanes), the output
// groups as N and the input groups as K; each row keeps the result of its
// own band and material.  BF16 keeps 8 mantissa bits, so both operands are
// split x = hi + lo (hi the BF16 rounding of x, lo that of the remainder)
// and the product is accumulated as hi*hi + hi*lo + lo*hi: relative error
// of order 2^-16.  That is not the FP64 source: the solve driver uses this
// only while the outer iteration is still far from converged and switches to
// the FP64 source for the final outer iterations (a mixed-precision
// refinement: the converged fixed point is the one of the FP64 source).
//
// Operands live in shared memory in the K-major layout without swizzle:
// 8-row x 16-byte core matrices, the two core matrices of one 16-element K
// step 128 bytes apart (leading byte offset), consecutive 8-row groups 256
// bytes apart (stride byte offset), K steps one after another.  The
// scattering operands of every band and material (built per call by
// tcb_table_kernel in that layout) are copied into shared memory once per
// CTA with bulk copies (cp.async.bulk, completion on an mbarrier).  The
// MMA rows are (cell, moment) pairs of whole cells, so the flux is read and
// the source written in whole per-cell lines of moments; conversion, MMA
// issue and the drain of the accumulators (tcgen05.ld) run in separate warps
// on double-buffered operands (see the kernel).  Every wait is bounded and
// records a timeout in the device error word.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "device_util.cuh"
#include "internal.h"

namespace snapb200 {
namespace {

constexpr int TCR = 128;   // cells per tile = MMA rows; 4 warps, warp w owns lanes 32w..32w+31

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

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
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

// A batch is CPB = floor(128 / cmom) cells with all their moments: MMA row
// r = (cell r / cmom, moment r % cmom).  For one input group the batch's flux
// is one contiguous run of CPB * cmom doubles, so a loader thread streams it
// into a shared-memory stage with one bulk copy per input group (S stages in
// flight); the converting threads read it from there.  Rows of different
// bands and materials need different B operands: each row is staged once per
// material with the rows of other materials zeroed, the batch's MMAs run
// once per (band, material) and accumulate the materials into one tile per
// band (nmom tiles of N columns), and each row keeps the tile of its own
// band, so the source is written in whole per-cell lines of moments too.
// Warp roles: warps 0-3 convert (thread = row), warps 4-7 drain the
// accumulators (warp w owns tensor-memory lanes 32(w-4)..32(w-4)+31), lane 0
// of warp 8 issues the MMAs, lane 0 of warp 9 loads.  Operands are
// double-buffered when two sets fit the shared memory (NA = 2; buffer =
// batch % NA), accumulators when two sets fit the 512 tensor-memory columns
// (TB = 2), with mbarriers
//   raw[st] / rawfree[st]: a stage holds a batch's flux / has been converted,
//   full[buf]:  the converted operands are in shared memory (128 arrivals),
//   mma[buf]:   the batch's MMAs are done (tcgen05.commit): the operands may
//               be overwritten and the accumulators read,
//   free[tbuf]: the accumulators have been read (128 arrivals),
// so loads run S batches ahead and the conversion of batch b+1 and the
// drain of batch b-1 overlap the MMAs of batch b.  S = 0 (no room for a
// stage, or runs not 16-byte aligned): the converting threads load the flux
// themselves.
constexpr int TC_THREADS = 10 * 32;
constexpr int TC_MAX_STAGES = 4;

__global__ void __launch_bounds__(TC_THREADS, 1)
    outer_source_tc_kernel(const double *__restrict__ qi, const __nv_bfloat16 *__restrict__ tab,
                           const int32_t *__restrict__ mat, const double *__restrict__ flux,
                           double *__restrict__ q2grp, int G, int N, int KP, int nmat, int nmom,
                           int M, int NA, int TB, int S, long long C, int tmem_cols, int *err,
                           long long timeout_ns) {
  extern __shared__ __align__(1024) unsigned char tc_smem[];
  const int CPB = TCR / M;   // cells per batch
  const size_t b_tile = (size_t)N * KP * 2, a_tile = (size_t)TCR * KP * 2;
  const size_t b_bytes = (size_t)nmom * nmat * 2 * b_tile;
  const size_t run = (size_t)CPB * M * sizeof(double), stage = run * G;
  unsigned char *sB = tc_smem;                       // [l][mat][hi, lo] N x KP
  unsigned char *sA = tc_smem + b_bytes;             // [buf][mat][hi, lo] 128 x KP
  const size_t a_buf = (size_t)nmat * 2 * a_tile;
  double *sQ = (double *)(sA + NA * a_buf);           // [2][cell][g]: qi of a batch (drain)
  const double *sR = sQ + (size_t)2 * CPB * G;        // [stage][g'][CPB * M]
  __shared__ __align__(8) uint64_t s_bar[7 + 2 * TC_MAX_STAGES];
  __shared__ uint32_t s_tmem;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t bar_tab = smem_u32(&s_bar[0]);
  auto bar_full = [&](int b) { return smem_u32(&s_bar[1 + b]); };
  auto bar_mma = [&](int b) { return smem_u32(&s_bar[3 + b]); };
  auto bar_free = [&](int b) { return smem_u32(&s_bar[5 + b]); };
  auto bar_raw = [&](int st) { return smem_u32(&s_bar[7 + st]); };
  auto bar_rawfree = [&](int st) { return smem_u32(&s_bar[7 + TC_MAX_STAGES + st]); };
  const int tcols = nmom * N;   // accumulator columns of one batch: a tile per band

  if (tid == 0) {
    mbar_init(bar_tab, 1);
    for (int b = 0; b < 2; ++b) {
      mbar_init(bar_full(b), TCR);
      mbar_init(bar_mma(b), 1);
      mbar_init(bar_free(b), TCR);
    }
    for (int st = 0; st < S; ++st) {
      mbar_init(bar_raw(st), 1);
      mbar_init(bar_rawfree(st), TCR);
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

  const long long nbatches = (C + CPB - 1) / CPB;
  const long long nb = blockIdx.x < nbatches ? (nbatches - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  auto batch_cell0 = [&](long long b) { return (blockIdx.x + b * (long long)gridDim.x) * CPB; };
  // a batch is staged when it has all its cells (the last may not)
  auto staged = [&](long long b) { return S > 0 && batch_cell0(b) + CPB <= C; };

  if (warp < 8) {
    // rows: thread tid (conversion) or lane row 32(warp-4) + lane (drain)
    const int row = warp < 4 ? tid : (warp - 4) * 32 + lane;
    const int rc = row / M, rm = row - rc * M;   // cell of the batch, moment
    int rl = 0;
    while ((rl + 1) * (rl + 1) <= rm) ++rl;      // band of the moment
    if (warp < 4) {
      // ---- conversion: row of each batch's operands (material of the
      // next batch's cell loaded a batch ahead)
      int mat_next = (nb > 0 && rc < CPB && batch_cell0(0) + rc < C) ? mat[batch_cell0(0) + rc] - 1 : -1;
      for (long long b = 0; b < nb; ++b) {
        const int buf = (int)(b % NA);
        const uint32_t use = (uint32_t)(b / NA);
        const int matr = mat_next;
        {
          const long long cn = batch_cell0(b + 1) + rc;
          mat_next = (b + 1 < nb && rc < CPB && cn < C) ? mat[cn] - 1 : -1;
        }
        if (use > 0 && !mbar_wait(bar_mma(buf), (use - 1) & 1u, err, timeout_ns)) break;
        const long long c = batch_cell0(b) + rc;
        const bool valid = rc < CPB && c < C;
        const bool from_stage = staged(b);
        const int st = S > 0 ? (int)(b % S) : 0;
        if (from_stage && !mbar_wait(bar_raw(st), (uint32_t)(b / S) & 1u, err, timeout_ns)) break;
        const double *src = from_stage ? sR + (size_t)st * (stage / sizeof(double)) + row
                                       : flux + ((size_t)(valid ? c : 0)) * M + rm;
        const size_t gstride = from_stage ? (size_t)CPB * M : (size_t)C * M;
        unsigned char *A = sA + (size_t)buf * a_buf;
        for (int k32 = 0; k32 < KP; k32 += 32) {
          // 32 input groups per thread loaded before any is converted: where
          // the flux is not staged (64 groups leave no shared memory for it)
          // the row's loads are latency-bound (64 groups: 3.17 -> 2.50 ms
          // against 8 in flight)
          double x[32];
#pragma unroll
          for (int e = 0; e < 32; ++e) {
            const int gi = k32 + e;
            x[e] = (valid && gi < G) ? (from_stage ? src[gi * gstride] : __ldg(src + gi * gstride))
                                     : 0.0;
          }
#pragma unroll
          for (int hh = 0; hh < 4; ++hh) {
            const int k8 = k32 + 8 * hh;
            if (k8 >= KP) break;
            __align__(16) __nv_bfloat16 h[8], lo[8];
#pragma unroll
            for (int e = 0; e < 8; ++e) split_bf16(x[8 * hh + e], h[e], lo[e]);
            const uint32_t off = kmajor_offset(TCR, row, k8);
            const uint4 zv = make_uint4(0, 0, 0, 0);
            for (int mi = 0; mi < nmat; ++mi) {
              unsigned char *t = A + (size_t)mi * 2 * a_tile;
              *(uint4 *)(t + off) = mi == matr ? *(const uint4 *)h : zv;
              *(uint4 *)(t + a_tile + off) = mi == matr ? *(const uint4 *)lo : zv;
            }
          }
        }
        if (S > 0) mbar_arrive(bar_rawfree(st));   // the stage may be refilled
        // visible to the tensor cores, then count this row in
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_arrive(bar_full(buf));
      }
    } else {
      // ---- drain: this lane's row keeps the tile of its band.  The
      // moment-0 row of each cell copies the cell's fixed source of the next
      // batch into shared memory (cp.async) while this batch is drained.
      const uint32_t lane_addr = tmem + ((uint32_t)((warp - 4) * 32) << 16);
      const bool owns_q = rm == 0 && rc < CPB;
      auto fetch_q = [&](long long b) {
        if (owns_q && b < nb) {
          const long long cq = batch_cell0(b) + rc;
          double *q = sQ + ((size_t)(b & 1) * CPB + rc) * G;
          for (int g = 0; g < G; ++g) {
            if (cq < C) {
              const unsigned sq = (unsigned)__cvta_generic_to_shared(q + g);
              asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(sq),
                           "l"(qi + (size_t)g * C + cq)
                           : "memory");
            } else {
              q[g] = 0.0;
            }
          }
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
      };
      fetch_q(0);
      for (long long b = 0; b < nb; ++b) {
        const int buf = (int)(b % NA), tbuf = (int)(b % TB);
        if (!mbar_wait(bar_mma(buf), (uint32_t)(b / NA) & 1u, err, timeout_ns)) break;
        fence_after_sync();
        const long long c = batch_cell0(b) + rc;
        const bool valid = rc < CPB && c < C;
        const uint32_t tb = lane_addr + (uint32_t)(tbuf * tcols);
        fetch_q(b + 1);
        asm volatile("cp.async.wait_group 1;" ::: "memory");   // this batch's copies are in
        for (int gb = 0; gb < N; gb += 16) {
          // the fixed source of the block's groups (moment-0 rows)
          const double *q = sQ + ((size_t)(b & 1) * CPB + (rc < CPB ? rc : 0)) * G;
          double qv[16];
#pragma unroll
          for (int j = 0; j < 16; ++j) qv[j] = (valid && rm == 0 && gb + j < G) ? q[gb + j] : 0.0;
          // every band's tile (at most 4), one wait, keep the row's band
          float u[4][16], v[16];
#pragma unroll
          for (int t = 0; t < 4; ++t)
            if (t < nmom) tmem_ld16(tb + (uint32_t)(t * N + gb), u[t]);
          tmem_wait_ld();
#pragma unroll
          for (int j = 0; j < 16; ++j)
            v[j] = rl == 0 ? u[0][j] : rl == 1 ? u[1][j] : rl == 2 ? u[2][j] : u[3][j];
          if (!valid) continue;
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const int g = gb + j;
            if (g >= G) break;
            q2grp[((size_t)g * C + c) * M + rm] = (double)v[j] + qv[j];
          }
        }
        fence_before_sync();
        mbar_arrive(bar_free(tbuf));
      }
      asm volatile("cp.async.wait_all;" ::: "memory");   // no copy outlives the CTA
    }
  } else if (warp == 8 && lane == 0) {
    // ---- MMA issue: band l (every material) -> columns tbuf * tcols + l * N
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
      const int buf = (int)(b % NA), tbuf = (int)(b % TB);
      if (!mbar_wait(bar_full(buf), (uint32_t)(b / NA) & 1u, err, timeout_ns)) break;
      const long long tuse = b / TB;   // earlier batches on these accumulators
      if (tuse > 0 && !mbar_wait(bar_free(tbuf), (uint32_t)(tuse - 1) & 1u, err, timeout_ns)) break;
      fence_after_sync();
      for (int l = 0; l < nmom; ++l) {
        const uint32_t d = tmem + (uint32_t)(tbuf * tcols + l * N);
        for (int mi = 0; mi < nmat; ++mi) {
          const uint32_t a_hi = smem_u32(sA + (size_t)buf * a_buf + (size_t)mi * 2 * a_tile),
                         a_lo = a_hi + (uint32_t)a_tile;
          const uint32_t b_hi = smem_u32(sB + ((size_t)l * nmat + mi) * 2 * b_tile),
                         b_lo = b_hi + (uint32_t)b_tile;
          for (int s = 0; s < KP / 16; ++s) {
            const uint32_t ao = (uint32_t)s * (TCR / 8) * 256, bo = (uint32_t)s * (N / 8) * 256;
            mma_bf16(d, smem_desc(a_hi + ao), smem_desc(b_hi + bo), idesc, mi > 0 || s > 0);
            mma_bf16(d, smem_desc(a_hi + ao), smem_desc(b_lo + bo), idesc, 1);
            mma_bf16(d, smem_desc(a_lo + ao), smem_desc(b_hi + bo), idesc, 1);
          }
        }
      }
      mma_commit(bar_mma(buf));
    }
  } else if (warp == 9 && lane == 0 && S > 0) {
    // ---- loads: batch b's flux into stage b % S, one bulk copy per input group
    for (long long b = 0; b < nb; ++b) {
      const int st = (int)(b % S);
      const long long use = b / S;
      if (use > 0 && !mbar_wait(bar_rawfree(st), (uint32_t)(use - 1) & 1u, err, timeout_ns)) break;
      if (!staged(b)) {
        mbar_arrive(bar_raw(st));   // the converting threads load this batch themselves
        continue;
      }
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_raw(st)),
                   "r"((uint32_t)stage)
                   : "memory");
      const unsigned char *src = (const unsigned char *)(flux + (size_t)batch_cell0(b) * M);
      const uint32_t dst = smem_u32(sR) + (uint32_t)(st * stage);
      for (int g = 0; g < G; ++g)
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                dst + (uint32_t)(g * run)),
            "l"(src + (size_t)g * C * M * sizeof(double)), "r"((uint32_t)run), "r"(bar_raw(st))
            : "memory");
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

// Launch plan: accumulator sets (TB = 2 when two sets of nmom tiles of N
// columns fit the 512 tensor-memory columns, else 1), the columns to
// allocate (a power of two >= 32), the flux stages (as many as fit, at most
// TC_MAX_STAGES; none when the per-group runs are not 16-byte aligned) and
// the shared-memory bytes (scattering operands, NA operand buffers, stages).
struct TcPlan {
  int N, KP, NA, TB, S, cols;
  size_t smem;
};

bool tc_plan(int G, int nmat, int nmom, long long C, TcPlan *pl) {
  const int M = nmom * nmom;
  pl->N = pad16(G);
  pl->KP = pad16(G);
  const long long tcols = (long long)nmom * pl->N;
  if (tcols > 512 || M > TCR || nmom > 4) return false;
  pl->TB = 2 * tcols <= 512 ? 2 : 1;
  pl->cols = 32;
  while (pl->cols < pl->TB * tcols) pl->cols <<= 1;
  const size_t b_bytes = (size_t)nmom * nmat * 2 * pl->N * pl->KP * 2,
               a_buf = (size_t)nmat * 2 * TCR * pl->KP * 2;
  const size_t q_bytes = 2 * (size_t)(TCR / M) * G * sizeof(double);   // two batches' qi
  pl->NA = b_bytes + 2 * a_buf + q_bytes <= 200 * 1024 ? 2 : 1;   // operand buffers
  const size_t base = b_bytes + pl->NA * a_buf + q_bytes;
  if (base > 200 * 1024) return false;
  const size_t run = (size_t)(TCR / M) * M * sizeof(double), stage = run * G;
  const bool aligned = run % 16 == 0 && (C * M * sizeof(double)) % 16 == 0;
  pl->S = 0;
  while (aligned && pl->S < TC_MAX_STAGES && base + (pl->S + 1) * stage <= 200 * 1024) ++pl->S;
  if (pl->S == 1) pl->S = 0;   // one stage would not run ahead
  pl->smem = base + pl->S * stage;
  return true;
}

}  // namespace

size_t outer_tc_table_words(int G, int nmat, int nmom) {
  // BF16 words, counted in 32-bit units
  return (size_t)nmom * nmat * 2 * pad16(G) * pad16(G) / 2;
}

bool outer_tc_supported(int G, int nmat, int nmom) {
  TcPlan pl;
  return tc_plan(G, nmat, nmom, 2, &pl);
}

bool outer_tc_preferred(int G, int nmat, int nmom) { return outer_tc_supported(G, nmat, nmom); }

cudaError_t k_outer_source_tc(const double *qi, const double *slgg, const int32_t *mat,
                              const double *flux, double *q2grp, uint32_t *tab, int G, int nmat,
                              int nmom, int M, long long C, int *err, long long timeout_ns,
                              cudaStream_t st) {
  TcPlan pl;
  if (!tc_plan(G, nmat, nmom, C, &pl)) return cudaErrorInvalidValue;
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
  const long long batches = (C + TCR / M - 1) / (TCR / M);
  const int grid = (int)std::min<long long>(batches, (long long)blocks * sms);
  outer_source_tc_kernel<<<grid, TC_THREADS, pl.smem, st>>>(qi, (const __nv_bfloat16 *)tab, mat, flux,
                                                     q2grp, G, pl.N, pl.KP, nmat, nmom, M, pl.NA, pl.TB,
                                                     pl.S, C, pl.cols, err, timeout_ns);
  return cudaGetLastError();
}

}  // namespace snapb200
