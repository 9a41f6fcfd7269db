// General FP64 sweep: one CTA per (octant, group), the CTA's threads over the
// angles, cells walked one at a time in the upwind order of the reference's
// CPU body (z, then y, then x fastest; sweep.cc:336-338).
//
// It covers what the tiled kernel (sweep.cuh) does not: any mesh extent (the
// tiled kernel needs nx % 8 == 0 and ny % 4 == 0), up to 2048 angles per
// octant (the tiled kernel holds at most 64 in registers; the reference's
// time-dependent benchmark decks use 32 to 1024, input/*_1x1x1.in), the
// time-dependent terms (vdelt * psi_t in the numerator and the denominator,
// the time face of the fixup, psi_t out; sweep.cc:413-419, 461-468, 473-518)
// and the manufactured per-angle source of the MMS check (sweep.cc:368-375).
//
// Each thread owns a fixed set of angles, so every face value it reads (the
// x face carried in a register along the pencil, the y face of the previous
// pencil, the z face of the previous plane, both in global scratch) was
// written by the same thread: cells need no barrier between them except for
// the fixup's cell-wide vote (the count of negative faces over all angles,
// sweep.cc:425-472, a CTA-wide sum here) and the per-pencil reduction of the
// flux moments (the angle sums of sweep.cc:565-590, combined over the warps
// in shared memory and added with one atomic per cell and moment).
//
// The arithmetic follows the reference's CPU body: correctly rounded
// division for the geometry parameter and the fixup (expxs.cc:384-385,
// sweep.cc:499-501), and every angle of a cell recomputed in each fixup pass.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>

#include "device_util.cuh"
#include "internal.h"

namespace snapb200 {
namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int MAX_THREADS = 512;
constexpr int MAX_WARPS = MAX_THREADS / 32;

// MAXT: the CTA size the register budget is sized for: 128 registers per
// thread at any size, so that 4 CTAs of 128 threads (or 2 of 256) are
// resident per SM.  A sweep is one walk over the cells per wave of resident
// CTAs (one CTA per octant and group), so the register footprint per angle
// sets the number of waves: the per-angle constants live in shared memory,
// the fixup flags in bit masks, and the angular source is recomputed in the
// rare fixup passes instead of being kept.
template <int APT, int MAXT>
__global__ void __launch_bounds__(MAXT, (MAXT >= 512 ? 1 : 512 / MAXT)) wide_sweep_kernel(const WideParams p) {
  extern __shared__ double s_dyn[];
  __shared__ int s_cnt[MAX_WARPS];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nwarps = blockDim.x >> 5;
  const int o_local = blockIdx.x / p.G, g = blockIdx.x - o_local * p.G;
  const int o = p.o_base + o_local;
  const bool sx = o & 1, sy = (o >> 1) & 1, sz = (o >> 2) & 1;
  const int nx = p.nx, ny = p.ny, nz = p.nz, A = p.A, M = p.M;
  const long long C = (long long)nx * ny * nz;
  const double *qg = p.qtot + (size_t)g * C * M;
  const double *tg = p.t_xs + (size_t)g * C;
  const double vd = p.td ? p.vdelt[g] : 0.0;
  // the time terms and the time face exist only where vdelt != 0 (sweep.cc:413, 461, 473, 513)
  const bool tt = vd != 0.0;
  const size_t field = ((size_t)o * p.G + g) * C;   // (octant, group) field of the per-angle arrays
  double *ypen = p.ypen + (size_t)blockIdx.x * nx * A;
  double *zpl = p.zpl + (size_t)blockIdx.x * nx * ny * A;
  const double *ec = p.ec + (size_t)o * M * A;
  double *s_red = s_dyn;                                   // [warps][nx][M] per-warp moment partials
  double *s_cx = s_red + (size_t)nwarps * nx * M;          // [A] hi*mu, then hj*eta, hk*xi, w
  double *s_cy = s_cx + A, *s_cz = s_cy + A, *s_w = s_cz + A;
  for (int a = tid; a < A; a += blockDim.x) {
    s_cx[a] = p.mu[a] * p.hi;
    s_cy[a] = p.eta[a] * p.hj;
    s_cz[a] = p.xi[a] * p.hk;
    s_w[a] = p.w[a];
  }
  __syncthreads();
  // this thread's angles: tid + k * blockDim.x
  auto angle = [&](int k) { return tid + k * (int)blockDim.x; };
  double xin[APT];   // x face carried along the pencil
#pragma unroll
  for (int k = 0; k < APT; ++k) xin[k] = 0.0;

  // The inputs of a cell (sigma_t, the scalar source, and per angle the
  // time-edge flux and the incoming y and z faces) are loaded one cell
  // ahead, while the cell before is computed.  The faces a cell reads were
  // written by this thread at an earlier cell, except when the mesh is one
  // cell wide (nx = 1: the y face of the next pencil is this cell's; nx =
  // ny = 1: so is the z face), where they are forwarded from registers.
  double n_sig = 0.0, n_q0 = 0.0;
  double n_iy[APT], n_iz[APT], n_it[APT];
  auto load_cell = [&](int xx, int yy, int zz) {
    const int x = sx ? xx : nx - 1 - xx, y = sy ? yy : ny - 1 - yy, z = sz ? zz : nz - 1 - zz;
    const long long c = ((long long)z * ny + y) * nx + x;
    n_sig = __ldg(tg + c);
    n_q0 = __ldg(qg + c * M);
#pragma unroll
    for (int k = 0; k < APT; ++k) {
      const int a = angle(k);
      const bool on = a < A;
      n_it[k] = (tt && on) ? p.tf_in[(field + c) * A + a] : 0.0;
      n_iy[k] = (yy == 0 || !on) ? 0.0 : ypen[(size_t)xx * A + a];
      n_iz[k] = (zz == 0 || !on) ? 0.0 : zpl[((size_t)yy * nx + xx) * A + a];
    }
  };
  load_cell(0, 0, 0);

  for (int zz = 0; zz < nz; ++zz) {
    const int z = sz ? zz : nz - 1 - zz;
    for (int yy = 0; yy < ny; ++yy) {
      const int y = sy ? yy : ny - 1 - yy;
      for (int xx = 0; xx < nx; ++xx) {
        const int x = sx ? xx : nx - 1 - xx;
        const long long c = ((long long)z * ny + y) * nx + x;
        const double *q = qg + c * M;
        const double sig = n_sig;
        const double q0 = n_q0;
        double pc[APT], iy[APT], iz[APT], it[APT];
#pragma unroll
        for (int k = 0; k < APT; ++k) {
          iy[k] = n_iy[k];
          iz[k] = n_iz[k];
          it[k] = n_it[k];
        }
        // the next cell's inputs
        const bool more = xx + 1 < nx || yy + 1 < ny || zz + 1 < nz;
        const int nxx = xx + 1 < nx ? xx + 1 : 0;
        const int nyy = xx + 1 < nx ? yy : (yy + 1 < ny ? yy + 1 : 0);
        const int nzz = (xx + 1 < nx || yy + 1 < ny) ? zz : zz + 1;
        if (more) load_cell(nxx, nyy, nzz);
        // angular source of angle k (sweep.cc:354-375); the same operations
        // in the same order wherever it is needed
        auto source = [&](int k) {
          const int a = angle(k);
          double s = q0;
          for (int m = 1; m < M; ++m) s += ec[(size_t)m * A + a] * __ldg(q + m);
          if (p.qim) s += p.qim[(field + c) * A + a];
          return s;
        };
        if (xx == 0) {
#pragma unroll
          for (int k = 0; k < APT; ++k) xin[k] = 0.0;   // vacuum x boundary (single chunk)
        }
        bool neg = false;
#pragma unroll
        for (int k = 0; k < APT; ++k) {
          const int a = angle(k);
          const bool on = a < A;
          const int ak = on ? a : 0;
          const double cx = s_cx[ak], cy = s_cy[ak], cz = s_cz[ak];
          // diamond difference with the geometry parameter (expxs.cc:384-385,
          // sweep.cc:377-423)
          double v = (on ? source(k) : 0.0) + xin[k] * cx;
          v += iy[k] * cy;
          v += iz[k] * cz;
          if (tt) v += vd * it[k];
          const double dinv = __drcp_rn(sig + vd + cx + cy + cz);
          v = on ? v * dinv : 0.0;
          pc[k] = v;
          const double v2 = 2.0 * v;
          neg = neg || (v2 - xin[k] < 0.0) || (v2 - iy[k] < 0.0) || (v2 - iz[k] < 0.0) ||
                (tt && v2 - it[k] < 0.0);
        }
        // negative-flux fixup (sweep.cc:425-533): flags per angle and face
        // (bit k of each mask: 1 = the face keeps its value), the count of
        // negative faces summed over every angle of the cell, every angle
        // recomputed until the count stops changing
        unsigned hxm = ~0u, hym = ~0u, hzm = ~0u, htm = ~0u;
        if (p.fixup && __syncthreads_or(neg)) {
          int old = 0;
          for (int iter = 0; iter < 4 * 2048 + 4; ++iter) {
            int cnt = 0;
#pragma unroll
            for (int k = 0; k < APT; ++k) {
              if (angle(k) >= A) continue;
              const double v2 = 2.0 * pc[k];
              if (v2 - xin[k] < 0.0) { hxm &= ~(1u << k); ++cnt; }
              if (v2 - iy[k] < 0.0) { hym &= ~(1u << k); ++cnt; }
              if (v2 - iz[k] < 0.0) { hzm &= ~(1u << k); ++cnt; }
              if (tt && v2 - it[k] < 0.0) { htm &= ~(1u << k); ++cnt; }
            }
            cnt = __reduce_add_sync(FULL, cnt);
            if (lane == 0) s_cnt[warp] = cnt;
            __syncthreads();
            int total = 0;
            for (int w2 = 0; w2 < nwarps; ++w2) total += s_cnt[w2];
            __syncthreads();
            if (total == old) break;
            old = total;
#pragma unroll
            for (int k = 0; k < APT; ++k) {
              const int a = angle(k);
              if (a >= A) continue;
              const double cx = s_cx[a], cy = s_cy[a], cz = s_cz[a];
              const double hx = (hxm >> k) & 1u ? 1.0 : 0.0, hy = (hym >> k) & 1u ? 1.0 : 0.0,
                           hz = (hzm >> k) & 1u ? 1.0 : 0.0, ht = (htm >> k) & 1u ? 1.0 : 0.0;
              double v = source(k) + 0.5 * (xin[k] * cx * (1.0 + hx) + iy[k] * cy * (1.0 + hy) +
                                           iz[k] * cz * (1.0 + hz) + it[k] * vd * (1.0 + ht));
              const double den = (v <= 0.0) ? 0.0 : sig + cx * hx + cy * hy + cz * hz + vd * ht;
              pc[k] = den < 1.0e-12 ? 0.0 : __ddiv_rn(v, den);
            }
          }
        }
        // outgoing faces (flags are all 1 without a fixup) and the moments
        double part0 = 0.0;
#pragma unroll
        for (int k = 0; k < APT; ++k) {
          const int a = angle(k);
          if (a >= A) continue;
          const double hx = (hxm >> k) & 1u ? 1.0 : 0.0, hy = (hym >> k) & 1u ? 1.0 : 0.0,
                       hz = (hzm >> k) & 1u ? 1.0 : 0.0, ht = (htm >> k) & 1u ? 1.0 : 0.0;
          const double v2 = 2.0 * pc[k];
          xin[k] = (v2 - xin[k]) * hx;
          const double oy = (v2 - iy[k]) * hy, oz = (v2 - iz[k]) * hz;
          ypen[(size_t)xx * A + a] = oy;
          zpl[((size_t)yy * nx + xx) * A + a] = oz;
          if (tt) p.tf_out[(field + c) * A + a] = (v2 - it[k]) * ht;
          part0 += s_w[a] * pc[k];
          // one-cell-wide meshes: the next cell's face is this cell's output
          if (nx == 1 && nyy > 0 && more) n_iy[k] = oy;
          if (nx == 1 && ny == 1 && nzz > 0 && more) n_iz[k] = oz;
        }
        // per-warp moment partials of this cell into shared memory
        double *red = s_red + ((size_t)warp * nx + xx) * M;
        {
          const double r = __shfl_xor_sync(FULL, part0, 16) + part0;
          double r2 = r + __shfl_xor_sync(FULL, r, 8);
          r2 += __shfl_xor_sync(FULL, r2, 4);
          r2 += __shfl_xor_sync(FULL, r2, 2);
          r2 += __shfl_xor_sync(FULL, r2, 1);
          if (lane == 0) red[0] = r2;
        }
        for (int m = 1; m < M; ++m) {
          double pm = 0.0;
#pragma unroll
          for (int k = 0; k < APT; ++k) {
            const int a = angle(k);
            if (a < A) pm += ec[(size_t)m * A + a] * (s_w[a] * pc[k]);
          }
          pm += __shfl_xor_sync(FULL, pm, 16);
          pm += __shfl_xor_sync(FULL, pm, 8);
          pm += __shfl_xor_sync(FULL, pm, 4);
          pm += __shfl_xor_sync(FULL, pm, 2);
          pm += __shfl_xor_sync(FULL, pm, 1);
          if (lane == 0) red[m] = pm;
        }
      }
      // the pencil's moments: sum the warps' partials, one atomic per
      // (cell, moment) into the flux (octants add in arrival order, as the
      // reference's relaxed reductions do)
      __syncthreads();
      for (int i = tid; i < nx * M; i += blockDim.x) {
        const int xx = i / M, m = i - xx * M;
        double s = 0.0;
        for (int w2 = 0; w2 < nwarps; ++w2) s += s_red[((size_t)w2 * nx + xx) * M + m];
        const int x = sx ? xx : nx - 1 - xx;
        const long long c = ((long long)z * ny + y) * nx + x;
        atomicAdd(p.flux + ((size_t)g * C + c) * M + m, s);
      }
      __syncthreads();
    }
  }
}

}  // namespace

// Angles per thread: enough for a CTA of at most 128 threads where four per
// thread suffice (fewer warps shorten the per-cell barrier and reductions:
// on the 4096-cell reference decks, 256 angles 8.3 -> 5.2 ms per sweep and
// 512 angles 18.9 -> 12.5 ms against one angle per thread), else four; more
// when SNAP_B200_WIDE_APT asks (2 or 4).
int wide_apt(int A) {
  int apt = A <= 128 ? 1 : A <= 256 ? 2 : 4;
  if (const char *e = getenv("SNAP_B200_WIDE_APT")) {
    const int want = atoi(e);
    if (want == 2 || want == 4) apt = std::max(apt, want);
  }
  return apt;
}

int wide_threads(int A) {
  const int apt = wide_apt(A);
  const int t = (A + apt - 1) / apt;
  return std::min(MAX_THREADS, ((t + 31) / 32) * 32);
}

size_t wide_smem_bytes(int A, int nx, int M) {
  return sizeof(double) * ((size_t)(wide_threads(A) / 32) * nx * M + 4 * (size_t)A);
}

bool wide_supported(int A, int nx, int M) {
  return A >= 1 && A <= 4 * MAX_THREADS && M >= 1 && M <= 16 &&
         wide_smem_bytes(A, nx, M) <= 200 * 1024;
}

template <int APT, int MAXT>
cudaError_t launch_apt(const WideParams &p, int n_blocks, int threads, size_t smem,
                       cudaStream_t st) {
  cudaError_t e = cudaFuncSetAttribute(wide_sweep_kernel<APT, MAXT>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  wide_sweep_kernel<APT, MAXT><<<n_blocks, threads, smem, st>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_sweep_wide(const WideParams &p, int n_blocks, cudaStream_t st) {
  if (!wide_supported(p.A, p.nx, p.M)) return cudaErrorInvalidValue;
  const int threads = wide_threads(p.A);
  const size_t smem = wide_smem_bytes(p.A, p.nx, p.M);
  // CTA sizes with their own instances (128 registers per thread in each)
  switch (wide_apt(p.A)) {
    case 1: return launch_apt<1, MAX_THREADS>(p, n_blocks, threads, smem, st);
    case 2:
      return threads <= 128 ? launch_apt<2, 128>(p, n_blocks, threads, smem, st)
                            : launch_apt<2, MAX_THREADS>(p, n_blocks, threads, smem, st);
    default:
      return threads <= 128   ? launch_apt<4, 128>(p, n_blocks, threads, smem, st)
             : threads <= 256 ? launch_apt<4, 256>(p, n_blocks, threads, smem, st)
                              : launch_apt<4, MAX_THREADS>(p, n_blocks, threads, smem, st);
  }
}

}  // namespace snapb200
