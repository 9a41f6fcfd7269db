// HBM-bound kernels around the sweep: cross-section expansion, outer and
// inner sources, the octant-slot reduction fused with the convergence test.
#include <algorithm>

#include "device_util.cuh"
#include "internal.h"

namespace snapb200 {
namespace {

constexpr int BLK = 256;

inline int grid_for(long long n, int per_block = BLK) {
  long long g = (n + per_block - 1) / per_block;
  if (g > 148LL * 32) g = 148LL * 32;   // grid-stride beyond 32 CTAs per SM
  return (int)(g < 1 ? 1 : g);
}

// Adds the CTA's count of violations and its largest change into the device
// words with one atomic each instead of one per warp (every CTA thread calls
// it; the launch is uniform in whether it does).  Non-negative floats order
// like their bit patterns.
__device__ __forceinline__ void flush_test(int bad, float dmax, int *violations, unsigned *maxdf) {
  __shared__ int s_bad[32];
  __shared__ unsigned s_max[32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  bad = __reduce_add_sync(0xffffffffu, bad);
  const unsigned m = __reduce_max_sync(0xffffffffu, __float_as_uint(dmax));
  if (lane == 0) {
    s_bad[w] = bad;
    s_max[w] = m;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int b = 0;
    unsigned mm = 0;
    for (int i = 0; i < nw; ++i) {
      b += s_bad[i];
      mm = s_max[i] > mm ? s_max[i] : mm;
    }
    if (b) atomicAdd(violations, b);
    if (maxdf && mm) atomicMax(maxdf, mm);
  }
}

__device__ __forceinline__ int band_of(int k) {
  int l = 0;
  while ((l + 1) * (l + 1) <= k) ++l;
  return l;
}

// expxs.cc:85-115 / gpu_expxs.cu:21-267
__global__ void expand_xs_kernel(const double *__restrict__ sig, const int32_t *__restrict__ mat,
                                 double *__restrict__ xs, int G, int nmat, long long C) {
  const long long n = (long long)G * C;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int g = (int)(i / C);
    const long long c = i - (long long)g * C;
    xs[i] = sig[g * nmat + (mat[c] - 1)];
  }
}

__global__ void scale_xs_kernel(double *__restrict__ xs, const double *__restrict__ scale, int G,
                                long long C) {
  const long long n = (long long)G * C;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    xs[i] *= scale[i % C];
}

// expxs.cc:220-250 / gpu_expxs.cu:269-534
__global__ void expand_scat_kernel(const double *__restrict__ slgg, const int32_t *__restrict__ mat,
                                   double *__restrict__ s_xs, int G, int nmat, int nmom,
                                   long long C) {
  const long long n = (long long)G * C * nmom;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int l = (int)(i % nmom);
    const long long gc = i / nmom;
    const int g = (int)(gc / C);
    const long long c = gc - (long long)g * C;
    s_xs[i] = slgg[(((size_t)g * nmat + (mat[c] - 1)) * G + g) * nmom + l];
  }
}

// outer.cc:107-217 / gpu_outer.cu:22-441, all cmom moments.  A CTA stages
// the flux of CELLS cells (all groups and moments) in shared memory and
// produces every (group, cell, moment) output of those cells.
// Destination groups g_lo .. g_lo+g_n-1 (qi and q2grp hold those groups
// only); the flux holds all G source groups.
template <int CELLS>
__global__ void outer_source_kernel(const double *__restrict__ qi, const double *__restrict__ slgg,
                                    const int32_t *__restrict__ mat,
                                    const double *__restrict__ flux, double *__restrict__ q2grp,
                                    int G, int nmat, int nmom, int M, long long C, int g_lo,
                                    int g_n) {
  extern __shared__ double sflux[];   // [G][CELLS][M]
  const long long ntiles = (C + CELLS - 1) / CELLS;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long c0 = tile * CELLS;
    const int nc = (int)min((long long)CELLS, C - c0);
    __syncthreads();
    for (int i = threadIdx.x; i < G * CELLS * M; i += blockDim.x) {
      const int m = i % M, cc = (i / M) % CELLS, g = i / (M * CELLS);
      sflux[i] = cc < nc ? flux[((size_t)g * C + c0 + cc) * M + m] : 0.0;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < g_n * CELLS * M; i += blockDim.x) {
      const int m = i % M, cc = (i / M) % CELLS, gl = i / (M * CELLS);
      if (cc >= nc) continue;
      const int g1 = g_lo + gl;
      const long long c = c0 + cc;
      const int l = band_of(m);
      const double *row = slgg + ((size_t)g1 * nmat + (mat[c] - 1)) * G * nmom + l;
      double acc = (m == 0) ? qi[(size_t)gl * C + c] : 0.0;
      for (int g2 = 0; g2 < G; ++g2) {
        if (g2 == g1) continue;
        acc += __ldg(row + (size_t)g2 * nmom) * sflux[(g2 * CELLS + cc) * M + m];
      }
      q2grp[((size_t)gl * C + c) * M + m] = acc;
    }
  }
}

// The same outer source with the group-to-group contraction on the FP64
// tensor cores (mma.m8n8k4.f64).  For one moment k of band l the outputs of
// 8 cells are an (output groups x 8 cells) block:
//   D[g][c] = sum_{g'} S_l,mat(c)[g][g'] phi[g'][c][k]
// with S the scattering matrix of band l with its diagonal zeroed (in-group
// scattering belongs to the inner source).  Rows of D = 8 output groups per
// MMA tile, columns = 8 cells, k = 4 input groups per MMA.  Cells of
// different materials share one accumulator: the B operand of material m is
// phi masked to the columns whose cell has material m, so each column
// accumulates exactly its own material's products.
// A warp takes a block of 8 cells and MTW output-group tiles and walks the
// bands; per band and 4 input groups each lane loads the band's moments of
// one (input group, cell) straight from the flux (the band's A fragment then
// serves all of the band's moments), and writes the band's moments of its
// (output group, 2 cells) as consecutive words.  A CTA owns one set of MTW
// output-group tiles and keeps their fragments of every band and material
// in shared memory (copied once from the table odm_table_kernel builds).
constexpr int ODM_WARPS = 8;

template <int NMOM, int MTW>
size_t odm_smem_bytes(int G, int nmat) {
  return sizeof(double) * (size_t)NMOM * nmat * MTW * ((G + 3) / 4) * 32;
}

// tab[l][m][mt][kt][lane] = S_l,m[8mt + lane/4][4kt + lane%4] (output group
// g_lo + row, input group col), zero on the diagonal and in the padding
__global__ void odm_table_kernel(const double *__restrict__ slgg, int G, int nmat, int nmom,
                                 int g_lo, int g_n, int GT, int GK, double *__restrict__ tab) {
  const long long n = (long long)nmom * nmat * GT * GK * 32;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int ln = (int)(i & 31);
    long long r = i >> 5;
    const int kt = (int)(r % GK);
    r /= GK;
    const int mt = (int)(r % GT);
    r /= GT;
    const int m = (int)(r % nmat);
    const int l = (int)(r / nmat);
    const int row = 8 * mt + (ln >> 2), col = 4 * kt + (ln & 3), go = g_lo + row;
    tab[i] = (row < g_n && col < G && go != col)
                 ? slgg[(((size_t)go * nmat + m) * G + col) * nmom + l]
                 : 0.0;
  }
}

template <int NMOM, int MTW>
__global__ void __launch_bounds__(ODM_WARPS * 32)
    outer_source_dmma_kernel(const double *__restrict__ qi, const double *__restrict__ tab,
                             const int32_t *__restrict__ mat, const double *__restrict__ flux,
                             double *__restrict__ q2grp, int G, int nmat, long long C, int g_n,
                             int GT, int n_mg) {
  constexpr int M = NMOM * NMOM, NKMAX = 2 * NMOM - 1;
  extern __shared__ __align__(16) double odm_smem[];   // [l][mat][j][kt][32]
  const int GK = (G + 3) / 4;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int mg = blockIdx.x % n_mg, p = blockIdx.x / n_mg, P = gridDim.x / n_mg;
  // this CTA's fragments: output-group tiles mg*MTW + j of every band and material
  for (int i = tid; i < NMOM * nmat * MTW * GK * 32; i += blockDim.x) {
    const int ln = i & 31, kt = (i >> 5) % GK, j = (i >> 5) / GK % MTW, lm = (i >> 5) / (GK * MTW);
    const int mt = mg * MTW + j;
    odm_smem[i] = mt < GT ? __ldg(tab + (((size_t)lm * GT + mt) * GK + kt) * 32 + ln) : 0.0;
  }
  __syncthreads();
  const long long nblocks = (C + 7) / 8;
  for (long long blk = (long long)p * ODM_WARPS + w; blk < nblocks; blk += (long long)P * ODM_WARPS) {
    // B column of this lane: cell blk*8 + lane/4, input group 4kt + lane%4
    const long long cb = blk * 8 + (lane >> 2);
    const int matb = cb < C ? mat[cb] - 1 : -1;
#pragma unroll
    for (int l = 0; l < NMOM; ++l) {
      const int k0 = l * l, nk = 2 * l + 1;
      double acc[MTW][NKMAX][2];
#pragma unroll
      for (int j = 0; j < MTW; ++j)
#pragma unroll
        for (int kk = 0; kk < NKMAX; ++kk) acc[j][kk][0] = acc[j][kk][1] = 0.0;
      // the band's moments of (input group 4kt + lane%4, cell cb), one
      // input-group step ahead of the MMAs that use them
      double bn[NKMAX];
      auto load_b = [&](int kt) {
        const int gb = 4 * kt + (lane & 3);
        const bool in = kt < GK && gb < G && cb < C;
        const double *src = flux + ((size_t)(in ? gb : 0) * C + (in ? cb : 0)) * M + k0;
#pragma unroll
        for (int kk = 0; kk < NKMAX; ++kk) bn[kk] = (kk < nk && in) ? __ldg(src + kk) : 0.0;
      };
      load_b(0);
      for (int kt = 0; kt < GK; ++kt) {
        double b[NKMAX];
#pragma unroll
        for (int kk = 0; kk < NKMAX; ++kk) b[kk] = bn[kk];
        load_b(kt + 1);
        for (int m = 0; m < nmat; ++m) {
          const double *a = odm_smem + ((size_t)(l * nmat + m) * MTW * GK + kt) * 32 + lane;
          const bool mine = matb == m;
          double bm[NKMAX];
#pragma unroll
          for (int kk = 0; kk < NKMAX; ++kk) bm[kk] = mine ? b[kk] : 0.0;
#pragma unroll
          for (int j = 0; j < MTW; ++j) {
            const double aj = a[(size_t)j * GK * 32];
#pragma unroll
            for (int kk = 0; kk < NKMAX; ++kk)
              if (kk < nk) dmma_8x8x4(acc[j][kk][0], acc[j][kk][1], aj, bm[kk]);
          }
        }
      }
      // D rows (output groups) 8mt + lane/4, columns (cells) 2(lane%4) + {0,1}
#pragma unroll
      for (int j = 0; j < MTW; ++j) {
        const int gl = 8 * (mg * MTW + j) + (lane >> 2);
        if (gl >= g_n) continue;
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const long long c = blk * 8 + 2 * (lane & 3) + e;
          if (c >= C) continue;
          double *dst = q2grp + ((size_t)gl * C + c) * M + k0;
#pragma unroll
          for (int kk = 0; kk < NKMAX; ++kk) {
            if (kk >= nk) continue;
            double v = acc[j][kk][e];
            if (l == 0) v += qi[(size_t)gl * C + c];
            dst[kk] = v;
          }
        }
      }
    }
  }
}

// inner.cc:106-160 / gpu_inner.cu:22-117
template <typename QT>
__global__ void inner_source_kernel(const double *__restrict__ s_xs,
                                    const double *__restrict__ q2grp,
                                    const double *__restrict__ flux, QT *__restrict__ qtot, int G,
                                    int nmom, int M, long long C) {
  const long long n = (long long)G * C * M;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int m = (int)(i % M);
    const long long gc = i / M;
    qtot[i] = (QT)(q2grp[i] + flux[i] * s_xs[gc * nmom + band_of(m)]);
  }
}

// inner source with the old scalar flux saved and the moments cleared
template <typename QT>
__global__ void inner_source_save_kernel(const double *__restrict__ s_xs,
                                         const double *__restrict__ q2grp, double *flux,
                                         QT *__restrict__ qtot, double *__restrict__ old0, int G,
                                         int nmom, int M, long long C) {
  const long long n = (long long)G * C * M;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int m = (int)(i % M);
    const long long gc = i / M;
    const double f = flux[i];
    qtot[i] = (QT)(q2grp[i] + f * s_xs[gc * nmom + band_of(m)]);
    if (m == 0) old0[gc] = f;
    flux[i] = 0.0;
  }
}

// inner.cc:283-324 against a saved scalar flux, with the largest change
__global__ void test_change_kernel(const double *__restrict__ flux, const double *__restrict__ old0,
                                   int M, long long n, double epsi, int *violations,
                                   unsigned *maxdf) {
  int bad = 0;
  float dmax = 0.0f;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    double p = old0[i];
    double df = 1.0;
    if (fabs(p) < 1.0e-12) {
      p = 1.0;
      df = 0.0;
    }
    df = fabs(flux[i * M] / p - df);
    if (df > epsi) ++bad;
    dmax = fmaxf(dmax, (float)df);
  }
  flush_test(bad, dmax, violations, maxdf);
}

// flux = sum of the octant slots.  With `test`, also the inner convergence
// test of inner.cc:283-324 against the previous scalar flux, which is read
// from flux64_out before it is overwritten.
template <typename ST, typename OT>
__global__ void reduce_slots_kernel(const ST *__restrict__ slots, int nslots, OT *flux_out,
                                    double *flux64_out, int G, int M, long long C, int test,
                                    double epsi, int *violations, unsigned *maxdf) {
  const long long n = (long long)G * C * M;
  int bad = 0;
  float dmax = 0.0f;   // largest relative change seen by this thread
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int k = 0; k < nslots; ++k) s += (double)slots[(size_t)k * n + i];
    if (test && (i % M) == 0) {
      double prev = flux64_out[i];
      double df = 1.0;
      if (fabs(prev) < 1.0e-12) {
        prev = 1.0;
        df = 0.0;
      }
      df = fabs(s / prev - df);
      if (df > epsi) ++bad;
      dmax = fmaxf(dmax, (float)df);   // NaN compares false: ignored, as in the count
    }
    if (flux_out) flux_out[i] = (OT)s;
    if (flux64_out && (void *)flux64_out != (void *)flux_out) flux64_out[i] = s;
  }
  if (test) flush_test(bad, dmax, violations, maxdf);
}

// inner.cc:283-324 / outer.cc:354-403
__global__ void count_violations_kernel(const double *__restrict__ flux,
                                        const double *__restrict__ prev, int M, long long n,
                                        double epsi, int *violations) {
  int bad = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    double p = prev[i * M];
    double df = 1.0;
    if (fabs(p) < 1.0e-12) {
      p = 1.0;
      df = 0.0;
    }
    df = fabs(flux[i * M] / p - df);
    if (df > epsi) ++bad;
  }
  flush_test(bad, 0.0f, violations, nullptr);
}

__global__ void copy_moment0_kernel(const double *__restrict__ flux, double *__restrict__ out,
                                    int M, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i * M] = flux[i * M];
}

// Adjoint of the scattering source (outer.cc:145-171 and inner.cc:130-146
// transposed): every group, in-group included.
template <int CELLS>
__global__ void adjoint_scatter_kernel(const double *__restrict__ r, const double *__restrict__ slgg,
                                       const int32_t *__restrict__ mat,
                                       const double *__restrict__ qbar, double *__restrict__ phib,
                                       int G, int nmat, int nmom, int M, long long C) {
  extern __shared__ double sq[];   // [G][CELLS][M]
  const long long ntiles = (C + CELLS - 1) / CELLS;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long c0 = tile * CELLS;
    const int nc = (int)min((long long)CELLS, C - c0);
    __syncthreads();
    for (int i = threadIdx.x; i < G * CELLS * M; i += blockDim.x) {
      const int m = i % M, cc = (i / M) % CELLS, g = i / (M * CELLS);
      sq[i] = cc < nc ? qbar[((size_t)g * C + c0 + cc) * M + m] : 0.0;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < G * CELLS * M; i += blockDim.x) {
      const int m = i % M, cc = (i / M) % CELLS, g2 = i / (M * CELLS);
      if (cc >= nc) continue;
      const long long c = c0 + cc;
      const int l = band_of(m), mt = mat[c] - 1;
      double acc = (m == 0) ? r[(size_t)g2 * C + c] : 0.0;
      for (int g = 0; g < G; ++g)
        acc += __ldg(slgg + (((size_t)g * nmat + mt) * G + g2) * nmom + l) *
               sq[(g * CELLS + cc) * M + m];
      phib[((size_t)g2 * C + c) * M + m] = acc;
    }
  }
}

// The adjoint source update in place: phib = r + S^T qbar (as
// adjoint_scatter_kernel), with max |new - old| and max |new| accumulated in
// norm[0..1] as bit patterns of non-negative doubles (NaN differences count
// as infinite).  QT/PT: the types of qbar and phib (the sweep precision).
template <int CELLS, typename QT, typename PT>
__global__ void adjoint_update_kernel(const double *__restrict__ r, const double *__restrict__ slgg,
                                      const int32_t *__restrict__ mat,
                                      const QT *__restrict__ qbar, PT *__restrict__ phib,
                                      unsigned long long *__restrict__ norm, int G, int nmat,
                                      int nmom, int M, long long C) {
  extern __shared__ double sq[];   // [G][CELLS][M]
  double md = 0.0, ma = 0.0;
  const long long ntiles = (C + CELLS - 1) / CELLS;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long c0 = tile * CELLS;
    const int nc = (int)min((long long)CELLS, C - c0);
    __syncthreads();
    for (int i = threadIdx.x; i < G * CELLS * M; i += blockDim.x) {
      const int m = i % M, cc = (i / M) % CELLS, g = i / (M * CELLS);
      sq[i] = cc < nc ? (double)qbar[((size_t)g * C + c0 + cc) * M + m] : 0.0;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < G * CELLS * M; i += blockDim.x) {
      const int m = i % M, cc = (i / M) % CELLS, g2 = i / (M * CELLS);
      if (cc >= nc) continue;
      const long long c = c0 + cc;
      const int l = band_of(m), mt = mat[c] - 1;
      double acc = (m == 0) ? r[(size_t)g2 * C + c] : 0.0;
      for (int g = 0; g < G; ++g)
        acc += __ldg(slgg + (((size_t)g * nmat + mt) * G + g2) * nmom + l) *
               sq[(g * CELLS + cc) * M + m];
      PT *dst = phib + ((size_t)g2 * C + c) * M + m;
      const PT nv = (PT)acc;
      const double d = fabs((double)nv - (double)*dst);
      md = (d != d) ? INFINITY : fmax(md, d);
      ma = fmax(ma, fabs((double)nv));
      *dst = nv;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    md = fmax(md, __shfl_xor_sync(0xffffffffu, md, o));
    ma = fmax(ma, __shfl_xor_sync(0xffffffffu, ma, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(norm, (unsigned long long)__double_as_longlong(md));
    atomicMax(norm + 1, (unsigned long long)__double_as_longlong(ma));
  }
}

template <typename QT>
__global__ void grad_sxs_kernel(const QT *__restrict__ qbar, const double *__restrict__ flux,
                                double *__restrict__ grad, int G, int nmom, int M, long long C) {
  const long long n = (long long)G * C * nmom;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int l = (int)(i % nmom);
    const long long gc = i / nmom;
    double acc = 0.0;
    for (int k = l * l; k < (l + 1) * (l + 1) && k < M; ++k)
      acc += (double)qbar[gc * M + k] * flux[gc * M + k];
    grad[i] = acc;
  }
}

template <typename IT>
__global__ void moment0_kernel(const IT *__restrict__ in, double *__restrict__ out, int M,
                               long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = in[i * M];
}

// max |a-b| and max |a| as bit patterns (non-negative doubles order like
// their unsigned bit patterns); NaN differences count as infinite
__global__ void max_abs_diff_kernel(const double *__restrict__ a, const double *__restrict__ b,
                                    long long n, unsigned long long *out) {
  double md = 0.0, ma = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double d = fabs(a[i] - b[i]);
    md = (d != d) ? INFINITY : fmax(md, d);
    ma = fmax(ma, fabs(a[i]));
  }
  for (int o = 16; o > 0; o >>= 1) {
    md = fmax(md, __shfl_xor_sync(0xffffffffu, md, o));
    ma = fmax(ma, __shfl_xor_sync(0xffffffffu, ma, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(out, (unsigned long long)__double_as_longlong(md));
    atomicMax(out + 1, (unsigned long long)__double_as_longlong(ma));
  }
}

// mms.cc:442-470 (MMSScale): x *= f
__global__ void scale_kernel(double *__restrict__ x, double f, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    x[i] *= f;
}

__global__ void to_f32_kernel(const double *__restrict__ in, float *__restrict__ out, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = (float)in[i];
}

}  // namespace

cudaError_t k_adjoint_scatter(const double *r, const double *slgg, const int32_t *mat,
                              const double *qbar, double *phi_bar, int G, int nmat, int nmom,
                              int M, long long C, cudaStream_t st) {
  constexpr int CELLS = 4;
  const size_t smem = sizeof(double) * G * CELLS * M;
  if (smem > 200 * 1024) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(adjoint_scatter_kernel<CELLS>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const long long tiles = (C + CELLS - 1) / CELLS;
  adjoint_scatter_kernel<CELLS><<<grid_for(tiles, 1), BLK, smem, st>>>(r, slgg, mat, qbar, phi_bar,
                                                                        G, nmat, nmom, M, C);
  return cudaGetLastError();
}

cudaError_t k_grad_sxs(const double *qbar, const double *flux, double *grad, int G, int nmom,
                       int M, long long C, cudaStream_t st) {
  return k_grad_sxs_any(qbar, 0, flux, grad, G, nmom, M, C, st);
}

cudaError_t k_grad_sxs_any(const void *qbar, int fp32, const double *flux, double *grad, int G,
                           int nmom, int M, long long C, cudaStream_t st) {
  const int grid = grid_for((long long)G * C * nmom);
  if (fp32)
    grad_sxs_kernel<float><<<grid, BLK, 0, st>>>((const float *)qbar, flux, grad, G, nmom, M, C);
  else
    grad_sxs_kernel<double><<<grid, BLK, 0, st>>>((const double *)qbar, flux, grad, G, nmom, M, C);
  return cudaGetLastError();
}

cudaError_t k_moment0(const double *in, double *out, int M, long long n, cudaStream_t st) {
  moment0_kernel<double><<<grid_for(n), BLK, 0, st>>>(in, out, M, n);
  return cudaGetLastError();
}

cudaError_t k_moment0_any(const void *in, int fp32, double *out, int M, long long n,
                          cudaStream_t st) {
  if (fp32)
    moment0_kernel<float><<<grid_for(n), BLK, 0, st>>>((const float *)in, out, M, n);
  else
    moment0_kernel<double><<<grid_for(n), BLK, 0, st>>>((const double *)in, out, M, n);
  return cudaGetLastError();
}

cudaError_t k_adjoint_update(const double *r, const double *slgg, const int32_t *mat,
                             const void *qbar, void *phib, int fp32, unsigned long long *norm,
                             int G, int nmat, int nmom, int M, long long C, cudaStream_t st) {
  constexpr int CELLS = 4;
  const size_t smem = sizeof(double) * G * CELLS * M;
  if (smem > 200 * 1024) return cudaErrorInvalidValue;
  const long long tiles = (C + CELLS - 1) / CELLS;
  cudaError_t e;
  if (fp32) {
    auto kern = adjoint_update_kernel<CELLS, float, float>;
    if ((e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)))
      return e;
    kern<<<grid_for(tiles, 1), BLK, smem, st>>>(r, slgg, mat, (const float *)qbar, (float *)phib,
                                                norm, G, nmat, nmom, M, C);
  } else {
    auto kern = adjoint_update_kernel<CELLS, double, double>;
    if ((e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)))
      return e;
    kern<<<grid_for(tiles, 1), BLK, smem, st>>>(r, slgg, mat, (const double *)qbar,
                                                (double *)phib, norm, G, nmat, nmom, M, C);
  }
  return cudaGetLastError();
}

cudaError_t k_max_abs_diff(const double *a, const double *b, long long n,
                           unsigned long long *out, cudaStream_t st) {
  max_abs_diff_kernel<<<grid_for(n), BLK, 0, st>>>(a, b, n, out);
  return cudaGetLastError();
}

cudaError_t k_to_f32(const double *in, float *out, long long n, cudaStream_t st) {
  to_f32_kernel<<<grid_for(n), BLK, 0, st>>>(in, out, n);
  return cudaGetLastError();
}

cudaError_t k_scale(double *x, double f, size_t n, cudaStream_t st) {
  scale_kernel<<<grid_for((long long)n), BLK, 0, st>>>(x, f, (long long)n);
  return cudaGetLastError();
}

cudaError_t k_expand_xs(const double *sig, const int32_t *mat, double *xs, int G, int nmat,
                        long long C, cudaStream_t st) {
  expand_xs_kernel<<<grid_for((long long)G * C), BLK, 0, st>>>(sig, mat, xs, G, nmat, C);
  return cudaGetLastError();
}

cudaError_t k_scale_xs(double *xs, const double *scale, int G, long long C, cudaStream_t st) {
  scale_xs_kernel<<<grid_for((long long)G * C), BLK, 0, st>>>(xs, scale, G, C);
  return cudaGetLastError();
}

cudaError_t k_expand_scat(const double *slgg, const int32_t *mat, double *s_xs, int G, int nmat,
                          int nmom, long long C, cudaStream_t st) {
  expand_scat_kernel<<<grid_for((long long)G * C * nmom), BLK, 0, st>>>(slgg, mat, s_xs, G, nmat,
                                                                          nmom, C);
  return cudaGetLastError();
}

namespace {

template <int NMOM, int MTW>
cudaError_t launch_outer_dmma(const double *qi, const double *tab, const int32_t *mat,
                              const double *flux, double *q2grp, int G, int nmat, long long C,
                              int g_n, cudaStream_t st) {
  auto kern = outer_source_dmma_kernel<NMOM, MTW>;
  const size_t smem = odm_smem_bytes<NMOM, MTW>(G, nmat);
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 0, blocks = 0;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kern, ODM_WARPS * 32, smem)) !=
      cudaSuccess)
    return e;
  const int GT = (g_n + 7) / 8, n_mg = (GT + MTW - 1) / MTW;
  // CTAs per output-group set: fill the device, at most one warp per cell block
  const long long nblocks = (C + 7) / 8;
  const long long per_set =
      std::max<long long>(1, std::min<long long>((long long)std::max(blocks, 1) * sms / n_mg,
                                                 (nblocks + ODM_WARPS - 1) / ODM_WARPS));
  kern<<<(int)(per_set * n_mg), ODM_WARPS * 32, smem, st>>>(qi, tab, mat, flux, q2grp, G, nmat, C,
                                                            g_n, GT, n_mg);
  return cudaGetLastError();
}

template <int NMOM>
cudaError_t launch_outer_dmma_mtw(const double *qi, const double *tab, const int32_t *mat,
                                  const double *flux, double *q2grp, int G, int nmat, long long C,
                                  int g_n, cudaStream_t st) {
  const int GT = (g_n + 7) / 8;
  if (GT == 1) return launch_outer_dmma<NMOM, 1>(qi, tab, mat, flux, q2grp, G, nmat, C, g_n, st);
  if (GT == 2) return launch_outer_dmma<NMOM, 2>(qi, tab, mat, flux, q2grp, G, nmat, C, g_n, st);
  return launch_outer_dmma<NMOM, 4>(qi, tab, mat, flux, q2grp, G, nmat, C, g_n, st);
}

}  // namespace

size_t outer_dmma_table_words(int G, int g_n, int nmat, int nmom) {
  return (size_t)nmom * nmat * ((g_n + 7) / 8) * ((G + 3) / 4) * 32;
}

cudaError_t k_outer_source_groups(const double *qi, const double *slgg, const int32_t *mat,
                                  const double *flux, double *q2grp, double *tab, int G, int nmat,
                                  int nmom, int M, long long C, int g_lo, int g_n, int *launches,
                                  cudaStream_t st) {
  *launches = 1;
  // tensor-core form when its fragments fit in shared memory
  const int GT = (g_n + 7) / 8, GK = (G + 3) / 4;
  const size_t dsmem = sizeof(double) * (size_t)nmom * nmat * std::min(GT, 4) * GK * 32;
  if (tab && dsmem <= 160 * 1024) {
    *launches = 2;
    odm_table_kernel<<<32, 256, 0, st>>>(slgg, G, nmat, nmom, g_lo, g_n, GT, GK, tab);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    switch (nmom) {
      case 1: return launch_outer_dmma_mtw<1>(qi, tab, mat, flux, q2grp, G, nmat, C, g_n, st);
      case 2: return launch_outer_dmma_mtw<2>(qi, tab, mat, flux, q2grp, G, nmat, C, g_n, st);
      case 3: return launch_outer_dmma_mtw<3>(qi, tab, mat, flux, q2grp, G, nmat, C, g_n, st);
      case 4: return launch_outer_dmma_mtw<4>(qi, tab, mat, flux, q2grp, G, nmat, C, g_n, st);
      default: *launches = 1; break;
    }
  }
  constexpr int CELLS = 4;
  const size_t smem = sizeof(double) * G * CELLS * M;
  if (smem > 200 * 1024) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(outer_source_kernel<CELLS>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const long long tiles = (C + CELLS - 1) / CELLS;
  outer_source_kernel<CELLS><<<grid_for(tiles, 1), BLK, smem, st>>>(qi, slgg, mat, flux, q2grp, G,
                                                                     nmat, nmom, M, C, g_lo, g_n);
  return cudaGetLastError();
}

cudaError_t k_inner_source(const double *s_xs, const double *q2grp, const double *flux, void *qtot,
                           int fp32, int G, int nmom, int M, long long C, cudaStream_t st) {
  const int grid = grid_for((long long)G * C * M);
  if (fp32)
    inner_source_kernel<float><<<grid, BLK, 0, st>>>(s_xs, q2grp, flux, (float *)qtot, G, nmom, M, C);
  else
    inner_source_kernel<double><<<grid, BLK, 0, st>>>(s_xs, q2grp, flux, (double *)qtot, G, nmom, M,
                                                      C);
  return cudaGetLastError();
}

cudaError_t k_inner_source_save(const double *s_xs, const double *q2grp, double *flux, void *qtot,
                                int fp32, double *old0, int G, int nmom, int M, long long C,
                                cudaStream_t st) {
  const int grid = grid_for((long long)G * C * M);
  if (fp32)
    inner_source_save_kernel<float><<<grid, BLK, 0, st>>>(s_xs, q2grp, flux, (float *)qtot, old0, G,
                                                          nmom, M, C);
  else
    inner_source_save_kernel<double><<<grid, BLK, 0, st>>>(s_xs, q2grp, flux, (double *)qtot, old0,
                                                           G, nmom, M, C);
  return cudaGetLastError();
}

cudaError_t k_test_change(const double *flux, const double *old0, int M, long long n, double epsi,
                          int *violations, unsigned *maxdf, cudaStream_t st) {
  test_change_kernel<<<grid_for(n), BLK, 0, st>>>(flux, old0, M, n, epsi, violations, maxdf);
  return cudaGetLastError();
}

cudaError_t k_reduce_slots(const void *slots, int nslots, int fp32, void *flux_out, int out_fp32,
                           double *flux64_out, int G, int M, long long C, int test, double epsi,
                           int *violations, cudaStream_t st, unsigned *maxdf) {
  const int grid = grid_for((long long)G * C * M);
  if (fp32) {
    if (out_fp32)
      reduce_slots_kernel<float, float><<<grid, BLK, 0, st>>>(
          (const float *)slots, nslots, (float *)flux_out, flux64_out, G, M, C, test, epsi,
          violations, maxdf);
    else
      reduce_slots_kernel<float, double><<<grid, BLK, 0, st>>>(
          (const float *)slots, nslots, (double *)flux_out, flux64_out, G, M, C, test, epsi,
          violations, maxdf);
  } else {
    reduce_slots_kernel<double, double><<<grid, BLK, 0, st>>>(
        (const double *)slots, nslots, (double *)flux_out, flux64_out, G, M, C, test, epsi,
        violations, maxdf);
  }
  return cudaGetLastError();
}

cudaError_t k_count_violations(const double *flux, const double *prev, int M, long long n,
                               double epsi, int *violations, cudaStream_t st) {
  count_violations_kernel<<<grid_for(n), BLK, 0, st>>>(flux, prev, M, n, epsi, violations);
  return cudaGetLastError();
}

cudaError_t k_copy_moment0(const double *flux, double *out, int M, long long n, cudaStream_t st) {
  copy_moment0_kernel<<<grid_for(n), BLK, 0, st>>>(flux, out, M, n);
  return cudaGetLastError();
}

}  // namespace snapb200
