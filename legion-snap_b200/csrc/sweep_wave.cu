// Wavefront form of the general FP64 sweep: one CTA per (octant, group), the
// cells of one diagonal plane (i + j + k = s in sweep order) in flight at
// once, one cell per warp (a warp holds all of a cell's angles, up to 128,
// four per lane), a CTA barrier between diagonals.
//
// The general kernel (sweep_wide.cu) walks the cells of an (octant, group)
// one at a time, so its time is the mesh's cell count times one cell's
// latency.  Cells on one diagonal do not depend on each other (each reads
// only the faces its upstream neighbours wrote on the previous diagonal),
// so here the chain is the number of diagonals (nx + ny + nz - 2) times the
// cells a cell group takes per diagonal.  Face planes: the x face leaving
// cell (i, j, k) is stored at slot (j, k) and read from there by cell
// (i+1, j, k) on the next diagonal; y faces at (i, k), z faces at (i, j).
// Within a diagonal a slot is read and then overwritten by the same cell
// only, so one copy of each plane suffices.
//
// The arithmetic is that of the general kernel and of the reference's CPU
// body (sweep.cc:354-591): correctly rounded division for the geometry
// parameter and the fixup, every angle of a cell recomputed in each fixup
// pass until the cell's count of negative faces stops changing (a warp
// reduction), the time-dependent terms and the manufactured source.
//
// Measured on the reference's small_4K deck (16^3 cells, 128 angles, 32
// groups): 1.71 ms per sweep against 3.83 ms cell by cell; 4 warps per CTA
// beat 2 (2.42 ms) and 8 (1.90 ms).  Spreading a cell's 256 angles over two
// warps (medium_4K) was slower than the cell-by-cell kernel at two angles
// per thread (6.6 against 5.2 ms), so larger angle counts stay there.  The flux moments of a cell are reduced over its
// angles and added with one atomic per moment (octants add in arrival
// order, as the reference's relaxed reductions do).
#include <cuda_runtime.h>

#include <algorithm>

#include "device_util.cuh"
#include "internal.h"

namespace snapb200 {
namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int WAVE_WARPS = 4;   // warps per CTA (cells in flight)

// APT angles per lane; MQ: the most flux moments held per cell (1, or 16
// for any nmom).
template <int APT, int MQ>
__global__ void __launch_bounds__(WAVE_WARPS * 32, 2) wave_sweep_kernel(const WideParams p) {
  constexpr int CG = WAVE_WARPS;   // cells in flight
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int cg = warp;
  const int o_local = blockIdx.x / p.G, g = blockIdx.x - o_local * p.G;
  const int o = p.o_base + o_local;
  const bool sx = o & 1, sy = (o >> 1) & 1, sz = (o >> 2) & 1;
  const int nx = p.nx, ny = p.ny, nz = p.nz, A = p.A, M = p.M;
  const long long C = (long long)nx * ny * nz;
  const double *qg = p.qtot + (size_t)g * C * M;
  const double *tg = p.t_xs + (size_t)g * C;
  const double vd = p.td ? p.vdelt[g] : 0.0;
  const bool tt = vd != 0.0;   // time terms and time face only where vdelt != 0
  const size_t field = ((size_t)o * p.G + g) * C;
  double *wx = p.wx + (size_t)blockIdx.x * ny * nz * A;   // [j][k][A]
  double *wy = p.wy + (size_t)blockIdx.x * nx * nz * A;   // [i][k][A]
  double *wz = p.wz + (size_t)blockIdx.x * nx * ny * A;   // [i][j][A]
  const double *ec = p.ec + (size_t)o * M * A;

  int ang[APT];
  bool on[APT];
  double cx[APT], cy[APT], cz[APT], wt[APT];
#pragma unroll
  for (int t = 0; t < APT; ++t) {
    ang[t] = lane + t * 32;
    on[t] = ang[t] < A;
    const int a = on[t] ? ang[t] : 0;
    cx[t] = p.mu[a] * p.hi;
    cy[t] = p.eta[a] * p.hj;
    cz[t] = p.xi[a] * p.hk;
    wt[t] = on[t] ? p.w[a] : 0.0;
  }

  // sum over the cell's angles (the warp) of per-thread counts
  auto group_sum_i = [&](int v) -> int { return __reduce_add_sync(FULL, v); };

  // inputs of a cell, loaded one cell ahead
  double n_sig = 0.0, n_q[MQ];
  double n_qim[APT], n_ix[APT], n_iy[APT], n_iz[APT], n_it[APT];
  auto load_cell = [&](int i, int j, int k) {
    const int x = sx ? i : nx - 1 - i, y = sy ? j : ny - 1 - j, z = sz ? k : nz - 1 - k;
    const long long c = ((long long)z * ny + y) * nx + x;
    n_sig = __ldg(tg + c);
#pragma unroll
    for (int m = 0; m < MQ; ++m) n_q[m] = m < M ? __ldg(qg + c * M + m) : 0.0;
#pragma unroll
    for (int t = 0; t < APT; ++t) {
      const int a = on[t] ? ang[t] : 0;
      n_qim[t] = (p.qim && on[t]) ? __ldg(p.qim + (field + c) * A + a) : 0.0;
      n_it[t] = (tt && on[t]) ? __ldg(p.tf_in + (field + c) * A + a) : 0.0;
      n_ix[t] = (i == 0 || !on[t]) ? 0.0 : wx[((size_t)j * nz + k) * A + a];
      n_iy[t] = (j == 0 || !on[t]) ? 0.0 : wy[((size_t)i * nz + k) * A + a];
      n_iz[t] = (k == 0 || !on[t]) ? 0.0 : wz[((size_t)i * ny + j) * A + a];
    }
  };

  const int nd = nx + ny + nz - 2;   // diagonals
  for (int s = 0; s < nd; ++s) {
    // this warp's cells of diagonal s: rows i = i_lo + warp, + CG, ...,
    // each with every valid j (k = s - i - j)
    const int i_lo = max(0, s - (ny - 1) - (nz - 1)), i_hi = min(nx - 1, s);
    auto j_lo = [&](int i) { return max(0, s - i - (nz - 1)); };
    auto j_hi = [&](int i) { return min(ny - 1, s - i); };
    int ci = i_lo + cg, cj = ci <= i_hi ? j_lo(ci) : 0;
    if (ci <= i_hi) load_cell(ci, cj, s - ci - cj);
    while (ci <= i_hi) {
      const int i = ci, j = cj, k = s - ci - cj;
      // the next cell of this group on this diagonal
      if (cj < j_hi(ci)) {
        ++cj;
      } else {
        ci += CG;
        cj = ci <= i_hi ? j_lo(ci) : 0;
      }
      const double sig = n_sig;
      double q[MQ];
#pragma unroll
      for (int m = 0; m < MQ; ++m) q[m] = n_q[m];
      double ix[APT], iy[APT], iz[APT], it[APT], qm[APT];
#pragma unroll
      for (int t = 0; t < APT; ++t) {
        ix[t] = n_ix[t];
        iy[t] = n_iy[t];
        iz[t] = n_iz[t];
        it[t] = n_it[t];
        qm[t] = n_qim[t];
      }
      if (ci <= i_hi) load_cell(ci, cj, s - ci - cj);
      const int x = sx ? i : nx - 1 - i, y = sy ? j : ny - 1 - j, z = sz ? k : nz - 1 - k;
      const long long c = ((long long)z * ny + y) * nx + x;

      double pc[APT], psi[APT];
      int neg = 0;
#pragma unroll
      for (int t = 0; t < APT; ++t) {
        const int a = on[t] ? ang[t] : 0;
        double sv = q[0];   // angular source (sweep.cc:354-375)
#pragma unroll
        for (int m = 1; m < MQ; ++m)
          if (m < M) sv += ec[(size_t)m * A + a] * q[m];
        if (p.qim) sv += qm[t];
        psi[t] = sv;
        double v = sv + ix[t] * cx[t];   // diamond difference (sweep.cc:377-423)
        v += iy[t] * cy[t];
        v += iz[t] * cz[t];
        if (tt) v += vd * it[t];
        const double dinv = __drcp_rn(sig + vd + cx[t] + cy[t] + cz[t]);
        v = on[t] ? v * dinv : 0.0;
        pc[t] = v;
        const double v2 = 2.0 * v;
        neg |= (v2 - ix[t] < 0.0) || (v2 - iy[t] < 0.0) || (v2 - iz[t] < 0.0) ||
               (tt && v2 - it[t] < 0.0);
      }
      // negative-flux fixup (sweep.cc:425-533), cell-wide over the warp
      double hx[APT], hy[APT], hz[APT], ht[APT];
#pragma unroll
      for (int t = 0; t < APT; ++t) hx[t] = hy[t] = hz[t] = ht[t] = 1.0;
      if (p.fixup && group_sum_i(neg) > 0) {
        int old = 0;
        for (int iter = 0; iter < 4 * 256 + 4; ++iter) {
          int cnt = 0;
#pragma unroll
          for (int t = 0; t < APT; ++t) {
            if (!on[t]) continue;
            const double v2 = 2.0 * pc[t];
            if (v2 - ix[t] < 0.0) { hx[t] = 0.0; ++cnt; }
            if (v2 - iy[t] < 0.0) { hy[t] = 0.0; ++cnt; }
            if (v2 - iz[t] < 0.0) { hz[t] = 0.0; ++cnt; }
            if (tt && v2 - it[t] < 0.0) { ht[t] = 0.0; ++cnt; }
          }
          const int total = group_sum_i(cnt);
          if (total == old) break;
          old = total;
#pragma unroll
          for (int t = 0; t < APT; ++t) {
            if (!on[t]) continue;
            const double v = psi[t] + 0.5 * (ix[t] * cx[t] * (1.0 + hx[t]) +
                                             iy[t] * cy[t] * (1.0 + hy[t]) +
                                             iz[t] * cz[t] * (1.0 + hz[t]) +
                                             it[t] * vd * (1.0 + ht[t]));
            const double den = (v <= 0.0) ? 0.0
                                          : sig + cx[t] * hx[t] + cy[t] * hy[t] + cz[t] * hz[t] +
                                                vd * ht[t];
            pc[t] = den < 1.0e-12 ? 0.0 : __ddiv_rn(v, den);
          }
        }
      }
      // outgoing faces (flags are all 1 without a fixup)
#pragma unroll
      for (int t = 0; t < APT; ++t) {
        if (!on[t]) continue;
        const int a = ang[t];
        const double v2 = 2.0 * pc[t];
        wx[((size_t)j * nz + k) * A + a] = (v2 - ix[t]) * hx[t];
        wy[((size_t)i * nz + k) * A + a] = (v2 - iy[t]) * hy[t];
        wz[((size_t)i * ny + j) * A + a] = (v2 - iz[t]) * hz[t];
        if (tt) p.tf_out[(field + c) * A + a] = (v2 - it[t]) * ht[t];
      }
      // flux moments of this octant (sweep.cc:565-590): one atomic per moment
#pragma unroll
      for (int m = 0; m < MQ; ++m) {
        if (m >= M) break;
        double pm = 0.0;
#pragma unroll
        for (int t = 0; t < APT; ++t)
          if (on[t]) pm += (m == 0 ? 1.0 : ec[(size_t)m * A + ang[t]]) * (wt[t] * pc[t]);
        pm += __shfl_xor_sync(FULL, pm, 16);
        pm += __shfl_xor_sync(FULL, pm, 8);
        pm += __shfl_xor_sync(FULL, pm, 4);
        pm += __shfl_xor_sync(FULL, pm, 2);
        pm += __shfl_xor_sync(FULL, pm, 1);
        if (lane == 0) atomicAdd(p.flux + ((size_t)g * C + c) * M + m, pm);
      }
    }
    __syncthreads();   // every face of diagonal s is written before s + 1 reads
  }
}

template <int APT>
cudaError_t launch(const WideParams &p, int n_blocks, cudaStream_t st) {
  if (p.M == 1)
    wave_sweep_kernel<APT, 1><<<n_blocks, WAVE_WARPS * 32, 0, st>>>(p);
  else
    wave_sweep_kernel<APT, 16><<<n_blocks, WAVE_WARPS * 32, 0, st>>>(p);
  return cudaGetLastError();
}

}  // namespace

bool wave_supported(int A, int M) { return A >= 1 && A <= 128 && M >= 1 && M <= 16; }

size_t wave_scratch_doubles(int nx, int ny, int nz, int A, int blocks) {
  return ((size_t)ny * nz + (size_t)nx * nz + (size_t)nx * ny) * A * blocks;
}

cudaError_t launch_sweep_wave(const WideParams &p, int n_blocks, cudaStream_t st) {
  if (!wave_supported(p.A, p.M)) return cudaErrorInvalidValue;
  // a cell's angles on one warp: one, two or four per lane
  if (p.A <= 32) return launch<1>(p, n_blocks, st);
  if (p.A <= 64) return launch<2>(p, n_blocks, st);
  return launch<4>(p, n_blocks, st);
}

}  // namespace snapb200
