// FP64 persistent sweep kernel: all octants and groups of one inner iteration.
//
// Replaces the reference's MiniKBATask GPU path (sweep.cc:1550-1620 ->
// run_gpu_sweep, gpu_sweep.cu:1395-2008, 2047-2295), which launches one
// cooperative kernel per (octant, group) on its own stream with one CTA per
// wavefront cell and a software grid barrier between wavefronts.
//
// Decomposition here: a work item is (octant, group, column tile of 8 x TY
// cells in the xy plane); a CTA walks the tile's whole z column with a 3-D
// skewed diagonal, so at step s the cell (i, j, k) with i + j + k = s is
// processed.  Warp j owns tile row j; lane l = 4*i + q owns cell row i of the
// warp and the angles 8*nt + 2*q + {0,1}, which is the accumulator layout of
// the FP64 m8n8k4 tensor-core MMA, so
//   - the angular source psi = sum_m ec[m][a] qtot[m] is one MMA chain with
//     the qtot of the warp's 8 cells as the A operand (sweep.cc:354-366), and
//   - the moment accumulation phi[m] += sum_a ec[m][a] w[a] pc[a] is a second
//     MMA chain that takes the diamond-difference result straight from the
//     accumulator registers as its A operand (sweep.cc:565-591).
// The x face moves one cell row per step by a lane shuffle, the z face stays
// in the lane's registers for the whole column, the y face passes between
// warps through shared memory.  Faces crossing a tile edge go through global
// memory (L2) with a device-scope progress counter per tile, published with a
// release store and awaited with a bounded acquire spin.  Work items are
// taken from a queue in an order where every item's upstream neighbours come
// first, so a running item only ever waits on items that are already running
// or done.  Each octant writes its own flux slot (no atomics; the octant sum
// is a separate deterministic reduction).
#include "device_util.cuh"
#include "internal.h"

namespace snapb200 {
namespace {

constexpr unsigned FULL = 0xffffffffu;

template <int NT, int MK, int TY>
struct Fp64Shape {
  static constexpr int AP = 8 * NT;            // padded angles
  static constexpr int S2 = 2 * NT;            // angle slots per lane
  static constexpr int MN = MK == 0 ? 0 : (MK + 1) / 2;
  static constexpr int B1 = MK * NT * 32;      // source fragments
  static constexpr int B2 = S2 * MN * 32;      // accumulation fragments
  static constexpr int SMEM_DOUBLES = B1 + B2 + 4 * AP + 2 * TY * 8 * AP;
};

// Diamond difference for one (cell, angle): sweep.cc:377-423 with the
// geometry parameter of expxs.cc:374-379 recomputed in place.
__device__ __forceinline__ double dd_fp64(double psi, double x, double y, double z, double cx,
                                          double cy, double cz, double sig) {
  const double den = ((sig + cx) + cy) + cz;
  const double dinv = 1.0 / den;
  double v = psi;
  v += x * cx;
  v += y * cy;
  v += z * cz;
  return v * dinv;
}

template <int NT, int MK, int TY>
__global__ void __launch_bounds__(TY * 32)
    sweep_fp64_kernel(const SweepParams p) {
  using S = Fp64Shape<NT, MK, TY>;
  constexpr int AP = S::AP, S2 = S::S2, MN = S::MN;
  extern __shared__ __align__(16) double smem[];
  double *sB1 = smem;
  double *sB2 = sB1 + S::B1;
  double *sC = sB2 + S::B2;        // [4][AP]: cx, cy, cz, w
  double *sY = sC + 4 * AP;        // [2][TY][8][AP] y faces between warps
  __shared__ int s_item, s_ok;

  const int tid = threadIdx.x, lane = tid & 31, j = tid >> 5;
  const int ci = lane >> 2, q = lane & 3;
  const long long C = (long long)p.nx * p.ny * p.nz;
  const int M = p.M;
  const int nsteps = p.nz + 7 + TY - 1;

  for (int i = tid; i < 4 * AP; i += blockDim.x) sC[i] = ((const double *)p.coef)[i];
  for (int i = tid; i < 2 * TY * 8 * AP; i += blockDim.x) sY[i] = 0.0;
  int cur_oct = -1;

  for (;;) {
    if (tid == 0) s_item = ld_volatile(p.error) ? -1 : atomicAdd(p.counter, 1);
    __syncthreads();
    const int item = s_item;
    if (item < 0 || item >= p.n_items) break;
    const int packed = p.item_table[item];
    const int sweep = packed >> 16, tx = (packed >> 8) & 255, ty = packed & 255;
    const int o_local = sweep / p.G, g = sweep - o_local * p.G;
    const int o = p.o_base + o_local;
    if (MK > 0 && o != cur_oct) {
      const double *b1 = (const double *)p.bt1 + (size_t)o * S::B1;
      const double *b2 = (const double *)p.bt2 + (size_t)o * S::B2;
      for (int i = tid; i < S::B1; i += blockDim.x) sB1[i] = b1[i];
      for (int i = tid; i < S::B2; i += blockDim.x) sB2[i] = b2[i];
      cur_oct = o;
    }
    const bool sx = o & 1, sy = (o >> 1) & 1, sz = (o >> 2) & 1;
    const int lx = tx * 8 + ci, ly = ty * TY + j;
    const int gx = sx ? lx : p.nx - 1 - lx;
    const int gy = sy ? ly : p.ny - 1 - ly;
    const int up_x = tx > 0 ? p.item_index[(sweep * p.tiles_x + tx - 1) * p.tiles_y + ty] : -1;
    const int up_y = ty > 0 ? p.item_index[(sweep * p.tiles_x + tx) * p.tiles_y + ty - 1] : -1;
    const size_t bxs = (size_t)p.nz * TY * AP, bys = (size_t)p.nz * 8 * AP;
    const double *bx_in = up_x >= 0 ? (const double *)p.bx + (size_t)up_x * bxs : nullptr;
    const double *by_in = up_y >= 0 ? (const double *)p.by + (size_t)up_y * bys : nullptr;
    double *bx_out = (tx + 1 < p.tiles_x) ? (double *)p.bx + (size_t)item * bxs : nullptr;
    double *by_out = (ty + 1 < p.tiles_y) ? (double *)p.by + (size_t)item * bys : nullptr;
    const double *qg = (const double *)p.qtot + (size_t)g * C * M;
    const double *tg = (const double *)p.t_xs + (size_t)g * C;
    double *phi = (double *)p.phi_slots + ((size_t)o_local * p.G + g) * C * M;

    double xf[S2], zf[S2], pc[S2];
#pragma unroll
    for (int t = 0; t < S2; ++t) xf[t] = zf[t] = pc[t] = 0.0;

    for (int s = 0; s < nsteps; ++s) {
      if (tid == 0) {
        bool ok = true;
        if (up_x >= 0)
          ok = bounded_wait_geq(p.progress + up_x, min(s + 8, nsteps), p.error, p.timeout_ns,
                                DEV_ERR_TIMEOUT);
        if (ok && up_y >= 0)
          ok = bounded_wait_geq(p.progress + up_y, min(s + TY, nsteps), p.error, p.timeout_ns,
                                DEV_ERR_TIMEOUT);
        s_ok = ok;
      }
      __syncthreads();
      if (!s_ok) break;

      const int k = s - ci - j;
      const bool act = (k >= 0) && (k < p.nz);
      // incoming x face: the outgoing face of cell row ci-1 at step s-1
#pragma unroll
      for (int t = 0; t < S2; ++t) xf[t] = __shfl_up_sync(FULL, xf[t], 4);
      if (ci == 0) {
        if (act && bx_in) {
          const double *src = bx_in + ((size_t)k * TY + j) * AP + 2 * q;
#pragma unroll
          for (int nt = 0; nt < NT; ++nt) {
            const double2 v = __ldcg((const double2 *)(src + 8 * nt));
            xf[2 * nt] = v.x;
            xf[2 * nt + 1] = v.y;
          }
        } else {
#pragma unroll
          for (int t = 0; t < S2; ++t) xf[t] = 0.0;
        }
      }
      const int gz = sz ? k : p.nz - 1 - k;
      const long long cell = act ? ((long long)gz * p.ny + gy) * p.nx + gx : 0;
      const double sig = act ? tg[cell] : 1.0;

      // angular source (tensor cores when there are higher moments)
      if constexpr (MK == 0) {
        const double q0 = act ? qg[cell] : 0.0;
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
          pc[2 * nt] = (8 * nt + 2 * q < p.A) ? q0 : 0.0;
          pc[2 * nt + 1] = (8 * nt + 2 * q + 1 < p.A) ? q0 : 0.0;
        }
      } else {
        double qa[MK];
        bool loaded = false;
        if constexpr (MK == 4) {
          if (M == 16) {  // lane q holds moments 4q..4q+3: two 16-byte loads
            const double2 *src = (const double2 *)(qg + cell * 16 + 4 * q);
            const double2 v0 = act ? __ldg(src) : make_double2(0.0, 0.0);
            const double2 v1 = act ? __ldg(src + 1) : make_double2(0.0, 0.0);
            qa[0] = v0.x;
            qa[1] = v0.y;
            qa[2] = v1.x;
            qa[3] = v1.y;
            loaded = true;
          }
        }
        if (!loaded) {
#pragma unroll
          for (int kt = 0; kt < MK; ++kt) {
            const int m = q * MK + kt;
            qa[kt] = (act && m < M) ? __ldg(qg + cell * M + m) : 0.0;
          }
        }
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
          double c0 = 0.0, c1 = 0.0;
#pragma unroll
          for (int kt = 0; kt < MK; ++kt) dmma_8x8x4(c0, c1, qa[kt], sB1[(kt * NT + nt) * 32 + lane]);
          pc[2 * nt] = c0;
          pc[2 * nt + 1] = c1;
        }
      }

      // incoming y face
      const double *ysrc = nullptr;
      bool y_global = false;
      if (j > 0) {
        ysrc = sY + ((((s - 1) & 1) * TY + (j - 1)) * 8 + ci) * AP;
      } else if (act && by_in) {
        ysrc = by_in + ((size_t)k * 8 + ci) * AP;
        y_global = true;
      }
      auto load_y = [&](int a0) -> double2 {
        if (!act || !ysrc) return make_double2(0.0, 0.0);
        return y_global ? __ldcg((const double2 *)(ysrc + a0)) : *(const double2 *)(ysrc + a0);
      };

      // diamond difference
      int neg = 0;
#pragma unroll
      for (int nt = 0; nt < NT; ++nt) {
        const int a0 = 8 * nt + 2 * q;
        const double2 cx = *(const double2 *)(sC + a0);
        const double2 cy = *(const double2 *)(sC + AP + a0);
        const double2 cz = *(const double2 *)(sC + 2 * AP + a0);
        const double2 yv = load_y(a0);
        pc[2 * nt] = dd_fp64(pc[2 * nt], xf[2 * nt], yv.x, zf[2 * nt], cx.x, cy.x, cz.x, sig);
        pc[2 * nt + 1] =
            dd_fp64(pc[2 * nt + 1], xf[2 * nt + 1], yv.y, zf[2 * nt + 1], cx.y, cy.y, cz.y, sig);
        if (p.fixup) {
          neg += (2.0 * pc[2 * nt] - xf[2 * nt] < 0.0) + (2.0 * pc[2 * nt] - yv.x < 0.0) +
                 (2.0 * pc[2 * nt] - zf[2 * nt] < 0.0);
          neg += (2.0 * pc[2 * nt + 1] - xf[2 * nt + 1] < 0.0) +
                 (2.0 * pc[2 * nt + 1] - yv.y < 0.0) + (2.0 * pc[2 * nt + 1] - zf[2 * nt + 1] < 0.0);
        }
      }

      // negative-flux fixup (sweep.cc:425-518): a cell-wide count over all of
      // its angles and faces, iterated until the count stops changing.  The
      // four lanes of a cell vote through shuffles; the loop is warp-uniform.
      unsigned hx = ~0u, hy = ~0u, hz = ~0u;
      bool fixed = false;
      if (p.fixup) {
        int cellneg = neg + __shfl_xor_sync(FULL, neg, 1);
        cellneg += __shfl_xor_sync(FULL, cellneg, 2);
        const bool cell_fix = act && cellneg > 0;
        if (__any_sync(FULL, cell_fix)) {
          fixed = true;
          double psi[S2];
#pragma unroll
          for (int nt = 0; nt < NT; ++nt)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              const int a = 8 * nt + 2 * q + h;
              double v = 0.0;
              if (act && a < p.A) {
                if constexpr (MK == 0) {
                  v = qg[cell];
                } else {
                  for (int m = 0; m < M; ++m) {
                    const double e = sB1[((m % MK) * NT + nt) * 32 + 4 * (2 * q + h) + m / MK];
                    v += e * qg[cell * M + m];
                  }
                }
              }
              psi[2 * nt + h] = v;
            }
          bool done = !cell_fix;
          int old = 0;
          for (int iter = 0; iter < 6 * S2 * 4 + 8; ++iter) {
            int cnt = 0;
            if (!done) {
#pragma unroll
              for (int nt = 0; nt < NT; ++nt) {
                const double2 yv = load_y(8 * nt + 2 * q);
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                  const int t = 2 * nt + h;
                  const double yy = h ? yv.y : yv.x;
                  if (2.0 * pc[t] - xf[t] < 0.0) { hx &= ~(1u << t); ++cnt; }
                  if (2.0 * pc[t] - yy < 0.0) { hy &= ~(1u << t); ++cnt; }
                  if (2.0 * pc[t] - zf[t] < 0.0) { hz &= ~(1u << t); ++cnt; }
                }
              }
            }
            cnt += __shfl_xor_sync(FULL, cnt, 1);
            cnt += __shfl_xor_sync(FULL, cnt, 2);
            if (!done) {
              if (cnt == old) done = true;
              else old = cnt;
            }
            if (__all_sync(FULL, done)) break;
            if (!done) {
#pragma unroll
              for (int nt = 0; nt < NT; ++nt) {
                const int a0 = 8 * nt + 2 * q;
                const double2 yv = load_y(a0);
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                  const int t = 2 * nt + h;
                  const double cx = sC[a0 + h], cy = sC[AP + a0 + h], cz = sC[2 * AP + a0 + h];
                  const double fx = (hx >> t) & 1 ? 1.0 : 0.0;
                  const double fy = (hy >> t) & 1 ? 1.0 : 0.0;
                  const double fz = (hz >> t) & 1 ? 1.0 : 0.0;
                  const double yy = h ? yv.y : yv.x;
                  const double v = psi[t] + 0.5 * (xf[t] * cx * (1.0 + fx) + yy * cy * (1.0 + fy) +
                                                   zf[t] * cz * (1.0 + fz));
                  const double den = (v <= 0.0) ? 0.0 : (sig + cx * fx + cy * fy + cz * fz);
                  pc[t] = (den < 1.0e-12) ? 0.0 : v / den;
                }
              }
            }
          }
        }
      }

      // outgoing faces
#pragma unroll
      for (int nt = 0; nt < NT; ++nt) {
        const int a0 = 8 * nt + 2 * q;
        const double2 yv = load_y(a0);
        double ox[2], oy[2], oz[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int t = 2 * nt + h;
          const double yy = h ? yv.y : yv.x;
          ox[h] = 2.0 * pc[t] - xf[t];
          oy[h] = 2.0 * pc[t] - yy;
          oz[h] = 2.0 * pc[t] - zf[t];
          if (fixed) {
            ox[h] *= (hx >> t) & 1 ? 1.0 : 0.0;
            oy[h] *= (hy >> t) & 1 ? 1.0 : 0.0;
            oz[h] *= (hz >> t) & 1 ? 1.0 : 0.0;
          }
          xf[t] = ox[h];
          if (act) zf[t] = oz[h];
        }
        if (j + 1 < TY) {
          *(double2 *)(sY + (((s & 1) * TY + j) * 8 + ci) * AP + a0) = make_double2(oy[0], oy[1]);
        } else if (by_out && act) {
          __stcg((double2 *)(by_out + ((size_t)k * 8 + ci) * AP + a0), make_double2(oy[0], oy[1]));
        }
        if (ci == 7 && bx_out && act)
          __stcg((double2 *)(bx_out + ((size_t)k * TY + j) * AP + a0), make_double2(ox[0], ox[1]));
      }

      // flux moments of this octant
      if constexpr (MK == 0) {
        double acc = 0.0;
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
          acc += sC[3 * AP + 8 * nt + 2 * q] * pc[2 * nt];
          acc += sC[3 * AP + 8 * nt + 2 * q + 1] * pc[2 * nt + 1];
        }
        acc += __shfl_xor_sync(FULL, acc, 1);
        acc += __shfl_xor_sync(FULL, acc, 2);
        if (act && q == 0) phi[cell] = p.accumulate ? phi[cell] + acc : acc;
      } else {
#pragma unroll
        for (int mt = 0; mt < MN; ++mt) {
          double c0 = 0.0, c1 = 0.0;
#pragma unroll
          for (int t = 0; t < S2; ++t) dmma_8x8x4(c0, c1, pc[t], sB2[(t * MN + mt) * 32 + lane]);
          if (act) {
            const int m = q * 2 * MN + 2 * mt;
            double *dst = phi + cell * M + m;
            if (m < M) dst[0] = p.accumulate ? dst[0] + c0 : c0;
            if (m + 1 < M) dst[1] = p.accumulate ? dst[1] + c1 : c1;
          }
        }
      }

      __syncthreads();
      if (tid == 0 && (bx_out || by_out)) {
        __threadfence();
        st_release_gpu(p.progress + item, s + 1);
      }
    }
    __syncthreads();
  }
}

template <int NT, int MK, int TY>
size_t smem_bytes_t() {
  return sizeof(double) * Fp64Shape<NT, MK, TY>::SMEM_DOUBLES;
}

template <int NT, int MK, int TY>
cudaError_t launch_t(const SweepParams &p, int grid, cudaStream_t st) {
  const size_t smem = smem_bytes_t<NT, MK, TY>();
  cudaError_t e = cudaFuncSetAttribute(sweep_fp64_kernel<NT, MK, TY>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  sweep_fp64_kernel<NT, MK, TY><<<grid, TY * 32, smem, st>>>(p);
  return cudaGetLastError();
}

template <int NT, int MK, int TY>
cudaError_t occupancy_t(int *blocks, size_t *smem) {
  *smem = smem_bytes_t<NT, MK, TY>();
  cudaError_t e = cudaFuncSetAttribute(sweep_fp64_kernel<NT, MK, TY>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)*smem);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, sweep_fp64_kernel<NT, MK, TY>,
                                                       TY * 32, *smem);
}

// Dispatch table over the compiled shapes: NT in {1..8}, MK in {0..4}, TY = 8.
template <int TY>
struct Dispatch {
  template <int NT, int MK>
  static cudaError_t go(int nt, int mk, int op, const SweepParams *p, int grid, cudaStream_t st,
                        int *blocks, size_t *smem) {
    if (nt == NT && mk == MK) {
      if (op == 0) return launch_t<NT, MK, TY>(*p, grid, st);
      if (op == 1) return occupancy_t<NT, MK, TY>(blocks, smem);
      *smem = smem_bytes_t<NT, MK, TY>();
      return cudaSuccess;
    }
    if constexpr (MK < 4) {
      return go<NT, MK + 1>(nt, mk, op, p, grid, st, blocks, smem);
    } else if constexpr (NT < 8) {
      return go<NT + 1, 0>(nt, mk, op, p, grid, st, blocks, smem);
    } else {
      return cudaErrorInvalidValue;
    }
  }
};

cudaError_t dispatch(const SweepShape &sh, int op, const SweepParams *p, int grid,
                     cudaStream_t st, int *blocks, size_t *smem) {
  if (sh.TY != 8 || sh.NT < 1 || sh.NT > 8 || sh.MK < 0 || sh.MK > 4)
    return cudaErrorInvalidValue;
  return Dispatch<8>::go<1, 0>(sh.NT, sh.MK, op, p, grid, st, blocks, smem);
}

}  // namespace

bool sweep_fp64_supported(const SweepShape &sh) {
  return sh.TY == 8 && sh.NT >= 1 && sh.NT <= 8 && sh.MK >= 0 && sh.MK <= 4;
}

cudaError_t launch_sweep_fp64(const SweepShape &sh, const SweepParams &p, int grid,
                              cudaStream_t st) {
  return dispatch(sh, 0, &p, grid, st, nullptr, nullptr);
}

cudaError_t sweep_fp64_occupancy(const SweepShape &sh, int *blocks_per_sm, size_t *smem) {
  return dispatch(sh, 1, nullptr, 0, nullptr, blocks_per_sm, smem);
}

size_t sweep_fp64_smem(const SweepShape &sh) {
  size_t smem = 0;
  dispatch(sh, 2, nullptr, 0, nullptr, nullptr, &smem);
  return smem;
}

}  // namespace snapb200
