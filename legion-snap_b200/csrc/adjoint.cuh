// Adjoint (transposed) sweep: the reverse-direction wavefront of the discrete
// adjoint of the diamond-difference sweep, all octants and groups in one
// persistent launch.  No counterpart in the reference, which has no
// sensitivity capability; the forward operator it transposes is
// sweep.cc:354-591 (with the fixup of sweep.cc:425-518 frozen at the forward
// solution).
//
// Forward, per (octant, angle, cell), with p_d the face flags the cell-average
// flux was last computed with and h_d those of the outgoing faces (all 1
// unless the fixup cleared them; the fixup's count-based stop can leave them
// different):
//   pc = (psi + 1/2 sum_d c_d (1+p_d) psi_in_d) / (sigma_t + sum_d c_d p_d)
//   psi_out_d = h_d (2 pc - psi_in_d),   phi_k += ec[k][a] w[a] pc,
//   psi = sum_k ec[k][a] qtot_k.
// Adjoint, walked from the forward outflow corner back to the inflow corner
// (octant direction bits flipped), with adjoint faces bar_out_d arriving from
// the forward-downstream cells:
//   bar_pc  = w[a] sum_k ec[k][a] bar_phi_k                 (MMA chain 1)
//   s       = (bar_pc + 2 sum_d h_d bar_out_d) / den_p       (0 if pc was zeroed)
//   bar_in_d = 1/2 c_d (1+p_d) s - h_d bar_out_d             (sent upstream)
//   bar_qtot_k += sum_a ec[k][a] s                           (MMA chain 2)
//   bar_sigma_t -= s * pc                                    (needs the forward pc)
// The tile/queue/flag machinery is the forward kernel's (sweep.cuh).
#pragma once

#include "sweep.cuh"

namespace snapb200 {
namespace adj {

using sw::FULL;
using sw::Vec2;
using sw::cp_async16;
using sw::cp_async_commit;
using sw::cp_async_wait;
using sw::recip_rn;
using sw::div_rn;

template <typename T, int NT, int MK, int TY>
struct Shape {
  static constexpr int AP = 8 * NT;
  static constexpr int S2 = 2 * NT;
  static constexpr int MN = MK == 0 ? 0 : (MK + 1) / 2;
  static constexpr int B1 = MK * NT * 32;
  static constexpr int B2 = S2 * MN * 32;
  static constexpr int YRING = 2 * TY * 8 * AP;
  static constexpr int XST = 2 * TY * AP;
  static constexpr int YST = 2 * 8 * AP;
  static constexpr size_t SMEM_BYTES =
      sizeof(double) * (B1 + B2) + sizeof(T) * (4 * AP + YRING + XST + YST);
  // CTAs per SM the register budget is sized for: 3 (168 registers; no
  // spills in FP32, at most a few bytes in FP64 up to 5 angle tiles), 1 for
  // FP64 from 6 angle tiles up, where 168 registers would spill
  static constexpr int MIN_BLOCKS = TY == 8 || (sizeof(T) == 8 && NT >= 6) ? 1 : 3;
};

template <typename T, int NT, int MK, int TY>
__global__ void __launch_bounds__(TY * 32, (Shape<T, NT, MK, TY>::MIN_BLOCKS)) adjoint_kernel(const SweepParams p) {
  using S = Shape<T, NT, MK, TY>;
  using T2 = typename Vec2<T>::type;
  constexpr int AP = S::AP, S2 = S::S2, MN = S::MN;
  constexpr bool F32 = sizeof(T) == 4;
  extern __shared__ __align__(16) double smem[];
  double *sB1 = smem;               // ec*w in the source-expansion layout
  double *sB2 = sB1 + S::B1;        // ec in the accumulation layout
  T *sC = (T *)(sB2 + S::B2);
  T *sY = sC + 4 * AP;
  T *sXs = sY + S::YRING;
  T *sYs = sXs + S::XST;
  __shared__ int s_item, s_ok;

  const int tid = threadIdx.x, lane = tid & 31, j = tid >> 5;
  const int ci = lane >> 2, q = lane & 3;
  const long long C = (long long)p.nx * p.ny * p.nz;
  const long long plane = (long long)p.nx * p.ny;
  const int M = p.M;
  const int nsteps = p.nz + 7 + TY - 1;

  for (int i = tid; i < 4 * AP; i += blockDim.x) sC[i] = ((const T *)p.coef)[i];
  for (int i = tid; i < S::YRING; i += blockDim.x) sY[i] = T(0);
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
    // the walk runs against the octant's direction of travel
    const int od = o ^ 7;
    const bool sx = od & 1, sy = (od >> 1) & 1, sz = (od >> 2) & 1;
    const int lx = tx * 8 + ci, ly = ty * TY + j;
    const int gx = sx ? lx : p.nx - 1 - lx;
    const int gy = sy ? ly : p.ny - 1 - ly;
    const int up_x = tx > 0 ? p.item_index[(sweep * p.tiles_x + tx - 1) * p.tiles_y + ty] : -1;
    const int up_y = ty > 0 ? p.item_index[(sweep * p.tiles_x + tx) * p.tiles_y + ty - 1] : -1;
    const size_t bxs = (size_t)p.nz * TY * AP, bys = (size_t)p.nz * 8 * AP;
    const T *bx_in = up_x >= 0 ? (const T *)p.bx + (size_t)up_x * bxs : nullptr;
    const T *by_in = up_y >= 0 ? (const T *)p.by + (size_t)up_y * bys : nullptr;
    T *bx_out = (tx + 1 < p.tiles_x) ? (T *)p.bx + (size_t)item * bxs : nullptr;
    T *by_out = (ty + 1 < p.tiles_y) ? (T *)p.by + (size_t)item * bys : nullptr;
    const bool publish = bx_out || by_out;
    const T *phib = (const T *)p.qtot + (size_t)g * C * M;       // adjoint moment source
    const T *tg = (const T *)p.t_xs + (size_t)g * C;
    T *qbar = (T *)p.phi_slots + ((size_t)o_local * p.G + g) * C * M;
    T *sbar = p.sigt_bar_slots ? (T *)p.sigt_bar_slots + ((size_t)o_local * p.G + g) * C : nullptr;
    const T *pcs = (const T *)p.pc_store;
    const uint8_t *fls = p.flag_store;
    const long long col = (long long)gy * p.nx + gx;
    auto cell_of = [&](int k) -> long long { return (sz ? k : p.nz - 1 - k) * plane + col; };

    const bool copier = !F32 || (q & 1) == 0;
    auto prefetch = [&](int st) {
      const int buf = st & 1;
      if (ci == 0 && bx_in && copier) {
        const int k = st - j;
        if (k >= 0 && k < p.nz) {
          const T *src = bx_in + ((size_t)k * TY + j) * AP + 2 * q;
          T *dst = sXs + (buf * TY + j) * AP + 2 * q;
#pragma unroll
          for (int nt = 0; nt < NT; ++nt) cp_async16(dst + 8 * nt, src + 8 * nt);
        }
      }
      if (j == 0 && by_in && copier) {
        const int k = st - ci;
        if (k >= 0 && k < p.nz) {
          const T *src = by_in + ((size_t)k * 8 + ci) * AP + 2 * q;
          T *dst = sYs + (buf * 8 + ci) * AP + 2 * q;
#pragma unroll
          for (int nt = 0; nt < NT; ++nt) cp_async16(dst + 8 * nt, src + 8 * nt);
        }
      }
      cp_async_commit();
    };
    auto need_x = [&](int st) { return min(st + 8, nsteps); };
    auto need_y = [&](int st) { return min(st + TY, nsteps); };

    if (tid == 0) {
      bool ok = true;
      if (up_x >= 0) ok = bounded_wait_geq(p.progress + up_x, need_x(1), p.error, p.timeout_ns,
                                           DEV_ERR_TIMEOUT);
      if (ok && up_y >= 0) ok = bounded_wait_geq(p.progress + up_y, need_y(1), p.error,
                                                 p.timeout_ns, DEV_ERR_TIMEOUT);
      s_ok = ok;
    }
    __syncthreads();
    if (!s_ok) continue;
    prefetch(0);
    prefetch(1);

    T xf[S2], zf[S2], sv[S2];
#pragma unroll
    for (int t = 0; t < S2; ++t) xf[t] = zf[t] = sv[t] = T(0);
    T qa[MK > 0 ? MK : 1];
    T sig_n = T(1);
    auto load_src = [&](int k) {
      const bool a = (k >= 0) && (k < p.nz);
      const long long cell = a ? cell_of(k) : 0;
      sig_n = a ? __ldg(tg + cell) : T(1);
      if constexpr (MK == 0) {
        qa[0] = a ? __ldg(phib + cell) : T(0);
      } else {
#pragma unroll
        for (int kt = 0; kt < MK; ++kt) {
          const int m = q * MK + kt;
          qa[kt] = (a && m < M) ? __ldg(phib + cell * M + m) : T(0);
        }
      }
    };
    load_src(0 - ci - j);
    int poll_x = 0, poll_y = 0;

    for (int s = 0; s < nsteps; ++s) {
      const int k = s - ci - j;
      const bool act = (k >= 0) && (k < p.nz);
      const long long cell = act ? cell_of(k) : 0;
      const T sig = sig_n;
      // adjoint of the moment accumulation: bar_pc = w sum_k ec bar_phi
      if constexpr (MK == 0) {
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
          sv[2 * nt] = sC[3 * AP + 8 * nt + 2 * q] * qa[0];
          sv[2 * nt + 1] = sC[3 * AP + 8 * nt + 2 * q + 1] * qa[0];
        }
      } else {
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
          double c0 = 0.0, c1 = 0.0;
#pragma unroll
          for (int kt = 0; kt < MK; ++kt)
            dmma_8x8x4(c0, c1, (double)qa[kt], sB1[(kt * NT + nt) * 32 + lane]);
          sv[2 * nt] = (T)c0;
          sv[2 * nt + 1] = (T)c1;
        }
      }
      load_src(k + 1);
      if (tid == 0) {
        if (up_x >= 0) poll_x = ld_acquire_gpu(p.progress + up_x);
        if (up_y >= 0) poll_y = ld_acquire_gpu(p.progress + up_y);
      }
      cp_async_wait<1>();
      if constexpr (F32) __syncwarp();
      const T2 zero2 = {T(0), T(0)};
#pragma unroll
      for (int t = 0; t < S2; ++t) xf[t] = __shfl_up_sync(FULL, xf[t], 4);
      if (ci == 0) {
        const T *src = sXs + ((s & 1) * TY + j) * AP + 2 * q;
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
          const T2 v = (act && bx_in) ? *(const T2 *)(src + 8 * nt) : zero2;
          xf[2 * nt] = v.x;
          xf[2 * nt + 1] = v.y;
        }
      }
      const T *ysrc = nullptr;
      if (j > 0) ysrc = sY + ((((s - 1) & 1) * TY + (j - 1)) * 8 + ci) * AP;
      else if (by_in) ysrc = sYs + ((s & 1) * 8 + ci) * AP;
      const size_t sbase = (((size_t)o * p.G + g) * C + cell) * AP + 2 * q;

      T sig_acc = T(0);
#pragma unroll
      for (int nt = 0; nt < NT; ++nt) {
        const int a0 = 8 * nt + 2 * q;
        const T2 cx = *(const T2 *)(sC + a0);
        const T2 cy = *(const T2 *)(sC + AP + a0);
        const T2 cz = *(const T2 *)(sC + 2 * AP + a0);
        const T2 yv = (act && ysrc) ? *(const T2 *)(ysrc + a0) : zero2;
        T2 pcf = zero2;
        if (sbar && act) pcf = *(const T2 *)(pcs + sbase + 8 * nt);
        T ox[2], oy[2], oz[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int t = 2 * nt + h;
          const T ccx = h ? cx.y : cx.x, ccy = h ? cy.y : cy.x, ccz = h ? cz.y : cz.x;
          const T yb = h ? yv.y : yv.x;
          const unsigned f = (p.fixup && act) ? fls[sbase + 8 * nt + h] : 0x77u;
          T sbar_v;
          if ((f & 0x7fu) == 0x77u) {
            sbar_v = (sv[t] + T(2) * (xf[t] + yb + zf[t])) * recip_rn(((sig + ccx) + ccy) + ccz);
            ox[h] = ccx * sbar_v - xf[t];
            oy[h] = ccy * sbar_v - yb;
            oz[h] = ccz * sbar_v - zf[t];
          } else {
            const T fx = (f & 1u) ? T(1) : T(0), fy = (f & 2u) ? T(1) : T(0),
                    fz = (f & 4u) ? T(1) : T(0);
            const T kx = (f & 16u) ? T(1) : T(0), ky = (f & 32u) ? T(1) : T(0),
                    kz = (f & 64u) ? T(1) : T(0);
            const T P = sv[t] + T(2) * (fx * xf[t] + fy * yb + fz * zf[t]);
            sbar_v = (f & 8u) ? T(0) : div_rn(P, sig + ccx * kx + ccy * ky + ccz * kz);
            ox[h] = T(0.5) * ccx * (T(1) + kx) * sbar_v - fx * xf[t];
            oy[h] = T(0.5) * ccy * (T(1) + ky) * sbar_v - fy * yb;
            oz[h] = T(0.5) * ccz * (T(1) + kz) * sbar_v - fz * zf[t];
          }
          sv[t] = act ? sbar_v : T(0);
          sig_acc -= sv[t] * (h ? pcf.y : pcf.x);
          xf[t] = ox[h];
          if (act) zf[t] = oz[h];
        }
        const T2 oy2 = {oy[0], oy[1]}, ox2 = {ox[0], ox[1]};
        if (j + 1 < TY) {
          *(T2 *)(sY + (((s & 1) * TY + j) * 8 + ci) * AP + a0) = oy2;
        } else if (by_out && act) {
          __stcg((T2 *)(by_out + ((size_t)k * 8 + ci) * AP + a0), oy2);
        }
        if (ci == 7 && bx_out && act) __stcg((T2 *)(bx_out + ((size_t)k * TY + j) * AP + a0), ox2);
      }

      // adjoint of the angular source: bar_qtot_k = sum_a ec[k][a] s
      if constexpr (MK == 0) {
        T acc = T(0);
#pragma unroll
        for (int t = 0; t < S2; ++t) acc += sv[t];
        acc += __shfl_xor_sync(FULL, acc, 1);
        acc += __shfl_xor_sync(FULL, acc, 2);
        if (act && q == 0) qbar[cell] = p.accumulate ? qbar[cell] + acc : acc;
      } else {
#pragma unroll
        for (int mt = 0; mt < MN; ++mt) {
          double a0 = 0.0, a1 = 0.0, b0 = 0.0, b1 = 0.0;
#pragma unroll
          for (int t = 0; t < S2; t += 2) {
            dmma_8x8x4(a0, a1, (double)sv[t], sB2[(t * MN + mt) * 32 + lane]);
            dmma_8x8x4(b0, b1, (double)sv[t + 1], sB2[((t + 1) * MN + mt) * 32 + lane]);
          }
          if (act) {
            const int m = q * 2 * MN + 2 * mt;
            T *dst = qbar + cell * M + m;
            const T c0 = (T)(a0 + b0), c1 = (T)(a1 + b1);
            if (m < M) dst[0] = p.accumulate ? dst[0] + c0 : c0;
            if (m + 1 < M) dst[1] = p.accumulate ? dst[1] + c1 : c1;
          }
        }
      }
      if (sbar) {
        sig_acc += __shfl_xor_sync(FULL, sig_acc, 1);
        sig_acc += __shfl_xor_sync(FULL, sig_acc, 2);
        if (act && q == 0) sbar[cell] = p.accumulate ? sbar[cell] + sig_acc : sig_acc;
      }

      if (tid == 0) {
        bool ok = true;
        const int st2 = s + 2;
        if (st2 < nsteps) {
          if (up_x >= 0 && poll_x < need_x(st2))
            ok = bounded_wait_geq(p.progress + up_x, need_x(st2), p.error, p.timeout_ns,
                                  DEV_ERR_TIMEOUT);
          if (ok && up_y >= 0 && poll_y < need_y(st2))
            ok = bounded_wait_geq(p.progress + up_y, need_y(st2), p.error, p.timeout_ns,
                                  DEV_ERR_TIMEOUT);
        }
        s_ok = ok;
      }
      __syncthreads();
      if (!s_ok) break;
      if (tid == 0 && publish) st_release_gpu(p.progress + item, s + 1);
      if (s + 2 < nsteps) prefetch(s + 2);
      else cp_async_commit();
    }
    cp_async_wait<0>();
    __syncthreads();
  }
}

template <typename T, int NT, int MK>
cudaError_t dispatch_mk(int op, const SweepParams *p, int grid, cudaStream_t st, int *blocks,
                        size_t *smem) {
  constexpr int TY = 4;
  const size_t bytes = Shape<T, NT, MK, TY>::SMEM_BYTES;
  if (smem) *smem = bytes;
  if (op == 2) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(adjoint_kernel<T, NT, MK, TY>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e != cudaSuccess) return e;
  if (op == 1)
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, adjoint_kernel<T, NT, MK, TY>,
                                                         TY * 32, bytes);
  adjoint_kernel<T, NT, MK, TY><<<grid, TY * 32, bytes, st>>>(*p);
  return cudaGetLastError();
}

// op 0: launch, 1: occupancy, 2: shared memory bytes.  Tiles are 8 x 4.
template <typename T, int NT>
cudaError_t dispatch_nt(int mk, int op, const SweepParams *p, int grid, cudaStream_t st,
                        int *blocks, size_t *smem) {
  switch (mk) {
    case 0: return dispatch_mk<T, NT, 0>(op, p, grid, st, blocks, smem);
    case 1: return dispatch_mk<T, NT, 1>(op, p, grid, st, blocks, smem);
    case 2: return dispatch_mk<T, NT, 2>(op, p, grid, st, blocks, smem);
    case 3: return dispatch_mk<T, NT, 3>(op, p, grid, st, blocks, smem);
    case 4: return dispatch_mk<T, NT, 4>(op, p, grid, st, blocks, smem);
  }
  return cudaErrorInvalidValue;
}

}  // namespace adj
}  // namespace snapb200
