// FP32 sweep kernel with the moment contractions on the TF32 tensor cores.
//
// Same path and same synchronisation as sweep_kernel (sweep.cuh; reference:
// MiniKBATask, sweep.cc:354-591, run_gpu_sweep, gpu_sweep.cu:1395-2008), but a
// work item is (octant, pair of energy groups, 8 x 4-cell column tile) and the
// warp computes both groups of the pair at once.  Both groups see the same
// geometry, octant and angles, so they share every index, every fragment
// table and every wavefront step; only the data differ.  That fills the
// 16-row operand of the m16n8k8 TF32 MMA: row g is (cell g, first group),
// row g + 8 is (cell g, second group).  Lane l = 4*g + t owns cell row g of
// the warp and the angles 8*nt + 2*t + {0,1} of both groups -- the MMA's
// accumulator layout -- so
//   - the angular source psi[r][a] = sum_m qtot[r][m] ec[m][a] takes the
//     moments of row r as the A operand (the k index runs over the moments in
//     the order 2t, 2t+1 within each k-tile of 8, which makes a lane's A
//     elements adjacent in memory), and
//   - the moment accumulation phi[r][m] = sum_a pc[r][a] (ec w)[a][m] takes the
//     diamond-difference result straight from the accumulator registers as its
//     A operand (the k index runs over the angles in the order 2t, 2t+1, which
//     is exactly where the accumulator holds them).
// TF32 keeps 10 mantissa bits, so every contraction is split (Dekker-style):
// x = x_hi + x_lo with x_hi the TF32 rounding of x, and a*b is accumulated as
// a_lo*b_hi + a_hi*b_lo + a_hi*b_hi in FP32, which leaves an error of order
// 2^-22 relative (the dropped a_lo*b_lo term and FP32 accumulation).  The
// fragment tables are split on the host; the per-step operands are split in
// registers.
//
// The diamond difference, the negative-flux fixup and all stored data are in
// FP32; octant sums, sources and convergence tests stay in FP64 (outside).
// A group count that is odd gets a phantom second member in its last pair: it
// computes on the first member's data and stores nothing.
#pragma once

#include "sweep.cuh"

namespace snapb200 {
namespace tc {

using sw::FULL;
using sw::cp_async16;
using sw::cp_async_commit;
using sw::cp_async_wait;
using sw::ld_acquire_cta;
using sw::st_release_cta;
using sw::cta_wait_value_geq;

// x rounded to TF32 (10 explicit mantissa bits, round to nearest, ties away)
__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}
// split x = hi + lo, both TF32 (x - hi is exact in FP32)
__device__ __forceinline__ void split_tf32(float x, uint32_t &hi, uint32_t &lo) {
  hi = to_tf32(x);
  lo = to_tf32(x - __uint_as_float(hi));
}

// D(16x8) += A(16x8, row) * B(8x8, col), TF32 inputs, FP32 accumulation.
// Lane l = 4g + t: A = {[g][t], [g+8][t], [g][t+4], [g+8][t+4]},
// B = {[t][g], [t+4][g]}, D = {[g][2t], [g][2t+1], [g+8][2t], [g+8][2t+1]}.
__device__ __forceinline__ void mma_tf32(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2,
                                         uint32_t a3, uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}
// the three split products, small terms first
__device__ __forceinline__ void mma_split(float (&d)[4], const uint32_t (&ah)[4],
                                          const uint32_t (&al)[4], uint4 b) {
  mma_tf32(d, al[0], al[1], al[2], al[3], b.x, b.y);
  mma_tf32(d, ah[0], ah[1], ah[2], ah[3], b.z, b.w);
  mma_tf32(d, ah[0], ah[1], ah[2], ah[3], b.x, b.y);
}

// NT angle tiles of 8; KT moment tiles of 8 (0: single moment, no MMA).
template <int NT, int KT>
struct Shape {
  static constexpr int TY = 4;                 // warps per CTA = tile rows
  static constexpr int AP = 8 * NT;            // padded angles
  static constexpr int S2 = 2 * NT;            // angle slots per lane and group
  static constexpr int F1 = KT * NT * 32;      // source fragments (uint4: hi0, hi1, lo0, lo1)
  static constexpr int F2 = NT * KT * 32;      // accumulation fragments
  static constexpr int R = 2;                  // y-face ring depth (steps)
  static constexpr int YRING = R * TY * 8 * 2 * AP;   // y faces between warps
  static constexpr int PSI = TY * 2 * S2 * 32;        // angular source stash
  static constexpr int XST = 2 * TY * 2 * AP;         // staged x faces
  static constexpr int YST = 2 * 8 * 2 * AP;          // staged y faces
  static constexpr int NC = 5;                        // cx, cy, cz, w, cx+cy+cz
  static constexpr int ZR = AP;                       // a row of zero faces
  static constexpr size_t SMEM_BYTES =
      sizeof(uint4) * (F1 + F2) + sizeof(float) * (NC * AP + YRING + PSI + XST + YST + ZR);
  // 168 registers at 3 CTAs per SM; 7 or more angle tiles need 255 (2 CTAs)
#ifndef SNAP_SWEEP_TC32_BLOCKS
#define SNAP_SWEEP_TC32_BLOCKS 3
#endif
  static constexpr int MIN_BLOCKS = NT >= 7 ? 2 : SNAP_SWEEP_TC32_BLOCKS;
};

template <int NT, int KT>
__global__ void __launch_bounds__(128, (Shape<NT, KT>::MIN_BLOCKS))
    sweep_tc32_kernel(const SweepParams p) {
  using S = Shape<NT, KT>;
  constexpr int TY = S::TY, AP = S::AP, S2 = S::S2, R = S::R;
  extern __shared__ __align__(16) uint4 smem4[];
  uint4 *sF1 = smem4;                   // [KT][NT][32]
  uint4 *sF2 = sF1 + S::F1;             // [NT][KT][32]
  float *sC = (float *)(sF2 + S::F2);   // [5][AP]: cx, cy, cz, w, cx + cy + cz
  float *sY = sC + S::NC * AP;          // [R][TY][8][2][AP]
  float *sPsi = sY + S::YRING;          // [TY][2][S2][32]
  float *sXs = sPsi + S::PSI;           // [2][TY][2][AP]
  float *sYs = sXs + S::XST;            // [2][8][2][AP]
  float *sZero = sYs + S::YST;          // [AP] zeros
  __shared__ int s_item;
  __shared__ int s_full[TY];            // ring slots filled by warp j (its completed steps)
  __shared__ int s_used[TY];            // ring data of warp j-1 consumed by warp j

  const int tid = threadIdx.x, lane = tid & 31, j = tid >> 5;
  const int ci = lane >> 2, q = lane & 3;
  const long long C = (long long)p.nx * p.ny * p.nz;
  const long long plane = (long long)p.nx * p.ny;
  const int M = p.M;
  const int GP = (p.G + 1) >> 1;        // group pairs
  float *psi_stash = sPsi + j * 2 * S2 * 32 + lane;   // slot (u, t) at (u * S2 + t) * 32

  for (int i = tid; i < 4 * AP; i += blockDim.x) sC[i] = ((const float *)p.coef)[i];
  for (int i = tid; i < AP; i += blockDim.x) sZero[i] = 0.0f;
  __syncthreads();
  for (int i = tid; i < AP; i += blockDim.x)
    sC[4 * AP + i] = i < p.A ? (sC[i] + sC[AP + i]) + sC[2 * AP + i] : 1.0f;
  int cur_oct = -1;

  for (;;) {
    if (tid == 0) s_item = ld_volatile(p.error) ? -1 : atomicAdd(p.counter, 1);
    if (lane == 0) {
      s_full[j] = 0;
      s_used[j] = 0;
    }
    __syncthreads();
    const int item = s_item;
    if (item < 0 || item >= p.n_items) break;
    const int packed = p.item_table[item];
    const int sweep = packed >> 16, tx = (packed >> 8) & 255, ty = packed & 255;
    const int o_local = sweep / GP, gp = sweep - o_local * GP;
    const int o = p.o_base + o_local;
    const int g0 = 2 * gp;
    const bool has1 = g0 + 1 < p.G;      // a real second group (else a phantom copy of g0)
    const int g1 = has1 ? g0 + 1 : g0;
    if (KT > 0 && o != cur_oct) {
      const uint4 *f1 = (const uint4 *)p.bt1 + (size_t)o * S::F1;
      const uint4 *f2 = (const uint4 *)p.bt2 + (size_t)o * S::F2;
      for (int i = tid; i < S::F1; i += blockDim.x) sF1[i] = f1[i];
      for (int i = tid; i < S::F2; i += blockDim.x) sF2[i] = f2[i];
      cur_oct = o;
      __syncthreads();
    }
    const bool sx = o & 1, sy = (o >> 1) & 1, sz = (o >> 2) & 1;
    const int lx = tx * 8 + ci, ly = ty * TY + j;
    const int gx = sx ? lx : p.nx - 1 - lx;
    const int gy = sy ? ly : p.ny - 1 - ly;
    const int up_x = tx > 0 ? p.item_index[(sweep * p.tiles_x + tx - 1) * p.tiles_y + ty] : -1;
    const int up_y =
        (j == 0 && ty > 0) ? p.item_index[(sweep * p.tiles_x + tx) * p.tiles_y + ty - 1] : -1;
    const bool x_out = tx + 1 < p.tiles_x;
    const bool y_out = j == TY - 1 && ty + 1 < p.tiles_y;
    const size_t bxs = (size_t)p.nz * TY * 2 * AP, bys = (size_t)p.nz * 8 * 2 * AP;
    const float *bx_in = up_x >= 0 ? (const float *)p.bx + (size_t)up_x * bxs : nullptr;
    const float *by_in = up_y >= 0 ? (const float *)p.by + (size_t)up_y * bys : nullptr;
    const int *prog_x = up_x >= 0 ? p.progress + (size_t)up_x * TY + j : nullptr;
    const int *prog_y = up_y >= 0 ? p.progress + (size_t)up_y * TY + (TY - 1) : nullptr;
    float *bx_out = x_out ? (float *)p.bx + (size_t)item * bxs : nullptr;
    float *by_out = y_out ? (float *)p.by + (size_t)item * bys : nullptr;
    int *prog_out = (x_out || y_out) ? p.progress + (size_t)item * TY + j : nullptr;
    const float *qg0 = (const float *)p.qtot + (size_t)g0 * C * M;
    const float *qg1 = (const float *)p.qtot + (size_t)g1 * C * M;
    const float *tg0 = (const float *)p.t_xs + (size_t)g0 * C;
    const float *tg1 = (const float *)p.t_xs + (size_t)g1 * C;
    float *phi0 = (float *)p.phi_slots + ((size_t)o_local * p.G + g0) * C * M;
    float *phi1 = (float *)p.phi_slots + ((size_t)o_local * p.G + g1) * C * M;
    const long long col = (long long)gy * p.nx + gx;
    auto cell_of = [&](int k) -> long long { return (sz ? k : p.nz - 1 - k) * plane + col; };
    const int s_first = j, s_last = j + p.nz + 6;

    // prefetch of the tile-edge faces of step `st` (both groups; the even
    // lane of a lane pair copies 16 bytes = the angles of both lanes)
    const bool copier = (q & 1) == 0;
    int seen_x = 0, seen_y = 0;
    bool ok = true;
    auto prefetch = [&](int st) {
      const int buf = st & 1;
      if (ci == 0 && bx_in && copier) {
        const int k = st - j;
        if (k >= 0 && k < p.nz) {
          if (seen_x < st + 8) {
            seen_x = wait_value_geq(prog_x, st + 8, p.error, p.timeout_ns, DEV_ERR_TIMEOUT);
            ok = ok && seen_x >= st + 8;
          }
          const float *src = bx_in + ((size_t)k * TY + j) * 2 * AP + 2 * q;
          float *dst = sXs + (buf * TY + j) * 2 * AP + 2 * q;
          if (ok) {
#pragma unroll
            for (int i = 0; i < 2 * NT; ++i) cp_async16(dst + 8 * i, src + 8 * i);
          }
        }
      }
      if (by_in && copier) {
        const int k = st - ci;
        if (k >= 0 && k < p.nz) {
          if (seen_y < st + TY) {
            seen_y = wait_value_geq(prog_y, st + TY, p.error, p.timeout_ns, DEV_ERR_TIMEOUT);
            ok = ok && seen_y >= st + TY;
          }
          const float *src = by_in + ((size_t)k * 8 + ci) * 2 * AP + 2 * q;
          float *dst = sYs + (buf * 8 + ci) * 2 * AP + 2 * q;
          if (ok) {
#pragma unroll
            for (int i = 0; i < 2 * NT; ++i) cp_async16(dst + 8 * i, src + 8 * i);
          }
        }
      }
      cp_async_commit();
    };

    prefetch(s_first);
    prefetch(s_first + 1);

    float xf[2][S2], zf[2][S2], pc[2][S2];
#pragma unroll
    for (int u = 0; u < 2; ++u)
#pragma unroll
      for (int t = 0; t < S2; ++t) xf[u][t] = zf[u][t] = pc[u][t] = 0.0f;
    // source and sigma_t of the next step, loaded one step ahead:
    // qa[u][kt] = moments 8kt + 2q, 8kt + 2q + 1 of group u
    float2 qa[2][KT > 0 ? KT : 1];
    float sig_n[2] = {1.0f, 1.0f};
    auto load_src = [&](int k) {
      const bool a = (k >= 0) && (k < p.nz);
      const long long cell = a ? cell_of(k) : 0;
      sig_n[0] = a ? __ldg(tg0 + cell) : 1.0f;
      sig_n[1] = a ? __ldg(tg1 + cell) : 1.0f;
      if constexpr (KT == 0) {
        qa[0][0].x = a ? __ldg(qg0 + cell) : 0.0f;
        qa[1][0].x = a ? __ldg(qg1 + cell) : 0.0f;
      } else {
#pragma unroll
        for (int kt = 0; kt < KT; ++kt) {
          const int m = 8 * kt + 2 * q;
          if ((M & 1) == 0) {
            const bool in = a && m < M;   // M even: m < M implies m + 1 < M
            const float2 z2 = {0.0f, 0.0f};
            qa[0][kt] = in ? __ldg((const float2 *)(qg0 + cell * M + m)) : z2;
            qa[1][kt] = in ? __ldg((const float2 *)(qg1 + cell * M + m)) : z2;
          } else {
            qa[0][kt].x = (a && m < M) ? __ldg(qg0 + cell * M + m) : 0.0f;
            qa[0][kt].y = (a && m + 1 < M) ? __ldg(qg0 + cell * M + m + 1) : 0.0f;
            qa[1][kt].x = (a && m < M) ? __ldg(qg1 + cell * M + m) : 0.0f;
            qa[1][kt].y = (a && m + 1 < M) ? __ldg(qg1 + cell * M + m + 1) : 0.0f;
          }
        }
      }
    };
    load_src(s_first - ci - j);
    int seen_full = 0, seen_used = 0;
    if (__all_sync(FULL, ok)) {
      for (int s = s_first; s <= s_last; ++s) {
        const int k = s - ci - j;
        const bool act = (k >= 0) && (k < p.nz);
        const long long cell = act ? cell_of(k) : 0;
        const float sig[2] = {sig_n[0], sig_n[1]};
        // angular source of both groups (split-TF32 tensor cores)
        if constexpr (KT == 0) {
#pragma unroll
          for (int u = 0; u < 2; ++u)
#pragma unroll
            for (int t = 0; t < S2; ++t)
              pc[u][t] = (8 * (t >> 1) + 2 * q + (t & 1) < p.A) ? qa[u][0].x : 0.0f;
        } else {
          uint32_t ah[KT][4], al[KT][4];
#pragma unroll
          for (int kt = 0; kt < KT; ++kt) {
            split_tf32(qa[0][kt].x, ah[kt][0], al[kt][0]);
            split_tf32(qa[1][kt].x, ah[kt][1], al[kt][1]);
            split_tf32(qa[0][kt].y, ah[kt][2], al[kt][2]);
            split_tf32(qa[1][kt].y, ah[kt][3], al[kt][3]);
          }
#pragma unroll
          for (int nt = 0; nt < NT; ++nt) {
            float d[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
            for (int kt = 0; kt < KT; ++kt) mma_split(d, ah[kt], al[kt], sF1[(kt * NT + nt) * 32 + lane]);
            pc[0][2 * nt] = d[0];
            pc[0][2 * nt + 1] = d[1];
            pc[1][2 * nt] = d[2];
            pc[1][2 * nt + 1] = d[3];
          }
        }
        load_src(k + 1);
        if (p.fixup) {
#pragma unroll
          for (int u = 0; u < 2; ++u)
#pragma unroll
            for (int t = 0; t < S2; ++t) psi_stash[(u * S2 + t) * 32] = pc[u][t];
        }

        // y faces of step s-1 from warp j-1 (ring) or the staged tile edge
        if (j > 0 && seen_full < s) {
          seen_full = cta_wait_value_geq(&s_full[j - 1], s, p.error, p.timeout_ns);
          if (!__all_sync(FULL, seen_full >= s)) break;
        }
        cp_async_wait<1>();
        __syncwarp();   // staged data copied by the partner lane
        // x faces: row ci-1's outgoing faces of step s-1, or the staged edge
#pragma unroll
        for (int u = 0; u < 2; ++u)
#pragma unroll
          for (int t = 0; t < S2; ++t) xf[u][t] = __shfl_up_sync(FULL, xf[u][t], 4);
        if (ci == 0) {
          const bool xin = act && bx_in;   // else zeros: vacuum edge or inactive cell
          const float *src = (xin ? sXs + ((s & 1) * TY + j) * 2 * AP : sZero) + 2 * q;
          const int ustride = xin ? AP : 0;
#pragma unroll
          for (int u = 0; u < 2; ++u)
#pragma unroll
            for (int nt = 0; nt < NT; ++nt) {
              const float2 v = *(const float2 *)(src + u * ustride + 8 * nt);
              xf[u][2 * nt] = v.x;
              xf[u][2 * nt + 1] = v.y;
            }
        }
        const float *ysrc = nullptr;
        if (j > 0) ysrc = sY + ((((s - 1) % R) * TY + (j - 1)) * 8 + ci) * 2 * AP;
        else if (by_in) ysrc = sYs + ((s & 1) * 8 + ci) * 2 * AP;
        auto load_y = [&](int u, int a0) -> float2 {
          if (!act || !ysrc) return float2{0.0f, 0.0f};
          return *(const float2 *)(ysrc + u * AP + a0);
        };

        // diamond difference (expxs.cc:374-379, sweep.cc:377-423)
        bool neg = false;
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
          const int a0 = 8 * nt + 2 * q;
          const float2 cx = *(const float2 *)(sC + a0);
          const float2 cy = *(const float2 *)(sC + AP + a0);
          const float2 cz = *(const float2 *)(sC + 2 * AP + a0);
          const float2 cs = *(const float2 *)(sC + 4 * AP + a0);
#pragma unroll
          for (int u = 0; u < 2; ++u) {
            const float2 yv = load_y(u, a0);
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              const int t = 2 * nt + h;
              const float ccx = h ? cx.y : cx.x, ccy = h ? cy.y : cy.x, ccz = h ? cz.y : cz.x;
              const float yy = h ? yv.y : yv.x;
              const float dinv = sw::recip(sig[u] + (h ? cs.y : cs.x));
              float v = pc[u][t];
              v = __fmaf_rn(xf[u][t], ccx, v);
              v = __fmaf_rn(yy, ccy, v);
              v = __fmaf_rn(zf[u][t], ccz, v);
              v *= dinv;
              pc[u][t] = v;
              const float v2 = v + v;
              neg = neg | (v2 < xf[u][t]) | (v2 < yy) | (v2 < zf[u][t]);
            }
          }
        }

        // negative-flux fixup (sweep.cc:425-518), per group: per-face flags,
        // cell-wide count (four lanes vote), flagged angles recomputed until
        // the count stops changing; warp-uniform loop over both groups
        unsigned hx[2] = {~0u, ~0u}, hy[2] = {~0u, ~0u}, hz[2] = {~0u, ~0u}, hzero[2] = {0u, 0u};
        unsigned px[2] = {~0u, ~0u}, py[2] = {~0u, ~0u}, pz[2] = {~0u, ~0u};
        const bool fixed = p.fixup && __any_sync(FULL, act && neg);
        if (fixed) {
          int old[2];
          bool done[2];
#pragma unroll
          for (int u = 0; u < 2; ++u) {
            int cnt = 0;
#pragma unroll
            for (int nt = 0; nt < NT; ++nt) {
              const float2 yv = load_y(u, 8 * nt + 2 * q);
#pragma unroll
              for (int h = 0; h < 2; ++h) {
                const int t = 2 * nt + h;
                const float yy = h ? yv.y : yv.x;
                const float v2 = pc[u][t] + pc[u][t];
                if (v2 < xf[u][t]) { hx[u] &= ~(1u << t); ++cnt; }
                if (v2 < yy) { hy[u] &= ~(1u << t); ++cnt; }
                if (v2 < zf[u][t]) { hz[u] &= ~(1u << t); ++cnt; }
              }
            }
            cnt += __shfl_xor_sync(FULL, cnt, 1);
            cnt += __shfl_xor_sync(FULL, cnt, 2);
            done[u] = !(act && cnt > 0);
            old[u] = cnt;
          }
          for (int iter = 0; iter < 3 * S2 * 4 + 4; ++iter) {
#pragma unroll
            for (int u = 0; u < 2; ++u) {
              int c2 = 0;
              if (!done[u]) {
                px[u] = hx[u];
                py[u] = hy[u];
                pz[u] = hz[u];
#pragma unroll
                for (int nt = 0; nt < NT; ++nt) {
                  const int a0 = 8 * nt + 2 * q;
                  const float2 yv = load_y(u, a0);
#pragma unroll
                  for (int h = 0; h < 2; ++h) {
                    const int t = 2 * nt + h;
                    if (((hx[u] & hy[u] & hz[u]) >> t) & 1) continue;
                    const float ccx = sC[a0 + h], ccy = sC[AP + a0 + h], ccz = sC[2 * AP + a0 + h];
                    const bool fx = (hx[u] >> t) & 1, fy = (hy[u] >> t) & 1, fz = (hz[u] >> t) & 1;
                    const float yy = h ? yv.y : yv.x;
                    const float tx_ = xf[u][t] * ccx, ty_ = yy * ccy, tz_ = zf[u][t] * ccz;
                    const float v = psi_stash[(u * S2 + t) * 32] +
                                    0.5f * ((fx ? tx_ + tx_ : tx_) + (fy ? ty_ + ty_ : ty_) +
                                            (fz ? tz_ + tz_ : tz_));
                    const float den = (v <= 0.0f) ? 0.0f
                                                  : sig[u] + (fx ? ccx : 0.0f) + (fy ? ccy : 0.0f) +
                                                        (fz ? ccz : 0.0f);
                    const bool z = den < 1.0e-12f;
                    pc[u][t] = z ? 0.0f : sw::divide(v, den);
                    hzero[u] = z ? (hzero[u] | (1u << t)) : (hzero[u] & ~(1u << t));
                    const float v2 = pc[u][t] + pc[u][t];
                    if (v2 < xf[u][t]) hx[u] &= ~(1u << t);
                    if (v2 < yy) hy[u] &= ~(1u << t);
                    if (v2 < zf[u][t]) hz[u] &= ~(1u << t);
                    c2 += (int)(v2 < xf[u][t]) + (int)(v2 < yy) + (int)(v2 < zf[u][t]);
                  }
                }
              }
              c2 += __shfl_xor_sync(FULL, c2, 1);
              c2 += __shfl_xor_sync(FULL, c2, 2);
              if (!done[u]) {
                if (c2 == old[u]) done[u] = true;
                else old[u] = c2;
              }
            }
            if (__all_sync(FULL, done[0] && done[1])) break;
          }
        }

        // outgoing faces (after warp j+1 has consumed what the ring slot held)
        if (j + 1 < TY && s - R >= j && seen_used < s - R + 2) {
          seen_used = cta_wait_value_geq(&s_used[j + 1], s - R + 2, p.error, p.timeout_ns);
          if (!__all_sync(FULL, seen_used >= s - R + 2)) break;
        }
        float *yring = sY + (((s % R) * TY + j) * 8 + ci) * 2 * AP;
#pragma unroll
        for (int u = 0; u < 2; ++u)
#pragma unroll
          for (int nt = 0; nt < NT; ++nt) {
            const int a0 = 8 * nt + 2 * q;
            const float2 yv = load_y(u, a0);
            float ox[2], oy[2];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              const int t = 2 * nt + h;
              const float yy = h ? yv.y : yv.x;
              const float v2 = pc[u][t] + pc[u][t];
              ox[h] = v2 - xf[u][t];
              oy[h] = v2 - yy;
              float oz = v2 - zf[u][t];
              if (fixed) {
                // fx_hv * hv with hv in {0, 1} (sweep.cc:519-525)
                ox[h] *= (hx[u] >> t) & 1 ? 1.0f : 0.0f;
                oy[h] *= (hy[u] >> t) & 1 ? 1.0f : 0.0f;
                oz *= (hz[u] >> t) & 1 ? 1.0f : 0.0f;
              }
              xf[u][t] = ox[h];
              if (act) zf[u][t] = oz;
            }
            const float2 oy2 = {oy[0], oy[1]}, ox2 = {ox[0], ox[1]};
            if (j + 1 < TY) {
              *(float2 *)(yring + u * AP + a0) = oy2;
            } else if (by_out && act) {
              __stcg((float2 *)(by_out + ((size_t)k * 8 + ci) * 2 * AP + u * AP + a0), oy2);
            }
            if (ci == 7 && bx_out && act)
              __stcg((float2 *)(bx_out + ((size_t)k * TY + j) * 2 * AP + u * AP + a0), ox2);
          }
        __syncwarp();
        if (lane == 0) {
          if (j + 1 < TY) st_release_cta(&s_full[j], s + 1);
          if (j > 0) st_release_cta(&s_used[j], s + 1);
          if (prog_out && ((s - s_first + 1) % SNAP_SWEEP_PUBLISH_EVERY == 0 || s == s_last))
            st_release_gpu(prog_out, s + 1);
        }

        // forward state for the adjoint (cell-average flux and fixup flags)
        if (p.pc_store && act) {
#pragma unroll
          for (int u = 0; u < 2; ++u) {
            if (u == 1 && !has1) break;
            const size_t base =
                (((size_t)o * p.G + (u ? g1 : g0)) * C + cell) * AP + 2 * q;
            float *pcs = (float *)p.pc_store + base;
            uint8_t *fls = p.flag_store + base;
#pragma unroll
            for (int nt = 0; nt < NT; ++nt) {
              *(float2 *)(pcs + 8 * nt) = float2{pc[u][2 * nt], pc[u][2 * nt + 1]};
#pragma unroll
              for (int h = 0; h < 2; ++h) {
                const int t = 2 * nt + h;
                fls[8 * nt + h] =
                    (uint8_t)(((hx[u] >> t) & 1) | (((hy[u] >> t) & 1) << 1) |
                              (((hz[u] >> t) & 1) << 2) | (((hzero[u] >> t) & 1) << 3) |
                              (((px[u] >> t) & 1) << 4) | (((py[u] >> t) & 1) << 5) |
                              (((pz[u] >> t) & 1) << 6));
              }
            }
          }
        }

        // flux moments of this octant, both groups
        if constexpr (KT == 0) {
          float acc[2] = {0.0f, 0.0f};
#pragma unroll
          for (int u = 0; u < 2; ++u) {
#pragma unroll
            for (int nt = 0; nt < NT; ++nt) {
              acc[u] += sC[3 * AP + 8 * nt + 2 * q] * pc[u][2 * nt];
              acc[u] += sC[3 * AP + 8 * nt + 2 * q + 1] * pc[u][2 * nt + 1];
            }
            acc[u] += __shfl_xor_sync(FULL, acc[u], 1);
            acc[u] += __shfl_xor_sync(FULL, acc[u], 2);
          }
          if (act && q == 0) {
            phi0[cell] = p.accumulate ? phi0[cell] + acc[0] : acc[0];
            if (has1) phi1[cell] = p.accumulate ? phi1[cell] + acc[1] : acc[1];
          }
        } else {
          float dm[KT][4];
#pragma unroll
          for (int mt = 0; mt < KT; ++mt) dm[mt][0] = dm[mt][1] = dm[mt][2] = dm[mt][3] = 0.0f;
#pragma unroll
          for (int nt = 0; nt < NT; ++nt) {
            uint32_t ph[4], pl[4];
            split_tf32(pc[0][2 * nt], ph[0], pl[0]);
            split_tf32(pc[1][2 * nt], ph[1], pl[1]);
            split_tf32(pc[0][2 * nt + 1], ph[2], pl[2]);
            split_tf32(pc[1][2 * nt + 1], ph[3], pl[3]);
#pragma unroll
            for (int mt = 0; mt < KT; ++mt) mma_split(dm[mt], ph, pl, sF2[(nt * KT + mt) * 32 + lane]);
          }
          if (act) {
#pragma unroll
            for (int mt = 0; mt < KT; ++mt) {
              const int m = 8 * mt + 2 * q;
              float *d0 = phi0 + cell * M + m;
              float *d1 = phi1 + cell * M + m;
              if (m < M) {
                d0[0] = p.accumulate ? d0[0] + dm[mt][0] : dm[mt][0];
                if (has1) d1[0] = p.accumulate ? d1[0] + dm[mt][2] : dm[mt][2];
              }
              if (m + 1 < M) {
                d0[1] = p.accumulate ? d0[1] + dm[mt][1] : dm[mt][1];
                if (has1) d1[1] = p.accumulate ? d1[1] + dm[mt][3] : dm[mt][3];
              }
            }
          }
        }

        // the staged edge faces of step s+2 (into the buffer read this step)
        __syncwarp();
        prefetch(s + 2);
        if (!__all_sync(FULL, ok)) break;
      }
    }
    cp_async_wait<0>();
    __syncthreads();
  }
}

template <int NT, int KT>
cudaError_t launch(const SweepParams &p, int grid, cudaStream_t st) {
  const size_t smem = Shape<NT, KT>::SMEM_BYTES;
  cudaError_t e = cudaFuncSetAttribute(sweep_tc32_kernel<NT, KT>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  sweep_tc32_kernel<NT, KT><<<grid, 128, smem, st>>>(p);
  return cudaGetLastError();
}

template <int NT, int KT>
cudaError_t occupancy(int *blocks, size_t *smem) {
  *smem = Shape<NT, KT>::SMEM_BYTES;
  cudaError_t e = cudaFuncSetAttribute(sweep_tc32_kernel<NT, KT>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)*smem);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, sweep_tc32_kernel<NT, KT>, 128,
                                                       *smem);
}

// op 0: launch, 1: occupancy, 2: shared memory bytes
template <int NT>
cudaError_t dispatch_nt(int kt, int op, const SweepParams *p, int grid, cudaStream_t st,
                        int *blocks, size_t *smem) {
#define SNAP_TC_CASE(KTV)                                                   \
  if (kt == KTV) {                                                          \
    if (op == 0) return launch<NT, KTV>(*p, grid, st);                      \
    if (op == 1) return occupancy<NT, KTV>(blocks, smem);                   \
    *smem = Shape<NT, KTV>::SMEM_BYTES;                                     \
    return cudaSuccess;                                                     \
  }
  SNAP_TC_CASE(0) SNAP_TC_CASE(1) SNAP_TC_CASE(2)
#undef SNAP_TC_CASE
  return cudaErrorInvalidValue;
}

}  // namespace tc

// one translation unit per pair of angle-tile counts; sweep_dispatch.cu picks
#define SNAP_TC_DECL(N)                                                                  \
  cudaError_t sweep_tc32_dispatch_nt##N(int, int, const SweepParams *, int, cudaStream_t, \
                                        int *, size_t *);
SNAP_TC_DECL(1) SNAP_TC_DECL(2) SNAP_TC_DECL(3) SNAP_TC_DECL(4)
SNAP_TC_DECL(5) SNAP_TC_DECL(6) SNAP_TC_DECL(7) SNAP_TC_DECL(8)
#undef SNAP_TC_DECL

}  // namespace snapb200
