// Internal declarations shared by the CUDA translation units of snap_b200.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "snap_b200.h"

namespace snapb200 {

// Order of the forward sweep's MMA operand tables (per octant; lane l of the
// m8n8k4 fragment).  Paired order (the FP64 sweep): for the source
// expansion, k-tile kt of angle tile nt, with an even k-tile count k-tiles
// 2i and 2i+1 of one angle tile are adjacent, so one 16-byte shared-memory
// load feeds two MMAs; for the moment accumulation, angle slot t and moment
// tile mt, the moment tiles of one slot are adjacent.  Otherwise (the FP32
// sweep, whose register budget keeps single loads) lane-minor.
__host__ __device__ inline int b1_slot(int kt, int nt, int l, int NT, int MK, bool paired) {
  return paired && MK % 2 == 0 ? (((kt >> 1) * NT + nt) * 32 + l) * 2 + (kt & 1)
                               : (kt * NT + nt) * 32 + l;
}
__host__ __device__ inline int b2_slot(int t, int mt, int l, int MN, bool paired) {
  return paired ? (t * 32 + l) * MN + mt : (t * MN + mt) * 32 + l;
}

// Parameters of one launch of the persistent sweep kernel.
struct SweepParams {
  int nx, ny, nz;
  int M;           // flux moments (cmom)
  int A;           // real angles per octant
  int G;           // groups
  int tiles_x, tiles_y;
  int n_items;     // work items of this launch
  int o_base;      // first octant of this launch
  int accumulate;  // add into the flux slots instead of storing
  int atomic_flux; // phi_slots is the FP64 flux [G][C][M]: every octant adds into it atomically
  int fixup;
  int withhold_item1;     // fault injection: work item + 1 whose warps never publish progress (0: none)
  int gchain = 1;  // groups per work item, walked as one chained z column (sweep kernel)
  long long timeout_ns;
  const int *item_table;  // item -> (sweep << 16) | (tx << 8) | ty; sweep = octant * chains + chain
  const int *item_index;  // [sweep][tx][ty] -> item
  const void *qtot;       // [G][C][M]
  const void *t_xs;       // [G][C]
  void *phi_slots;        // [octants per launch][G][C][M]
  void *bx;               // [item][nz][TY][AP] x-faces leaving a tile
  void *by;               // [item][nz][8][AP]  y-faces leaving a tile
  int *progress;          // completed steps: [item][TY] (forward sweep), [item] (adjoint)
  int *counter;           // work-queue head
  int *error;             // device error word
  const void *bt1;        // [8][MK][NT][32] source-expansion fragments
  const void *bt2;        // [8][2NT][MN][32] moment-accumulation fragments
  const void *coef;       // [4][AP]: hi*mu, hj*eta, hk*xi, w
  // Optional forward-state store for the adjoint (null when not wanted):
  // cell-average angular flux and fixup flags of every (octant, group, cell,
  // padded angle): bits 0-2 = outgoing face x, y, z kept, bit 3 = flux forced
  // to 0, bits 4-6 = faces kept in the last recompute of the flux.
  void *pc_store;         // [8][G][C][AP]
  uint8_t *flag_store;    // [8][G][C][AP]
  // Adjoint sweep only: the adjoint of t_xs per octant slot, [P][G][C].
  void *sigt_bar_slots;
  // Time-dependent form only (FP64, one moment; null otherwise): vdelt [G]
  // and per (octant, group, cell, angle) the time-edge flux in and out and
  // the manufactured source (may be null), [8][G][C][A].
  const double *vdelt;
  const double *tf_in;
  double *tf_out;
  const double *qim;
};

// Parameters of the general sweep (sweep_wide.cu): one CTA per (octant,
// group), threads over angles, cells one at a time.  FP64 throughout.
struct WideParams {
  int nx, ny, nz;
  int A;            // angles per octant
  int M;            // flux moments (cmom)
  int G;            // groups
  int o_base;       // first octant of this launch (the grid covers octants o_base.. x G)
  int fixup;
  int td;           // time dependent: vdelt, tf_in and tf_out are used
  double hi, hj, hk;
  const double *mu, *eta, *xi, *w;   // [A]
  const double *ec;                  // [8][M][A]
  const double *qtot;                // [G][C][M]
  const double *t_xs;                // [G][C]
  const double *vdelt;               // [G]
  const double *tf_in;               // [8][G][C][A] angular flux at the start of the time step
  double *tf_out;                    // [8][G][C][A] angular flux at its end
  const double *qim;                 // [8][G][C][A] manufactured per-angle source, or null
  double *flux;                      // [G][C][M], every octant added atomically
  double *ypen;                      // scratch [blocks][nx][A]
  double *zpl;                       // scratch [blocks][ny*nx][A]
  // face planes of the wavefront form (sweep_wave.cu)
  double *wx;                        // scratch [blocks][ny*nz][A]
  double *wy;                        // scratch [blocks][nx*nz][A]
  double *wz;                        // scratch [blocks][nx*ny][A]
};
int wide_threads(int A);
size_t wide_smem_bytes(int A, int nx, int M);
bool wide_supported(int A, int nx, int M);
cudaError_t launch_sweep_wide(const WideParams &p, int n_blocks, cudaStream_t st);
// the wavefront form of the general sweep: up to 128 angles per octant
bool wave_supported(int A, int M);
size_t wave_scratch_doubles(int nx, int ny, int nz, int A, int blocks);
cudaError_t launch_sweep_wave(const WideParams &p, int n_blocks, cudaStream_t st);

// The manufactured-solution check (mms.cu).
struct MmsGeometry {
  int nx, ny, nz, A, G, nmat;
  int chunk[3];            // cells per spatial chunk along x, y, z
  double lx, ly, lz;
  int timedep;
  double tf, dt;
  const double *quad[3];   // host mu, eta, xi [A]
};
size_t mms_scratch_words(int nx, int ny, int nz, int A);
cudaError_t mms_init(const MmsGeometry &geo, const int32_t *mat, const double *sigt,
                     const double *slgg, double *ref, double *qim, double *qi, double *scratch,
                     cudaStream_t st);
// out = {max, min, sum} of |flux/ref - 1|; scratch: 3 words of device memory
cudaError_t mms_compare(const double *flux, int M, const double *ref, long long n, void *scratch,
                        double out[3], cudaStream_t st);

// Per-precision static configuration picked at context creation.
struct SweepShape {
  int NT;   // angle tiles of 8 (AP = 8*NT padded angles)
  int MK;   // source k-tiles of 4 moments (0: single moment)
  int MN;   // moment n-tiles of 8
  int TY;   // warps per CTA = tile rows in y
  int KT;   // moment tiles of 8 of the split-TF32 FP32 kernel (0: single moment)
};

// Records the message snap_last_error() returns; returns `code`.
int set_last_error(int code, const std::string &msg);

// Error codes written to the device error word.
enum : int { DEV_ERR_NONE = 0, DEV_ERR_TIMEOUT = 1 };

// sweep kernels (sweep_fp64.cu / sweep_fp32.cu)
// the time-dependent form of the tiled kernel (FP64, one moment: MK = 0)
cudaError_t launch_sweep_fp64_td(const SweepShape &sh, const SweepParams &p, int grid,
                                 cudaStream_t st);
cudaError_t sweep_fp64_td_occupancy(const SweepShape &sh, int *blocks_per_sm, size_t *smem);
cudaError_t launch_sweep_fp64(const SweepShape &sh, const SweepParams &p, int grid,
                              cudaStream_t st);
cudaError_t sweep_fp64_occupancy(const SweepShape &sh, int *blocks_per_sm, size_t *smem);
size_t sweep_fp64_smem(const SweepShape &sh);
bool sweep_fp64_supported(const SweepShape &sh);

cudaError_t launch_sweep_fp32(const SweepShape &sh, const SweepParams &p, int grid,
                              cudaStream_t st);
cudaError_t sweep_fp32_occupancy(const SweepShape &sh, int *blocks_per_sm, size_t *smem);
size_t sweep_fp32_smem(const SweepShape &sh);
bool sweep_fp32_supported(const SweepShape &sh);

// FP32 sweep on the TF32 tensor cores (sweep_tc.cuh): work items are
// (octant, group pair, tile), fragment tables from build_tc_tables
bool sweep_tc32_supported(const SweepShape &sh);
cudaError_t launch_sweep_tc32(const SweepShape &sh, const SweepParams &p, int grid,
                              cudaStream_t st);
cudaError_t sweep_tc32_occupancy(const SweepShape &sh, int *blocks_per_sm, size_t *smem);

// adjoint sweep kernels (adjoint_dispatch.cu); op 0 launch, 1 occupancy, 2 smem
bool adjoint_supported(const SweepShape &sh);
cudaError_t adjoint_dispatch(int fp32, const SweepShape &sh, int op, const SweepParams *p, int grid,
                             cudaStream_t st, int *blocks, size_t *smem);

// small kernels (kernels.cu)
cudaError_t k_expand_xs(const double *sig, const int32_t *mat, double *xs, int G, int nmat,
                        long long C, cudaStream_t st);
cudaError_t k_scale_xs(double *xs, const double *scale, int G, long long C, cudaStream_t st);
cudaError_t k_expand_scat(const double *slgg, const int32_t *mat, double *s_xs, int G, int nmat,
                          int nmom, long long C, cudaStream_t st);
// outer source of output groups g_lo .. g_lo+g_n-1 from the flux of G groups:
// the FP64 tensor-core form when `tab` (outer_dmma_table_words() doubles of
// scratch) is given and the shape fits, else the SIMT form; *launches = the
// kernels launched
size_t outer_dmma_table_words(int G, int g_n, int nmat, int nmom);
cudaError_t k_outer_source_groups(const double *qi, const double *slgg, const int32_t *mat,
                                  const double *flux, double *q2grp, double *tab, int G, int nmat,
                                  int nmom, int M, long long C, int g_lo, int g_n, int *launches,
                                  cudaStream_t st);
// outer source with the group-to-group contraction on the tcgen05 tensor
// cores, split BF16 operands (outer_tc.cu); `tab` holds
// outer_tc_table_words() 32-bit words of scratch; its waits record a timeout
// in *err after timeout_ns
size_t outer_tc_table_words(int G, int nmat, int nmom);
bool outer_tc_supported(int G, int nmat, int nmom);
// whether the plan batches 4 moments (32-byte runs per input line); with
// fewer the FP64 tensor-core form is the faster one
bool outer_tc_preferred(int G, int nmat, int nmom);
cudaError_t k_outer_source_tc(const double *qi, const double *slgg, const int32_t *mat,
                              const double *flux, double *q2grp, uint32_t *tab, int G, int nmat,
                              int nmom, int M, long long C, int *err, long long timeout_ns,
                              cudaStream_t st);
// qtot as k_inner_source, and in the same pass the old scalar flux saved to
// old0[g*C + c] and the flux moments cleared (for sweeps that add octants
// straight into the flux)
cudaError_t k_inner_source_save(const double *s_xs, const double *q2grp, double *flux, void *qtot,
                                int fp32, double *old0, int G, int nmom, int M, long long C,
                                cudaStream_t st);
// inner test of the new scalar flux flux[i*M] against old0[i]: violation
// count and the largest relative change (float bits)
cudaError_t k_test_change(const double *flux, const double *old0, int M, long long n, double epsi,
                          int *violations, unsigned *maxdf, cudaStream_t st);
cudaError_t k_inner_source(const double *s_xs, const double *q2grp, const double *flux,
                           void *qtot, int fp32, int G, int nmom, int M, long long C,
                           cudaStream_t st);
// flux = sum of `slots` partial slots; optionally counts convergence violations
// of the new scalar flux against the old one (read before it is overwritten)
// and records the largest relative change (float bits, atomicMax) in *maxdf.
cudaError_t k_reduce_slots(const void *slots, int nslots, int fp32, void *flux_out,
                           int out_fp32, double *flux64_out, int G, int M, long long C,
                           int test, double epsi, int *violations, cudaStream_t st,
                           unsigned *maxdf = nullptr);
cudaError_t k_count_violations(const double *flux, const double *prev, int M, long long n,
                               double epsi, int *violations, cudaStream_t st);
cudaError_t k_to_f32(const double *in, float *out, long long n, cudaStream_t st);
// x[i] *= f
cudaError_t k_scale(double *x, double f, size_t n, cudaStream_t st);
// phi_bar[g'][c][k] = r[g'][c] (k = 0) + sum_g slgg[g][mat][g'][l(k)] qbar[g][c][k]
cudaError_t k_adjoint_scatter(const double *r, const double *slgg, const int32_t *mat,
                              const double *qbar, double *phi_bar, int G, int nmat, int nmom,
                              int M, long long C, cudaStream_t st);
// phi_bar = r + S^T qbar in place (qbar and phi_bar float when fp32, else
// double), norm[0] = max |change|, norm[1] = max |phi_bar| (bit patterns;
// norm must start at zero)
cudaError_t k_adjoint_update(const double *r, const double *slgg, const int32_t *mat,
                             const void *qbar, void *phib, int fp32, unsigned long long *norm,
                             int G, int nmat, int nmom, int M, long long C, cudaStream_t st);
cudaError_t k_grad_sxs_any(const void *qbar, int fp32, const double *flux, double *grad, int G,
                           int nmom, int M, long long C, cudaStream_t st);
cudaError_t k_moment0_any(const void *in, int fp32, double *out, int M, long long n,
                          cudaStream_t st);
// grad[g][c][l] = sum_{k in band l} qbar[g][c][k] flux[g][c][k]
cudaError_t k_grad_sxs(const double *qbar, const double *flux, double *grad, int G, int nmom,
                       int M, long long C, cudaStream_t st);
// out[i] = in[i*M] (moment 0)
cudaError_t k_moment0(const double *in, double *out, int M, long long n, cudaStream_t st);
// out[0] = max |a - b|, out[1] = max |a| over n values (as ordered bit patterns
// of non-negative doubles, combined with atomicMax; out must start at zero)
cudaError_t k_max_abs_diff(const double *a, const double *b, long long n,
                           unsigned long long *out, cudaStream_t st);
cudaError_t k_copy_moment0(const double *flux, double *out, int M, long long n, cudaStream_t st);

}  // namespace snapb200
