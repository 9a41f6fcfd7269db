/*
 * snap_b200: B200-native (sm_100a) steady-state solve path of Legion-SNAP.
 *
 * A thin C ABI over hand-written CUDA kernels.  Each entry point replaces one
 * of the reference's task-level operations on the solve path; the reference
 * implements them as Legion task variants whose GPU bodies call the host
 * launchers cited beside each declaration (file:line in the reference tree).
 *
 * Conventions
 *  - Every array argument is a DEVICE pointer owned by the caller, except
 *    where a parameter is documented as host memory.  `stream` is a
 *    cudaStream_t passed as void*; all work is stream-ordered.
 *  - Cells are single-chunk, x fastest: c = (z*ny + y)*nx + x.
 *  - mat[c]: int32, 1-based material id (the reference's mat field).
 *  - sig[g*nmat + m-1]: per-group, per-material cross section.
 *  - slgg[((g_to*nmat + m-1)*ng + g_from)*nmom + l]: scattering matrix
 *    (the reference's slgg field g_to at point (m, g_from), Legendre order l).
 *  - Per-cell per-group arrays are group-major: xs[g*C + c].
 *  - Moment arrays hold cmom = nmom*nmom flux moments per cell and group,
 *    moment 0 being the scalar flux: flux[(g*C + c)*cmom + k].
 *  - s_xs[(g*C + c)*nmom + l]: in-group scattering per Legendre order.
 *  - Floating point: SNAP_FP64 arrays are double; SNAP_FP32 contexts take
 *    float arrays for the sweep-side data (qtot, t_xs, flux) and double for
 *    the convergence/residual data (see the per-function notes).
 *  - Every function returns a snap_status; none exits the process.
 */
#ifndef SNAP_B200_H
#define SNAP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  SNAP_OK = 0,
  SNAP_ERR_BAD_ARG = 1,
  SNAP_ERR_UNSUPPORTED = 2,
  SNAP_ERR_OOM = 3,
  SNAP_ERR_DEVICE_TIMEOUT = 4, /* a bounded device-side wait gave up */
  SNAP_ERR_CUDA = 5
} snap_status;

typedef enum { SNAP_FP64 = 0, SNAP_FP32 = 1 } snap_precision;

typedef struct {
  int nx, ny, nz;      /* cells of the single spatial chunk */
  int nang;            /* angles per octant */
  int ng;              /* energy groups */
  int nmom;            /* Legendre orders (1..4); cmom = nmom*nmom moments */
  int nmat;            /* materials in the sig/slgg tables */
  int fixup;           /* negative-flux fixup (sweep.cc:425-518) */
  int precision;       /* snap_precision */
  double hi, hj, hk;   /* 2/dx, 2/dy, 2/dz (snap.cc:1178-1180) */
  /* HOST arrays, copied at create time: quadrature and moment coefficients
   * (snap.cc:1208-1337; ec laid out [octant][cmom][nang]) */
  const double *mu, *eta, *xi, *w;
  const double *ec;
} snap_config;

typedef struct snap_ctx snap_ctx;

/* Creates a context on `device`: uploads the quadrature, builds the per-octant
 * coefficient tables and allocates the sweep's scratch (per-octant flux
 * slots, tile-boundary faces, progress flags).  Shapes outside the tiled
 * sweep kernel (nx not a multiple of 8, ny not a multiple of 4, more than 64
 * angles per octant) run every forward sweep on the general kernel (one CTA
 * per octant and group; up to 128 angles the cells of a diagonal plane in
 * flight, one warp per cell, else cell by cell up to 2048 angles; FP64
 * contexts only; no adjoint).  SNAP_B200_WAVE=0 selects the cell-by-cell
 * form always.  The tiled kernel's inner-iteration sweeps walk several
 * groups' z columns per work item (a chain of groups, sized at creation);
 * SNAP_B200_GROUP_CHAIN=n sets the chain length (a divisor of ng; 1: none).
 * Replaces InitGPUSweep -> initialize_gpu_context (init.cc:215-236,
 * gpu_sweep.cu:71-273). */
int snap_create(const snap_config *cfg, int device, snap_ctx **out);
int snap_destroy(snap_ctx *ctx);

/* Bytes of device scratch the context holds now (the per-octant flux slots
 * are allocated on the first call that needs them: snap_sweep, the adjoint
 * entry points; inner iterations and snap_transport_solve need none). */
size_t snap_scratch_bytes(const snap_ctx *ctx);

/* xs[g*C + c] = sig[g*nmat + mat[c]-1]
 * Replaces ExpandCrossSection (expxs.cc:118-160 -> run_expand_cross_section,
 * gpu_expxs.cu:21-267).  Always double. */
int snap_expand_xs(snap_ctx *ctx, const double *sig, const int32_t *mat, double *xs,
                   void *stream);

/* s_xs[(g*C + c)*nmom + l] = slgg[g][mat[c]][g][l]
 * Replaces ExpandScatteringCrossSection (expxs.cc:253-290 ->
 * run_expand_scattering_cross_section, gpu_expxs.cu:269-534).  Always double. */
int snap_expand_scattering_xs(snap_ctx *ctx, const double *slgg, const int32_t *mat,
                              double *s_xs, void *stream);

/* q2grp[(g*C+c)*cmom + 0] = qi[g*C+c] + sum_{g'!=g} slgg[g][mat][g'][0] flux[g'][c][0]
 * q2grp[(g*C+c)*cmom + k] = sum_{g'!=g} slgg[g][mat][g'][l(k)] flux[g'][c][k]
 * Replaces CalcOuterSource (outer.cc:220-284 -> run_flux0_outer_source /
 * run_fluxm_outer_source, gpu_outer.cu:76-441).  Always double; the
 * contraction runs on the FP64 tensor cores (mma.m8n8k4.f64) up to 64 groups
 * per launch, so sums are taken in a different order than the reference's
 * loop (rounding-level differences). */
int snap_calc_outer_source(snap_ctx *ctx, const double *qi, const double *slgg,
                           const int32_t *mat, const double *flux, double *q2grp,
                           void *stream);

/* The same outer source with the group-to-group contraction on the
 * fifth-generation tensor cores (tcgen05.mma kind::f16, accumulators in
 * tensor memory): both operands split into two BF16 parts (three products,
 * FP32 accumulation), relative error of order 1e-5 of the scattering term;
 * qi is added in FP64.  Replaces CalcOuterSource (outer.cc:220-284) where a
 * low-precision source is acceptable: snap_transport_solve uses it in FP32
 * contexts only while the outer iteration is far from converged, and only
 * where its launch plan batches four moments (up to 32 groups with two
 * materials, 64 with one).  Its waits are bounded: a timeout sets the
 * device error word, which the next synchronising call reports.
 * SNAP_ERR_UNSUPPORTED when the accumulators of one moment (groups rounded
 * up to 16, times materials, twice) exceed the 512 tensor-memory columns or
 * the operands the shared memory. */
int snap_calc_outer_source_tc(snap_ctx *ctx, const double *qi, const double *slgg,
                              const int32_t *mat, const double *flux, double *q2grp,
                              void *stream);

/* The outer source of a group shard, for a solve whose energy groups are
 * split over several contexts (one per GPU): the context's ng groups are
 * groups g_lo .. g_lo+ng-1 of ng_total.  qi and q2grp hold the shard's groups
 * ([ng][C] and [ng][C][cmom]); slgg is the full table (ng_total groups) and
 * flux_all the all-gathered flux of every group ([ng_total][C][cmom]).
 * Same arithmetic as snap_calc_outer_source (outer.cc:107-217); the
 * reference has no group sharding (it couples groups through Legion regions). */
int snap_calc_outer_source_groups(snap_ctx *ctx, int g_lo, int ng_total, const double *qi,
                                  const double *slgg, const int32_t *mat,
                                  const double *flux_all, double *q2grp, void *stream);

/* qtot[k] = q2grp[k] + flux[k] * s_xs[l(k)]
 * Replaces CalcInnerSource (inner.cc:163-215 -> run_inner_source_*,
 * gpu_inner.cu:22-117).  FP64 context: qtot double.  FP32 context: qtot float. */
int snap_calc_inner_source(snap_ctx *ctx, const double *s_xs, const double *q2grp,
                           const double *flux, void *qtot, void *stream);

/* One full sweep of all 8 octants and all groups with vacuum boundaries:
 * flux = sum over octants and angles (zeroed first).  One persistent kernel
 * covers every octant and group.
 * Replaces perform_sweeps' MiniKBATask launches (snap.cc:849-887,
 * sweep.cc:1524-1620 -> run_gpu_sweep, gpu_sweep.cu:2047-2295).
 * FP64 context: qtot/t_xs/flux double.  FP32 context: float. */
int snap_sweep(snap_ctx *ctx, const void *qtot, const void *t_xs, void *flux, void *stream);

/* The time-dependent sweep of all 8 octants and groups (the MiniKBATask
 * body with its time-flux and MMS regions, sweep.cc:354-591): as snap_sweep
 * (flux zeroed first) with vdelt[g] * psi_t_in added to each angle's
 * diamond-difference numerator and vdelt[g] to its denominator, the outgoing
 * time face psi_t_out = 2 pc - psi_t_in (a fourth face of the fixup, with
 * its own flag), and qim added to the angular source when not NULL; groups
 * with vdelt == 0 sweep as in steady state.  vdelt [ng]; psi_t_in,
 * psi_t_out and qim [octant][g][c][nang]; all device, FP64 contexts.  Runs
 * the tiled kernel's time-dependent form where the context has one flux
 * moment and a tiled shape (at most 64 angles), else the general kernel
 * (SNAP_B200_TD_GENERAL=1 selects the general kernel always).  Replaces
 * run_gpu_sweep with time dependence (gpu_sweep.cu:738-1393). */
int snap_sweep_td(snap_ctx *ctx, const double *qtot, const double *t_xs, const double *vdelt,
                  const double *psi_t_in, double *psi_t_out, const double *qim, double *flux,
                  void *stream);

/* converged = every scalar flux satisfies |flux/prev - 1| <= epsi (or
 * |flux| <= epsi where |prev| < 1e-12).  kind 0: inner test (epsi as given);
 * kind 1: outer test, which the caller runs with 100*epsi and only when the
 * inner loop converged.  `flux`/`prev` hold cmom moments per cell (moment 0
 * tested).  *converged is HOST memory; the call synchronises `stream`.
 * Replaces TestInnerConvergence / TestOuterConvergence (inner.cc:327-367,
 * outer.cc:405-451 -> run_inner_convergence / run_outer_convergence,
 * gpu_inner.cu:119-236, gpu_outer.cu:443-563).  Always double. */
int snap_test_convergence(snap_ctx *ctx, int kind, const double *flux, const double *prev,
                          double epsi, int *converged, void *stream);

/* One inner iteration on device-resident data, the body of the reference's
 * inner loop (snap.cc:487-503: CalcInnerSource, save_fluxes, MiniKBATask for
 * every octant and group, TestInnerConvergence):
 *   qtot  = q2grp + flux * s_xs            (scratch supplied by the caller,
 *                                           sweep precision, G*C*cmom words)
 *   flux  = sweep(qtot, t_xs)              (in place, double, cmom moments)
 *   *converged = inner test of the new scalar flux against the old one.
 * t_xs has the sweep precision.  *converged is HOST memory; the call
 * synchronises `stream`.  In FP32 contexts the inner test uses
 * max(epsi, 32 * 2^-24): the FP32 sweep's rounding changes some scalar flux
 * by about 1e-6 relative on every inner iteration, so a tighter test passes
 * only by chance. */
int snap_inner_iteration(snap_ctx *ctx, const double *s_xs, const double *q2grp,
                         const void *t_xs, double *flux, void *qtot, double epsi,
                         int *converged, void *stream);

typedef struct {
  double sweep_ms;          /* device time of the sweep kernels (CUDA events) */
  long long sweep_calls;    /* sweeps timed */
  long long kernel_launches;/* kernels this library launched */
} snap_timing;

/* Accumulated timing of this context since creation or the last reset. */
int snap_get_timing(snap_ctx *ctx, snap_timing *out, int reset);

/* One line of the reference's convergence log (convergence.cc:154-232). */
typedef struct {
  int kind;            /* 0: an inner iteration and its inner test, 1: an outer test */
  int time_step, outer, inner;   /* 0-based numbers, as the reference prints them */
  int converged;
  double us;           /* host wall time: the inner iteration, or the whole outer iteration */
} snap_iter_record;

typedef struct {
  double epsi;
  int iitm, oitm;
  /* outputs */
  int inner_total, outer_total, converged;
  int inners_per_outer[1024];
  double sweep_ms;     /* device time spent in the sweep kernels */
  double total_ms;     /* device time of the whole solve */
  int outers_lowp;     /* outer iterations whose source came from snap_calc_outer_source_tc */
  /* optional HOST array for the iteration log: records_cap entries, NULL
   * for none; records_len reports how many were written */
  snap_iter_record *records;
  int records_cap, records_len;
} snap_solve_info;

/* Full steady-state fixed-source solve, the sequential semantics of the
 * reference's predicated loop (snap.cc:409-541): cross-section expansion,
 * outer source, inner source, sweep, inner/outer convergence.  flux (cmom
 * moments, double) holds the result; it is zeroed first (snap.cc:313-316).
 * Replaces Snap::transport_solve's loop body for one time step.
 * FP32 contexts (the precision form) take the outer source from
 * snap_calc_outer_source_tc while the last outer iteration changed some
 * scalar flux by more than 1000*epsi relative (ten times the outer
 * convergence tolerance), and from the FP64 source after that; convergence
 * is only declared on an outer iteration with the FP64 source, so the
 * solution is the fixed point of the FP64 source (set
 * SNAP_B200_FP32_EXACT_OUTER=1 to use the FP64 source throughout). */
int snap_transport_solve(snap_ctx *ctx, const int32_t *mat, const double *qi,
                         const double *sigt, const double *slgg, const double *sigt_scale,
                         double *flux, snap_solve_info *info, void *stream);

/* Time stepping of a time-dependent solve (the reference's timedep = 1
 * decks: input/*_1x1x1.in, input/mms.in). */
typedef struct {
  int nsteps;            /* time steps (the time loop of snap.cc:409-541) */
  double dt;             /* time-step length, tf / nsteps (snap.cc:1174) */
  const double *vdelt;   /* DEVICE [ng]: 2 / (dt v_g); NULL: the reference's
                            speeds v_g = ng - g (snap.cc:717-739) */
  double *psi_t;         /* DEVICE scratch of 2 * 8 * ng * C * nang doubles: the
                            angular flux at the two edges of a time step, laid
                            out [2][octant][g][c][angle] (the reference's
                            time_flux_even / time_flux_odd, snap.cc:288-298);
                            NULL: allocated and freed by the call */
  int psi_t_initialised; /* 0: psi_t is zeroed first (snap.cc:341-344);
                            1: its first half holds the initial angular flux */
  double *qim;           /* DEVICE [octant][g][c][angle] per-angle source added
                            to the angular source (the MMS source,
                            sweep.cc:368-375), or NULL */
  int qim_time_scaled;   /* 1: qim is multiplied in place at the start of
                            every time step by the reference's MMS factors
                            (dt/2, then (2cy+1)/(2cy-1); snap.cc:451-466) */
} snap_time_config;

/* Time-dependent solve: tc->nsteps time steps of the steady-state loop of
 * snap_transport_solve (outer source, inner source, sweep, inner and outer
 * tests per step; the flux carries over between steps), with the
 * time-dependent sweep: vdelt * psi_t_in added to the diamond-difference
 * numerator and vdelt to its denominator, psi_t_out = 2 pc - psi_t_in as a
 * fourth outgoing face (with its own fixup flag), the two halves of psi_t
 * swapping roles every step.  Replaces Snap::transport_solve with
 * time_dependent = true (snap.cc:409-541, sweep.cc:413-419, 461-468, 473-518).
 * The sweep is that of snap_sweep_td (the tiled kernel for one moment and
 * at most 64 angles, else the general kernel: any mesh, up to 2048 angles
 * per octant).  FP64 contexts.  info->inners_per_outer lists the outer iterations of all
 * steps in order. */
int snap_transport_solve_td(snap_ctx *ctx, const int32_t *mat, const double *qi,
                            const double *sigt, const double *slgg, const double *sigt_scale,
                            const snap_time_config *tc, double *flux, snap_solve_info *info,
                            void *stream);

/* ---- Manufactured-solution check (the reference's src_opt = 3 decks) ---- */

/* The manufactured solution of the reference's MMS check for the context's
 * mesh (nmom = 1): ref_flux [G][C] = (g+1) X(x) Y(y) Z(z), the cell averages
 * of sin(pi x/lx) sin(pi y/ly) sin(pi z/lz) (mms.cc:83-179), and the per-angle
 * source qim [8][G][C][nang] that makes it the solution: its streaming term
 * in each octant's direction, the removal sigt * ref, minus the scattering
 * of every group into g (mms.cc:211-359).  timedep != 0: qi [G][C] =
 * ref_flux / v_g and ref_flux scaled to tf - dt/2, the solution at the middle
 * of the last step (mms.cc:387-418); then pass qim to snap_transport_solve_td
 * with qim_time_scaled = 1.  sigt [G][nmat] and slgg as for the solve.
 * chunk_cells = cells per spatial chunk along x, y, z (the deck's nx/ichunk,
 * ny/npey, nz/npez; NULL: one chunk): each chunk's cell edges start at its
 * first cell times that axis's spacing and then step by dx, as the
 * reference's per-chunk tasks compute them, which differs from one chunk
 * only when the spacings differ.  Replaces MMSInitFlux, MMSInitSource and
 * MMSInitTimeDependent (snap.cc:373-388).  Synchronises `stream`. */
int snap_mms_init(snap_ctx *ctx, const int32_t *mat, const double *sigt, const double *slgg,
                  double lx, double ly, double lz, const int *chunk_cells, int timedep,
                  double tf, double dt, double *ref_flux, double *qim, double *qi,
                  void *stream);

/* out[0], out[1], out[2] = max, min and sum over cells and groups of
 * |flux/ref - 1| (|flux| where ref < 1e-12); flux holds cmom moments per
 * cell (the scalar one is compared).  The reference fails the check when the
 * max exceeds 0.1 or the sum / (cells * chunks * groups) exceeds 1e-3
 * (snap.cc:542-560; its divisor multiplies the global cell count by the
 * number of chunks).
 * Replaces MMSCompare (mms.cc:498-545).  Synchronises `stream`. */
int snap_mms_compare(snap_ctx *ctx, const double *flux, const double *ref_flux, double *out,
                     void *stream);

/* ---- Sensitivities (no counterpart in the reference) ------------------ */

/* A forward sweep (as snap_sweep) that also records, for the adjoint, the
 * cell-average angular flux and the fixup face flags of every octant, angle,
 * group and cell in the context (8*G*C*padded-angles words + bytes). */
int snap_record_forward(snap_ctx *ctx, const void *qtot, const void *t_xs, void *flux,
                        void *stream);

/* One adjoint sweep of all octants and groups: the transpose of the sweep
 * operator (reverse-direction wavefront, transposed diamond difference with
 * the recorded fixup flags frozen) applied to the adjoint flux moments
 * phi_bar [G][C][cmom] (sweep precision): qtot_bar [G][C][cmom] (double) =
 * M^T L^-T D^T phi_bar.  With sigt_bar != NULL also the sensitivity to the
 * expanded total cross section, sigt_bar [G][C] = -sum_{octant,angle} s*pc,
 * from the recorded forward state.  Needs snap_record_forward first when the
 * fixup is on or sigt_bar is wanted.  Synchronises `stream`. */
int snap_adjoint_sweep(snap_ctx *ctx, const void *phi_bar, const void *t_xs, double *qtot_bar,
                       double *sigt_bar, void *stream);

/* Discrete adjoint of the converged steady-state solve.  Given the expanded
 * total cross section t_xs [G][C] (double) the forward solve used, the
 * converged forward flux (double, cmom moments) and a response J = sum
 * r[g][c] * flux[g][c][0], iterates phi_bar = r + S^T M^T L^-T D^T phi_bar
 * (S: the full group-to-group scattering, in-group included; fixup flags
 * frozen at the forward state) until max|change| <= info->epsi *
 * max|phi_bar| (at most iitm*oitm iterations; info->inner_total reports
 * them) and returns dJ/dt_xs [G][C] (per-cell, per-group total cross
 * section), dJ/dqi [G][C] (fixed source) and, when grad_sxs != NULL,
 * dJ/ds_xs [G][C][nmom] (per-cell in-group scattering).  Angular fluxes are
 * never stored across iterations: the forward state is recomputed once from
 * the flux moments. */
int snap_adjoint_solve(snap_ctx *ctx, const int32_t *mat, const double *qi, const double *t_xs,
                       const double *slgg, const double *flux, const double *response,
                       double *grad_sigt, double *grad_qi, double *grad_sxs,
                       snap_solve_info *info, void *stream);

/* Size of the static device scratch that snap_sweep_noalloc works in. */
#define SNAP_NOALLOC_SCRATCH_BYTES (48u << 20)

/* The FP64 sweep of snap_sweep (all octants and groups; flux zeroed first)
 * for callers that cannot allocate device memory: code running where
 * cudaMalloc is unavailable or forbidden (inside another library's
 * allocator-free section, a host callback, a process whose device memory
 * pool belongs to someone else, a real-time loop that must not touch the
 * allocator), which therefore cannot call snap_create.
 * Takes the configuration directly (cfg->precision must be SNAP_FP64; host
 * quadrature arrays as for snap_create) and device qtot, t_xs and flux
 * arrays as snap_sweep does.  It allocates nothing: its scratch is one
 * static device array of SNAP_NOALLOC_SCRATCH_BYTES bytes, and problems
 * needing more return SNAP_ERR_UNSUPPORTED with the size in
 * snap_last_error().  CUDA loads code lazily, so the array and the sweep's
 * code are placed on a device when first used there and held until the
 * process exits: call once with qtot, t_xs and flux all NULL (set-up only:
 * nothing is launched), with the device current, outside any section that
 * must not allocate; otherwise the first sweep does this.  Every call shares
 * that array (it keeps the last call's contents; each call clears what must
 * start at zero), so calls that overlap on the GPU race.  The first call on
 * a device looks the array's device address up and keeps it; make it before
 * any stream capture on that device, and make no call after a
 * cudaDeviceReset of it.  Synchronises `stream` (except the set-up call).
 * No counterpart in the reference. */
int snap_sweep_noalloc(const snap_config *cfg, const double *qtot, const double *t_xs,
                       double *flux, void *stream);

/* Self-test of the sweep's division arithmetic (no counterpart in the
 * reference).  The sweep divides by Newton-Raphson refinement of the
 * hardware reciprocal approximation instead of the correctly rounded
 * operations; this entry point exposes both for comparison.  For n operand
 * pairs (a[i], b[i]) in device memory (double for SNAP_FP64, float for
 * SNAP_FP32) it writes out[4i] = the sweep's 1/b[i], out[4i+1] = the
 * correctly rounded 1/b[i], out[4i+2] = the sweep's a[i]/b[i] and
 * out[4i+3] = the correctly rounded a[i]/b[i].  Does not synchronise. */
int snap_selftest_division(int precision, const void *a, const void *b, long long n, void *out,
                           void *stream);

/* Fault injection for tests of the bounded device-side waits (no
 * counterpart in the reference): in the next sweep launch of this context,
 * the warps of work item `item` (0 .. items per launch - 1; item 0 is the
 * first tile of the first octant and group) never publish their tile-edge
 * progress, so the tiles downstream of it wait until their limit
 * (SNAP_B200_TIMEOUT_MS, read at snap_create), give up, and the call returns
 * SNAP_ERR_DEVICE_TIMEOUT.  One launch only; the context stays usable. */
int snap_inject_stall(snap_ctx *ctx, int item);

/* Last error message of this thread (static storage). */
const char *snap_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
