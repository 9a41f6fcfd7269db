/*
 * CPU oracle for the SNAP steady-state solve path (TEST INFRASTRUCTURE ONLY).
 *
 * This is a plain-C, FP64 restatement of the reference's CPU task bodies.
 * It exists to check the CUDA path; nothing in the product links it.  Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
 *
 * Parity status: pinned against the reference's own CPU task variants
 * (compiled from the reference sources through oracle/refshim, see
 * oracle/Makefile) for nmom = 1.  For nmom > 1 the reference's moment
 * machinery is broken (3-slot MomentTriple, ec stored with stride nmom,
 * fluxm never re-zeroed), so for nmom > 1 this restatement generalises the
 * moment bands to cmom = nmom^2 and is pinned only by self-consistency
 * checks in tests/ ("parity unpinned" against the reference for nmom > 1).
 *
 * Data layout (shared with the CUDA path):
 *   cell c = (z*ny + y)*nx + x          (x fastest, Fortran order)
 *   mat[c]                    int32, 1-based material id
 *   sigt[g*nmat + m-1]        total cross section per group/material
 *   slgg[((gto*nmat + m-1)*ng + gfrom)*nmom + l]   scattering matrix
 *   qi[g*C + c]               fixed source
 *   t_xs[g*C + c]             expanded total xs
 *   s_xs[(g*C + c)*nmom + l]  expanded in-group scattering per Legendre order
 *   q2grp/qtot/flux[(g*C + c)*cmom + k]    moment k (k = 0 is the scalar)
 *   ec[(oct*cmom + k)*nang + a]            moment expansion coefficients
 */
#ifndef SNAP_ORACLE_H
#define SNAP_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int nx, ny, nz;
  int nang;      /* angles per octant */
  int ng;        /* energy groups */
  int nmom;      /* Legendre orders */
  int cmom;      /* flux moments = nmom*nmom in 3-D */
  int nmat;
  int fixup;     /* negative-flux fixup on/off */
  double hi, hj, hk;
  const double *mu, *eta, *xi, *w;   /* [nang] */
  const double *ec;                  /* [8][cmom][nang] */
} oracle_geom;

/* snap.cc:1171-1342 (num_dims = 3 branch), moment bands stored with stride
 * cmom.  Fills mu/eta/xi/w [nang] and ec [8*cmom*nang]. */
void oracle_quadrature(int nang, int nmom, double *mu, double *eta, double *xi,
                       double *w, double *ec);

/* expxs.cc:85-115 */
void oracle_expand_xs(const oracle_geom *g, const double *sig, const int32_t *mat,
                      double *xs);
/* expxs.cc:220-250 */
void oracle_expand_scattering(const oracle_geom *g, const double *slgg,
                              const int32_t *mat, double *s_xs);
/* outer.cc:107-217 (moment bands generalised to cmom) */
void oracle_outer_source(const oracle_geom *g, const double *qi, const double *slgg,
                         const int32_t *mat, const double *flux, double *q2grp);
/* inner.cc:106-160 (moment bands generalised to cmom) */
void oracle_inner_source(const oracle_geom *g, const double *s_xs,
                         const double *q2grp, const double *flux, double *qtot);
/* sweep.cc:242-616: one octant ("corner") of one group, accumulating into
 * flux.  Vacuum incoming faces. */
void oracle_sweep_octant_group(const oracle_geom *g, int corner, int group,
                               const double *qtot, const double *t_xs,
                               double *flux);
/* all 8 octants x all groups (flux zeroed first).  Groups are independent
 * sweeps (snap.cc:865-887 launches one task per octant and group chunk); with
 * oracle_set_threads(n > 1) they are spread over n POSIX threads, each group's
 * octants still summed in octant order, so the result does not depend on n. */
void oracle_sweep(const oracle_geom *g, const double *qtot, const double *t_xs,
                  double *flux);
/* Adjoint of oracle_sweep with the fixup flags frozen at the forward state
 * of qtot (no reference counterpart): qtot_bar [G][C][cmom] = transpose of
 * the sweep applied to phi_bar [G][C][cmom], and (sigt_bar != NULL) the
 * sensitivity to t_xs, sigt_bar [G][C].  Both are zeroed first. */
void oracle_adjoint_octant_group(const oracle_geom *g, int corner, int group,
                                 const double *qtot, const double *t_xs,
                                 const double *phi_bar, double *qtot_bar,
                                 double *sigt_bar);
void oracle_adjoint_sweep(const oracle_geom *g, const double *qtot, const double *t_xs,
                          const double *phi_bar, double *qtot_bar, double *sigt_bar);
/* host threads used by oracle_sweep and oracle_outer_source (default 1) */
void oracle_set_threads(int n);
/* inner.cc:283-324 / outer.cc:354-403: returns 1 if converged */
int oracle_test_convergence(const oracle_geom *g, const double *flux,
                            const double *flux_prev, double epsi);

typedef struct {
  double epsi;
  int iitm, oitm;
  int inner_total;       /* out: inner iterations executed */
  int outer_total;       /* out: outer iterations executed */
  int converged;         /* out: outer convergence reached */
  int inners_per_outer[1024]; /* out */
} oracle_solve_info;

/* snap.cc:409-541 sequential semantics of the predicated loop. flux must be
 * zero on entry (snap.cc:313-316). */
void oracle_transport_solve(const oracle_geom *g, const double *qi,
                            const double *slgg, const int32_t *mat,
                            const double *t_xs, const double *s_xs,
                            double *flux, oracle_solve_info *info);

#ifdef __cplusplus
}
#endif
#endif
