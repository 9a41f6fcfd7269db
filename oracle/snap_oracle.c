/*
 * CPU oracle for the SNAP steady-state solve path (TEST INFRASTRUCTURE ONLY).
 * See snap_oracle.h for the layout and the parity status.  Every function
 * cites the reference file:line it restates.
 */
#include "snap_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

static int g_threads = 1;
void oracle_set_threads(int n) { g_threads = n < 1 ? 1 : (n > 256 ? 256 : n); }

/* Runs body(arg, i) for i in [0, n) on g_threads POSIX threads (strided). */
typedef struct {
  void (*body)(void *, int);
  void *arg;
  int n, stride, first;
} par_job;

static void *par_worker(void *p) {
  par_job *j = (par_job *)p;
  for (int i = j->first; i < j->n; i += j->stride) j->body(j->arg, i);
  return NULL;
}

static void par_for(int n, void (*body)(void *, int), void *arg) {
  const int t = g_threads < n ? g_threads : n;
  if (t <= 1) {
    for (int i = 0; i < n; i++) body(arg, i);
    return;
  }
  pthread_t th[256];
  par_job jobs[256];
  for (int k = 0; k < t; k++) {
    jobs[k].body = body; jobs[k].arg = arg; jobs[k].n = n; jobs[k].stride = t; jobs[k].first = k;
    pthread_create(&th[k], NULL, par_worker, &jobs[k]);
  }
  for (int k = 0; k < t; k++) pthread_join(th[k], NULL);
}

static inline int band_of(int k) {
  /* moment k of the 3-D expansion belongs to Legendre band l with
   * l*l <= k < (l+1)*(l+1): band l holds 2l+1 moments (lma, snap.cc:1320) */
  int l = 0;
  while ((l + 1) * (l + 1) <= k) l++;
  return l;
}

/* snap.cc:1171-1342, num_dims == 3 */
void oracle_quadrature(int nang, int nmom, double *mu, double *eta, double *xi,
                       double *w, double *ec) {
  const int cmom = nmom * nmom;
  const double dm = 1.0 / (double)nang;
  mu[0] = 0.5 * dm; /* snap.cc:1208-1210 */
  for (int i = 1; i < nang; i++) mu[i] = mu[i - 1] + dm;
  eta[0] = 1.0 - 0.5 * dm; /* snap.cc:1212-1214 */
  for (int i = 1; i < nang; i++) eta[i] = eta[i - 1] - dm;
  for (int i = 0; i < nang; i++) { /* snap.cc:1217-1220 */
    const double t = mu[i] * mu[i] + eta[i] * eta[i];
    xi[i] = sqrt(1.0 - t);
  }
  for (int i = 0; i < nang; i++) w[i] = 0.125 / (double)nang; /* snap.cc:1232 */
  /* snap.cc:1298-1337: oct = 4*kd + 2*jd + id, sign -1 for bit clear */
  for (int oct = 0; oct < 8; oct++) {
    const double is = (oct & 1) ? 1.0 : -1.0;
    const double js = (oct & 2) ? 1.0 : -1.0;
    const double ks = (oct & 4) ? 1.0 : -1.0;
    double *e = ec + (size_t)oct * cmom * nang;
    for (int a = 0; a < nang; a++) e[a] = 1.0;
    int moment = 1;
    for (int l = 1; l < nmom; l++) {
      for (int m = 0; m < 2 * l + 1; m++) {
        for (int a = 0; a < nang; a++)
          e[(size_t)moment * nang + a] =
              pow(is * mu[a], (double)(2 * l - 1)) * pow(ks * xi[a] * js * eta[a], (double)m);
        moment++;
      }
    }
  }
}

/* expxs.cc:85-115: xs[g][c] = sig[g][mat[c]] */
void oracle_expand_xs(const oracle_geom *g, const double *sig, const int32_t *mat,
                      double *xs) {
  const size_t C = (size_t)g->nx * g->ny * g->nz;
  for (int grp = 0; grp < g->ng; grp++)
    for (size_t c = 0; c < C; c++)
      xs[grp * C + c] = sig[grp * g->nmat + (mat[c] - 1)];
}

/* expxs.cc:220-250: s_xs[g][c] = slgg[g][mat[c]][g] (all Legendre orders) */
void oracle_expand_scattering(const oracle_geom *g, const double *slgg,
                              const int32_t *mat, double *s_xs) {
  const size_t C = (size_t)g->nx * g->ny * g->nz;
  const int ng = g->ng, nmat = g->nmat, nmom = g->nmom;
  for (int grp = 0; grp < ng; grp++)
    for (size_t c = 0; c < C; c++) {
      const double *src = slgg + (((size_t)grp * nmat + (mat[c] - 1)) * ng + grp) * nmom;
      for (int l = 0; l < nmom; l++) s_xs[(grp * C + c) * nmom + l] = src[l];
    }
}

/* outer.cc:107-217.  qo0 = qi + sum_{g2 != g1} slgg[g1][mat][g2][0]*flux0[g2]
 * (outer.cc:160-171); higher moments k use the Legendre order of their band
 * (outer.cc:196-207, generalised to all cmom-1 moments). */
typedef struct {
  const oracle_geom *g;
  const double *qi, *slgg, *flux;
  const int32_t *mat;
  double *q2grp;
} outer_args;

static void outer_group(void *arg, int g1) {
  const outer_args *x = (const outer_args *)arg;
  const oracle_geom *g = x->g;
  const double *qi = x->qi, *slgg = x->slgg, *flux = x->flux;
  const int32_t *mat = x->mat;
  double *q2grp = x->q2grp;
  const size_t C = (size_t)g->nx * g->ny * g->nz;
  const int ng = g->ng, nmat = g->nmat, nmom = g->nmom, cmom = g->cmom;
  {
    for (size_t c = 0; c < C; c++) {
      const int m = mat[c] - 1;
      double q0 = qi[g1 * C + c];
      for (int g2 = 0; g2 < ng; g2++) {
        if (g1 == g2) continue;
        q0 += slgg[(((size_t)g1 * nmat + m) * ng + g2) * nmom + 0] *
              flux[(g2 * C + c) * cmom + 0];
      }
      q2grp[(g1 * C + c) * cmom + 0] = q0;
      for (int k = 1; k < cmom; k++) {
        const int l = band_of(k);
        double qk = 0.0;
        for (int g2 = 0; g2 < ng; g2++) {
          if (g1 == g2) continue;
          qk += slgg[(((size_t)g1 * nmat + m) * ng + g2) * nmom + l] *
                flux[(g2 * C + c) * cmom + k];
        }
        q2grp[(g1 * C + c) * cmom + k] = qk;
      }
    }
  }
}

void oracle_outer_source(const oracle_geom *g, const double *qi, const double *slgg,
                         const int32_t *mat, const double *flux, double *q2grp) {
  outer_args x = {g, qi, slgg, flux, mat, q2grp};
  par_for(g->ng, outer_group, &x);
}

/* inner.cc:106-160: qtot[0] = q2grp0 + flux0*s_xs[0];
 * qtot[k] = q2grpm[k] + fluxm[k]*s_xs[l(k)] (inner.cc:139-144) */
void oracle_inner_source(const oracle_geom *g, const double *s_xs,
                         const double *q2grp, const double *flux, double *qtot) {
  const size_t C = (size_t)g->nx * g->ny * g->nz;
  const int cmom = g->cmom, nmom = g->nmom;
  for (int grp = 0; grp < g->ng; grp++)
    for (size_t c = 0; c < C; c++) {
      const size_t base = (grp * C + c) * cmom;
      const double *sx = s_xs + (grp * C + c) * nmom;
      qtot[base] = q2grp[base] + flux[base] * sx[0];
      for (int k = 1; k < cmom; k++)
        qtot[base + k] = q2grp[base + k] + flux[base + k] * sx[band_of(k)];
    }
}

/* sweep.cc:242-616 (MiniKBATask::cpu_implementation), steady state
 * (vdelt == 0), single spatial chunk, vacuum incoming faces. */
void oracle_sweep_octant_group(const oracle_geom *g, int corner, int group,
                               const double *qtot, const double *t_xs,
                               double *flux) {
  const int nx = g->nx, ny = g->ny, nz = g->nz, A = g->nang, cmom = g->cmom;
  const size_t C = (size_t)nx * ny * nz;
  const int sx = (corner & 1) != 0, sy = (corner & 2) != 0, sz = (corner & 4) != 0;
  const double tolr = 1.0e-12;
  const double *ec = g->ec + (size_t)corner * cmom * A;

  double *buf = (double *)calloc((size_t)A * 13 + (size_t)A * nx + (size_t)A * nx * ny, sizeof(double));
  double *psi = buf, *pc = psi + A, *psii = pc + A, *psij = psii + A, *psik = psij + A;
  double *hv_x = psik + A, *hv_y = hv_x + A, *hv_z = hv_y + A;
  double *fx = hv_z + A, *fy = fx + A, *fz = fy + A, *dinv = fz + A, *pw = dinv + A;
  double *ypencil = pw + A;          /* sweep.cc:301 */
  double *zplane = ypencil + (size_t)A * nx; /* sweep.cc:302 */

  for (int zz = 0; zz < nz; zz++) {
    const int z = sz ? zz : nz - 1 - zz;
    for (int yy = 0; yy < ny; yy++) {
      const int y = sy ? yy : ny - 1 - yy;
      for (int xx = 0; xx < nx; xx++) {
        const int x = sx ? xx : nx - 1 - xx;
        const size_t c = ((size_t)z * ny + y) * nx + x;
        const double *q = qtot + (group * C + c) * cmom;
        const double sig = t_xs[group * C + c];
        /* angular source, sweep.cc:354-366 (band stride cmom) */
        for (int a = 0; a < A; a++) psi[a] = q[0];
        for (int k = 1; k < cmom; k++)
          for (int a = 0; a < A; a++) psi[a] += ec[(size_t)k * A + a] * q[k];
        /* geometry parameter, expxs.cc:374-379 (vdelt = 0) */
        for (int a = 0; a < A; a++)
          dinv[a] = 1.0 / (sig + 0.0 + g->hi * g->mu[a] + g->hj * g->eta[a] + g->hk * g->xi[a]);
        for (int a = 0; a < A; a++) pc[a] = psi[a];
        if (xx == 0) memset(psii, 0, sizeof(double) * A); /* vacuum ghost */
        for (int a = 0; a < A; a++) pc[a] += psii[a] * g->mu[a] * g->hi;
        if (yy == 0) memset(psij, 0, sizeof(double) * A);
        else memcpy(psij, ypencil + (size_t)xx * A, sizeof(double) * A);
        for (int a = 0; a < A; a++) pc[a] += psij[a] * g->eta[a] * g->hj;
        if (zz == 0) memset(psik, 0, sizeof(double) * A);
        else memcpy(psik, zplane + ((size_t)yy * nx + xx) * A, sizeof(double) * A);
        for (int a = 0; a < A; a++) pc[a] += psik[a] * g->xi[a] * g->hk;
        for (int a = 0; a < A; a++) pc[a] *= dinv[a];

        if (g->fixup) { /* sweep.cc:425-518 */
          unsigned old_neg = 0;
          for (int a = 0; a < A; a++) { hv_x[a] = 1.0; hv_y[a] = 1.0; hv_z[a] = 1.0; }
          for (;;) {
            unsigned neg = 0;
            for (int a = 0; a < A; a++) {
              fx[a] = 2.0 * pc[a] - psii[a];
              if (fx[a] < 0.0) { hv_x[a] = 0.0; neg++; }
            }
            for (int a = 0; a < A; a++) {
              fy[a] = 2.0 * pc[a] - psij[a];
              if (fy[a] < 0.0) { hv_y[a] = 0.0; neg++; }
            }
            for (int a = 0; a < A; a++) {
              fz[a] = 2.0 * pc[a] - psik[a];
              if (fz[a] < 0.0) { hv_z[a] = 0.0; neg++; }
            }
            if (neg == old_neg) break;
            old_neg = neg;
            for (int a = 0; a < A; a++) {
              pc[a] = psi[a] + 0.5 * (psii[a] * g->mu[a] * g->hi * (1.0 + hv_x[a]) +
                                      psij[a] * g->eta[a] * g->hj * (1.0 + hv_y[a]) +
                                      psik[a] * g->xi[a] * g->hk * (1.0 + hv_z[a]));
              const double den = (pc[a] <= 0.0) ? 0.0
                  : (sig + g->mu[a] * g->hi * hv_x[a] + g->eta[a] * g->hj * hv_y[a] +
                     g->xi[a] * g->hk * hv_z[a]);
              if (den < tolr) pc[a] = 0.0;
              else pc[a] /= den;
            }
          }
          for (int a = 0; a < A; a++) {
            psii[a] = fx[a] * hv_x[a];
            psij[a] = fy[a] * hv_y[a];
            psik[a] = fz[a] * hv_z[a];
          }
        } else {
          for (int a = 0; a < A; a++) {
            psii[a] = 2.0 * pc[a] - psii[a];
            psij[a] = 2.0 * pc[a] - psij[a];
            psik[a] = 2.0 * pc[a] - psik[a];
          }
        }
        /* psii carries to the next x; psij/psik go to the pencil/plane
         * (sweep.cc:536-562; outgoing domain faces are not needed) */
        memcpy(ypencil + (size_t)xx * A, psij, sizeof(double) * A);
        memcpy(zplane + ((size_t)yy * nx + xx) * A, psik, sizeof(double) * A);

        /* moment accumulation, sweep.cc:565-591 */
        double *f = flux + (group * C + c) * cmom;
        double total = 0.0;
        for (int a = 0; a < A; a++) { pw[a] = g->w[a] * pc[a]; total += pw[a]; }
        f[0] += total;
        for (int k = 1; k < cmom; k++) {
          total = 0.0;
          for (int a = 0; a < A; a++) total += ec[(size_t)k * A + a] * pw[a];
          f[k] += total;
        }
      }
    }
  }
  free(buf);
}

typedef struct {
  const oracle_geom *g;
  const double *qtot, *t_xs;
  double *flux;
} sweep_args;

static void sweep_group(void *arg, int grp) {
  const sweep_args *x = (const sweep_args *)arg;
  for (int corner = 0; corner < 8; corner++)
    oracle_sweep_octant_group(x->g, corner, grp, x->qtot, x->t_xs, x->flux);
}

void oracle_sweep(const oracle_geom *g, const double *qtot, const double *t_xs,
                  double *flux) {
  const size_t C = (size_t)g->nx * g->ny * g->nz;
  /* snap.cc:494 zeroes flux0 before the sweeps; the restatement zeroes every
   * moment (the reference leaves fluxm stale, a bug for nmom > 1). */
  memset(flux, 0, sizeof(double) * C * g->ng * g->cmom);
  sweep_args x = {g, qtot, t_xs, flux};
  par_for(g->ng, sweep_group, &x);   /* groups: snap.cc:872; octants in order: :865 */
}

/* Adjoint of one (octant, group) sweep with the fixup flags frozen at the
 * forward state (no reference counterpart; the transpose of
 * oracle_sweep_octant_group): a forward pass over the cells in upwind order
 * records, per cell and angle, pc, the face flags the last fixup recompute
 * used (p_d), the flags of the outgoing faces (h_d), and whether pc was set
 * to zero; the reverse pass walks the cells downstream-first with the
 * adjoint faces and adds
 *   pc_bar   = sum_k ec[k][a] w[a] phi_bar[k] + 2 sum_d h_d out_bar_d
 *   s        = pc_bar / den          (0 where pc was set to zero)
 *   in_bar_d = -h_d out_bar_d + s (1 + p_d) c_d / 2
 *   qtot_bar[k] += ec[k][a] s,  sigt_bar -= s pc
 * where pc = (psi + sum_d c_d in_d (1 + p_d) / 2) / (sigma_t + sum_d c_d p_d)
 * (all p_d = 1: the diamond difference) and out_d = (2 pc - in_d) h_d. */
void oracle_adjoint_octant_group(const oracle_geom *g, int corner, int group,
                                 const double *qtot, const double *t_xs,
                                 const double *phi_bar, double *qtot_bar,
                                 double *sigt_bar) {
  const int nx = g->nx, ny = g->ny, nz = g->nz, A = g->nang, cmom = g->cmom;
  const size_t C = (size_t)nx * ny * nz;
  const int sx = (corner & 1) != 0, sy = (corner & 2) != 0, sz = (corner & 4) != 0;
  const double tolr = 1.0e-12;
  const double *ec = g->ec + (size_t)corner * cmom * A;
  /* recorded forward state, indexed by the cell's position in sweep order */
  double *rpc = (double *)calloc(C * A, sizeof(double));
  double *rden = (double *)calloc(C * A, sizeof(double));
  unsigned char *rflag = (unsigned char *)calloc(C * A, 1);   /* p x,y,z bits 0-2, h bits 3-5, zero bit 6 */
  double *buf = (double *)calloc((size_t)A * 14 + (size_t)A * nx + (size_t)A * nx * ny, sizeof(double));
  double *psi = buf, *pc = psi + A, *psii = pc + A, *psij = psii + A, *psik = psij + A;
  double *hv_x = psik + A, *hv_y = hv_x + A, *hv_z = hv_y + A;
  double *fx = hv_z + A, *fy = fx + A, *fz = fy + A, *pvx = fz + A, *pvy = pvx + A, *pvz = pvy + A;
  double *ypencil = pvz + A, *zplane = ypencil + (size_t)A * nx;
  unsigned char *zero = (unsigned char *)calloc(A, 1);
  size_t n = 0;   /* cell position in sweep order */
  for (int zz = 0; zz < nz; zz++) {
    const int z = sz ? zz : nz - 1 - zz;
    for (int yy = 0; yy < ny; yy++) {
      const int y = sy ? yy : ny - 1 - yy;
      for (int xx = 0; xx < nx; xx++, n++) {
        const int x = sx ? xx : nx - 1 - xx;
        const size_t c = ((size_t)z * ny + y) * nx + x;
        const double *q = qtot + (group * C + c) * cmom;
        const double sig = t_xs[group * C + c];
        for (int a = 0; a < A; a++) psi[a] = q[0];
        for (int k = 1; k < cmom; k++)
          for (int a = 0; a < A; a++) psi[a] += ec[(size_t)k * A + a] * q[k];
        if (xx == 0) memset(psii, 0, sizeof(double) * A);
        if (yy == 0) memset(psij, 0, sizeof(double) * A);
        else memcpy(psij, ypencil + (size_t)xx * A, sizeof(double) * A);
        if (zz == 0) memset(psik, 0, sizeof(double) * A);
        else memcpy(psik, zplane + ((size_t)yy * nx + xx) * A, sizeof(double) * A);
        for (int a = 0; a < A; a++) {
          const double den = sig + g->hi * g->mu[a] + g->hj * g->eta[a] + g->hk * g->xi[a];
          pc[a] = (psi[a] + psii[a] * g->mu[a] * g->hi + psij[a] * g->eta[a] * g->hj +
                   psik[a] * g->xi[a] * g->hk) / den;
          rden[n * A + a] = den;
          hv_x[a] = hv_y[a] = hv_z[a] = 1.0;
          pvx[a] = pvy[a] = pvz[a] = 1.0;
          zero[a] = 0;
        }
        if (g->fixup) {
          unsigned old_neg = 0;
          for (;;) {
            unsigned neg = 0;
            for (int a = 0; a < A; a++) {
              fx[a] = 2.0 * pc[a] - psii[a];
              if (fx[a] < 0.0) { hv_x[a] = 0.0; neg++; }
              fy[a] = 2.0 * pc[a] - psij[a];
              if (fy[a] < 0.0) { hv_y[a] = 0.0; neg++; }
              fz[a] = 2.0 * pc[a] - psik[a];
              if (fz[a] < 0.0) { hv_z[a] = 0.0; neg++; }
            }
            if (neg == old_neg) break;
            old_neg = neg;
            for (int a = 0; a < A; a++) {
              pvx[a] = hv_x[a];
              pvy[a] = hv_y[a];
              pvz[a] = hv_z[a];
              const double v = psi[a] + 0.5 * (psii[a] * g->mu[a] * g->hi * (1.0 + hv_x[a]) +
                                                psij[a] * g->eta[a] * g->hj * (1.0 + hv_y[a]) +
                                                psik[a] * g->xi[a] * g->hk * (1.0 + hv_z[a]));
              const double den = (v <= 0.0) ? 0.0
                  : (sig + g->mu[a] * g->hi * hv_x[a] + g->eta[a] * g->hj * hv_y[a] +
                     g->xi[a] * g->hk * hv_z[a]);
              rden[n * A + a] = den;
              zero[a] = den < tolr;
              pc[a] = zero[a] ? 0.0 : v / den;
            }
          }
        }
        for (int a = 0; a < A; a++) {
          rpc[n * A + a] = pc[a];
          rflag[n * A + a] = (unsigned char)((pvx[a] != 0.0) | ((pvy[a] != 0.0) << 1) |
                                             ((pvz[a] != 0.0) << 2) | ((hv_x[a] != 0.0) << 3) |
                                             ((hv_y[a] != 0.0) << 4) | ((hv_z[a] != 0.0) << 5) |
                                             (zero[a] << 6));
          psii[a] = (2.0 * pc[a] - psii[a]) * hv_x[a];
          psij[a] = (2.0 * pc[a] - psij[a]) * hv_y[a];
          psik[a] = (2.0 * pc[a] - psik[a]) * hv_z[a];
        }
        memcpy(ypencil + (size_t)xx * A, psij, sizeof(double) * A);
        memcpy(zplane + ((size_t)yy * nx + xx) * A, psik, sizeof(double) * A);
      }
    }
  }
  /* reverse pass: adjoint faces, downstream cells first */
  double *bx = psii, *by = psij, *bz = psik;   /* adjoint of the cell's outgoing faces */
  for (int zz = nz - 1; zz >= 0; zz--) {
    const int z = sz ? zz : nz - 1 - zz;
    for (int yy = ny - 1; yy >= 0; yy--) {
      const int y = sy ? yy : ny - 1 - yy;
      for (int xx = nx - 1; xx >= 0; xx--) {
        n--;
        const int x = sx ? xx : nx - 1 - xx;
        const size_t c = ((size_t)z * ny + y) * nx + x;
        /* nothing downstream of the last cell along an axis */
        if (xx == nx - 1) memset(bx, 0, sizeof(double) * A);
        if (yy == ny - 1) memset(by, 0, sizeof(double) * A);
        else memcpy(by, ypencil + (size_t)xx * A, sizeof(double) * A);
        if (zz == nz - 1) memset(bz, 0, sizeof(double) * A);
        else memcpy(bz, zplane + ((size_t)yy * nx + xx) * A, sizeof(double) * A);
        const double *pb = phi_bar + (group * C + c) * cmom;
        double *qb = qtot_bar + (group * C + c) * cmom;
        double sb = 0.0;
        for (int a = 0; a < A; a++) {
          const unsigned f = rflag[n * A + a];
          double pcb = pb[0] * g->w[a];
          for (int k = 1; k < cmom; k++) pcb += ec[(size_t)k * A + a] * g->w[a] * pb[k];
          const double hx = (f >> 3) & 1, hy = (f >> 4) & 1, hz = (f >> 5) & 1;
          pcb += 2.0 * (hx * bx[a] + hy * by[a] + hz * bz[a]);
          const double s = ((f >> 6) & 1) ? 0.0 : pcb / rden[n * A + a];
          const double px = f & 1, py = (f >> 1) & 1, pz = (f >> 2) & 1;
          /* adjoint of the incoming faces = adjoint of the upstream cells' outgoing faces */
          bx[a] = -hx * bx[a] + s * 0.5 * (1.0 + px) * g->mu[a] * g->hi;
          by[a] = -hy * by[a] + s * 0.5 * (1.0 + py) * g->eta[a] * g->hj;
          bz[a] = -hz * bz[a] + s * 0.5 * (1.0 + pz) * g->xi[a] * g->hk;
          qb[0] += s;
          for (int k = 1; k < cmom; k++) qb[k] += ec[(size_t)k * A + a] * s;
          sb -= s * rpc[n * A + a];
        }
        if (sigt_bar) sigt_bar[group * C + c] += sb;
        /* bx carries to the upstream x neighbour; by, bz to the pencil/plane */
        memcpy(ypencil + (size_t)xx * A, by, sizeof(double) * A);
        memcpy(zplane + ((size_t)yy * nx + xx) * A, bz, sizeof(double) * A);
      }
    }
  }
  free(buf);
  free(zero);
  free(rflag);
  free(rden);
  free(rpc);
}

typedef struct {
  const oracle_geom *g;
  const double *qtot, *t_xs, *phi_bar;
  double *qtot_bar, *sigt_bar;
} adjoint_args;

static void adjoint_group(void *arg, int grp) {
  const adjoint_args *x = (const adjoint_args *)arg;
  for (int corner = 0; corner < 8; corner++)
    oracle_adjoint_octant_group(x->g, corner, grp, x->qtot, x->t_xs, x->phi_bar, x->qtot_bar,
                                x->sigt_bar);
}

void oracle_adjoint_sweep(const oracle_geom *g, const double *qtot, const double *t_xs,
                          const double *phi_bar, double *qtot_bar, double *sigt_bar) {
  const size_t C = (size_t)g->nx * g->ny * g->nz;
  memset(qtot_bar, 0, sizeof(double) * C * g->ng * g->cmom);
  if (sigt_bar) memset(sigt_bar, 0, sizeof(double) * C * g->ng);
  adjoint_args x = {g, qtot, t_xs, phi_bar, qtot_bar, sigt_bar};
  par_for(g->ng, adjoint_group, &x);
}

/* inner.cc:283-324 and outer.cc:354-403 (scalar moment only) */
int oracle_test_convergence(const oracle_geom *g, const double *flux,
                            const double *flux_prev, double epsi) {
  const size_t C = (size_t)g->nx * g->ny * g->nz;
  const double tolr = 1.0e-12;
  for (int grp = 0; grp < g->ng; grp++)
    for (size_t c = 0; c < C; c++) {
      double prev = flux_prev[(grp * C + c) * g->cmom];
      double df = 1.0;
      if (fabs(prev) < tolr) { prev = 1.0; df = 0.0; }
      df = fabs(flux[(grp * C + c) * g->cmom] / prev - df);
      if (df > epsi) return 0;
    }
  return 1;
}

/* snap.cc:472-540 with the predicates resolved sequentially */
void oracle_transport_solve(const oracle_geom *g, const double *qi,
                            const double *slgg, const int32_t *mat,
                            const double *t_xs, const double *s_xs,
                            double *flux, oracle_solve_info *info) {
  const size_t C = (size_t)g->nx * g->ny * g->nz;
  const size_t n = C * g->ng * g->cmom;
  double *q2grp = (double *)calloc(n, sizeof(double));
  double *qtot = (double *)calloc(n, sizeof(double));
  double *fpo = (double *)calloc(n, sizeof(double));
  double *fpi = (double *)calloc(n, sizeof(double));
  info->inner_total = 0;
  info->outer_total = 0;
  info->converged = 0;
  for (int o = 0; o < info->oitm; o++) {
    oracle_outer_source(g, qi, slgg, mat, flux, q2grp);   /* snap.cc:477 */
    memcpy(fpo, flux, sizeof(double) * n);                /* snap.cc:481 */
    int inner_conv = 0, inners = 0;
    for (int i = 0; i < info->iitm; i++) {
      oracle_inner_source(g, s_xs, q2grp, flux, qtot);    /* snap.cc:490 */
      memcpy(fpi, flux, sizeof(double) * n);              /* snap.cc:493 */
      oracle_sweep(g, qtot, t_xs, flux);                  /* snap.cc:494-499 */
      inners++;
      inner_conv = oracle_test_convergence(g, flux, fpi, info->epsi); /* :501 */
      if (inner_conv) break;
    }
    if (o < 1024) info->inners_per_outer[o] = inners;
    info->inner_total += inners;
    info->outer_total++;
    if (o == 0) continue;                                 /* snap.cc:521 */
    if (inner_conv && oracle_test_convergence(g, flux, fpo, 100.0 * info->epsi)) {
      info->converged = 1;                                /* outer.cc:361-365 */
      break;
    }
  }
  free(q2grp); free(qtot); free(fpo); free(fpi);
}
