/*
 * svof_oracle3d.c -- CPU restatement of the hot path in 3D, FP64.
 * TEST INFRASTRUCTURE ONLY (see svof_oracle3d.h).
 *
 * Every expression is the 2D reference expression (oracle/svof_oracle.c, which
 * cites the reference line by line) with its z counterpart appended after the
 * x and y terms, so that z-invariant fields (uz = 0, no z variation) add exact
 * zeros: z advection and diffusion terms vanish exactly, the Poisson kz = 0
 * mode carries the 2D problem scaled by powers of two.  Corner-normal sums and
 * the curvature use the 2D 2x2 expressions on the two bounding corner planes.
 */
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "svof_fft.h"
#include "svof_oracle3d.h"

static const double RK_A[3] = {32. / 60., 25. / 60., 45. / 60.};
static const double RK_B[3] = {0. / 60., -17. / 60., -25. / 60.};
static double rk_g(int s) { return RK_A[s] + RK_B[s]; }
static const double GAUSS_P[2] = {-0.2886751345948129, +0.2886751345948129};
static const double GAUSS_W[2] = {+0.5, +0.5};
static const double VOFBETA = 1.;
static const double VOFMIN = 1.e-8;
static const double G_PI = 3.14159265358979324;

struct svo3_ctx {
  svo3_params_t prm;
  int nx, ny, nz;
  double *xf, *xc, *dxf, *dxc;
  double dy, dz;
  double *ux, *uy, *uz, *p, *psi, *t;
  double *srcux[3], *srcuy[3], *srcuz[3], *srct[3];
  double *vof, *ifrcx, *ifrcy, *ifrcz, *dvof, *normal, *curv, *flxx, *flxy, *flxz, *src[2];
  long n_ux, n_cc, n_vof, n_dvof, n_normal, n_flxx, n_flxy, n_flxz, n_srcx, n_src;
  double *lapx_ux, *lapx_cc;  /* 3 per row; uy, uz and t share lapx_cc */
  double lapy[3], lapz[3];
  double *x1pncl;
  double *tdm_l, *tdm_c, *tdm_u, *tdm_v;
  double *spec;               /* [kz][i][ky] complex */
  double *line;               /* 2 * max(ny, nz) */
  svof_fft_plan_t *plan_y, *plan_z;
  double *evy, *evz, *pl, *pu;
  /* time-averaged statistics: ux1 ux2 uy1 uy2 uz1 uz2 t1 t2 uxt, made on the
   * first collection */
  double *stat[9];
  long stat_num;
  /* extension (absent from the reference; off while grav_vof == 0): the
   * Boussinesq buoyancy of the volume fraction along y, srcuy += grav_vof
   * (vof_face - vof_ref), as the 2D restatement's svo_set_gravity */
  double grav_vof, vof_ref;
};

#define NX (c->nx)
#define NY (c->ny)
#define NZ (c->nz)
#define UX(i, j, k) c->ux[(i) - 1 + (long)(NX + 1) * ((j) + (long)(NY + 2) * (k))]
#define CC(a, i, j, k) (a)[(i) + (long)(NX + 2) * ((j) + (long)(NY + 2) * (k))]
#define VOF(i, j, k) c->vof[(i) + (long)(NX + 2) * (((j) + 1) + (long)(NY + 4) * ((k) + 1))]
#define DVOF(i, j, k, m) c->dvof[3 * ((i) - 1 + (long)(NX + 1) * ((j) + (long)(NY + 3) * (k))) + (m)]
#define NRM(i, j, k, m) c->normal[4 * ((i) - 1 + (long)NX * ((j) + (long)(NY + 2) * (k))) + (m)]
#define SRCX(a, i, j, k) (a)[(i) - 2 + (long)(NX - 1) * (((j) - 1) + (long)NY * ((k) - 1))]
#define SRC(a, i, j, k) (a)[(i) - 1 + (long)NX * (((j) - 1) + (long)NY * ((k) - 1))]
#define FLXX(i, j, k) c->flxx[(i) - 1 + (long)(NX + 1) * (((j) - 1) + (long)NY * ((k) - 1))]
#define FLXY(i, j, k) c->flxy[(i) - 1 + (long)NX * (((j) - 1) + (long)(NY + 1) * ((k) - 1))]
#define FLXZ(i, j, k) c->flxz[(i) - 1 + (long)NX * (((j) - 1) + (long)NY * ((k) - 1))]
#define DXF(i) c->dxf[(i) - 1]
#define DXC(i) c->dxc[(i) - 1]

static double *dalloc(long n) { return calloc((size_t)(n > 0 ? n : 1), sizeof(double)); }

svo3_ctx_t *svo3_create(const svo3_params_t *prm, const double *xf, const double *xc) {
  if (prm->nx < 3 || prm->ny < 3 || prm->nz < 3) return NULL;
  svo3_ctx_t *c = calloc(1, sizeof(*c));
  c->prm = *prm;
  c->nx = prm->nx;
  c->ny = prm->ny;
  c->nz = prm->nz;
  const int nx = NX, ny = NY, nz = NZ;
  c->xf = dalloc(nx + 1);
  c->xc = dalloc(nx + 2);
  memcpy(c->xf, xf, sizeof(double) * (size_t)(nx + 1));
  memcpy(c->xc, xc, sizeof(double) * (size_t)(nx + 2));
  c->dxf = dalloc(nx);
  c->dxc = dalloc(nx + 1);
  for (int i = 1; i <= nx; i++) DXF(i) = c->xf[i] - c->xf[i - 1];
  for (int i = 1; i <= nx + 1; i++) DXC(i) = c->xc[i] - c->xc[i - 1];
  c->dy = prm->ly / ny;
  c->dz = prm->lz / nz;
  c->n_ux = (long)(nx + 1) * (ny + 2) * (nz + 2);
  c->n_cc = (long)(nx + 2) * (ny + 2) * (nz + 2);
  c->n_vof = (long)(nx + 2) * (ny + 4) * (nz + 4);
  c->n_dvof = 3L * (nx + 1) * (ny + 3) * (nz + 3);
  c->n_normal = 4L * nx * (ny + 2) * (nz + 2);
  c->n_flxx = (long)(nx + 1) * ny * nz;
  c->n_flxy = (long)nx * (ny + 1) * nz;
  c->n_flxz = (long)nx * ny * (nz + 1);
  c->n_srcx = (long)(nx - 1) * ny * nz;
  c->n_src = (long)nx * ny * nz;
  c->ux = dalloc(c->n_ux);
  c->uy = dalloc(c->n_cc);
  c->uz = dalloc(c->n_cc);
  c->p = dalloc(c->n_cc);
  c->psi = dalloc(c->n_cc);
  c->t = dalloc(c->n_cc);
  for (int k = 0; k < 3; k++) {
    c->srcux[k] = dalloc(c->n_srcx);
    c->srcuy[k] = dalloc(c->n_src);
    c->srcuz[k] = dalloc(c->n_src);
    c->srct[k] = dalloc(c->n_src);
  }
  c->vof = dalloc(c->n_vof);
  c->ifrcx = dalloc(c->n_srcx);
  c->ifrcy = dalloc(c->n_src);
  c->ifrcz = dalloc(c->n_src);
  c->dvof = dalloc(c->n_dvof);
  c->normal = dalloc(c->n_normal);
  c->curv = dalloc(c->n_cc);
  c->flxx = dalloc(c->n_flxx);
  c->flxy = dalloc(c->n_flxy);
  c->flxz = dalloc(c->n_flxz);
  c->src[0] = dalloc(c->n_src);
  c->src[1] = dalloc(c->n_src);
  c->lapx_ux = dalloc(3L * (nx - 1));
  for (int i = 2; i <= nx; i++) {
    const double l = 1. / DXF(i - 1) / DXC(i);
    const double u = 1. / DXF(i) / DXC(i);
    c->lapx_ux[3 * (i - 2) + 0] = l;
    c->lapx_ux[3 * (i - 2) + 1] = -l - u;
    c->lapx_ux[3 * (i - 2) + 2] = u;
  }
  c->lapx_cc = dalloc(3L * nx);
  for (int i = 1; i <= nx; i++) {
    const double l = 1. / DXC(i) / DXF(i);
    const double u = 1. / DXC(i + 1) / DXF(i);
    c->lapx_cc[3 * (i - 1) + 0] = l;
    c->lapx_cc[3 * (i - 1) + 1] = -l - u;
    c->lapx_cc[3 * (i - 1) + 2] = u;
  }
  c->lapy[0] = +1. / c->dy / c->dy;
  c->lapy[1] = -2. / c->dy / c->dy;
  c->lapy[2] = +1. / c->dy / c->dy;
  c->lapz[0] = +1. / c->dz / c->dz;
  c->lapz[1] = -2. / c->dz / c->dz;
  c->lapz[2] = +1. / c->dz / c->dz;
  c->x1pncl = dalloc((long)nx * ny * nz);
  c->tdm_l = dalloc(nx);
  c->tdm_c = dalloc(nx);
  c->tdm_u = dalloc(nx);
  c->tdm_v = dalloc(nx);
  const int nky = ny / 2 + 1;
  c->spec = dalloc(2L * nx * nky * nz);
  c->line = dalloc(2L * (ny > nz ? ny : nz) + 2);
  c->plan_y = svof_fft_plan_create((size_t)ny);
  c->plan_z = svof_fft_plan_create((size_t)nz);
  c->evy = dalloc(nky);
  c->evz = dalloc(nz);
  for (size_t j = 0; j < (size_t)nky; j++) {
    c->evy[j] = -4. / pow(prm->ly / ny, 2.) * pow(sin(G_PI * j / (double)ny), 2.);
  }
  for (size_t k = 0; k < (size_t)nz; k++) {
    c->evz[k] = -4. / pow(prm->lz / nz, 2.) * pow(sin(G_PI * k / (double)nz), 2.);
  }
  c->pl = dalloc(nx);
  c->pu = dalloc(nx);
  for (int i = 1; i <= nx; i++) {
    c->pl[i - 1] = 1. / DXC(i) / DXF(i);
    c->pu[i - 1] = 1. / DXC(i + 1) / DXF(i);
  }
  return c;
}

void svo3_destroy(svo3_ctx_t *c) {
  if (c)
    for (int q = 0; q < 9; q++) free(c->stat[q]);
  if (!c) return;
  double *bufs[] = {c->xf, c->xc, c->dxf, c->dxc, c->ux, c->uy, c->uz, c->p, c->psi, c->t, c->vof,
                    c->ifrcx, c->ifrcy, c->ifrcz, c->dvof, c->normal, c->curv, c->flxx, c->flxy, c->flxz,
                    c->src[0], c->src[1], c->lapx_ux, c->lapx_cc, c->x1pncl, c->tdm_l, c->tdm_c, c->tdm_u,
                    c->tdm_v, c->spec, c->line, c->evy, c->evz, c->pl, c->pu};
  for (size_t k = 0; k < sizeof(bufs) / sizeof(bufs[0]); k++) free(bufs[k]);
  for (int k = 0; k < 3; k++) {
    free(c->srcux[k]);
    free(c->srcuy[k]);
    free(c->srcuz[k]);
    free(c->srct[k]);
  }
  svof_fft_plan_destroy(c->plan_y);
  svof_fft_plan_destroy(c->plan_z);
  free(c);
}

double *svo3_field(svo3_ctx_t *c, const char *name, long *count) {
  struct { const char *n; double *p; long k; } tab[] = {
    {"ux", c->ux, c->n_ux}, {"uy", c->uy, c->n_cc}, {"uz", c->uz, c->n_cc}, {"p", c->p, c->n_cc},
    {"psi", c->psi, c->n_cc}, {"t", c->t, c->n_cc}, {"vof", c->vof, c->n_vof}, {"curv", c->curv, c->n_cc},
    {"normal", c->normal, c->n_normal}, {"dvof", c->dvof, c->n_dvof}, {"ifrcx", c->ifrcx, c->n_srcx},
    {"ifrcy", c->ifrcy, c->n_src}, {"ifrcz", c->ifrcz, c->n_src}, {"srcux0", c->srcux[0], c->n_srcx},
    {"srcuy0", c->srcuy[0], c->n_src}, {"srcuz0", c->srcuz[0], c->n_src}, {"srct0", c->srct[0], c->n_src},
    {"srcux1", c->srcux[1], c->n_srcx}, {"srcuy1", c->srcuy[1], c->n_src}, {"srcuz1", c->srcuz[1], c->n_src},
    {"srct1", c->srct[1], c->n_src}, {"src0", c->src[0], c->n_src}, {"src1", c->src[1], c->n_src},
  };
  for (size_t k = 0; k < sizeof(tab) / sizeof(tab[0]); k++) {
    if (0 == strcmp(name, tab[k].n)) {
      if (count) *count = tab[k].k;
      return tab[k].p;
    }
  }
  if (count) *count = -1;
  return NULL;
}

/* ---------------- boundaries: y halo on the interior z planes, then z halo on
 * whole planes, then the x wall values of the interior rows */
static void halo_yz(double *a, long w, int nh, int ny, int nz) {
  const long rows = ny + 2 * nh;
  const long plane = w * rows;
  for (int k = nh; k < nh + nz; k++) {
    double *pl = a + plane * k;
    memmove(pl, pl + w * ny, sizeof(double) * (size_t)(w * nh));
    memmove(pl + w * (ny + nh), pl + w * nh, sizeof(double) * (size_t)(w * nh));
  }
  memmove(a, a + plane * nz, sizeof(double) * (size_t)(plane * nh));
  memmove(a + plane * (nz + nh), a + plane * nh, sizeof(double) * (size_t)(plane * nh));
}

enum { W_ZERO, W_DIRICHLET, W_NEUMANN };

static void walls(svo3_ctx_t *c, double *a, long w, int nh, int kind, double lo, double hi) {
  const long rows = NY + 2 * nh;
  for (int k = nh; k < nh + NZ; k++) {
    for (int j = nh; j < nh + NY; j++) {
      double *r = a + w * (j + rows * k);
      if (W_ZERO == kind) {
        r[0] = 0.;
        r[w - 1] = 0.;
      } else if (W_DIRICHLET == kind) {
        r[0] = lo;
        r[w - 1] = hi;
      } else {
        r[0] = r[1];
        r[w - 1] = r[w - 2];
      }
    }
  }
}

static void bc_ux(svo3_ctx_t *c) {
  halo_yz(c->ux, NX + 1, 1, NY, NZ);
  walls(c, c->ux, NX + 1, 1, W_ZERO, 0., 0.);
}
static void bc_uy(svo3_ctx_t *c) {
  halo_yz(c->uy, NX + 2, 1, NY, NZ);
  walls(c, c->uy, NX + 2, 1, W_DIRICHLET, c->prm.uy_xm, c->prm.uy_xp);
}
static void bc_uz(svo3_ctx_t *c) {
  halo_yz(c->uz, NX + 2, 1, NY, NZ);
  walls(c, c->uz, NX + 2, 1, W_DIRICHLET, c->prm.uz_xm, c->prm.uz_xp);
}
static void bc_t(svo3_ctx_t *c) {
  halo_yz(c->t, NX + 2, 1, NY, NZ);
  walls(c, c->t, NX + 2, 1, W_DIRICHLET, c->prm.t_xm, c->prm.t_xp);
}
static void bc_neumann(svo3_ctx_t *c, double *a) {
  halo_yz(a, NX + 2, 1, NY, NZ);
  walls(c, a, NX + 2, 1, W_NEUMANN, 0., 0.);
}
static void bc_vof(svo3_ctx_t *c) {
  halo_yz(c->vof, NX + 2, 2, NY, NZ);
  const long n = (long)(NY + 4) * (NZ + 4);
  for (long r = 0; r < n; r++) {
    c->vof[(NX + 2) * r] = 0.;
    c->vof[(NX + 2) * r + NX + 1] = 0.;
  }
}

int svo3_init_boundaries(svo3_ctx_t *c) {
  bc_ux(c);
  bc_uy(c);
  bc_uz(c);
  bc_neumann(c, c->p);
  bc_t(c);
  bc_vof(c);
  return 0;
}

/* ---------------- time step */
int svo3_decide_dt(svo3_ctx_t *c, double *dt) {
  const double small = 1.e-8;
  double dta = 1.;
  for (int k = 1; k <= NZ; k++)
    for (int j = 1; j <= NY; j++)
      for (int i = 2; i <= NX; i++) dta = fmin(dta, DXC(i) / (fabs(UX(i, j, k)) + small));
  for (int k = 1; k <= NZ; k++)
    for (int j = 1; j <= NY; j++)
      for (int i = 1; i <= NX; i++) dta = fmin(dta, c->dy / (fabs(CC(c->uy, i, j, k)) + small));
  for (int k = 1; k <= NZ; k++)
    for (int j = 1; j <= NY; j++)
      for (int i = 1; i <= NX; i++) dta = fmin(dta, c->dz / (fabs(CC(c->uz, i, j, k)) + small));
  dta *= c->prm.coef_dt_adv;
  const int ndims = 3;
  const double cd = c->prm.coef_dt_dif;
  double r = dta;
  r = fmin(r, cd / c->prm.m_dif * 0.5 / ndims * pow(c->dy, 2.));
  r = fmin(r, cd / c->prm.m_dif * 0.5 / ndims * pow(c->dz, 2.));
  r = fmin(r, cd / c->prm.t_dif * 0.5 / ndims * pow(c->dy, 2.));
  r = fmin(r, cd / c->prm.t_dif * 0.5 / ndims * pow(c->dz, 2.));
  *dt = r;
  return 0;
}

/* ---------------- interface geometry */
static double plane_dx(const double v00, const double v10, const double v01, const double v11) {
  return -v00 + v10 - v01 + v11;
}
static double plane_dy(const double v00, const double v10, const double v01, const double v11) {
  return -v00 - v10 + v01 + v11;
}
static double plane_sum(const double v00, const double v10, const double v01, const double v11) {
  return +v00 + v10 + v01 + v11;
}

static void compute_gradient(svo3_ctx_t *c) {
  for (int k = 0; k <= NZ + 2; k++) {
    for (int j = 0; j <= NY + 2; j++) {
      for (int i = 1; i <= NX + 1; i++) {
        double a[2][4];
        for (int q = 0; q < 2; q++) {
          const int kk = k - 1 + q;
          a[q][0] = VOF(i - 1, j - 1, kk);
          a[q][1] = VOF(i, j - 1, kk);
          a[q][2] = VOF(i - 1, j, kk);
          a[q][3] = VOF(i, j, kk);
        }
        const double dvofdx = 1. / DXC(i) * (plane_dx(a[0][0], a[0][1], a[0][2], a[0][3]) +
                                             plane_dx(a[1][0], a[1][1], a[1][2], a[1][3]));
        const double dvofdy = 1. / c->dy * (plane_dy(a[0][0], a[0][1], a[0][2], a[0][3]) +
                                            plane_dy(a[1][0], a[1][1], a[1][2], a[1][3]));
        const double dvofdz = 1. / c->dz * (plane_sum(a[1][0], a[1][1], a[1][2], a[1][3]) -
                                            plane_sum(a[0][0], a[0][1], a[0][2], a[0][3]));
        const double norm = sqrt(+dvofdx * dvofdx + dvofdy * dvofdy + dvofdz * dvofdz);
        const double norminv = 1. / fmax(norm, DBL_EPSILON);
        DVOF(i, j, k, 0) = dvofdx * norminv;
        DVOF(i, j, k, 1) = dvofdy * norminv;
        DVOF(i, j, k, 2) = dvofdz * norminv;
      }
    }
  }
}

static double compute_intercept3(const double vof, const double n0, const double n1, const double n2) {
  const int cntmax = 8;
  const double resmax = 1.e-12;
  double exps[8];
  for (int kk = 0; kk < 2; kk++)
    for (int jj = 0; jj < 2; jj++)
      for (int ii = 0; ii < 2; ii++)
        exps[(kk * 2 + jj) * 2 + ii] =
            exp(-2. * VOFBETA * (+n0 * GAUSS_P[ii] + n1 * GAUSS_P[jj] + n2 * GAUSS_P[kk]));
  double val = 1. / vof - 1.;
  for (int cnt = 0; cnt < cntmax; cnt++) {
    double f0 = -1. * vof;
    double f1 = 0.;
    for (int kk = 0; kk < 2; kk++) {
      for (int jj = 0; jj < 2; jj++) {
        for (int ii = 0; ii < 2; ii++) {
          const double weight = GAUSS_W[ii] * GAUSS_W[jj] * GAUSS_W[kk];
          const double p = exps[(kk * 2 + jj) * 2 + ii];
          const double denom = 1. / (1. + p * val);
          f0 += weight * denom;
          f1 -= weight * p * denom * denom;
        }
      }
    }
    val -= f0 / f1;
    if (fabs(f0) < resmax) break;
  }
  return -0.5 / VOFBETA * log(val);
}

static void compute_normal(svo3_ctx_t *c) {
  for (int k = 0; k <= NZ + 1; k++) {
    for (int j = 0; j <= NY + 1; j++) {
      for (int i = 1; i <= NX; i++) {
        const double lvof = VOF(i, j, k);
        if (lvof < VOFMIN || 1. - VOFMIN < lvof) continue;
        double n[3];
        for (int m = 0; m < 3; m++) {
          n[m] = plane_sum(DVOF(i, j, k, m), DVOF(i + 1, j, k, m), DVOF(i, j + 1, k, m), DVOF(i + 1, j + 1, k, m)) +
                 plane_sum(DVOF(i, j, k + 1, m), DVOF(i + 1, j, k + 1, m), DVOF(i, j + 1, k + 1, m),
                           DVOF(i + 1, j + 1, k + 1, m));
        }
        n[0] /= DXF(i);
        n[1] /= c->dy;
        n[2] /= c->dz;
        const double norm = sqrt(+n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        const double norminv = 1. / fmax(norm, DBL_EPSILON);
        n[0] *= norminv;
        n[1] *= norminv;
        n[2] *= norminv;
        NRM(i, j, k, 0) = n[0];
        NRM(i, j, k, 1) = n[1];
        NRM(i, j, k, 2) = n[2];
        NRM(i, j, k, 3) = compute_intercept3(lvof, n[0], n[1], n[2]);
      }
    }
  }
}

static void compute_curvature(svo3_ctx_t *c) {
  for (int k = 0; k <= NZ + 1; k++) {
    for (int j = 0; j <= NY + 1; j++) {
      for (int i = 1; i <= NX; i++) {
        const double dnxdx =
            1. / DXF(i) * (plane_dx(DVOF(i, j, k, 0), DVOF(i + 1, j, k, 0), DVOF(i, j + 1, k, 0), DVOF(i + 1, j + 1, k, 0)) +
                           plane_dx(DVOF(i, j, k + 1, 0), DVOF(i + 1, j, k + 1, 0), DVOF(i, j + 1, k + 1, 0),
                                    DVOF(i + 1, j + 1, k + 1, 0)));
        const double dnydy =
            1. / c->dy * (plane_dy(DVOF(i, j, k, 1), DVOF(i + 1, j, k, 1), DVOF(i, j + 1, k, 1), DVOF(i + 1, j + 1, k, 1)) +
                          plane_dy(DVOF(i, j, k + 1, 1), DVOF(i + 1, j, k + 1, 1), DVOF(i, j + 1, k + 1, 1),
                                   DVOF(i + 1, j + 1, k + 1, 1)));
        const double dnzdz =
            1. / c->dz * (plane_sum(DVOF(i, j, k + 1, 2), DVOF(i + 1, j, k + 1, 2), DVOF(i, j + 1, k + 1, 2),
                                    DVOF(i + 1, j + 1, k + 1, 2)) -
                          plane_sum(DVOF(i, j, k, 2), DVOF(i + 1, j, k, 2), DVOF(i, j + 1, k, 2), DVOF(i + 1, j + 1, k, 2)));
        CC(c->curv, i, j, k) = 0.25 * (-dnxdx - dnydy - dnzdz);
      }
    }
  }
}

int svo3_curvature_tensor(svo3_ctx_t *c) {
  compute_gradient(c);
  compute_normal(c);
  compute_curvature(c);
  return 0;
}

int svo3_force(svo3_ctx_t *c) {
  const double tension = c->prm.tension;
  for (int k = 1; k <= NZ; k++) {
    for (int j = 1; j <= NY; j++) {
      for (int i = 1; i <= NX; i++) {
        const double vc = VOF(i, j, k), cc = CC(c->curv, i, j, k);
        if (i >= 2) {
          const double grad = 1. / DXC(i) * (-VOF(i - 1, j, k) + vc);
          const double kappa = 0.5 * (+CC(c->curv, i - 1, j, k) + cc);
          SRCX(c->ifrcx, i, j, k) = tension * grad * kappa;
        }
        {
          const double grad = 1. / c->dy * (-VOF(i, j - 1, k) + vc);
          const double kappa = 0.5 * (+CC(c->curv, i, j - 1, k) + cc);
          SRC(c->ifrcy, i, j, k) = tension * grad * kappa;
        }
        {
          const double grad = 1. / c->dz * (-VOF(i, j, k - 1) + vc);
          const double kappa = 0.5 * (+CC(c->curv, i, j, k - 1) + cc);
          SRC(c->ifrcz, i, j, k) = tension * grad * kappa;
        }
      }
    }
  }
  return 0;
}

/* ---------------- vof update */
static double indicator3(const double *n, const double x0, const double x1, const double x2) {
  return 1. / (1. + exp(-2. * VOFBETA * (+n[0] * x0 + n[1] * x1 + n[2] * x2 + n[3])));
}

int svo3_update_vof(svo3_ctx_t *c, int rkstep, double dt) {
  if (0 != rkstep) {
    double *tmp = c->src[0];
    c->src[0] = c->src[1];
    c->src[1] = tmp;
  }
  memset(c->src[0], 0, sizeof(double) * (size_t)c->n_src);
  for (int k = 1; k <= NZ; k++) {
    for (int j = 1; j <= NY; j++) {
      for (int i = 2; i <= NX; i++) {
        const double vel = UX(i, j, k);
        const int ii = vel < 0. ? i : i - 1;
        const double x = vel < 0. ? -0.5 : +0.5;
        const double lvof = VOF(ii, j, k);
        if (lvof < VOFMIN || 1. - VOFMIN < lvof) {
          FLXX(i, j, k) = vel * lvof;
          continue;
        }
        double flux = 0.;
        for (int kk = 0; kk < 2; kk++)
          for (int jj = 0; jj < 2; jj++)
            flux += GAUSS_W[jj] * GAUSS_W[kk] * indicator3(&NRM(ii, j, k, 0), x, GAUSS_P[jj], GAUSS_P[kk]);
        FLXX(i, j, k) = vel * flux;
      }
    }
  }
  for (int k = 1; k <= NZ; k++) {
    for (int j = 1; j <= NY + 1; j++) {
      for (int i = 1; i <= NX; i++) {
        const double vel = CC(c->uy, i, j, k);
        const int jj = vel < 0. ? j : j - 1;
        const double y = vel < 0. ? -0.5 : +0.5;
        const double lvof = VOF(i, jj, k);
        if (lvof < VOFMIN || 1. - VOFMIN < lvof) {
          FLXY(i, j, k) = vel * lvof;
          continue;
        }
        double flux = 0.;
        for (int kk = 0; kk < 2; kk++)
          for (int ii = 0; ii < 2; ii++)
            flux += GAUSS_W[ii] * GAUSS_W[kk] * indicator3(&NRM(i, jj, k, 0), GAUSS_P[ii], y, GAUSS_P[kk]);
        FLXY(i, j, k) = vel * flux;
      }
    }
  }
  for (int k = 1; k <= NZ + 1; k++) {
    for (int j = 1; j <= NY; j++) {
      for (int i = 1; i <= NX; i++) {
        const double vel = CC(c->uz, i, j, k);
        const int kk = vel < 0. ? k : k - 1;
        const double z = vel < 0. ? -0.5 : +0.5;
        const double lvof = VOF(i, j, kk);
        if (lvof < VOFMIN || 1. - VOFMIN < lvof) {
          FLXZ(i, j, k) = vel * lvof;
          continue;
        }
        double flux = 0.;
        for (int jj = 0; jj < 2; jj++)
          for (int ii = 0; ii < 2; ii++)
            flux += GAUSS_W[ii] * GAUSS_W[jj] * indicator3(&NRM(i, j, kk, 0), GAUSS_P[ii], GAUSS_P[jj], z);
        FLXZ(i, j, k) = vel * flux;
      }
    }
  }
  for (int k = 1; k <= NZ; k++) {
    for (int j = 1; j <= NY; j++) {
      for (int i = 1; i <= NX; i++) {
        double s = 0.;
        s += 1. / DXF(i) * (+FLXX(i, j, k) - FLXX(i + 1, j, k));
        s += 1. / c->dy * (+FLXY(i, j, k) - FLXY(i, j + 1, k));
        s += 1. / c->dz * (+FLXZ(i, j, k) - FLXZ(i, j, k + 1));
        SRC(c->src[0], i, j, k) = s;
        double v = VOF(i, j, k);
        v += dt * RK_A[rkstep] * s;
        if (0 != rkstep) v += dt * RK_B[rkstep] * SRC(c->src[1], i, j, k);
        VOF(i, j, k) = v;
      }
    }
  }
  bc_vof(c);
  return 0;
}

/* ---------------- Thomas */
static void gtsv(const int n, const double *l, const double *cc, const double *u, double *v, double *q,
                 const int stride) {
#define Q(i) q[(size_t)(i) * stride]
  v[0] = u[0] / cc[0];
  Q(0) = Q(0) / cc[0];
  for (int i = 1; i < n - 1; i++) {
    const double val = 1. / (cc[i] - l[i] * v[i - 1]);
    v[i] = val * (u[i]);
    Q(i) = val * (Q(i) - l[i] * Q(i - 1));
  }
  const double val = cc[n - 1] - l[n - 1] * v[n - 2];
  Q(n - 1) = fabs(val) > DBL_EPSILON ? 1. / val * (Q(n - 1) - l[n - 1] * Q(n - 2)) : 0.;
  for (int i = n - 2; i >= 0; i--) Q(i) -= v[i] * Q(i + 1);
#undef Q
}

/* ---------------- momentum / scalar predictor */
static void swap_reset(double **s, long n, int rkstep) {
  if (0 != rkstep) {
    double *tmp = s[0];
    s[0] = s[1];
    s[1] = tmp;
  }
  memset(s[0], 0, sizeof(double) * (size_t)n);
  memset(s[2], 0, sizeof(double) * (size_t)n);
}

static void rhs_all(svo3_ctx_t *c) {
  const double dy = c->dy, dz = c->dz, md = c->prm.m_dif, td = c->prm.t_dif;
  const double *uy = c->uy, *uz = c->uz, *p = c->p, *t = c->t;
  const double *ly = c->lapy, *lz = c->lapz;
  for (int k = 1; k <= NZ; k++) {
    for (int j = 1; j <= NY; j++) {
      for (int i = 1; i <= NX; i++) {
        const double dxf = DXF(i);
        if (i >= 2) {  /* ux */
          const double dxc = DXC(i);
          const double xm = UX(i - 1, j, k), xc = UX(i, j, k), xp = UX(i + 1, j, k);
          const double ys = UX(i, j - 1, k), yn = UX(i, j + 1, k), zs = UX(i, j, k - 1), zn = UX(i, j, k + 1);
          double sa = 0., sg = 0.;
          {
            const double ul = +0.5 * xm + 0.5 * xc, uu = +0.5 * xc + 0.5 * xp;
            const double l = +0.5 / dxc * ul, u = -0.5 / dxc * uu, cc = -l - u;
            sa += +l * xm + cc * xc + u * xp;
          }
          const double w_xm = 0.5 * DXF(i - 1) / dxc, w_xp = 0.5 * dxf / dxc;
          {
            const double ul = w_xm * CC(uy, i - 1, j, k) + w_xp * CC(uy, i, j, k);
            const double uu = w_xm * CC(uy, i - 1, j + 1, k) + w_xp * CC(uy, i, j + 1, k);
            const double l = +0.5 / dy * ul, u = -0.5 / dy * uu, cc = -l - u;
            sa += +l * ys + cc * xc + u * yn;
          }
          {
            const double ul = w_xm * CC(uz, i - 1, j, k) + w_xp * CC(uz, i, j, k);
            const double uu = w_xm * CC(uz, i - 1, j, k + 1) + w_xp * CC(uz, i, j, k + 1);
            const double l = +0.5 / dz * ul, u = -0.5 / dz * uu, cc = -l - u;
            sa += +l * zs + cc * xc + u * zn;
          }
          const double *lx = c->lapx_ux + 3 * (i - 2);
          sg += md * (+lx[0] * xm + lx[1] * xc + lx[2] * xp);
          sa += md * (+ly[0] * ys + ly[1] * xc + ly[2] * yn);
          sa += md * (+lz[0] * zs + lz[1] * xc + lz[2] * zn);
          sg -= 1. / dxc * (-CC(p, i - 1, j, k) + CC(p, i, j, k));
          if (c->prm.add_buoyancy) sa += +0.5 * CC(t, i - 1, j, k) + 0.5 * CC(t, i, j, k);
          sa += SRCX(c->ifrcx, i, j, k);
          SRCX(c->srcux[0], i, j, k) = sa;
          SRCX(c->srcux[2], i, j, k) = sg;
        }
        const double *lx = c->lapx_cc + 3 * (i - 1);
        {  /* uy */
          const double xm = CC(uy, i - 1, j, k), xc = CC(uy, i, j, k), xp = CC(uy, i + 1, j, k);
          const double ys = CC(uy, i, j - 1, k), yn = CC(uy, i, j + 1, k);
          const double zs = CC(uy, i, j, k - 1), zn = CC(uy, i, j, k + 1);
          double sa = 0., sg = 0.;
          {
            const double ul = +0.5 * UX(i, j - 1, k) + 0.5 * UX(i, j, k);
            const double uu = +0.5 * UX(i + 1, j - 1, k) + 0.5 * UX(i + 1, j, k);
            const double l = +0.5 / dxf * ul, u = -0.5 / dxf * uu, cc = -l - u;
            sa += +l * xm + cc * xc + u * xp;
          }
          {
            const double ul = +0.5 * ys + 0.5 * xc, uu = +0.5 * xc + 0.5 * yn;
            const double l = +0.5 / dy * ul, u = -0.5 / dy * uu, cc = -l - u;
            sa += +l * ys + cc * xc + u * yn;
          }
          {
            const double ul = +0.5 * CC(uz, i, j - 1, k) + 0.5 * CC(uz, i, j, k);
            const double uu = +0.5 * CC(uz, i, j - 1, k + 1) + 0.5 * CC(uz, i, j, k + 1);
            const double l = +0.5 / dz * ul, u = -0.5 / dz * uu, cc = -l - u;
            sa += +l * zs + cc * xc + u * zn;
          }
          sg += md * (+lx[0] * xm + lx[1] * xc + lx[2] * xp);
          sa += md * (+ly[0] * ys + ly[1] * xc + ly[2] * yn);
          sa += md * (+lz[0] * zs + lz[1] * xc + lz[2] * zn);
          sg -= 1. / dy * (-CC(p, i, j - 1, k) + CC(p, i, j, k));
          sa += SRC(c->ifrcy, i, j, k);
          /* extension: buoyancy of the volume fraction, the face value of
           * vof averaged from the two cells beside the uy face (the vof
           * after this substep's advection, as in 2D) */
          if (0. != c->grav_vof) sa += c->grav_vof * (0.5 * VOF(i, j - 1, k) + 0.5 * VOF(i, j, k) - c->vof_ref);
          SRC(c->srcuy[0], i, j, k) = sa;
          SRC(c->srcuy[2], i, j, k) = sg;
        }
        {  /* uz */
          const double xm = CC(uz, i - 1, j, k), xc = CC(uz, i, j, k), xp = CC(uz, i + 1, j, k);
          const double ys = CC(uz, i, j - 1, k), yn = CC(uz, i, j + 1, k);
          const double zs = CC(uz, i, j, k - 1), zn = CC(uz, i, j, k + 1);
          double sa = 0., sg = 0.;
          {
            const double ul = +0.5 * UX(i, j, k - 1) + 0.5 * UX(i, j, k);
            const double uu = +0.5 * UX(i + 1, j, k - 1) + 0.5 * UX(i + 1, j, k);
            const double l = +0.5 / dxf * ul, u = -0.5 / dxf * uu, cc = -l - u;
            sa += +l * xm + cc * xc + u * xp;
          }
          {
            const double ul = +0.5 * CC(uy, i, j, k - 1) + 0.5 * CC(uy, i, j, k);
            const double uu = +0.5 * CC(uy, i, j + 1, k - 1) + 0.5 * CC(uy, i, j + 1, k);
            const double l = +0.5 / dy * ul, u = -0.5 / dy * uu, cc = -l - u;
            sa += +l * ys + cc * xc + u * yn;
          }
          {
            const double ul = +0.5 * zs + 0.5 * xc, uu = +0.5 * xc + 0.5 * zn;
            const double l = +0.5 / dz * ul, u = -0.5 / dz * uu, cc = -l - u;
            sa += +l * zs + cc * xc + u * zn;
          }
          sg += md * (+lx[0] * xm + lx[1] * xc + lx[2] * xp);
          sa += md * (+ly[0] * ys + ly[1] * xc + ly[2] * yn);
          sa += md * (+lz[0] * zs + lz[1] * xc + lz[2] * zn);
          sg -= 1. / dz * (-CC(p, i, j, k - 1) + CC(p, i, j, k));
          sa += SRC(c->ifrcz, i, j, k);
          SRC(c->srcuz[0], i, j, k) = sa;
          SRC(c->srcuz[2], i, j, k) = sg;
        }
        {  /* t */
          const double xm = CC(t, i - 1, j, k), xc = CC(t, i, j, k), xp = CC(t, i + 1, j, k);
          const double ys = CC(t, i, j - 1, k), yn = CC(t, i, j + 1, k);
          const double zs = CC(t, i, j, k - 1), zn = CC(t, i, j, k + 1);
          double sa = 0., sg = 0.;
          {
            const double l = +0.5 / dxf * UX(i, j, k), u = -0.5 / dxf * UX(i + 1, j, k), cc = -l - u;
            sa += +l * xm + cc * xc + u * xp;
          }
          {
            const double l = +0.5 / dy * CC(uy, i, j, k), u = -0.5 / dy * CC(uy, i, j + 1, k), cc = -l - u;
            sa += +l * ys + cc * xc + u * yn;
          }
          {
            const double l = +0.5 / dz * CC(uz, i, j, k), u = -0.5 / dz * CC(uz, i, j, k + 1), cc = -l - u;
            sa += +l * zs + cc * xc + u * zn;
          }
          sg += td * (+lx[0] * xm + lx[1] * xc + lx[2] * xp);
          sa += td * (+ly[0] * ys + ly[1] * xc + ly[2] * yn);
          sa += td * (+lz[0] * zs + lz[1] * xc + lz[2] * zn);
          SRC(c->srct[0], i, j, k) = sa;
          SRC(c->srct[2], i, j, k) = sg;
        }
      }
    }
  }
}

static void predict_field(svo3_ctx_t *c, double *const *s, const long nitems, const int n, const double *lapx,
                          const double dif, const int rkstep, const double dt) {
  const double ca = RK_A[rkstep], cb = RK_B[rkstep], cg = rk_g(rkstep);
  for (long m = 0; m < nitems; m++) c->x1pncl[m] = +ca * dt * s[0][m] + cb * dt * s[1][m] + cg * dt * s[2][m];
  const double prefactor = 0.5 * cg * dt * dif;
  for (int i = 0; i < n; i++) {
    c->tdm_l[i] = -prefactor * lapx[3 * i + 0];
    c->tdm_c[i] = 1. - prefactor * lapx[3 * i + 1];
    c->tdm_u[i] = -prefactor * lapx[3 * i + 2];
  }
  for (long line = 0; line < (long)NY * NZ; line++) {
    gtsv(n, c->tdm_l, c->tdm_c, c->tdm_u, c->tdm_v, c->x1pncl + line * n, 1);
  }
}

int svo3_predict(svo3_ctx_t *c, int rkstep, double dt) {
  swap_reset(c->srcux, c->n_srcx, rkstep);
  swap_reset(c->srcuy, c->n_src, rkstep);
  swap_reset(c->srcuz, c->n_src, rkstep);
  swap_reset(c->srct, c->n_src, rkstep);
  rhs_all(c);
  /* ux */
  predict_field(c, c->srcux, c->n_srcx, NX - 1, c->lapx_ux, c->prm.m_dif, rkstep, dt);
  for (int k = 1; k <= NZ; k++)
    for (int j = 1; j <= NY; j++)
      for (int i = 2; i <= NX; i++) UX(i, j, k) += SRCX(c->x1pncl, i, j, k);
  bc_ux(c);
  predict_field(c, c->srcuy, c->n_src, NX, c->lapx_cc, c->prm.m_dif, rkstep, dt);
  for (int k = 1; k <= NZ; k++)
    for (int j = 1; j <= NY; j++)
      for (int i = 1; i <= NX; i++) CC(c->uy, i, j, k) += SRC(c->x1pncl, i, j, k);
  bc_uy(c);
  predict_field(c, c->srcuz, c->n_src, NX, c->lapx_cc, c->prm.m_dif, rkstep, dt);
  for (int k = 1; k <= NZ; k++)
    for (int j = 1; j <= NY; j++)
      for (int i = 1; i <= NX; i++) CC(c->uz, i, j, k) += SRC(c->x1pncl, i, j, k);
  bc_uz(c);
  predict_field(c, c->srct, c->n_src, NX, c->lapx_cc, c->prm.t_dif, rkstep, dt);
  for (int k = 1; k <= NZ; k++)
    for (int j = 1; j <= NY; j++)
      for (int i = 1; i <= NX; i++) CC(c->t, i, j, k) += SRC(c->x1pncl, i, j, k);
  bc_t(c);
  return 0;
}

/* ---------------- Poisson: r2c y, c2c z, complex Thomas x; spec[kz][i][ky] */
int svo3_potential(svo3_ctx_t *c, int rkstep, double dt) {
  const int nx = NX, ny = NY, nz = NZ, nky = ny / 2 + 1;
  const double prefactor = 1. / (rk_g(rkstep) * dt) / (1. * ny * nz);
  double *line = c->line;
  double *rhs = c->x1pncl;  /* ny reals per (i, k) */
  /* right-hand side and r2c along y, for each (i, k) */
  for (int k = 1; k <= nz; k++) {
    for (int i = 1; i <= nx; i++) {
      for (int j = 1; j <= ny; j++) {
        const double dx = DXF(i);
        rhs[j - 1] = prefactor * (+(UX(i + 1, j, k) - UX(i, j, k)) / dx +
                                  (CC(c->uy, i, j + 1, k) - CC(c->uy, i, j, k)) / c->dy +
                                  (CC(c->uz, i, j, k + 1) - CC(c->uz, i, j, k)) / c->dz);
      }
      svof_fft_r2c(c->plan_y, rhs, c->spec + 2 * ((size_t)(k - 1) * nx * nky + (size_t)(i - 1) * nky));
    }
  }
  /* forward DFT along z for each (i, ky) */
  for (int i = 0; i < nx; i++) {
    for (int ky = 0; ky < nky; ky++) {
      for (int k = 0; k < nz; k++) {
        const size_t o = 2 * ((size_t)k * nx * nky + (size_t)i * nky + ky);
        line[2 * k] = c->spec[o];
        line[2 * k + 1] = c->spec[o + 1];
      }
      svof_fft_c2c(c->plan_z, line, -1);
      for (int k = 0; k < nz; k++) {
        const size_t o = 2 * ((size_t)k * nx * nky + (size_t)i * nky + ky);
        c->spec[o] = line[2 * k];
        c->spec[o + 1] = line[2 * k + 1];
      }
    }
  }
  /* complex Neumann Thomas along x for each (ky, kz) */
  for (int kz = 0; kz < nz; kz++) {
    for (int ky = 0; ky < nky; ky++) {
      const double lam = c->evy[ky] + c->evz[kz];
      for (int n = 0; n < nx; n++) c->tdm_c[n] = -c->pl[n] - c->pu[n] + lam;
      c->tdm_c[0] += c->pl[0];
      c->tdm_c[nx - 1] += c->pu[nx - 1];
      double *q = c->spec + 2 * ((size_t)kz * nx * nky + ky);
      gtsv(nx, c->pl, c->tdm_c, c->pu, c->tdm_v, q + 0, 2 * nky);
      gtsv(nx, c->pl, c->tdm_c, c->pu, c->tdm_v, q + 1, 2 * nky);
    }
  }
  /* backward DFT along z */
  for (int i = 0; i < nx; i++) {
    for (int ky = 0; ky < nky; ky++) {
      for (int k = 0; k < nz; k++) {
        const size_t o = 2 * ((size_t)k * nx * nky + (size_t)i * nky + ky);
        line[2 * k] = c->spec[o];
        line[2 * k + 1] = c->spec[o + 1];
      }
      svof_fft_c2c(c->plan_z, line, +1);
      for (int k = 0; k < nz; k++) {
        const size_t o = 2 * ((size_t)k * nx * nky + (size_t)i * nky + ky);
        c->spec[o] = line[2 * k];
        c->spec[o + 1] = line[2 * k + 1];
      }
    }
  }
  /* c2r along y and psi */
  for (int k = 1; k <= nz; k++) {
    for (int i = 1; i <= nx; i++) {
      svof_fft_c2r(c->plan_y, c->spec + 2 * ((size_t)(k - 1) * nx * nky + (size_t)(i - 1) * nky), rhs);
      for (int j = 1; j <= ny; j++) CC(c->psi, i, j, k) = rhs[j - 1];
    }
  }
  bc_neumann(c, c->psi);
  return 0;
}

int svo3_correct(svo3_ctx_t *c, int rkstep, double dt) {
  const double prefactor = rk_g(rkstep) * dt;
  for (int k = 1; k <= NZ; k++)
    for (int j = 1; j <= NY; j++)
      for (int i = 2; i <= NX; i++)
        UX(i, j, k) -= prefactor / DXC(i) * (+CC(c->psi, i, j, k) - CC(c->psi, i - 1, j, k));
  bc_ux(c);
  for (int k = 1; k <= NZ; k++)
    for (int j = 1; j <= NY; j++)
      for (int i = 1; i <= NX; i++)
        CC(c->uy, i, j, k) -= prefactor / c->dy * (+CC(c->psi, i, j, k) - CC(c->psi, i, j - 1, k));
  bc_uy(c);
  for (int k = 1; k <= NZ; k++)
    for (int j = 1; j <= NY; j++)
      for (int i = 1; i <= NX; i++)
        CC(c->uz, i, j, k) -= prefactor / c->dz * (+CC(c->psi, i, j, k) - CC(c->psi, i, j, k - 1));
  bc_uz(c);
  return 0;
}

int svo3_update_pressure(svo3_ctx_t *c, int rkstep, double dt) {
  const double prefactor = 0.5 * rk_g(rkstep) * dt * c->prm.m_dif;
  for (int k = 1; k <= NZ; k++) {
    for (int j = 1; j <= NY; j++) {
      for (int i = 1; i <= NX; i++) {
        const double psc = CC(c->psi, i, j, k);
        double v = CC(c->p, i, j, k);
        v += psc;
        const double dm = (-CC(c->psi, i - 1, j, k) + psc) / DXC(i);
        const double dp = (-psc + CC(c->psi, i + 1, j, k)) / DXC(i + 1);
        v -= prefactor / DXF(i) * (-dm + dp);
        CC(c->p, i, j, k) = v;
      }
    }
  }
  bc_neumann(c, c->p);
  return 0;
}

int svo3_integrate(svo3_ctx_t *c, double *dt) {
  svo3_decide_dt(c, dt);
  for (int rk = 0; rk < 3; rk++) {
    svo3_curvature_tensor(c);
    svo3_force(c);
    svo3_update_vof(c, rk, *dt);
    svo3_predict(c, rk, *dt);
    svo3_potential(c, rk, *dt);
    svo3_correct(c, rk, *dt);
    svo3_update_pressure(c, rk, *dt);
  }
  return 0;
}

int svo3_set_gravity(svo3_ctx_t *c, double grav_vof, double vof_ref) {
  c->grav_vof = grav_vof;
  c->vof_ref = vof_ref;
  return 0;
}

int svo3_run(svo3_ctx_t *c, int nsteps, double *dts) {
  for (int n = 0; n < nsteps; n++) {
    double dt = 0.;
    svo3_integrate(c, &dt);
    if (dts) dts[n] = dt;
  }
  return 0;
}

/* ---------- time-averaged statistics ---------- */

/* the 2D collection of src/statistics.c:117-204 with a k loop and uz added;
 * arrays nz x ny x width, no halo, width nx+1 for ux1 ux2 uxt (q = 0, 1, 8)
 * and nx+2 for the others */
static int stat_width3(const svo3_ctx_t *c, int q) { return (0 == q || 1 == q || 8 == q) ? NX + 1 : NX + 2; }

int svo3_stat_collect(svo3_ctx_t *c) {
  if (!c->stat[0])
    for (int q = 0; q < 9; q++) c->stat[q] = calloc((size_t)stat_width3(c, q) * NY * NZ, sizeof(double));
  const double *UY = c->uy, *UZ = c->uz, *T = c->t;
#define SX(a, i, j, k) (a)[(i) - 1 + (long)(NX + 1) * (((j) - 1) + (long)NY * ((k) - 1))]
#define SC(a, i, j, k) (a)[(i) + (long)(NX + 2) * (((j) - 1) + (long)NY * ((k) - 1))]
  for (int k = 1; k <= NZ; k++)
    for (int j = 1; j <= NY; j++)
      for (int i = 1; i <= NX + 1; i++) {
        SX(c->stat[0], i, j, k) += pow(UX(i, j, k), 1.);
        SX(c->stat[1], i, j, k) += pow(UX(i, j, k), 2.);
      }
  for (int k = 1; k <= NZ; k++)
    for (int j = 1; j <= NY; j++)
      for (int i = 0; i <= NX + 1; i++) {
        SC(c->stat[2], i, j, k) += pow(CC(UY, i, j, k), 1.);
        SC(c->stat[3], i, j, k) += pow(CC(UY, i, j, k), 2.);
        SC(c->stat[4], i, j, k) += pow(CC(UZ, i, j, k), 1.);
        SC(c->stat[5], i, j, k) += pow(CC(UZ, i, j, k), 2.);
        SC(c->stat[6], i, j, k) += pow(CC(T, i, j, k), 1.);
        SC(c->stat[7], i, j, k) += pow(CC(T, i, j, k), 2.);
      }
  for (int k = 1; k <= NZ; k++)
    for (int j = 1; j <= NY; j++)
      for (int i = 1; i <= NX + 1; i++) {
        const double t_ = +0.5 * CC(T, i - 1, j, k) + 0.5 * CC(T, i, j, k);
        SX(c->stat[8], i, j, k) += UX(i, j, k) * t_;
      }
#undef SX
#undef SC
  c->stat_num += 1;
  return 0;
}

/* reduce_and_write (src/statistics.c:232-281) over y and z: the sum over j of
 * each z plane, in order from zero, then the sum of the planes in z order
 * from zero */
int svo3_stat_reduce(const svo3_ctx_t *c, int q, double *out) {
  if (q < 0 || q > 8) return 1;
  const int w = stat_width3(c, q);
  for (int i = 0; i < w; i++) out[i] = 0.;
  if (!c->stat[0]) return 0;
  double *plane = calloc((size_t)w, sizeof(double));
  for (int k = 0; k < NZ; k++) {
    for (int i = 0; i < w; i++) plane[i] = 0.;
    for (int j = 0; j < NY; j++)
      for (int i = 0; i < w; i++) plane[i] += c->stat[q][((long)k * NY + j) * w + i];
    for (int i = 0; i < w; i++) out[i] += plane[i];
  }
  free(plane);
  return 0;
}

long svo3_stat_num(const svo3_ctx_t *c) { return c->stat_num; }
