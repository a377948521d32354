/*
 * svof_oracle.c -- CPU restatement of SimpleVOFSolver's per-step hot path,
 * 2D, FP64.  TEST INFRASTRUCTURE ONLY (see svof_oracle.h).
 *
 * Each function below states the reference file:line it restates.  The
 * floating-point expressions keep the reference's operation order and
 * association (for example "1. / dx * (a - b)" is computed as (1/dx)*(a-b)),
 * sums start from the zeroed source arrays as in the reference, and the
 * tri-diagonal sweeps follow src/tdm.c exactly, so that this restatement
 * reproduces the compiled reference bit for bit (checked by
 * tests/test_oracle_pin.py).  The FFTW transforms are computed by
 * svof_fft.c (FFTW's unnormalised definitions).
 *
 * Unlike the reference, all state lives in an explicit context (the
 * reference keeps Laplacian tables, Poisson plans and line-solver buffers in
 * function-local statics), so several domains can coexist in one process.
 */
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "svof_fft.h"
#include "svof_oracle.h"

/* src/runge_kutta.c:8-15 */
static const double RK_A[3] = {32. / 60., 25. / 60., 45. / 60.};
static const double RK_B[3] = {0. / 60., -17. / 60., -25. / 60.};
static double rk_g(int s) { return RK_A[s] + RK_B[s]; }

/* src/interface/common.c:4-14, src/interface/internal.h:4 */
#define NGAUSS 2
static const double GAUSS_P[NGAUSS] = {-0.2886751345948129, +0.2886751345948129};
static const double GAUSS_W[NGAUSS] = {+0.5, +0.5};
static const double VOFBETA = 1.;
static const double VOFMIN = 1.e-8;

/* src/fluid/compute_potential/dct.c:20 */
static const double G_PI = 3.14159265358979324;

struct svo_ctx {
  svo_params_t prm;
  int nx, ny;
  double *xf, *xc, *dxf, *dxc;
  double dy;
  int uniform;
  /* fields */
  double *ux, *uy, *p, *psi, *t;
  double *srcux[3], *srcuy[3], *srct[3];
  double *vof, *ifrcx, *ifrcy, *dvof, *normal, *curv, *flxx, *flxy, *src[2];
  long n_ux, n_cc, n_vof, n_dvof, n_normal, n_flxx, n_flxy, n_ifrcx, n_ifrcy, n_srcux, n_src;
  /* Laplacian tables of src/fluid/predict/{ux,uy,t}.c (init_lap) */
  double *lapx_ux, *lapx_uy, *lapx_t; /* 3 per row */
  double lapy[3];
  /* line-solver buffers (src/linear_system.c, src/tdm.c) */
  double *x1pncl;                  /* nx*ny increments */
  double *tdm_l, *tdm_c, *tdm_u, *tdm_v, *tdm_q1;
  /* Poisson buffers and plans */
  double *pbuf0, *pbuf1;
  svof_fft_plan_t *plan_x, *plan_y;
  double *evals_dct, *evals_dft;
  double *plap_l, *plap_u;         /* DFT path x-Laplacian */
  /* time-averaged statistics (src/statistics.c:40-47): ux1 ux2 uy1 uy2 t1
   * t2 uxt, allocated on the first collection */
  double *stat[7];
  long stat_num;
  /* buoyancy of the volume fraction on uy (an extension, not in the
   * reference; off while grav_vof == 0): srcuy += grav_vof (vof_face - vof_ref) */
  double grav_vof, vof_ref;
};

/* ---------- index maps (reference include/array_macros/) ---------- */
#define NX (c->nx)
#define NY (c->ny)
#define UX(i, j) c->ux[(i) - 1 + (NX + 1) * (j)]
#define CC(a, i, j) (a)[(i) + (NX + 2) * (j)]
#define VOF(i, j) c->vof[(i) + (NX + 2) * ((j) + 1)]
#define DVOF(i, j, k) c->dvof[2 * ((i) - 1 + (NX + 1) * (j)) + (k)]
#define NORMAL(i, j, k) c->normal[3 * ((i) - 1 + NX * (j)) + (k)]
#define FLXX(i, j) c->flxx[(i) - 1 + (NX + 1) * ((j) - 1)]
#define FLXY(i, j) c->flxy[(i) - 1 + NX * ((j) - 1)]
#define IFRCX(i, j) c->ifrcx[(i) - 2 + (NX - 1) * ((j) - 1)]
#define IFRCY(i, j) c->ifrcy[(i) - 1 + NX * ((j) - 1)]
#define DXF(i) c->dxf[(i) - 1]
#define DXC(i) c->dxc[(i) - 1]

static double *dalloc(long n) { return calloc((size_t)(n > 0 ? n : 1), sizeof(double)); }

svo_ctx_t *svo_create(const svo_params_t *prm, const double *xf, const double *xc) {
  if (prm->nx < 3 || prm->ny < 3) return NULL;
  svo_ctx_t *c = calloc(1, sizeof(*c));
  c->prm = *prm;
  c->nx = prm->nx;
  c->ny = prm->ny;
  const int nx = c->nx, ny = c->ny;
  c->xf = dalloc(nx + 1);
  c->xc = dalloc(nx + 2);
  memcpy(c->xf, xf, sizeof(double) * (size_t)(nx + 1));
  memcpy(c->xc, xc, sizeof(double) * (size_t)(nx + 2));
  /* src/domain.c:107-143 */
  c->dxf = dalloc(nx);
  c->dxc = dalloc(nx + 1);
  for (int i = 1; i <= nx; i++) DXF(i) = c->xf[i] - c->xf[i - 1];
  for (int i = 1; i <= nx + 1; i++) DXC(i) = c->xc[i] - c->xc[i - 1];
  /* src/domain.c:190-192 */
  c->dy = prm->ly / ny;
  /* src/domain.c:75-98 */
  {
    double mn = +1. * DBL_MAX, mx = -1. * DBL_MAX;
    for (int i = 0; i < nx; i++) {
      mn = fmin(mn, c->dxf[i]);
      mx = fmax(mx, c->dxf[i]);
    }
    c->uniform = fabs(mx - mn) < 1.e-15;
  }
  c->n_ux = (long)(nx + 1) * (ny + 2);
  c->n_cc = (long)(nx + 2) * (ny + 2);
  c->n_vof = (long)(nx + 2) * (ny + 4);
  c->n_dvof = 2L * (nx + 1) * (ny + 3);
  c->n_normal = 3L * nx * (ny + 2);
  c->n_flxx = (long)(nx + 1) * ny;
  c->n_flxy = (long)nx * (ny + 1);
  c->n_ifrcx = (long)(nx - 1) * ny;
  c->n_ifrcy = (long)nx * ny;
  c->n_srcux = (long)(nx - 1) * ny;
  c->n_src = (long)nx * ny;
  c->ux = dalloc(c->n_ux);
  c->uy = dalloc(c->n_cc);
  c->p = dalloc(c->n_cc);
  c->psi = dalloc(c->n_cc);
  c->t = dalloc(c->n_cc);
  for (int k = 0; k < 3; k++) {
    c->srcux[k] = dalloc(c->n_srcux);
    c->srcuy[k] = dalloc(c->n_src);
    c->srct[k] = dalloc(c->n_src);
  }
  c->vof = dalloc(c->n_vof);
  c->ifrcx = dalloc(c->n_ifrcx);
  c->ifrcy = dalloc(c->n_ifrcy);
  c->dvof = dalloc(c->n_dvof);
  c->normal = dalloc(c->n_normal);
  c->curv = dalloc(c->n_cc);
  c->flxx = dalloc(c->n_flxx);
  c->flxy = dalloc(c->n_flxy);
  c->src[0] = dalloc(c->n_src);
  c->src[1] = dalloc(c->n_src);
  /* Laplacians: src/fluid/predict/ux.c:34-61, uy.c:34-61, t.c:34-61 */
  c->lapx_ux = dalloc(3L * (nx - 1));
  for (int i = 2; i <= nx; i++) {
    const double l = 1. / DXF(i - 1) / DXC(i);
    const double u = 1. / DXF(i) / DXC(i);
    const double cc = -l - u;
    c->lapx_ux[3 * (i - 2) + 0] = l;
    c->lapx_ux[3 * (i - 2) + 1] = cc;
    c->lapx_ux[3 * (i - 2) + 2] = u;
  }
  c->lapx_uy = dalloc(3L * nx);
  c->lapx_t = dalloc(3L * nx);
  for (int i = 1; i <= nx; i++) {
    const double l = 1. / DXC(i) / DXF(i);
    const double u = 1. / DXC(i + 1) / DXF(i);
    const double cc = -l - u;
    c->lapx_uy[3 * (i - 1) + 0] = l;
    c->lapx_uy[3 * (i - 1) + 1] = cc;
    c->lapx_uy[3 * (i - 1) + 2] = u;
    c->lapx_t[3 * (i - 1) + 0] = l;
    c->lapx_t[3 * (i - 1) + 1] = cc;
    c->lapx_t[3 * (i - 1) + 2] = u;
  }
  c->lapy[0] = +1. / c->dy / c->dy;
  c->lapy[1] = -2. / c->dy / c->dy;
  c->lapy[2] = +1. / c->dy / c->dy;
  /* line-solver buffers */
  const int nmax = nx > ny ? nx : ny;
  c->x1pncl = dalloc((long)nx * ny);
  c->tdm_l = dalloc(nmax);
  c->tdm_c = dalloc(nmax);
  c->tdm_u = dalloc(nmax);
  c->tdm_v = dalloc(nmax);
  c->tdm_q1 = dalloc(nmax);
  /* Poisson: complex buffers large enough for both paths */
  c->pbuf0 = dalloc(2L * nx * (ny / 2 + 1) + (long)nx * ny);
  c->pbuf1 = dalloc(2L * nx * (ny / 2 + 1) + (long)nx * ny);
  c->plan_x = svof_fft_plan_create((size_t)nx);
  c->plan_y = svof_fft_plan_create((size_t)ny);
  /* eigenvalues: src/fluid/compute_potential/dct.c:233-261 */
  c->evals_dct = dalloc(nx);
  {
    const double signal_length = 2. * nx;
    const double gridsize = prm->lx / nx;
    for (size_t i = 0; i < (size_t)nx; i++) {
      c->evals_dct[i] = -4. / pow(gridsize, 2.) * pow(sin(G_PI * i / signal_length), 2.);
    }
  }
  /* src/fluid/compute_potential/dft.c:263-291 */
  c->evals_dft = dalloc(ny / 2 + 1);
  {
    const double signal_length = (double)ny;
    const double gridsize = prm->ly / ny;
    for (size_t j = 0; j < (size_t)(ny / 2 + 1); j++) {
      c->evals_dft[j] = -4. / pow(gridsize, 2.) * pow(sin(G_PI * j / signal_length), 2.);
    }
  }
  /* src/fluid/compute_potential/dft.c:191-196 */
  c->plap_l = dalloc(nx);
  c->plap_u = dalloc(nx);
  for (int i = 1; i <= nx; i++) {
    c->plap_l[i - 1] = 1. / DXC(i) / DXF(i);
    c->plap_u[i - 1] = 1. / DXC(i + 1) / DXF(i);
  }
  return c;
}

void svo_destroy(svo_ctx_t *c) {
  if (c)
    for (int q = 0; q < 7; q++) free(c->stat[q]);
  if (!c) return;
  double *bufs[] = {c->xf, c->xc, c->dxf, c->dxc, c->ux, c->uy, c->p, c->psi, c->t,
                    c->vof, c->ifrcx, c->ifrcy, c->dvof, c->normal, c->curv, c->flxx, c->flxy,
                    c->src[0], c->src[1], c->lapx_ux, c->lapx_uy, c->lapx_t, c->x1pncl,
                    c->tdm_l, c->tdm_c, c->tdm_u, c->tdm_v, c->tdm_q1, c->pbuf0, c->pbuf1,
                    c->evals_dct, c->evals_dft, c->plap_l, c->plap_u};
  for (size_t k = 0; k < sizeof(bufs) / sizeof(bufs[0]); k++) free(bufs[k]);
  for (int k = 0; k < 3; k++) {
    free(c->srcux[k]);
    free(c->srcuy[k]);
    free(c->srct[k]);
  }
  svof_fft_plan_destroy(c->plan_x);
  svof_fft_plan_destroy(c->plan_y);
  free(c);
}

double *svo_field(svo_ctx_t *c, const char *name, long *count) {
  struct { const char *n; double *p; long k; } tab[] = {
    {"ux", c->ux, c->n_ux}, {"uy", c->uy, c->n_cc}, {"p", c->p, c->n_cc},
    {"psi", c->psi, c->n_cc}, {"t", c->t, c->n_cc},
    {"srcux0", c->srcux[0], c->n_srcux}, {"srcux1", c->srcux[1], c->n_srcux},
    {"srcux2", c->srcux[2], c->n_srcux}, {"srcuy0", c->srcuy[0], c->n_src},
    {"srcuy1", c->srcuy[1], c->n_src}, {"srcuy2", c->srcuy[2], c->n_src},
    {"srct0", c->srct[0], c->n_src}, {"srct1", c->srct[1], c->n_src},
    {"srct2", c->srct[2], c->n_src}, {"vof", c->vof, c->n_vof},
    {"ifrcx", c->ifrcx, c->n_ifrcx}, {"ifrcy", c->ifrcy, c->n_ifrcy},
    {"dvof", c->dvof, c->n_dvof}, {"normal", c->normal, c->n_normal},
    {"curv", c->curv, c->n_cc}, {"flxx", c->flxx, c->n_flxx}, {"flxy", c->flxy, c->n_flxy},
    {"src0", c->src[0], c->n_src}, {"src1", c->src[1], c->n_src},
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

int svo_x_grid_is_uniform(svo_ctx_t *c) { return c->uniform; }

/* ---------------- boundaries: src/halo.c:18-76 + src/fluid/boundary ---------------- */

/* periodic y halo of an array with row width w, nh halo rows on each side and
 * ny interior rows (src/halo.c:51-74: both exchanges copy whole rows, x ghost
 * cells included, before the x boundary values are assigned) */
static void halo_y(double *a, long w, int nh, int ny) {
  memmove(a, a + w * ny, sizeof(double) * (size_t)(w * nh));
  memmove(a + w * (ny + nh), a + w * nh, sizeof(double) * (size_t)(w * nh));
}

static void bc_ux(svo_ctx_t *c) {
  /* src/fluid/boundary/ux.c:7-39 */
  halo_y(c->ux, NX + 1, 1, NY);
  for (int j = 1; j <= NY; j++) {
    UX(1, j) = 0.;
    UX(NX + 1, j) = 0.;
  }
}

static void bc_uy(svo_ctx_t *c) {
  /* src/fluid/boundary/uy.c:8-40 */
  halo_y(c->uy, NX + 2, 1, NY);
  for (int j = 1; j <= NY; j++) {
    CC(c->uy, 0, j) = c->prm.uy_xm;
    CC(c->uy, NX + 1, j) = c->prm.uy_xp;
  }
}

static void bc_neumann(svo_ctx_t *c, double *a) {
  /* src/fluid/boundary/p.c:7-39, psi.c:7-39 */
  halo_y(a, NX + 2, 1, NY);
  for (int j = 1; j <= NY; j++) {
    CC(a, 0, j) = CC(a, 1, j);
    CC(a, NX + 1, j) = CC(a, NX, j);
  }
}

static void bc_t(svo_ctx_t *c) {
  /* src/fluid/boundary/t.c:8-40 */
  halo_y(c->t, NX + 2, 1, NY);
  for (int j = 1; j <= NY; j++) {
    CC(c->t, 0, j) = c->prm.t_xm;
    CC(c->t, NX + 1, j) = c->prm.t_xp;
  }
}

static void bc_vof(svo_ctx_t *c) {
  /* src/interface/boundary.c:7-39 */
  halo_y(c->vof, NX + 2, 2, NY);
  for (int j = -1; j <= NY + 2; j++) {
    VOF(0, j) = 0.;
    VOF(NX + 1, j) = 0.;
  }
}

int svo_init_boundaries(svo_ctx_t *c) {
  /* src/fluid/init.c:85-88, src/interface/init.c:63 */
  bc_ux(c);
  bc_uy(c);
  bc_neumann(c, c->p);
  bc_t(c);
  bc_vof(c);
  return 0;
}

/* ---------------- time step: src/fluid/decide_dt.c ---------------- */
int svo_decide_dt(svo_ctx_t *c, double *dt) {
  /* decide_dt_adv, :28-64 */
  const double small = 1.e-8;
  double dta = 1.;
  for (int j = 1; j <= NY; j++) {
    for (int i = 2; i <= NX; i++) {
      const double dx = DXC(i);
      const double vel = fabs(UX(i, j)) + small;
      dta = fmin(dta, dx / vel);
    }
  }
  for (int j = 1; j <= NY; j++) {
    for (int i = 1; i <= NX; i++) {
      const double vel = fabs(CC(c->uy, i, j)) + small;
      dta = fmin(dta, c->dy / vel);
    }
  }
  dta *= c->prm.coef_dt_adv;
  /* decide_dt_dif, :73-94 (only y is explicit: src/param/implicit.c:3-7) */
  const int ndims = 2;
  const double dt_dif_m_y = c->prm.coef_dt_dif / c->prm.m_dif * 0.5 / ndims * pow(c->dy, 2.);
  const double dt_dif_t_y = c->prm.coef_dt_dif / c->prm.t_dif * 0.5 / ndims * pow(c->dy, 2.);
  /* fluid_decide_dt, :129-143 */
  double r = dta;
  r = fmin(r, dt_dif_m_y);
  r = fmin(r, dt_dif_t_y);
  *dt = r;
  return 0;
}

/* ---------------- interface geometry: src/interface/curvature_tensor.c ---------------- */

/* compute_gradient, :14-48 */
static void compute_gradient(svo_ctx_t *c) {
  const double dy = c->dy;
  for (int j = 0; j <= NY + 2; j++) {
    for (int i = 1; i <= NX + 1; i++) {
      const double dx = DXC(i);
      const double dvofdx = 1. / dx * (-VOF(i - 1, j - 1) + VOF(i, j - 1) - VOF(i - 1, j) + VOF(i, j));
      const double dvofdy = 1. / dy * (-VOF(i - 1, j - 1) - VOF(i, j - 1) + VOF(i - 1, j) + VOF(i, j));
      const double norm = sqrt(+pow(dvofdx, 2.) + pow(dvofdy, 2.));
      const double norminv = 1. / fmax(norm, DBL_EPSILON);
      DVOF(i, j, 0) = dvofdx * norminv;
      DVOF(i, j, 1) = dvofdy * norminv;
    }
  }
}

/* compute_intercept, :50-92 */
static double compute_intercept(const double vof, const double n0, const double n1) {
  const int cntmax = 8;
  const double resmax = 1.e-12;
  double exps[NGAUSS * NGAUSS] = {0.};
  for (int jj = 0; jj < NGAUSS; jj++) {
    for (int ii = 0; ii < NGAUSS; ii++) {
      exps[jj * NGAUSS + ii] = exp(-2. * VOFBETA * (+n0 * GAUSS_P[ii] + n1 * GAUSS_P[jj]));
    }
  }
  double val = 1. / vof - 1.;
  for (int cnt = 0; cnt < cntmax; cnt++) {
    double f0 = -1. * vof;
    double f1 = 0.;
    for (int jj = 0; jj < NGAUSS; jj++) {
      for (int ii = 0; ii < NGAUSS; ii++) {
        const double weight = GAUSS_W[ii] * GAUSS_W[jj];
        const double p = exps[jj * NGAUSS + ii];
        const double denom = 1. / (1. + p * val);
        f0 += weight * denom;
        f1 -= weight * p * denom * denom;
      }
    }
    val -= f0 / f1;
    if (fabs(f0) < resmax) break;
  }
  return -0.5 / VOFBETA * log(val);
}

/* compute_normal, :94-145 */
static void compute_normal(svo_ctx_t *c) {
  const double dy = c->dy;
  for (int j = 0; j <= NY + 1; j++) {
    for (int i = 1; i <= NX; i++) {
      const double dx = DXF(i);
      const double lvof = VOF(i, j);
      if (lvof < VOFMIN || 1. - VOFMIN < lvof) continue;
      double nx = (+DVOF(i, j, 0) + DVOF(i + 1, j, 0) + DVOF(i, j + 1, 0) + DVOF(i + 1, j + 1, 0));
      double ny = (+DVOF(i, j, 1) + DVOF(i + 1, j, 1) + DVOF(i, j + 1, 1) + DVOF(i + 1, j + 1, 1));
      nx /= dx;
      ny /= dy;
      const double norm = sqrt(+pow(nx, 2.) + pow(ny, 2.));
      const double norminv = 1. / fmax(norm, DBL_EPSILON);
      nx *= norminv;
      ny *= norminv;
      const double seg = compute_intercept(lvof, nx, ny);
      NORMAL(i, j, 0) = nx;
      NORMAL(i, j, 1) = ny;
      NORMAL(i, j, 2) = seg;
    }
  }
}

/* compute_curvature, :147-176 */
static void compute_curvature(svo_ctx_t *c) {
  const double dy = c->dy;
  for (int j = 0; j <= NY + 1; j++) {
    for (int i = 1; i <= NX; i++) {
      const double dx = DXF(i);
      const double dnxdx = 1. / dx * (-DVOF(i, j, 0) + DVOF(i + 1, j, 0) - DVOF(i, j + 1, 0) + DVOF(i + 1, j + 1, 0));
      const double dnydy = 1. / dy * (-DVOF(i, j, 1) - DVOF(i + 1, j, 1) + DVOF(i, j + 1, 1) + DVOF(i + 1, j + 1, 1));
      CC(c->curv, i, j) = 0.5 * (-dnxdx - dnydy);
    }
  }
}

int svo_curvature_tensor(svo_ctx_t *c) {
  /* :178-186 */
  compute_gradient(c);
  compute_normal(c);
  compute_curvature(c);
  return 0;
}

/* src/interface/force.c:11-76 */
int svo_force(svo_ctx_t *c) {
  const double tension = c->prm.tension;
  for (int j = 1; j <= NY; j++) {
    for (int i = 2; i <= NX; i++) {
      const double dx = DXC(i);
      const double grad = 1. / dx * (-VOF(i - 1, j) + VOF(i, j));
      const double kappa = 0.5 * (+CC(c->curv, i - 1, j) + CC(c->curv, i, j));
      IFRCX(i, j) = tension * grad * kappa;
    }
  }
  for (int j = 1; j <= NY; j++) {
    for (int i = 1; i <= NX; i++) {
      const double grad = 1. / c->dy * (-VOF(i, j - 1) + VOF(i, j));
      const double kappa = 0.5 * (+CC(c->curv, i, j - 1) + CC(c->curv, i, j));
      IFRCY(i, j) = tension * grad * kappa;
    }
  }
  return 0;
}

/* ---------------- vof update: src/interface/update ---------------- */

/* indicator, update/main.c:16-26 */
static double indicator(const double *n, const double x0, const double x1) {
  return 1. / (1. + exp(-2. * VOFBETA * (+n[0] * x0 + n[1] * x1 + n[2])));
}

static void vof_rhs_advect(svo_ctx_t *c, int rkstep, double dt);

int svo_update_vof(svo_ctx_t *c, int rkstep, double dt) {
  /* reset_srcs, update/main.c:28-45 */
  if (0 != rkstep) {
    double *tmp = c->src[0];
    c->src[0] = c->src[1];
    c->src[1] = tmp;
  }
  memset(c->src[0], 0, sizeof(double) * (size_t)c->n_src);
  /* compute_flux_x, update/flxx.c:11-44 */
  for (int j = 1; j <= NY; j++) {
    for (int i = 2; i <= NX; i++) {
      const double vel = UX(i, j);
      const int ii = vel < 0. ? i : i - 1;
      const double x = vel < 0. ? -0.5 : +0.5;
      const double lvof = VOF(ii, j);
      if (lvof < VOFMIN || 1. - VOFMIN < lvof) {
        FLXX(i, j) = vel * lvof;
        continue;
      }
      double flux = 0.;
      for (int jj = 0; jj < NGAUSS; jj++) {
        flux += GAUSS_W[jj] * indicator(&NORMAL(ii, j, 0), x, GAUSS_P[jj]);
      }
      FLXX(i, j) = vel * flux;
    }
  }
  /* compute_flux_y, update/flxy.c:11-44 */
  for (int j = 1; j <= NY + 1; j++) {
    for (int i = 1; i <= NX; i++) {
      const double vel = CC(c->uy, i, j);
      const int jj = vel < 0. ? j : j - 1;
      const double y = vel < 0. ? -0.5 : +0.5;
      const double lvof = VOF(i, jj);
      if (lvof < VOFMIN || 1. - VOFMIN < lvof) {
        FLXY(i, j) = vel * lvof;
        continue;
      }
      double flux = 0.;
      for (int ii = 0; ii < NGAUSS; ii++) {
        flux += GAUSS_W[ii] * indicator(&NORMAL(i, jj, 0), GAUSS_P[ii], y);
      }
      FLXY(i, j) = vel * flux;
    }
  }
  vof_rhs_advect(c, rkstep, dt);
  return 0;
}

/* interface_compute_rhs + interface_advect_vof + the boundary update
 * (update/main.c:47-110, boundary.c:7-39): linear in the fluxes, src_b and
 * vof, so the tangent-linear model runs it on its own context as well */
static void vof_rhs_advect(svo_ctx_t *c, int rkstep, double dt) {
  /* interface_compute_rhs, update/main.c:47-78 */
  double *src = c->src[0];
  for (int j = 1; j <= NY; j++) {
    for (int i = 1; i <= NX; i++) {
      const double dx = DXF(i);
      src[(i - 1) + NX * (j - 1)] += 1. / dx * (+FLXX(i, j) - FLXX(i + 1, j));
    }
  }
  for (int j = 1; j <= NY; j++) {
    for (int i = 1; i <= NX; i++) {
      src[(i - 1) + NX * (j - 1)] += 1. / c->dy * (+FLXY(i, j) - FLXY(i, j + 1));
    }
  }
  /* interface_advect_vof, update/main.c:80-110 */
  {
    const double coef = RK_A[rkstep];
    for (int j = 1; j <= NY; j++) {
      for (int i = 1; i <= NX; i++) VOF(i, j) += dt * coef * c->src[0][(i - 1) + NX * (j - 1)];
    }
  }
  if (0 != rkstep) {
    const double coef = RK_B[rkstep];
    for (int j = 1; j <= NY; j++) {
      for (int i = 1; i <= NX; i++) VOF(i, j) += dt * coef * c->src[1][(i - 1) + NX * (j - 1)];
    }
  }
  bc_vof(c);
}

/* ---------------- Thomas solvers: src/tdm.c ---------------- */

/* gtsv, :17-50; stride lets the complex variant run on interleaved data
 * (the reference's fftw_complex instantiation is component-wise) */
static void gtsv(const int n, const double *l, const double *cc, const double *u, double *v,
                 double *q, const int stride) {
#define Q(i) q[(size_t)(i) * stride]
  v[0] = u[0] / cc[0];
  Q(0) = Q(0) / cc[0];
  for (int i = 1; i < n - 1; i++) {
    const double val = 1. / (cc[i] - l[i] * v[i - 1]);
    v[i] = val * (u[i]);
    Q(i) = val * (Q(i) - l[i] * Q(i - 1));
  }
  const double val = cc[n - 1] - l[n - 1] * v[n - 2];
  if (fabs(val) > DBL_EPSILON) {
    Q(n - 1) = 1. / val * (Q(n - 1) - l[n - 1] * Q(n - 2));
  } else {
    Q(n - 1) = 0.;
  }
  for (int i = n - 2; i >= 0; i--) Q(i) -= v[i] * Q(i + 1);
#undef Q
}

/* tdm_solve (periodic, nrhs = 1), :78-99 */
static void tdm_periodic(const int n, const double *l, const double *cc, const double *u,
                         double *v, double *q, double *q1) {
  for (int i = 0; i < n - 1; i++) {
    q1[i] = i == 0 ? -l[i] : i == n - 2 ? -u[i] : 0.;
  }
  gtsv(n - 1, l, cc, u, v, q1, 1);
  double *q0 = q;
  gtsv(n - 1, l, cc, u, v, q0, 1);
  const double num = q0[n - 1] - u[n - 1] * q0[0] - l[n - 1] * q0[n - 2];
  const double den = cc[n - 1] + u[n - 1] * q1[0] + l[n - 1] * q1[n - 2];
  q0[n - 1] = fabs(den) < DBL_EPSILON ? 0. : num / den;
  for (int i = 0; i < n - 1; i++) q0[i] = q0[i] + q0[n - 1] * q1[i];
}

/* ---------------- momentum / scalar predictor: src/fluid/predict ---------------- */

/* x-implicit line solve of one field (solve_in_x of {ux,uy,t}.c) on
 * x1pncl (size lines of length n, nrhs = ny) */
static void solve_in_x(svo_ctx_t *c, const double prefactor, const double *lapx, const int n) {
  for (int i = 0; i < n; i++) {
    c->tdm_l[i] = -prefactor * lapx[3 * i + 0];
    c->tdm_c[i] = 1. - prefactor * lapx[3 * i + 1];
    c->tdm_u[i] = -prefactor * lapx[3 * i + 2];
  }
  for (int j = 0; j < NY; j++) {
    gtsv(n, c->tdm_l, c->tdm_c, c->tdm_u, c->tdm_v, c->x1pncl + (size_t)j * n, 1);
  }
}

static void reset_srcs3(svo_ctx_t *c, double **s, long n, int rkstep) {
  /* src/fluid/predict/main.c:9-29 */
  if (0 != rkstep) {
    double *tmp = s[0];
    s[0] = s[1];
    s[1] = tmp;
  }
  memset(s[0], 0, sizeof(double) * (size_t)n);
  memset(s[2], 0, sizeof(double) * (size_t)n);
  (void)c;
}

static void rhs_ux(svo_ctx_t *c) {
  /* compute_rhs_ux, ux.c:218-249 */
  const double dy = c->dy;
  const double dif = c->prm.m_dif;
  double *srca = c->srcux[0], *srcg = c->srcux[2];
  const double *uy = c->uy, *p = c->p, *t = c->t;
  int cnt;
  /* advection_x, :71-92 */
  cnt = 0;
  for (int j = 1; j <= NY; j++) {
    for (int i = 2; i <= NX; i++, cnt++) {
      const double ux_l = +0.5 * UX(i - 1, j) + 0.5 * UX(i, j);
      const double ux_u = +0.5 * UX(i, j) + 0.5 * UX(i + 1, j);
      const double l = +0.5 / DXC(i) * ux_l;
      const double u = -0.5 / DXC(i) * ux_u;
      const double cc = -l - u;
      srca[cnt] += +l * UX(i - 1, j) + cc * UX(i, j) + u * UX(i + 1, j);
    }
  }
  /* advection_y, :94-120 */
  cnt = 0;
  for (int j = 1; j <= NY; j++) {
    for (int i = 2; i <= NX; i++, cnt++) {
      const double w_xm = 0.5 * DXF(i - 1) / DXC(i);
      const double w_xp = 0.5 * DXF(i) / DXC(i);
      const double uy_l = w_xm * CC(uy, i - 1, j) + w_xp * CC(uy, i, j);
      const double uy_u = w_xm * CC(uy, i - 1, j + 1) + w_xp * CC(uy, i, j + 1);
      const double l = +0.5 / dy * uy_l;
      const double u = -0.5 / dy * uy_u;
      const double cc = -l - u;
      srca[cnt] += +l * UX(i, j - 1) + cc * UX(i, j) + u * UX(i, j + 1);
    }
  }
  /* diffusion_x (implicit: srcg), :123-141 */
  cnt = 0;
  for (int j = 1; j <= NY; j++) {
    for (int i = 2; i <= NX; i++, cnt++) {
      const double *lx = c->lapx_ux + 3 * (i - 2);
      srcg[cnt] += dif * (+lx[0] * UX(i - 1, j) + lx[1] * UX(i, j) + lx[2] * UX(i + 1, j));
    }
  }
  /* diffusion_y (explicit: srca), :143-161 */
  cnt = 0;
  for (int j = 1; j <= NY; j++) {
    for (int i = 2; i <= NX; i++, cnt++) {
      srca[cnt] += dif * (+c->lapy[0] * UX(i, j - 1) + c->lapy[1] * UX(i, j) + c->lapy[2] * UX(i, j + 1));
    }
  }
  /* pressure (srcg), :164-179 */
  cnt = 0;
  for (int j = 1; j <= NY; j++) {
    for (int i = 2; i <= NX; i++, cnt++) {
      srcg[cnt] -= 1. / DXC(i) * (-CC(p, i - 1, j) + CC(p, i, j));
    }
  }
  /* buoyancy, :181-197 */
  if (c->prm.add_buoyancy) {
    cnt = 0;
    for (int j = 1; j <= NY; j++) {
      for (int i = 2; i <= NX; i++, cnt++) srca[cnt] += +0.5 * CC(t, i - 1, j) + 0.5 * CC(t, i, j);
    }
  }
  /* surface, :199-210 */
  cnt = 0;
  for (int j = 1; j <= NY; j++) {
    for (int i = 2; i <= NX; i++, cnt++) srca[cnt] += c->ifrcx[cnt];
  }
}

static void rhs_uy(svo_ctx_t *c) {
  /* compute_rhs_uy, uy.c:195-221 */
  const double dy = c->dy;
  const double dif = c->prm.m_dif;
  double *srca = c->srcuy[0], *srcg = c->srcuy[2];
  const double *uy = c->uy, *p = c->p;
  int cnt;
  /* advection_x, :70-92 */
  cnt = 0;
  for (int j = 1; j <= NY; j++) {
    for (int i = 1; i <= NX; i++, cnt++) {
      const double ux_l = +0.5 * UX(i, j - 1) + 0.5 * UX(i, j);
      const double ux_u = +0.5 * UX(i + 1, j - 1) + 0.5 * UX(i + 1, j);
      const double l = +0.5 / DXF(i) * ux_l;
      const double u = -0.5 / DXF(i) * ux_u;
      const double cc = -l - u;
      srca[cnt] += +l * CC(uy, i - 1, j) + cc * CC(uy, i, j) + u * CC(uy, i + 1, j);
    }
  }
  /* advection_y, :94-115 */
  cnt = 0;
  for (int j = 1; j <= NY; j++) {
    for (int i = 1; i <= NX; i++, cnt++) {
      const double uy_l = +0.5 * CC(uy, i, j - 1) + 0.5 * CC(uy, i, j);
      const double uy_u = +0.5 * CC(uy, i, j) + 0.5 * CC(uy, i, j + 1);
      const double l = +0.5 / dy * uy_l;
      const double u = -0.5 / dy * uy_u;
      const double cc = -l - u;
      srca[cnt] += +l * CC(uy, i, j - 1) + cc * CC(uy, i, j) + u * CC(uy, i, j + 1);
    }
  }
  /* diffusion_x (srcg), :118-136 */
  cnt = 0;
  for (int j = 1; j <= NY; j++) {
    for (int i = 1; i <= NX; i++, cnt++) {
      const double *lx = c->lapx_uy + 3 * (i - 1);
      srcg[cnt] += dif * (+lx[0] * CC(uy, i - 1, j) + lx[1] * CC(uy, i, j) + lx[2] * CC(uy, i + 1, j));
    }
  }
  /* diffusion_y (srca), :138-156 */
  cnt = 0;
  for (int j = 1; j <= NY; j++) {
    for (int i = 1; i <= NX; i++, cnt++) {
      srca[cnt] += dif * (+c->lapy[0] * CC(uy, i, j - 1) + c->lapy[1] * CC(uy, i, j) + c->lapy[2] * CC(uy, i, j + 1));
    }
  }
  /* pressure (srcg), :159-174 */
  cnt = 0;
  for (int j = 1; j <= NY; j++) {
    for (int i = 1; i <= NX; i++, cnt++) srcg[cnt] -= 1. / dy * (-CC(p, i, j - 1) + CC(p, i, j));
  }
  /* surface, :176-187 */
  cnt = 0;
  for (int j = 1; j <= NY; j++) {
    for (int i = 1; i <= NX; i++, cnt++) srca[cnt] += c->ifrcy[cnt];
  }
  /* extension: Boussinesq buoyancy of the volume fraction along y, the
   * face value of vof averaged from the two cells beside the uy face; absent
   * from the reference, whose only body force is the temperature buoyancy
   * along x (ux.c:181-197) */
  if (0. != c->grav_vof) {
    cnt = 0;
    for (int j = 1; j <= NY; j++) {
      for (int i = 1; i <= NX; i++, cnt++) {
        srca[cnt] += c->grav_vof * (0.5 * VOF(i, j - 1) + 0.5 * VOF(i, j) - c->vof_ref);
      }
    }
  }
}

static void rhs_t(svo_ctx_t *c) {
  /* compute_rhs_t, t.c:160-182 */
  const double dy = c->dy;
  const double dif = c->prm.t_dif;
  double *srca = c->srct[0], *srcg = c->srct[2];
  const double *uy = c->uy, *t = c->t;
  int cnt;
  /* advection_x, :68-89 */
  cnt = 0;
  for (int j = 1; j <= NY; j++) {
    for (int i = 1; i <= NX; i++, cnt++) {
      const double l = +0.5 / DXF(i) * UX(i, j);
      const double u = -0.5 / DXF(i) * UX(i + 1, j);
      const double cc = -l - u;
      srca[cnt] += +l * CC(t, i - 1, j) + cc * CC(t, i, j) + u * CC(t, i + 1, j);
    }
  }
  /* advection_y, :91-112 */
  cnt = 0;
  for (int j = 1; j <= NY; j++) {
    for (int i = 1; i <= NX; i++, cnt++) {
      const double l = +0.5 / dy * CC(uy, i, j);
      const double u = -0.5 / dy * CC(uy, i, j + 1);
      const double cc = -l - u;
      srca[cnt] += +l * CC(t, i, j - 1) + cc * CC(t, i, j) + u * CC(t, i, j + 1);
    }
  }
  /* diffusion_x (srcg), :115-133 */
  cnt = 0;
  for (int j = 1; j <= NY; j++) {
    for (int i = 1; i <= NX; i++, cnt++) {
      const double *lx = c->lapx_t + 3 * (i - 1);
      srcg[cnt] += dif * (+lx[0] * CC(t, i - 1, j) + lx[1] * CC(t, i, j) + lx[2] * CC(t, i + 1, j));
    }
  }
  /* diffusion_y (srca), :135-153 */
  cnt = 0;
  for (int j = 1; j <= NY; j++) {
    for (int i = 1; i <= NX; i++, cnt++) {
      srca[cnt] += dif * (+c->lapy[0] * CC(t, i, j - 1) + c->lapy[1] * CC(t, i, j) + c->lapy[2] * CC(t, i, j + 1));
    }
  }
}

/* increments of predict_{ux,uy,t}, e.g. ux.c:330-347 */
static void increments(svo_ctx_t *c, double *const *s, const long nitems, const int rkstep, const double dt) {
  const double coef_a = RK_A[rkstep], coef_b = RK_B[rkstep], coef_g = rk_g(rkstep);
  for (long n = 0; n < nitems; n++) {
    c->x1pncl[n] = +coef_a * dt * s[0][n] + coef_b * dt * s[1][n] + coef_g * dt * s[2][n];
  }
}

static void predict_tail(svo_ctx_t *c, int rkstep, double dt);

int svo_predict(svo_ctx_t *c, int rkstep, double dt) {
  /* fluid_predict_field, src/fluid/predict/main.c:62-79 */
  reset_srcs3(c, c->srcux, c->n_srcux, rkstep);
  reset_srcs3(c, c->srcuy, c->n_src, rkstep);
  reset_srcs3(c, c->srct, c->n_src, rkstep);
  rhs_ux(c);
  rhs_uy(c);
  rhs_t(c);
  predict_tail(c, rkstep, dt);
  return 0;
}

/* increments, x-implicit solves, updates and boundary updates of
 * predict_{ux,uy,t}: linear in the sources and fields, so the tangent-linear
 * model runs it on its own context as well */
static void predict_tail(svo_ctx_t *c, int rkstep, double dt) {
  /* predict_ux, ux.c:306-388 */
  {
    increments(c, c->srcux, c->n_srcux, rkstep, dt);
    const double prefactor = 0.5 * rk_g(rkstep) * dt * c->prm.m_dif;
    solve_in_x(c, prefactor, c->lapx_ux, NX - 1);
    int cnt = 0;
    for (int j = 1; j <= NY; j++) {
      for (int i = 2; i <= NX; i++, cnt++) UX(i, j) += c->x1pncl[cnt];
    }
    bc_ux(c);
  }
  /* predict_uy, uy.c:278-360 */
  {
    increments(c, c->srcuy, c->n_src, rkstep, dt);
    const double prefactor = 0.5 * rk_g(rkstep) * dt * c->prm.m_dif;
    solve_in_x(c, prefactor, c->lapx_uy, NX);
    int cnt = 0;
    for (int j = 1; j <= NY; j++) {
      for (int i = 1; i <= NX; i++, cnt++) CC(c->uy, i, j) += c->x1pncl[cnt];
    }
    bc_uy(c);
  }
  /* predict_t, t.c:239-321 */
  {
    increments(c, c->srct, c->n_src, rkstep, dt);
    const double prefactor = 0.5 * rk_g(rkstep) * dt * c->prm.t_dif;
    solve_in_x(c, prefactor, c->lapx_t, NX);
    int cnt = 0;
    for (int j = 1; j <= NY; j++) {
      for (int i = 1; i <= NX; i++, cnt++) CC(c->t, i, j) += c->x1pncl[cnt];
    }
    bc_t(c);
  }
}

/* ---------------- Poisson: src/fluid/compute_potential/{dct,dft}.c ---------------- */

/* assign_input, dct.c:285-315 / dft.c:315-345 (norm differs) */
static void assign_input(svo_ctx_t *c, const int rkstep, const double dt, const double norm, double *rhs) {
  const double dy = c->dy;
  const double prefactor = 1. / (rk_g(rkstep) * dt) / norm;
  int cnt = 0;
  for (int j = 1; j <= NY; j++) {
    for (int i = 1; i <= NX; i++, cnt++) {
      const double dx = DXF(i);
      const double ux_xm = UX(i, j);
      const double ux_xp = UX(i + 1, j);
      const double uy_ym = CC(c->uy, i, j);
      const double uy_yp = CC(c->uy, i, j + 1);
      rhs[cnt] = prefactor * (+(ux_xp - ux_xm) / dx + (uy_yp - uy_ym) / dy);
    }
  }
}

/* extract_output, dct.c:317-332 / dft.c:347-362 */
static void extract_output(svo_ctx_t *c, const double *rhs) {
  int cnt = 0;
  for (int j = 1; j <= NY; j++) {
    for (int i = 1; i <= NX; i++, cnt++) CC(c->psi, i, j) = rhs[cnt];
  }
  bc_neumann(c, c->psi);
}

/* fluid_compute_potential_dct, dct.c:373-421 */
int svo_potential_dct(svo_ctx_t *c, int rkstep, double dt) {
  const int nx = NX, ny = NY;
  double *buf0 = c->pbuf0, *buf1 = c->pbuf1;
  assign_input(c, rkstep, dt, 2. * nx, buf0);
  /* REDFT10 along x for every row, buf0 -> buf1 */
  for (int j = 0; j < ny; j++) svof_dct2(c->plan_x, buf0 + (size_t)j * nx, buf1 + (size_t)j * nx);
  /* x1 -> y1 transpose, buf1 -> buf0: element (k, j) at k * ny + j */
  for (int j = 0; j < ny; j++) {
    for (int k = 0; k < nx; k++) buf0[(size_t)k * ny + j] = buf1[(size_t)j * nx + k];
  }
  /* solve_linear_systems, dct.c:334-362 */
  for (int j = 0; j < ny; j++) {
    c->tdm_l[j] = 1. / c->dy / c->dy;
    c->tdm_u[j] = 1. / c->dy / c->dy;
  }
  for (int m = 0; m < nx; m++) {
    for (int n = 0; n < ny; n++) c->tdm_c[n] = -c->tdm_l[n] - c->tdm_u[n] + c->evals_dct[m];
    tdm_periodic(ny, c->tdm_l, c->tdm_c, c->tdm_u, c->tdm_v, buf0 + (size_t)m * ny, c->tdm_q1);
  }
  /* y1 -> x1 transpose, buf0 -> buf1 */
  for (int j = 0; j < ny; j++) {
    for (int k = 0; k < nx; k++) buf1[(size_t)j * nx + k] = buf0[(size_t)k * ny + j];
  }
  /* REDFT01 along x, buf1 -> buf0 */
  for (int j = 0; j < ny; j++) svof_dct3(c->plan_x, buf1 + (size_t)j * nx, buf0 + (size_t)j * nx);
  extract_output(c, buf0);
  return 0;
}

/* fluid_compute_potential_dft, dft.c:406-468 */
int svo_potential_dft(svo_ctx_t *c, int rkstep, double dt) {
  const int nx = NX, ny = NY, nky = ny / 2 + 1;
  double *buf0 = c->pbuf0, *buf1 = c->pbuf1;
  assign_input(c, rkstep, dt, 1. * ny, buf0);
  /* x1 -> y1 (real), buf0 -> buf1: element (i, j) at i * ny + j */
  for (int j = 0; j < ny; j++) {
    for (int i = 0; i < nx; i++) buf1[(size_t)i * ny + j] = buf0[(size_t)j * nx + i];
  }
  /* r2c along y, buf1 -> buf0: element (i, ky) at i * nky + ky (complex) */
  for (int i = 0; i < nx; i++) svof_fft_r2c(c->plan_y, buf1 + (size_t)i * ny, buf0 + 2 * (size_t)i * nky);
  /* y1 -> x1 (complex), buf0 -> buf1: element (i, ky) at ky * nx + i */
  for (int i = 0; i < nx; i++) {
    for (int k = 0; k < nky; k++) {
      buf1[2 * ((size_t)k * nx + i) + 0] = buf0[2 * ((size_t)i * nky + k) + 0];
      buf1[2 * ((size_t)k * nx + i) + 1] = buf0[2 * ((size_t)i * nky + k) + 1];
    }
  }
  /* solve_linear_systems, dft.c:364-395 (complex Thomas, component-wise) */
  for (int m = 0; m < nky; m++) {
    for (int n = 0; n < nx; n++) c->tdm_c[n] = -c->plap_l[n] - c->plap_u[n] + c->evals_dft[m];
    c->tdm_c[0] += c->plap_l[0];
    c->tdm_c[nx - 1] += c->plap_u[nx - 1];
    gtsv(nx, c->plap_l, c->tdm_c, c->plap_u, c->tdm_v, buf1 + 2 * (size_t)m * nx + 0, 2);
    gtsv(nx, c->plap_l, c->tdm_c, c->plap_u, c->tdm_v, buf1 + 2 * (size_t)m * nx + 1, 2);
  }
  /* x1 -> y1 (complex), buf1 -> buf0 */
  for (int i = 0; i < nx; i++) {
    for (int k = 0; k < nky; k++) {
      buf0[2 * ((size_t)i * nky + k) + 0] = buf1[2 * ((size_t)k * nx + i) + 0];
      buf0[2 * ((size_t)i * nky + k) + 1] = buf1[2 * ((size_t)k * nx + i) + 1];
    }
  }
  /* c2r along y, buf0 -> buf1 */
  for (int i = 0; i < nx; i++) svof_fft_c2r(c->plan_y, buf0 + 2 * (size_t)i * nky, buf1 + (size_t)i * ny);
  /* y1 -> x1 (real), buf1 -> buf0 */
  for (int j = 0; j < ny; j++) {
    for (int i = 0; i < nx; i++) buf0[(size_t)j * nx + i] = buf1[(size_t)i * ny + j];
  }
  extract_output(c, buf0);
  return 0;
}

/* ---------------- projection: src/fluid/correct_velocity ---------------- */
int svo_correct(svo_ctx_t *c, int rkstep, double dt) {
  /* main.c:15-27 */
  const double prefactor = rk_g(rkstep) * dt;
  /* ux.c:16-41 */
  for (int j = 1; j <= NY; j++) {
    for (int i = 2; i <= NX; i++) {
      const double dx = DXC(i);
      const double psi_xm = CC(c->psi, i - 1, j);
      const double psi_xp = CC(c->psi, i, j);
      UX(i, j) -= prefactor / dx * (+psi_xp - psi_xm);
    }
  }
  bc_ux(c);
  /* uy.c:15-39 */
  for (int j = 1; j <= NY; j++) {
    for (int i = 1; i <= NX; i++) {
      const double psi_ym = CC(c->psi, i, j - 1);
      const double psi_yp = CC(c->psi, i, j);
      CC(c->uy, i, j) -= prefactor / c->dy * (+psi_yp - psi_ym);
    }
  }
  bc_uy(c);
  return 0;
}

/* src/fluid/update_pressure.c:12-109 (x implicit, y explicit) */
int svo_update_pressure(svo_ctx_t *c, int rkstep, double dt) {
  for (int j = 1; j <= NY; j++) {
    for (int i = 1; i <= NX; i++) CC(c->p, i, j) += CC(c->psi, i, j);
  }
  const double prefactor = 0.5 * rk_g(rkstep) * dt * c->prm.m_dif;
  for (int j = 1; j <= NY; j++) {
    for (int i = 1; i <= NX; i++) {
      const double dpsidx_xm = (-CC(c->psi, i - 1, j) + CC(c->psi, i, j)) / DXC(i);
      const double dpsidx_xp = (-CC(c->psi, i, j) + CC(c->psi, i + 1, j)) / DXC(i + 1);
      CC(c->p, i, j) -= prefactor / DXF(i) * (-dpsidx_xm + dpsidx_xp);
    }
  }
  bc_neumann(c, c->p);
  return 0;
}

/* ---------------- one step: src/integrate.c:11-68 ---------------- */
int svo_integrate(svo_ctx_t *c, double *dt) {
  if (0 != svo_decide_dt(c, dt)) return 1;
  for (int rkstep = 0; rkstep < 3; rkstep++) {
    svo_curvature_tensor(c);
    svo_force(c);
    svo_update_vof(c, rkstep, *dt);
    svo_predict(c, rkstep, *dt);
    if (c->uniform) {
      svo_potential_dct(c, rkstep, *dt);
    } else {
      svo_potential_dft(c, rkstep, *dt);
    }
    svo_correct(c, rkstep, *dt);
    svo_update_pressure(c, rkstep, *dt);
  }
  return 0;
}

/* one step with a given dt (the time-step sequence of a differentiated run
 * is held fixed) */
int svo_integrate_fixed(svo_ctx_t *c, double dt) {
  for (int rkstep = 0; rkstep < 3; rkstep++) {
    svo_curvature_tensor(c);
    svo_force(c);
    svo_update_vof(c, rkstep, dt);
    svo_predict(c, rkstep, dt);
    if (c->uniform) {
      svo_potential_dct(c, rkstep, dt);
    } else {
      svo_potential_dft(c, rkstep, dt);
    }
    svo_correct(c, rkstep, dt);
    svo_update_pressure(c, rkstep, dt);
  }
  return 0;
}

int svo_set_gravity(svo_ctx_t *c, double grav_vof, double vof_ref) {
  c->grav_vof = grav_vof;
  c->vof_ref = vof_ref;
  return 0;
}

int svo_run(svo_ctx_t *c, int nsteps, double *dts) {
  for (int n = 0; n < nsteps; n++) {
    double dt = 0.;
    if (0 != svo_integrate(c, &dt)) return 1;
    if (dts) dts[n] = dt;
  }
  return 0;
}

/* ---------------- logging reductions: src/logging/{momentum,energy}.c and src/logging/nusselt/ ----------------
 * out = {x momentum, y momentum (momentum.c:38-54); kinetic energy of ux, of uy,
 * thermal energy (energy.c:41-65); Nusselt numbers from the wall heat flux
 * (nusselt/heat_flux.c:22-41), the kinetic energy injection
 * (kinetic_energy_injection.c:25-49), the kinetic energy dissipation
 * (kinetic_energy_dissipation.c:11-163) and the thermal energy dissipation
 * (thermal_energy_dissipation.c:10-95)}, each normalised by the laminar heat
 * flux t_dif ly (reference.c:4-12); the sums in the reference's loop order */
int svo_logging(svo_ctx_t *c, double out[9]) {
  const double dy = c->dy, md = c->prm.m_dif, td = c->prm.t_dif;
  const double *T = c->t, *UY = c->uy;
#define TT(i, j) CC(T, i, j)
#define VY(i, j) CC(UY, i, j)
  double mx = 0., my = 0.;
  for (int j = 1; j <= NY; j++)
    for (int i = 2; i <= NX; i++) mx += UX(i, j) * (DXC(i) * dy);
  for (int j = 1; j <= NY; j++)
    for (int i = 1; i <= NX; i++) my += VY(i, j) * (DXF(i) * dy);
  double ex = 0., ey = 0., et = 0.;
  for (int j = 1; j <= NY; j++)
    for (int i = 2; i <= NX; i++) ex += 0.5 * pow(UX(i, j), 2.) * (DXC(i) * dy);
  for (int j = 1; j <= NY; j++)
    for (int i = 1; i <= NX; i++) ey += 0.5 * pow(VY(i, j), 2.) * (DXF(i) * dy);
  for (int j = 1; j <= NY; j++)
    for (int i = 1; i <= NX; i++) et += 0.5 * pow(TT(i, j), 2.) * (DXF(i) * dy);
  const double ref = td * c->prm.ly;
  /* heat flux through the two walls */
  double hf = 0.;
  for (int j = 1; j <= NY; j++) {
    const double dtdx_xm = (+TT(1, j) - TT(0, j)) / DXC(1);
    const double dtdx_xp = (+TT(NX + 1, j) - TT(NX, j)) / DXC(NX + 1);
    hf -= 0.5 * td * (dtdx_xm + dtdx_xp) * dy;
  }
  /* kinetic energy injection */
  double inj = 0.;
  for (int j = 1; j <= NY; j++)
    for (int i = 2; i <= NX; i++) {
      const double t_ = +0.5 * TT(i - 1, j) + 0.5 * TT(i, j);
      inj += UX(i, j) * t_ * (DXC(i) * dy);
    }
  /* kinetic energy dissipation: ux-x, ux-y, uy-x, uy-y */
  double kd[4] = {0., 0., 0., 0.};
  for (int j = 1; j <= NY; j++)
    for (int i = 1; i <= NX + 1; i++) {
      const double cs = DXC(i) * dy;
      if (1 != i) {
        const double d = 1. / DXF(i - 1) * (UX(i, j) - UX(i - 1, j));
        const double w = DXF(i - 1) / DXC(i);
        kd[0] += md * 0.5 * w * pow(d, 2.) * cs;
      }
      if (NX + 1 != i) {
        const double d = 1. / DXF(i) * (UX(i + 1, j) - UX(i, j));
        const double w = DXF(i) / DXC(i);
        kd[0] += md * 0.5 * w * pow(d, 2.) * cs;
      }
    }
  for (int j = 1; j <= NY; j++)
    for (int i = 1; i <= NX + 1; i++) {
      const double cs = DXC(i) * dy;
      const double dm = 1. / dy * (UX(i, j) - UX(i, j - 1));
      kd[1] += md * 0.5 * pow(dm, 2.) * cs;
      const double dp = 1. / dy * (UX(i, j + 1) - UX(i, j));
      kd[1] += md * 0.5 * pow(dp, 2.) * cs;
    }
  for (int j = 1; j <= NY; j++)
    for (int i = 1; i <= NX; i++) {
      const double cs = DXF(i) * dy;
      {
        const double d = 1. / DXC(i) * (VY(i, j) - VY(i - 1, j));
        const double w0 = DXC(i) / DXF(i), w1 = 1 == i ? 2. : 1.;
        kd[2] += md * 0.5 * w0 * w1 * pow(d, 2.) * cs;
      }
      {
        const double d = 1. / DXC(i + 1) * (VY(i + 1, j) - VY(i, j));
        const double w0 = DXC(i + 1) / DXF(i), w1 = NX == i ? 2. : 1.;
        kd[2] += md * 0.5 * w0 * w1 * pow(d, 2.) * cs;
      }
    }
  for (int j = 1; j <= NY; j++)
    for (int i = 1; i <= NX; i++) {
      const double cs = DXF(i) * dy;
      const double dm = 1. / dy * (VY(i, j) - VY(i, j - 1));
      kd[3] += md * 0.5 * pow(dm, 2.) * cs;
      const double dp = 1. / dy * (VY(i, j + 1) - VY(i, j));
      kd[3] += md * 0.5 * pow(dp, 2.) * cs;
    }
  /* thermal energy dissipation: x, y */
  double th[2] = {0., 0.};
  for (int j = 1; j <= NY; j++)
    for (int i = 1; i <= NX; i++) {
      const double cs = DXF(i) * dy;
      {
        const double d = 1. / DXC(i) * (TT(i, j) - TT(i - 1, j));
        const double w0 = DXC(i) / DXF(i), w1 = 1 == i ? 2. : 1.;
        th[0] += td * 0.5 * w0 * w1 * pow(d, 2.) * cs;
      }
      {
        const double d = 1. / DXC(i + 1) * (TT(i + 1, j) - TT(i, j));
        const double w0 = DXC(i + 1) / DXF(i), w1 = NX == i ? 2. : 1.;
        th[0] += td * 0.5 * w0 * w1 * pow(d, 2.) * cs;
      }
    }
  for (int j = 1; j <= NY; j++)
    for (int i = 1; i <= NX; i++) {
      const double cs = DXF(i) * dy;
      const double dm = 1. / dy * (TT(i, j) - TT(i, j - 1));
      th[1] += td * 0.5 * pow(dm, 2.) * cs;
      const double dp = 1. / dy * (TT(i, j + 1) - TT(i, j));
      th[1] += td * 0.5 * pow(dp, 2.) * cs;
    }
#undef TT
#undef VY
  double kdis = 0.;
  kdis += kd[0];
  kdis += kd[1];
  kdis += kd[2];
  kdis += kd[3];
  double tdis = 0.;
  tdis += th[0];
  tdis += th[1];
  out[0] = mx;
  out[1] = my;
  out[2] = ex;
  out[3] = ey;
  out[4] = et;
  out[5] = hf / ref;
  out[6] = inj / ref + 1.;
  out[7] = kdis / ref + 1.;
  out[8] = tdis / ref;
  return 0;
}


/* ---------- time-averaged statistics (src/statistics.c) ---------- */

/* widths of the statistics arrays (array_macros/statistics/ux1.h .. uxt.h): ux1, ux2
 * and uxt hold i = 1 .. nx+1, the others i = 0 .. nx+1; rows j = 1 .. ny,
 * no halo */
static int stat_width(const svo_ctx_t *c, int q) { return (0 == q || 1 == q || 6 == q) ? NX + 1 : NX + 2; }

/* one sample: collect_mean_ux, collect_mean_uy, collect_mean_t and
 * collect_uxt (src/statistics.c:117-204), pow() as the reference calls it */
int svo_stat_collect(svo_ctx_t *c) {
  if (!c->stat[0])
    for (int q = 0; q < 7; q++) c->stat[q] = dalloc((long)stat_width(c, q) * NY);
  const double *T = c->t, *UY = c->uy;
  double *ux1 = c->stat[0], *ux2 = c->stat[1], *uy1 = c->stat[2], *uy2 = c->stat[3];
  double *t1 = c->stat[4], *t2 = c->stat[5], *uxt = c->stat[6];
#define SX(a, i, j) (a)[(i) - 1 + (NX + 1) * ((j) - 1)]
#define SC(a, i, j) (a)[(i) + (NX + 2) * ((j) - 1)]
  for (int j = 1; j <= NY; j++)
    for (int i = 1; i <= NX + 1; i++) {
      SX(ux1, i, j) += pow(UX(i, j), 1.);
      SX(ux2, i, j) += pow(UX(i, j), 2.);
    }
  for (int j = 1; j <= NY; j++)
    for (int i = 0; i <= NX + 1; i++) {
      SC(uy1, i, j) += pow(CC(UY, i, j), 1.);
      SC(uy2, i, j) += pow(CC(UY, i, j), 2.);
    }
  for (int j = 1; j <= NY; j++)
    for (int i = 0; i <= NX + 1; i++) {
      SC(t1, i, j) += pow(CC(T, i, j), 1.);
      SC(t2, i, j) += pow(CC(T, i, j), 2.);
    }
  for (int j = 1; j <= NY; j++)
    for (int i = 1; i <= NX + 1; i++) {
      const double t_ = +0.5 * CC(T, i - 1, j) + 0.5 * CC(T, i, j);
      SX(uxt, i, j) += UX(i, j) * t_;
    }
#undef SX
#undef SC
  c->stat_num += 1;
  return 0;
}

/* reduce_and_write (src/statistics.c:232-281): out[i] = sum over the rows in
 * order, starting from zero; out holds stat_width() values */
int svo_stat_reduce(const svo_ctx_t *c, int q, double *out) {
  if (q < 0 || q > 6) return 1;
  const int w = stat_width(c, q);
  for (int i = 0; i < w; i++) out[i] = 0.;
  if (!c->stat[0]) return 0;
  for (int j = 0; j < NY; j++)
    for (int i = 0; i < w; i++) out[i] += c->stat[q][(long)j * w + i];
  return 0;
}

long svo_stat_num(const svo_ctx_t *c) { return c->stat_num; }

#include "svof_oracle_tl.inc"
