/*
 * svof_oracle.h -- CPU restatement of SimpleVOFSolver's per-step hot path
 * (2D, FP64).  TEST INFRASTRUCTURE ONLY: this is the checker for the CUDA
 * library; only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg may load it.
 *
 * Every array is stored exactly as the reference stores it (the index maps of
 * include/array_macros/ in the reference): x fastest, one row per y index,
 * x ghost cells and y halo rows included.  With nx, ny the interior sizes:
 *
 *   ux    (nx+1) x (ny+2)   i in [1, nx+1], j in [0, ny+1]
 *   uy, p, psi, t, curv
 *         (nx+2) x (ny+2)   i in [0, nx+1], j in [0, ny+1]
 *   vof   (nx+2) x (ny+4)   i in [0, nx+1], j in [-1, ny+2]
 *   dvof  2 x (nx+1) x (ny+3)   corners, i in [1, nx+1], j in [0, ny+2]
 *   normal 3 x nx x (ny+2)      i in [1, nx], j in [0, ny+1]
 *   flxx  (nx+1) x ny,  flxy nx x (ny+1)
 *   ifrcx, srcux[3]  (nx-1) x ny  (i in [2, nx]);  ifrcy, srcuy[3], srct[3],
 *   src[2]  nx x ny
 */
#ifndef SVOF_ORACLE_H
#define SVOF_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int nx, ny;
  double lx, ly;
  double m_dif, t_dif;       /* sqrt(Pr)/sqrt(Ra), 1/(sqrt(Pr) sqrt(Ra)) */
  double tension;            /* 1 / We */
  double coef_dt_adv, coef_dt_dif;
  int add_buoyancy;          /* reference param_add_buoyancy */
  double uy_xm, uy_xp;       /* wall velocities (param_uy_x[mp]) */
  double t_xm, t_xp;         /* wall temperatures (param_t_x[mp]) */
} svo_params_t;

typedef struct svo_ctx svo_ctx_t;

svo_ctx_t *svo_create(const svo_params_t *params, const double *xf, const double *xc);
void svo_destroy(svo_ctx_t *ctx);
/* pointer to the storage of a field (names as the reference's members:
 * ux uy p psi t srcux0..2 srcuy0..2 srct0..2 vof ifrcx ifrcy dvof normal curv
 * flxx flxy src0 src1); *count receives the number of doubles */
double *svo_field(svo_ctx_t *ctx, const char *name, long *count);
/* boundary/halo update of ux uy p t vof, as fluid_init/interface_init do */
int svo_init_boundaries(svo_ctx_t *ctx);
int svo_x_grid_is_uniform(svo_ctx_t *ctx);

int svo_decide_dt(svo_ctx_t *ctx, double *dt);
int svo_curvature_tensor(svo_ctx_t *ctx);
int svo_force(svo_ctx_t *ctx);
int svo_update_vof(svo_ctx_t *ctx, int rkstep, double dt);
int svo_predict(svo_ctx_t *ctx, int rkstep, double dt);
int svo_potential_dct(svo_ctx_t *ctx, int rkstep, double dt);
int svo_potential_dft(svo_ctx_t *ctx, int rkstep, double dt);
int svo_correct(svo_ctx_t *ctx, int rkstep, double dt);
int svo_update_pressure(svo_ctx_t *ctx, int rkstep, double dt);
int svo_integrate(svo_ctx_t *ctx, double *dt);
int svo_run(svo_ctx_t *ctx, int nsteps, double *dts);
/* one step with a given dt (no CFL decision) */
int svo_integrate_fixed(svo_ctx_t *ctx, double dt);
/* extension absent from the reference: buoyancy of the volume fraction on uy,
 * srcuy_a += grav_vof * (vof at the uy face - vof_ref); grav_vof = g_y (1 -
 * density ratio) in the Boussinesq form, vof_ref the domain-mean volume
 * fraction (zero net force).  Off (the reference's physics) while grav_vof is 0. */
int svo_set_gravity(svo_ctx_t *ctx, double grav_vof, double vof_ref);

/* Tangent-linear model of one step (linearisation of every function above
 * about the current state of `c`).  `d` is a second context on the same grid
 * and parameters, with zero wall values, whose arrays hold the tangents
 * (directional derivatives) of c's fields; `dtension` is the tangent of the
 * surface tension coefficient 1/We, `dgrav` that of the vof buoyancy
 * coefficient grav_vof.  The time step is held fixed.  Advances
 * both contexts by one step. */
int svo_tl_integrate_fixed(svo_ctx_t *c, svo_ctx_t *d, double dt, double dtension, double dgrav);
/* the linearised functions one by one: each reads the primal state of c at
 * the function's input, so it runs before the primal function of the same
 * name; the linear functions (potential, correct, update_pressure) are the
 * primal functions applied to d */
int svo_tl_curvature_tensor(svo_ctx_t *c, svo_ctx_t *d);
int svo_tl_force(svo_ctx_t *c, svo_ctx_t *d, double dtension);
int svo_tl_update_vof(svo_ctx_t *c, svo_ctx_t *d, int rkstep, double dt);
int svo_tl_predict(svo_ctx_t *c, svo_ctx_t *d, int rkstep, double dt, double dgrav);
/* logging reductions of the current fields (src/logging/momentum.c,
 * energy.c, nusselt/ sources): out = {momentum x, y; energy ux, uy, t; Nusselt from
 * the wall heat flux, kinetic energy injection, kinetic and thermal energy
 * dissipation} */
int svo_logging(svo_ctx_t *ctx, double out[9]);
/* time-averaged statistics (src/statistics.c:117-281): one sample of ux1 ux2
 * uy1 uy2 t1 t2 uxt (q = 0 .. 6), the row sum of one quantity (nx+1 values
 * for ux1 ux2 uxt, nx+2 for the others), the number of samples */
int svo_stat_collect(svo_ctx_t *ctx);
int svo_stat_reduce(const svo_ctx_t *ctx, int q, double *out);
long svo_stat_num(const svo_ctx_t *ctx);

#ifdef __cplusplus
}
#endif

#endif
