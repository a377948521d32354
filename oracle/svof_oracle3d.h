/*
 * svof_oracle3d.h -- CPU restatement of the per-step hot path in 3D (FP64).
 * TEST INFRASTRUCTURE ONLY: the checker of the CUDA library's 3D path.
 *
 * The mounted reference is its 2D branch; its 3D branch is absent.  This
 * restatement extends the 2D algorithm (oracle/svof_oracle.c, pinned to the
 * reference) with z treated like y: periodic, uniform dz, the same stencils
 * and THINC/QQ reconstruction with 2 x 2 x 2 Gauss points, CSF in z, and a
 * Poisson solve by r2c along y, complex DFT along z and a complex Thomas
 * sweep along x (the general path of src/fluid/compute_potential/dft.c with a
 * second periodic direction).  Array layouts follow the reference's layout
 * generator (tools/define_arrays.py:192-229): x fastest, then y, then z;
 * halo widths ux (0,1)(1,1)(1,1), uy uz p psi t curv (1,1)(1,1)(1,1),
 * vof (1,1)(2,2)(2,2), normal 4 values per cell.  Parity against the reference
 * is therefore unpinned in 3D; tests/test_oracle3d.py checks that z-invariant
 * fields reproduce the pinned 2D path.
 */
#ifndef SVOF_ORACLE3D_H
#define SVOF_ORACLE3D_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int nx, ny, nz;
  double lx, ly, lz;
  double m_dif, t_dif, tension, coef_dt_adv, coef_dt_dif;
  int add_buoyancy;
  double uy_xm, uy_xp, uz_xm, uz_xp, t_xm, t_xp;
} svo3_params_t;

typedef struct svo3_ctx svo3_ctx_t;

svo3_ctx_t *svo3_create(const svo3_params_t *params, const double *xf, const double *xc);
void svo3_destroy(svo3_ctx_t *ctx);
double *svo3_field(svo3_ctx_t *ctx, const char *name, long *count);
int svo3_init_boundaries(svo3_ctx_t *ctx);
int svo3_decide_dt(svo3_ctx_t *ctx, double *dt);
int svo3_curvature_tensor(svo3_ctx_t *ctx);
int svo3_force(svo3_ctx_t *ctx);
int svo3_update_vof(svo3_ctx_t *ctx, int rkstep, double dt);
int svo3_predict(svo3_ctx_t *ctx, int rkstep, double dt);
int svo3_potential(svo3_ctx_t *ctx, int rkstep, double dt);
int svo3_correct(svo3_ctx_t *ctx, int rkstep, double dt);
int svo3_update_pressure(svo3_ctx_t *ctx, int rkstep, double dt);
int svo3_integrate(svo3_ctx_t *ctx, double *dt);
int svo3_run(svo3_ctx_t *ctx, int nsteps, double *dts);
/* extension: vof buoyancy on uy, srcuy += grav_vof (vof_face - vof_ref) (0 = off) */
int svo3_set_gravity(svo3_ctx_t *ctx, double grav_vof, double vof_ref);
/* time-averaged statistics: one sample of ux1 ux2 uy1 uy2 uz1 uz2 t1 t2 uxt
 * (q = 0 .. 8), the y-z sum of one quantity (nx+1 values for ux1 ux2 uxt,
 * nx+2 for the others), the number of samples */
int svo3_stat_collect(svo3_ctx_t *ctx);
int svo3_stat_reduce(const svo3_ctx_t *ctx, int q, double *out);
long svo3_stat_num(const svo3_ctx_t *ctx);

#ifdef __cplusplus
}
#endif

#endif
