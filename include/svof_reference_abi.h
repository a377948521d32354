/*
 * svof_reference_abi.h -- the reference's own solver entry points, with the
 * reference's signatures and struct layouts, implemented by libsvof_b200.so
 * on the GPU (drop-in boundary).
 *
 * A host program written against SimpleVOFSolver's headers (its main.c,
 * logging, save and statistics code, compiled with -DNDIMS=2) links this
 * library instead of the reference's solver sources (src/fluid/*,
 * src/interface/*, src/integrate.c, src/linear_system.c, src/tdm.c,
 * src/runge_kutta.c, src/param/*) and runs unchanged.  The structs below
 * reproduce the reference's layouts (include/array.h:10-23,
 * include/domain.h:19-28, include/fluid.h:20-31, include/interface.h:13-24,
 * include/linear_system.h:24-35) so both sides agree on every offset.
 *
 * Memory: fluid_init / interface_init allocate every array_t.data in CUDA
 * managed memory.  The host reads the fields through these pointers exactly as
 * the reference's logging and save code does; each entry point returns only
 * after its device work finished.  As in the reference (reset_srcs,
 * src/fluid/predict/main.c:9-29), the data pointers of arrays the solver
 * double-buffers change between calls: read fluid->ux.data afresh each time.
 *
 * Parameters: Ra, Pr, We, coef_dt_adv, coef_dt_dif from the environment, read
 * where the reference reads them.  The reference's compile-time parameters
 * (include/param.h:10-34) default to its values (src/param/*.c: buoyancy on,
 * wall velocities 0, wall temperatures +0.5 / -0.5) and may be overridden by
 * the environment variables SVOF_ADD_BUOYANCY, SVOF_UY_XM, SVOF_UY_XP,
 * SVOF_T_XM, SVOF_T_XP.  Diffusion is implicit in x, explicit in y
 * (src/param/implicit.c:3-7); other choices are refused.
 *
 * Scope: one process, one GPU (domain->mysizes must equal glsizes).
 */
#ifndef SVOF_REFERENCE_ABI_H
#define SVOF_REFERENCE_ABI_H

#include <stdbool.h>
#include <stddef.h>

#ifndef NDIMS
#define NDIMS 2
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct sdecomp_info_t_ sdecomp_info_t;
typedef struct sdecomp_transpose_plan_t_ sdecomp_transpose_plan_t;
typedef struct tdm_info_t_ tdm_info_t;

/* include/array.h:10-23 */
typedef struct {
  size_t size;
  int (*nadds)[2];
  size_t datasize;
  void *data;
} array_t;

/* include/domain.h:19-28 */
typedef struct {
  sdecomp_info_t *info;
  size_t glsizes[NDIMS];
  size_t mysizes[NDIMS];
  size_t offsets[NDIMS];
  double lengths[NDIMS];
  double *xf, *xc;
  double *dxf, *dxc;
  double dy;
} domain_t;

/* include/fluid.h:20-31 */
typedef struct {
  array_t ux;
  array_t uy;
  array_t p;
  array_t psi;
  array_t t;
  array_t srcux[3];
  array_t srcuy[3];
  array_t srct[3];
  double Ra, Pr;
  double m_dif, t_dif;
} fluid_t;

/* include/interface.h:13-24 */
typedef struct {
  array_t vof;
  array_t ifrcx;
  array_t ifrcy;
  array_t dvof;
  array_t normal;
  array_t curv;
  array_t flxx;
  array_t flxy;
  array_t src[2];
  double tension;
} interface_t;

/* include/linear_system.h:24-35 */
typedef struct {
  bool is_initialised;
  bool implicit[NDIMS];
  double *x1pncl;
  double *y1pncl;
  size_t x1pncl_mysizes[NDIMS];
  size_t y1pncl_mysizes[NDIMS];
  tdm_info_t *tdm_x;
  tdm_info_t *tdm_y;
  sdecomp_transpose_plan_t *transposer_x1_to_y1;
  sdecomp_transpose_plan_t *transposer_y1_to_x1;
} linear_system_t;

/* include/fluid_solver.h:10-99 */
int fluid_init(const char dirname_ic[], const domain_t *domain, fluid_t *fluid);
int fluid_save(const char dirname[], const domain_t *domain, const fluid_t *fluid);
int fluid_decide_dt(const domain_t *domain, const fluid_t *fluid, double *dt);
int fluid_predict_field(const domain_t *domain, const size_t rkstep, const double dt, fluid_t *fluid,
                        const interface_t *interface);
int fluid_compute_potential_dft(const domain_t *domain, const size_t rkstep, const double dt, fluid_t *fluid);
int fluid_compute_potential_dct(const domain_t *domain, const size_t rkstep, const double dt, fluid_t *fluid);
int fluid_correct_velocity(const domain_t *domain, const size_t rkstep, const double dt, fluid_t *fluid);
int fluid_update_pressure(const domain_t *domain, const size_t rkstep, const double dt, fluid_t *fluid);
int fluid_update_boundaries_ux(const domain_t *domain, array_t *ux);
int fluid_update_boundaries_uy(const domain_t *domain, array_t *uy);
int fluid_update_boundaries_p(const domain_t *domain, array_t *p);
int fluid_update_boundaries_psi(const domain_t *domain, array_t *psi);
int fluid_update_boundaries_t(const domain_t *domain, array_t *t);

/* include/interface_solver.h:8-41 */
int interface_init(const char dirname_ic[], const domain_t *domain, interface_t *interface);
int interface_save(const char dirname[], const domain_t *domain, const interface_t *interface);
int interface_compute_curvature_tensor(const domain_t *domain, interface_t *interface);
int interface_compute_force(const domain_t *domain, interface_t *interface);
int interface_update_vof(const domain_t *domain, const size_t rkstep, const double dt, const fluid_t *fluid,
                         interface_t *interface);
int interface_update_boundaries_vof(const domain_t *domain, array_t *vof);

/* include/linear_system.h:37-46: the line solves run on the device, so the
 * struct holds only the pencil buffers and sizes; tdm_x / tdm_y stay NULL */
int linear_system_init(const sdecomp_info_t *info, const bool implicit[NDIMS], const size_t glsizes[NDIMS],
                       linear_system_t *linear_system);
int linear_system_finalise(linear_system_t *linear_system);

/* include/integrate.h:5-10: one time step as one CUDA-graph launch */
int integrate(const domain_t *domain, fluid_t *fluid, interface_t *interface, double *dt);

#ifdef __cplusplus
}
#endif

#endif
