/*
 * svof3d_b200.h -- C ABI of the B200 library's 3D path (FP64).
 *
 * The 3D solver's step functions, with the reference 2D entry points'
 * semantics and call order (include/fluid_solver.h:10-99,
 * include/interface_solver.h:8-41, include/integrate.h:5-10), carried to a
 * third, periodic z direction that is treated like y.  The mounted reference is
 * its 2D branch, so no reference 3D entry point is replaced one to one.  The
 * field layouts follow the reference's 3D layout generator
 * (tools/define_arrays.py:192-229): x fastest, then y, then z, with halo
 * widths ux (0,1)(1,1)(1,1), uy uz p psi t curv (1,1)(1,1)(1,1),
 * vof (1,1)(2,2)(2,2) in (x)(y)(z).
 *
 *   ux        (nz+2) x (ny+2) x (nx+1)    UX(i,j,k), i = 1 .. nx+1
 *   uy uz p t psi curv
 *             (nz+2) x (ny+2) x (nx+2)    i = 0 .. nx+1
 *   vof       (nz+4) x (ny+4) x (nx+2)    j, k = -1 .. n+2
 *   normal    (nz+2) x (ny+2) x nx x 4    (nx, ny, nz, intercept) per cell
 *   ifrcx, srcux_*   nz x ny x (nx-1)     i = 2 .. nx
 *   ifrcy, ifrcz, srcuy_*, srcuz_*, srct_*, src_*   nz x ny x nx
 *
 * Every function returns 0 on success and non-zero on failure, with a message
 * in svof3d_last_error().  All device work runs on the solver's own stream,
 * except the host copies of the queued loads and stores, which run on two
 * copy streams the solver makes for them.
 * A solver is not reentrant: one host thread drives it at a time.
 *
 * Failure detection as in svof_b200.h: a non-finite velocity met by the CFL
 * reduction, or a time step that is not a positive finite number, makes the
 * next call that waits for the solver's stream (svof3d_fluid_decide_dt,
 * svof3d_run, svof3d_integrate, svof3d_last_dt, svof3d_io_wait,
 * svof3d_synchronize) return non-zero; SVOF_FAIL_ALLOC=N fails the N-th
 * device buffer allocation of svof3d_create.  Two health counters that are
 * not failures (the reference carries on silently in both cases) accumulate
 * on the device and are read by svof3d_health.
 */
#ifndef SVOF3D_B200_H
#define SVOF3D_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct svof3d_solver svof3d_solver_t;

typedef struct {
  int nx, ny, nz;               /* cells; ny and nz powers of two, nx >= 4 */
  double lx, ly, lz;            /* domain lengths */
  double m_dif, t_dif;          /* momentum and thermal diffusivities */
  double tension;               /* surface tension coefficient 1 / We */
  double coef_dt_adv, coef_dt_dif;
  int add_buoyancy;             /* +T on the x momentum */
  double uy_xm, uy_xp;          /* wall values of uy at x = 0, lx */
  double uz_xm, uz_xp;          /* wall values of uz */
  double t_xm, t_xp;            /* wall values of t */
  int precision;                /* SVOF3_FP64, SVOF3_MIXED or SVOF3_MIXED_DC */
} svof3d_params_t;

/* precision of svof3d_params_t:
 *   SVOF3_FP64   every array and every operation in FP64 (follows the
 *                restatement's rounding; only exp / log may differ)
 *   SVOF3_MIXED  velocities, pressure, psi, t, vof and the vof sources stay
 *                FP64; curvature, normals, forces, momentum sources and the
 *                predictor's sweep scratch are FP32; interface geometry and
 *                THINC compute in FP32; the momentum stencils, the x line
 *                solves, the vof update and the whole Poisson solve (the
 *                FP64 path's kernels, one pass, its y transforms carrying
 *                two columns per complex line) in FP64.  Fields stored in
 *                FP32 are converted to FP64 by svof3d_download_field / from
 *                FP64 by svof3d_upload_field.
 *   SVOF3_MIXED_DC as SVOF3_MIXED, with the Poisson solve in the form of a
 *                defect correction: an FP32 pass (FP32 spectrum, twiddles
 *                and transforms; the x line solve computing in FP64), the
 *                FP64 residual of its psi against the operator the solve
 *                inverts, and a second FP32 pass on the residual added to
 *                psi. */
enum { SVOF3_FP64 = 0, SVOF3_MIXED = 1, SVOF3_MIXED_DC = 2 };

enum {
  SVOF3_UX = 0,
  SVOF3_UY,
  SVOF3_UZ,
  SVOF3_P,
  SVOF3_T,
  SVOF3_VOF,
  SVOF3_PSI,
  SVOF3_CURV,
  SVOF3_NORMAL,
  SVOF3_IFRCX,
  SVOF3_IFRCY,
  SVOF3_IFRCZ,
  SVOF3_SRCUX_A,  /* momentum / scalar sources of the current substep (src_a) */
  SVOF3_SRCUX_B,  /* ... and of the previous substep (src_b) */
  SVOF3_SRCUY_A,
  SVOF3_SRCUY_B,
  SVOF3_SRCUZ_A,
  SVOF3_SRCUZ_B,
  SVOF3_SRCT_A,
  SVOF3_SRCT_B,
  SVOF3_SRC_A,    /* vof sources */
  SVOF3_SRC_B,
  SVOF3_NFIELDS
};

/* kernel kinds of svof3d_profile_step */
enum {
  SVOF3_K_DT = 0,
  SVOF3_K_GEOM,
  SVOF3_K_FORCE,
  SVOF3_K_VOF,
  SVOF3_K_PREDICT,
  SVOF3_K_POISSON_FWD,   /* divergence + r2c along y */
  SVOF3_K_POISSON_Z,     /* complex DFT along z, both directions */
  SVOF3_K_POISSON_SOLVE, /* complex Thomas along x */
  SVOF3_K_POISSON_INV,   /* c2r along y + psi boundaries */
  SVOF3_K_PROJECT,
  SVOF3_NKINDS
};

const char *svof3d_last_error(void);

/* xf: nx+1 face positions, xc: nx+2 centre positions (restart-file xf, xc) */
int svof3d_create(const svof3d_params_t *params, const double *xf, const double *xc, svof3d_solver_t **out);
int svof3d_destroy(svof3d_solver_t *s);

/* whole storage arrays (layouts above) */
int svof3d_field_count(const svof3d_solver_t *s, int field, size_t *count);
int svof3d_upload_field(svof3d_solver_t *s, int field, const double *host, size_t count);
int svof3d_download_field(svof3d_solver_t *s, int field, double *host, size_t count);
int svof3d_device_field(svof3d_solver_t *s, int field, double **dptr);

/* restart-file layout: interior y and z rows, x ghost cells included,
 * nz x ny x (nx+1) for ux and nz x ny x (nx+2) for uy, uz, p, t, psi, vof;
 * loading applies the field's halo and wall update */
int svof3d_load_interior(svof3d_solver_t *s, int field, const double *host, size_t count);
int svof3d_store_interior(svof3d_solver_t *s, int field, double *host, size_t count);

/* Queued forms of the two calls above, for streaming restart states through
 * one solver (load, enqueue steps, store, repeat) without waiting in between.
 * Each call returns once its copy is queued; in device order it sits after
 * the steps queued before it and before the steps queued after it.  The host
 * copy runs on a copy stream of its own (one per direction) through a
 * staging buffer in device memory, so host-to-device copies, device-to-host
 * copies and steps overlap; the host buffer must be page-locked for that and
 * must stay valid, and a load's buffer unchanged, until svof3d_io_wait()
 * returns.  The staging buffers (one per field and direction, restart-layout
 * size) are made on first use and freed by svof3d_destroy().  The restart
 * files they stand in for are read by fluid_init / interface_init and
 * written by fluid_save / interface_save (src/fluid/init.c:72,
 * src/fluid/save.c:8, src/interface/init.c:55, src/interface/save.c:7),
 * called from src/main.c:29-30 and src/main.c:78-82. */
int svof3d_load_interior_async(svof3d_solver_t *s, int field, const double *host, size_t count);
int svof3d_store_interior_async(svof3d_solver_t *s, int field, double *host, size_t count);
/* waits for every queued load, step and store */
int svof3d_io_wait(svof3d_solver_t *s);

/* the step functions; rkstep in 0 .. 2 */
int svof3d_fluid_decide_dt(svof3d_solver_t *s, double *dt);
int svof3d_interface_compute_curvature_tensor(svof3d_solver_t *s);
int svof3d_interface_compute_force(svof3d_solver_t *s);
int svof3d_interface_update_vof(svof3d_solver_t *s, size_t rkstep, double dt);
int svof3d_fluid_predict_field(svof3d_solver_t *s, size_t rkstep, double dt);
int svof3d_fluid_compute_potential_dft(svof3d_solver_t *s, size_t rkstep, double dt);
int svof3d_fluid_correct_velocity(svof3d_solver_t *s, size_t rkstep, double dt);
int svof3d_fluid_update_pressure(svof3d_solver_t *s, size_t rkstep, double dt);

/* one full step (decide_dt + 3 substeps) as one CUDA graph launch */
int svof3d_integrate(svof3d_solver_t *s, double *dt);
/* nsteps steps; dts (may be NULL) receives each step's dt */
int svof3d_run(svof3d_solver_t *s, int nsteps, double *dts);
/* nsteps steps queued on the solver's stream without waiting */
int svof3d_enqueue_steps(svof3d_solver_t *s, int nsteps);
/* dt of the last completed step; waits for the stream */
int svof3d_last_dt(svof3d_solver_t *s, double *dt);

/* max |div u| over the interior cells, vof min / max and total volume sum(vof dx dy dz) */
int svof3d_diagnostics(svof3d_solver_t *s, double *divmax, double *vofmin, double *vofmax, double *volume);
/* Time-averaged statistics on the device, the 2D collection of
 * src/statistics.c:117-204 carried to 3D (the reference's 3D statistics code
 * is not in the mounted sources): each svof3d_statistics_collect() adds one
 * sample of the current fields, queued on the solver's stream,
 *   ux1 += ux, ux2 += ux^2, uy1 += uy, uy2 += uy^2, uz1 += uz, uz2 += uz^2,
 *   t1 += t, t2 += t^2, uxt += ux (t(i-1) + t(i)) / 2
 * over the interior rows (j = 1 .. ny, k = 1 .. nz), i = 1 .. nx+1 for ux1
 * ux2 uxt and i = 0 .. nx+1 for the others; arrays nz x ny x (nx+1) or
 * nz x ny x (nx+2), no halo.  Squares are the correctly rounded products. */
enum {
  SVOF3_STAT_UX1 = 0,
  SVOF3_STAT_UX2,
  SVOF3_STAT_UY1,
  SVOF3_STAT_UY2,
  SVOF3_STAT_UZ1,
  SVOF3_STAT_UZ2,
  SVOF3_STAT_T1,
  SVOF3_STAT_T2,
  SVOF3_STAT_UXT,
  SVOF3_NSTATS
};
int svof3d_statistics_collect(svof3d_solver_t *s);
int svof3d_statistics_reset(svof3d_solver_t *s);
int svof3d_statistics_count(svof3d_solver_t *s, size_t *num);
/* the reduction of reduce_and_write (src/statistics.c:232-281) over y and z:
 * out[i] = sum over k = 1 .. nz, in order from zero, of the plane sums (each
 * the sum over j = 1 .. ny, in order from zero) at column i; count = nx+1
 * (ux1 ux2 uxt) or nx+2 */
int svof3d_statistics_reduce(svof3d_solver_t *s, int quantity, double *out, size_t count);
/* the accumulated array itself */
int svof3d_statistics_field(svof3d_solver_t *s, int quantity, double *out, size_t count);

/* ---- differentiation form (FP64 path; no counterpart in the reference) ----
 * The 2D form of svof_b200.h carried to 3D.  A differentiated run holds the
 * time-step sequence fixed: svof3d_integrate_fixed takes one step with the
 * given dt (no decide_dt) and, when tape is not NULL, records the primal
 * inputs of its three substeps (ux, uy, uz, vof in storage layouts) there:
 * svof3d_tape_count() doubles of device memory.  svof3d_adjoint_step maps
 * the adjoint of a step's outputs to the adjoint of its inputs, in place in
 * the adjoint fields, and accumulates the adjoint of the surface-tension
 * coefficient.  The per-function entry points apply one function's
 * transpose about the solver's current fields (the adjoint of its outputs in,
 * of its inputs out; the adjoints of fields a function does not read pass
 * through): update_pressure (p', psi -> p, psi), correct_velocity (u', psi
 * -> u, psi), compute_potential_dft (psi -> u; psi_bar cleared),
 * predict_field (u', src_a of the next substep -> u, p, the forces, src_a of
 * the previous substep), update_vof (vof', src of the next substep -> u,
 * vof, the normals, src of the previous substep), compute_force (the forces
 * -> vof, curvature, tension), compute_curvature_tensor (normals, curvature
 * -> vof); predict_field also maps to vof and the vof buoyancy coefficient
 * while the extension is on.  A tape (svof3d_tape_count() doubles) holds the
 * three substeps' inputs and the step's final vof.  Adjoint fields are compact: ux faces nz x ny x (nx-1), cells
 * nz x ny x nx, normal nz x ny x nx x 4, tension one value per cell (summed
 * by svof3d_adjoint_tension).  Requires add_buoyancy 0; the temperature is
 * not differentiated.  The adjoint computes in FP64 on every precision: with
 * SVOF3_MIXED / SVOF3_MIXED_DC it is the FP64 step's transpose about the
 * mixed trajectory (the taped FP64 fields), the interface transposes reading
 * normals, intercepts and curvature recomputed in FP64 from vof. */
enum {
  SVOF3_ADJ_UX = 0,
  SVOF3_ADJ_UY,
  SVOF3_ADJ_UZ,
  SVOF3_ADJ_P,
  SVOF3_ADJ_VOF,
  SVOF3_ADJ_PSI,
  SVOF3_ADJ_IFRCX,
  SVOF3_ADJ_IFRCY,
  SVOF3_ADJ_IFRCZ,
  SVOF3_ADJ_CURV,
  SVOF3_ADJ_NORMAL,
  SVOF3_ADJ_SRCUX_A,  /* momentum sources' adjoints (between substeps) */
  SVOF3_ADJ_SRCUY_A,
  SVOF3_ADJ_SRCUZ_A,
  SVOF3_ADJ_SRC_A,    /* vof source's adjoint */
  SVOF3_ADJ_TENSION,
  SVOF3_ADJ_GRAVITY   /* the vof buoyancy coefficient's adjoint, per cell */
};
/* the surface-tension coefficient 1/We of the following steps */
int svof3d_set_tension(svof3d_solver_t *s, double tension);
/* extension (absent from the reference; 0 = off, the default): Boussinesq
 * buoyancy of the volume fraction along y, src_a of uy += grav_vof
 * (0.5 vof(j-1) + 0.5 vof(j) - vof_ref), vof after the substep's advection;
 * with grav_vof = -(1 - r) / Fr^2 it models a density ratio r under gravity
 * along -y (the 2D svof_set_gravity carried to 3D) */
int svof3d_set_gravity(svof3d_solver_t *s, double grav_vof, double vof_ref);
int svof3d_tape_count(const svof3d_solver_t *s, size_t *count);
int svof3d_integrate_fixed(svof3d_solver_t *s, double dt, double *tape);
/* device pointer and element count of an adjoint field (made on first use) */
int svof3d_adjoint_field(svof3d_solver_t *s, int which, double **dptr, size_t *count);
int svof3d_adjoint_reset(svof3d_solver_t *s);
/* the adjoint's gradient floor tau: a corner whose vof gradient times its
 * smallest spacing is below tau (a vof variation below tau across a cell)
 * counts as flat and its normal's transpose (I - n n^T) / |g| as zero.  0,
 * the default of SVOF3_FP64, is the exact transpose; the mixed paths default
 * to 1e-5, below which their FP32 fluxes' vof noise (about 1e-8 beside the
 * interface) would make those transposes grow without bound over steps. */
int svof3d_adjoint_set_gradient_floor(svof3d_solver_t *s, double tau);
/* fp32 != 0: the adjoint's intermediates (the adjoints of the momentum
 * sources, forces, curvature, normals and corner gradients, and the sources'
 * pending terms) stored in FP32; the adjoint fields of the state (u, p, vof,
 * psi), the tension and gravity accumulators, the arithmetic, the x line
 * recurrences and the Poisson solve stay FP64.  Default 0.  Changing it
 * discards the adjoint's buffers (they are made again on the next adjoint
 * call; set it before svof3d_adjoint_reset).  With fp32 the intermediates
 * are not readable through svof3d_adjoint_field, and the gradient floor
 * defaults to 1e-5 on every path (the exact transpose's intermediates reach
 * ~1e9 at corners of round-off gradients, beyond FP32's resolution). */
int svof3d_adjoint_set_precision(svof3d_solver_t *s, int fp32);
int svof3d_adjoint_step(svof3d_solver_t *s, const double *tape, double dt);
int svof3d_adjoint_fluid_update_pressure(svof3d_solver_t *s, size_t rkstep, double dt);
int svof3d_adjoint_fluid_correct_velocity(svof3d_solver_t *s, size_t rkstep, double dt);
int svof3d_adjoint_fluid_compute_potential_dft(svof3d_solver_t *s, size_t rkstep, double dt);
int svof3d_adjoint_fluid_predict_field(svof3d_solver_t *s, size_t rkstep, double dt);
int svof3d_adjoint_interface_update_vof(svof3d_solver_t *s, size_t rkstep, double dt);
int svof3d_adjoint_interface_compute_force(svof3d_solver_t *s);
int svof3d_adjoint_interface_compute_curvature_tensor(svof3d_solver_t *s);
int svof3d_adjoint_tension(svof3d_solver_t *s, double *out);
int svof3d_adjoint_gravity(svof3d_solver_t *s, double *out);

/* one step launched kernel by kernel with events between; ms[k], launches[k] per kind */
int svof3d_profile_step(svof3d_solver_t *s, double *ms, int *launches, int nkinds);
int svof3d_synchronize(svof3d_solver_t *s);
/* health counters since creation or the last reset (waits for the stream;
 * either output may be NULL; reset != 0 clears both after reading):
 * newton_unconverged  THINC intercepts (svof3d_interface_compute_curvature_tensor
 *                     and the steps) whose Newton iteration did not reach the
 *                     1e-12 residual in 8 iterations (the reference keeps the
 *                     last iterate: src/interface/curvature_tensor.c:50-92)
 * small_pivots        Poisson x line solves (svof3d_fluid_compute_potential_dft
 *                     and the steps) other than the singular ky = kz = 0 line
 *                     that met a pivot of magnitude <= DBL_EPSILON (the
 *                     reference zeroes such a last pivot, src/tdm.c:39) */
int svof3d_health(svof3d_solver_t *s, unsigned long long *newton_unconverged, unsigned long long *small_pivots,
                  int reset);
int svof3d_stream(svof3d_solver_t *s, void **stream);

#ifdef __cplusplus
}
#endif

#endif
