/*
 * svof_b200.h -- C ABI of the B200 (sm_100a) implementation of
 * SimpleVOFSolver's per-step hot path.
 *
 * Plain pointers and sizes only.  All entry points return 0 on success and a
 * non-zero code on failure (the reference's convention, src/main.c:66-99);
 * svof_last_error() describes the last failure of the calling thread.
 *
 * Failure detection (absent from the reference, whose dt ignores NaN): the
 * CFL reduction of every step sets a device status word when it meets a
 * non-finite velocity (NaN or Inf) or yields a time step that is not a
 * positive finite number; the calls that wait for the solver's stream
 * (svof_fluid_decide_dt, svof_run, svof_integrate, svof_last_dt,
 * svof_synchronize) then return non-zero with that message, and clear the
 * word.  SVOF_FAIL_ALLOC=N in the environment makes the N-th device buffer
 * allocation of svof_create fail (a test hook: no allocation happens).
 *
 * Data layout: every field is stored on the device exactly as the reference
 * stores it in memory (reference include/array_macros/**): float64, x
 * fastest, x ghost cells and y halo rows included.  For nx x ny interior
 * cells:
 *   SVOF_UX                    (ny+2) rows x (nx+1)
 *   SVOF_UY, SVOF_P, SVOF_PSI, SVOF_T, SVOF_CURV
 *                              (ny+2) rows x (nx+2)
 *   SVOF_VOF                   (ny+4) rows x (nx+2)
 *   SVOF_NORMAL                (ny+2) rows x nx x 3   (nx, ny, intercept)
 *   SVOF_IFRCX, SVOF_SRCUX_A/B ny rows x (nx-1)
 *   SVOF_IFRCY, SVOF_SRCUY_A/B, SVOF_SRCT_A/B, SVOF_SRC_A/B
 *                              ny rows x nx
 * The restart (NPY) files of the reference hold rows 1..ny of ux, uy, p, t,
 * vof (src/array.c:80-206); svof_load_interior() accepts exactly that part.
 *
 * Threading: one solver is used by one host thread at a time; all device
 * work is issued on the solver's own CUDA stream.
 */
#ifndef SVOF_B200_H
#define SVOF_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct svof_solver svof_solver_t;

/* run-time form of the reference's compile-time and env parameters:
 * include/param.h:10-34 (buoyancy, wall values), src/fluid/init.c:90-93
 * (m_dif = sqrt(Pr)/sqrt(Ra), t_dif = 1/(sqrt(Pr) sqrt(Ra))),
 * src/interface/init.c:66-68 (tension = 1/We),
 * src/fluid/decide_dt.c:109-112 (coef_dt_adv, coef_dt_dif).
 * Diffusion is implicit in x and explicit in y (src/param/implicit.c:3-7). */
typedef struct {
  int nx, ny;             /* interior cells; the FFT direction must be a power of two */
  double lx, ly;          /* domain lengths */
  double m_dif, t_dif;    /* momentum / temperature diffusivities */
  double tension;         /* surface tension coefficient, 1/We */
  double coef_dt_adv;     /* CFL safety factors */
  double coef_dt_dif;
  int add_buoyancy;       /* add +T to the ux source (Boussinesq) */
  double uy_xm, uy_xp;    /* wall velocity in y at x = 0, x = lx */
  double t_xm, t_xp;      /* wall temperature at x = 0, x = lx */
} svof_params_t;

enum {
  SVOF_UX = 0,
  SVOF_UY = 1,
  SVOF_P = 2,
  SVOF_PSI = 3,
  SVOF_T = 4,
  SVOF_VOF = 5,
  SVOF_CURV = 6,
  SVOF_NORMAL = 7,
  SVOF_IFRCX = 8,
  SVOF_IFRCY = 9,
  SVOF_SRCUX_A = 10, /* current RK source (explicit part), srcux[rk_a] */
  SVOF_SRCUX_B = 11, /* previous RK source, srcux[rk_b] */
  SVOF_SRCUY_A = 12,
  SVOF_SRCUY_B = 13,
  SVOF_SRCT_A = 14,
  SVOF_SRCT_B = 15,
  SVOF_SRC_A = 16,   /* vof sources, interface src[rk_a], src[rk_b] */
  SVOF_SRC_B = 17,
  SVOF_NFIELDS = 18
};

/* Creates a solver for the grid xf[nx+1], xc[nx+2] (reference domain_t,
 * include/domain.h:19-28; dxf, dxc and dy are derived as src/domain.c:170-209
 * does).  Allocates all device memory.  Replaces the allocation and set-up
 * parts of fluid_init (include/fluid_solver.h:10-14), interface_init
 * (include/interface_solver.h:8-12) and linear_system_init
 * (include/linear_system.h:37-42). */
int svof_create(const svof_params_t *params, const double *xf, const double *xc,
                svof_solver_t **solver);
/* replaces linear_system_finalise (include/linear_system.h:44-46) and frees
 * everything svof_create allocated */
int svof_destroy(svof_solver_t *solver);

/* number of doubles in a field's device storage (layout above) */
int svof_field_count(const svof_solver_t *solver, int field, size_t *count);
/* whole-storage copies between host memory and the device field */
int svof_upload_field(svof_solver_t *solver, int field, const double *host, size_t count);
int svof_download_field(svof_solver_t *solver, int field, double *host, size_t count);
/* device address of a field's current storage (valid until the next call
 * that advances the solution) */
int svof_device_field(svof_solver_t *solver, int field, double **device_ptr);
/* Loads rows 1..ny (the restart-file part, shape (ny, nx+nadds)) of ux, uy,
 * p, t or vof from host memory and imposes that field's boundary and halo
 * values, as array.load + fluid_update_boundaries_* / interface_update_
 * boundaries_vof do in fluid_init (src/fluid/init.c:82-88) and
 * interface_init (src/interface/init.c:60-63). */
int svof_load_interior(svof_solver_t *solver, int field, const double *host, size_t count);
/* copies rows 1..ny of ux, uy, p, t or vof to host memory (the part
 * fluid_save / interface_save write, src/fluid/save.c:18-25) */
int svof_store_interior(svof_solver_t *solver, int field, double *host, size_t count);

/* 1 if |max dxf - min dxf| < 1e-15 (src/domain.c:75-98): the Poisson solve
 * uses the DCT path, otherwise the DFT path (src/integrate.c:49-57) */
int svof_x_grid_is_uniform(const svof_solver_t *solver, int *is_uniform);

/* ---- the reference's solver entry points (include/fluid_solver.h,
 *      include/interface_solver.h), one kernel sequence each ---- */
/* fluid_decide_dt (include/fluid_solver.h:24-28); *dt is read back */
int svof_fluid_decide_dt(svof_solver_t *solver, double *dt);
/* interface_compute_curvature_tensor (include/interface_solver.h:20-23) */
int svof_interface_compute_curvature_tensor(svof_solver_t *solver);
/* interface_compute_force (include/interface_solver.h:25-28) */
int svof_interface_compute_force(svof_solver_t *solver);
/* interface_update_vof (include/interface_solver.h:30-36) */
int svof_interface_update_vof(svof_solver_t *solver, size_t rkstep, double dt);
/* fluid_predict_field (include/fluid_solver.h:31-37) */
int svof_fluid_predict_field(svof_solver_t *solver, size_t rkstep, double dt);
/* fluid_compute_potential_dct / _dft (include/fluid_solver.h:41-55) */
int svof_fluid_compute_potential_dct(svof_solver_t *solver, size_t rkstep, double dt);
int svof_fluid_compute_potential_dft(svof_solver_t *solver, size_t rkstep, double dt);
/* fluid_correct_velocity (include/fluid_solver.h:58-63) */
int svof_fluid_correct_velocity(svof_solver_t *solver, size_t rkstep, double dt);
/* fluid_update_pressure (include/fluid_solver.h:66-71) */
int svof_fluid_update_pressure(svof_solver_t *solver, size_t rkstep, double dt);

/* integrate (reference include/integrate.h:5-10): one full time step
 * (dt + 3 Runge-Kutta substeps) as one CUDA-graph launch; *dt is read back */
int svof_integrate(svof_solver_t *solver, double *dt);
/* nsteps calls of svof_integrate without host synchronisation between
 * steps; dts (optional, nsteps entries) receives every dt */
int svof_run(svof_solver_t *solver, int nsteps, double *dts);

/* enqueues nsteps time steps (graph launches plus the 8-byte dt read-back)
 * on the solver's stream and returns without waiting; svof_last_dt waits and
 * returns the last dt.  Same semantics as svof_run, for callers that overlap
 * host work or time the device with events. */
int svof_enqueue_steps(svof_solver_t *solver, int nsteps);
int svof_last_dt(svof_solver_t *solver, double *dt);

/* diagnostics of src/logging/divergence.c:36-50 and src/logging/interface.c:
 * 22-39 computed on the device: max |div u|, and vof min, max and
 * sum(vof dx dy) / sum(dx dy) */
int svof_diagnostics(svof_solver_t *solver, double *divmax, double *vofmin, double *vofmax,
                     double *vofmean);

/* the logging reductions of src/logging/momentum.c:38-54, src/logging/
 * energy.c:41-65 and src/logging/nusselt/ (heat_flux.c:22-41,
 * kinetic_energy_injection.c:25-49, kinetic_energy_dissipation.c:11-163,
 * thermal_energy_dissipation.c:10-95, reference.c:4-12) computed on the
 * device from the current fields, without moving them to the host.  out[0..8]
 * (nout >= 9) = {x momentum, y momentum, kinetic energy of ux, of uy, thermal
 * energy, Nusselt number from the wall heat flux, from the kinetic energy
 * injection, from the kinetic energy dissipation, from the thermal energy
 * dissipation}: the values the reference writes to momentum.dat, energy.dat
 * and nusselt.dat.  The sums are compensated (TwoSum) and deterministic; they
 * differ from the reference's sequential sums only by round-off. */
int svof_logging_quantities(svof_solver_t *solver, double *out, int nout);

/* Time-averaged statistics on the device (src/statistics.c).  Each
 * svof_statistics_collect() adds one sample of the current fields to FP64
 * accumulators (collect_mean_ux, collect_mean_uy, collect_mean_t,
 * collect_uxt, src/statistics.c:117-204), queued on the solver's stream:
 *   ux1 += ux, ux2 += ux^2, uy1 += uy, uy2 += uy^2, t1 += t, t2 += t^2,
 *   uxt += ux (t(i-1) + t(i)) / 2
 * over the interior rows j = 1 .. ny, for i = 1 .. nx+1 (ux1 ux2 uxt) and
 * i = 0 .. nx+1 (the others), in the reference's statistics layouts
 * (include/array_macros/statistics/ux1.h .. uxt.h: ny x (nx+1) and
 * ny x (nx+2), no halo).  The squares are the correctly rounded products;
 * the reference's pow(x, 2.) is within one unit in the last place of them.
 * The caller keeps the sampling schedule, as src/main.c:137-140 does.  The
 * accumulators (7 arrays) are allocated on the first collection. */
enum {
  SVOF_STAT_UX1 = 0,
  SVOF_STAT_UX2,
  SVOF_STAT_UY1,
  SVOF_STAT_UY2,
  SVOF_STAT_T1,
  SVOF_STAT_T2,
  SVOF_STAT_UXT,
  SVOF_NSTATS
};
int svof_statistics_collect(svof_solver_t *solver);
/* zero the accumulators and the sample count */
int svof_statistics_reset(svof_solver_t *solver);
/* samples since creation or the last reset (the reference's g_num) */
int svof_statistics_count(svof_solver_t *solver, size_t *num);
/* the reduced output of reduce_and_write (src/statistics.c:232-281):
 * out[i] = sum over the rows j = 1 .. ny, in that order from zero, of the
 * accumulated quantity at column i; count = nx+1 (ux1 ux2 uxt) or nx+2 */
int svof_statistics_reduce(svof_solver_t *solver, int quantity, double *out, size_t count);
/* the accumulated array itself (the unreduced array.dump output) */
int svof_statistics_field(svof_solver_t *solver, int quantity, double *out, size_t count);

/* kernel kinds of svof_profile_step */
enum {
  SVOF_K_DT = 0,            /* CFL reduction + dt (2 launches) */
  SVOF_K_GEOM = 1,          /* normals, intercept, curvature */
  SVOF_K_FORCE = 2,         /* CSF force */
  SVOF_K_VOF = 3,           /* THINC fluxes + vof update */
  SVOF_K_PREDICT = 4,       /* momentum / scalar RHS + x Thomas + update */
  SVOF_K_POISSON_FWD = 5,   /* divergence + forward transform */
  SVOF_K_POISSON_SOLVE = 6, /* spectral line solves */
  SVOF_K_POISSON_INV = 7,   /* inverse transform + psi boundaries */
  SVOF_K_PROJECT = 8,       /* velocity correction + pressure update */
  SVOF_NKINDS = 9
};
/* One time step launched kernel by kernel (no graph), timed with CUDA events
 * on the solver's stream: ms[k] / launches[k] accumulate per kind k.  The
 * solution advances exactly as with svof_integrate.  No reference
 * counterpart (measurement aid). */
int svof_profile_step(svof_solver_t *solver, double *ms, int *launches, int nkinds);

/* Pressure Poisson solve of the uniform-x (DCT) path for callers that cannot
 * allocate device memory -- for example a host whose device memory belongs to
 * a pool or budget it does not control, code running where a device
 * allocation is not allowed, or a plug-in that is handed only its input and
 * output buffers.  No counterpart in the reference: it computes what
 * svof_fluid_compute_potential_dct computes, but needs no svof_create and
 * calls no cudaMalloc, cudaFree or other allocating routine.
 *
 * Inputs: params->nx, ny, lx, ly; xf (host, nx+1 faces of a uniform grid);
 * ux, uy (device, reference layouts); rkstep and dt.  Output: psi (device,
 * (ny+2) x (nx+2), interior, Neumann walls and halo rows; its four halo corner
 * cells keep their previous values, as in the reference).  Work is enqueued
 * on `stream` (a cudaStream_t, or NULL for the default stream).
 *
 * Scratch: one file-scope device array of about 2.2 MB, held by every GPU that
 * loads this library until the process exits.  Limits: nx a power of two,
 * 4 <= nx, ny <= 1024, nx * ny <= 65536; larger grids are refused with a
 * non-zero return and a message on stderr.  The first call on a device looks
 * up that device's address of the array (cudaGetSymbolAddress) and should
 * come before any stream capture.  A call whose grid differs from the previous
 * call's on that device builds the line-solve tables on the host, uploads them
 * and waits for `stream`; other calls only enqueue work.  All calls share the
 * array, which keeps the last call's tables, dt and spectrum: calls that
 * overlap on the GPU race.  The host part of a call holds a process-wide lock,
 * so host threads may call at the same time, but their GPU work must not
 * overlap. */
int svof_poisson_dct_noalloc(const svof_params_t *params, const double *xf, const double *ux,
                             const double *uy, double *psi, size_t rkstep, double dt, void *stream);

/* ---------------------------------------------------------------------
 * Differentiation form (FP64).  No counterpart in the reference: the adjoint
 * of one time step, for gradients of an objective of the final state with
 * respect to the initial velocities and vof, the surface-tension
 * coefficient 1/We and the vof buoyancy coefficient grav_vof.  The time-step sequence of a differentiated run is held
 * fixed (svof_integrate_fixed); branches of the method (upwind side of a face,
 * interfacial-cell test, clamps of vanishing gradients) follow the primal
 * state.  Requires add_buoyancy = 0: the temperature is not differentiated.
 * -------------------------------------------------------------------- */

/* Extension absent from the reference (whose only body force is the
 * temperature buoyancy along x): Boussinesq buoyancy of the volume fraction
 * on uy, srcuy_a += grav_vof * (vof at the uy face - vof_ref), with vof after
 * the substep's advection.  grav_vof = g_y (1 - density ratio) with g_y =
 * -1/Fr^2 for gravity along -y; vof_ref = the domain-mean volume fraction
 * (zero net force in the periodic direction).  0 (the default) is the
 * reference's physics, bit for bit. */
int svof_set_gravity(svof_solver_t *solver, double grav_vof, double vof_ref);

/* replaces the run-time parameters (same grid), for example the surface
 * tension 1/We of a differentiated run; waits for the solver's stream */
int svof_set_params(svof_solver_t *solver, const svof_params_t *params);

/* doubles of one step's tape: the inputs ux, uy, vof (storage layouts) of the
 * three Runge-Kutta substeps, then the step's final vof */
int svof_tape_count(const svof_solver_t *solver, size_t *count);
/* one time step with the given dt (no CFL decision), enqueued on the solver's
 * stream (svof_synchronize waits for it); when tape (device memory,
 * svof_tape_count doubles) is not NULL it records the step's substep inputs
 * and final vof.
 * Replaces integrate() (include/integrate.h:5-10) in a differentiated run. */
int svof_integrate_fixed(svof_solver_t *solver, double dt, double *tape);

/* adjoint fields, device memory owned by the solver (made on first use),
 * compact layouts: SVOF_ADJ_UX and SVOF_ADJ_IFRCX ny rows x (nx-1) (faces
 * i = 2..nx), SVOF_ADJ_NORMAL ny x nx x 3, the others ny x nx.  The adjoint of
 * a step's output is written into UX, UY, P, VOF; svof_adjoint_step turns it
 * into the adjoint of the step's input in place.  TENSION holds per-cell
 * contributions to the adjoint of 1/We (svof_adjoint_tension sums them),
 * GRAVITY those to the adjoint of grav_vof (svof_adjoint_gravity).  The
 * pointer of SVOF_ADJ_VOF and SVOF_ADJ_SRC_A changes after each interface
 * adjoint (they alternate between two buffers): ask again. */
enum {
  SVOF_ADJ_UX = 0,
  SVOF_ADJ_UY = 1,
  SVOF_ADJ_P = 2,
  SVOF_ADJ_VOF = 3,
  SVOF_ADJ_PSI = 4,
  SVOF_ADJ_IFRCX = 5,
  SVOF_ADJ_IFRCY = 6,
  SVOF_ADJ_CURV = 7,
  SVOF_ADJ_NORMAL = 8,     /* (nx, ny, intercept) of the cell normal */
  SVOF_ADJ_SRCUX_A = 9,    /* pending adjoints of the substep's src_a (from the next substep's beta term) */
  SVOF_ADJ_SRCUY_A = 10,
  SVOF_ADJ_SRC_A = 11,
  SVOF_ADJ_TENSION = 12,
  SVOF_ADJ_GRAVITY = 13
};
int svof_adjoint_field(svof_solver_t *solver, int which, double **dptr, size_t *count);
/* zero every adjoint field (enqueued) */
int svof_adjoint_reset(svof_solver_t *solver);
/* the adjoint of one svof_integrate_fixed(dt, tape) step, enqueued: (UX, UY,
 * P, VOF) of the step's output -> of its input, TENSION and GRAVITY += their
 * contributions.
 * Per substep in reverse: the projection and pressure update, the Poisson
 * solve (its adjoint is a second Poisson solve of psi_bar / dxf: the x grid's
 * metric weights), the implicit-x line solves, the momentum right-hand sides,
 * the THINC/QQ fluxes and vof update, the CSF force, the intercepts (implicit
 * function theorem), the normals and the curvature. */
int svof_adjoint_step(svof_solver_t *solver, const double *tape, double dt);
/* the same pieces one by one, each the adjoint of the reference function of
 * the same name about the primal state in the solver's current fields (that
 * function's input), in place on the adjoint fields; each waits for its work */
int svof_adjoint_fluid_update_pressure(svof_solver_t *solver, size_t rkstep, double dt);
int svof_adjoint_fluid_correct_velocity(svof_solver_t *solver, size_t rkstep, double dt);
int svof_adjoint_fluid_compute_potential(svof_solver_t *solver, size_t rkstep, double dt);
int svof_adjoint_fluid_predict_field(svof_solver_t *solver, size_t rkstep, double dt);
int svof_adjoint_interface_update_vof(svof_solver_t *solver, size_t rkstep, double dt);
int svof_adjoint_interface_compute_force(svof_solver_t *solver);
int svof_adjoint_interface_compute_curvature_tensor(svof_solver_t *solver);
/* the accumulated adjoint of 1/We (waits) */
int svof_adjoint_tension(svof_solver_t *solver, double *out);
/* the accumulated adjoint of grav_vof (waits); for a density ratio r and
 * Froude number Fr, d/dr = grav_bar / Fr^2 (grav_vof = -(1 - r) / Fr^2) */
int svof_adjoint_gravity(svof_solver_t *solver, double *out);

/* wait for all work of the solver's stream */
int svof_synchronize(svof_solver_t *solver);
/* CUDA stream the solver issues its work on (cudaStream_t) */
int svof_stream(svof_solver_t *solver, void **stream);
const char *svof_last_error(void);

/* Guard zones (a debugging aid in place of a memory checker).  With
 * SVOF_GUARD_BYTES=N in the environment when the solvers allocate (N > 0,
 * rounded up to a multiple of 256), every device buffer of the 2D and 3D
 * solvers gets N bytes before and after it, filled with a canary byte.
 * svof_guard_bytes() returns the band in effect (0: off, the default).
 * svof_guard_check() waits for the device, scans every live guard zone of
 * the process and returns 0 when all are intact; otherwise non-zero, with
 * the number of changed bytes in *bad_bytes (may be NULL) and the first
 * changed zone named in svof_last_error().  Writes outside a buffer are
 * detected; reads are not. */
size_t svof_guard_bytes(void);
int svof_guard_check(size_t *bad_bytes);

#ifdef __cplusplus
}
#endif

#endif
