/*
 * ref_harness.c -- drives the reference's own, unmodified solver sources
 * (SimpleVOFSolver src/*.c, compiled against the single-rank shims in
 * oracle/shims) from Python through ctypes.  TEST INFRASTRUCTURE ONLY.
 *
 * The reference's main loop (src/main.c:110-141) has no step limit and stops
 * only on simulation/wall time, so this harness calls integrate()
 * (src/integrate.c:11-68) a given number of times instead.  Initialisation
 * follows src/main.c:58-84: fileio.init, domain_init, fluid_init,
 * interface_init, which read the NPY initial-condition directory and the
 * environment variables Ra, Pr, We (and coef_dt_adv, coef_dt_dif on the first
 * fluid_decide_dt call).
 *
 * The reference keeps solver state in function-local statics that are
 * initialised once per process, so one process drives one domain.
 */
#include <stdio.h>
#include <string.h>
#include <stdbool.h>
#include "domain.h"
#include "fluid.h"
#include "fluid_solver.h"
#include "interface.h"
#include "interface_solver.h"
#include "integrate.h"
#include "fileio.h"

static domain_t g_domain;
static fluid_t g_fluid;
static interface_t g_interface;
static int g_ready = 0;

int ref_init(const char *dirname_ic) {
  if (g_ready) return 1;
  if (0 != fileio.init()) return 1;
  if (0 != domain_init(dirname_ic, &g_domain)) return 1;
  if (0 != fluid_init(dirname_ic, &g_domain, &g_fluid)) return 1;
  if (0 != interface_init(dirname_ic, &g_domain, &g_interface)) return 1;
  g_ready = 1;
  return 0;
}

static array_t *lookup(const char *name) {
  if (0 == strcmp(name, "ux")) return &g_fluid.ux;
  if (0 == strcmp(name, "uy")) return &g_fluid.uy;
  if (0 == strcmp(name, "p")) return &g_fluid.p;
  if (0 == strcmp(name, "psi")) return &g_fluid.psi;
  if (0 == strcmp(name, "t")) return &g_fluid.t;
  if (0 == strncmp(name, "srcux", 5)) return &g_fluid.srcux[name[5] - '0'];
  if (0 == strncmp(name, "srcuy", 5)) return &g_fluid.srcuy[name[5] - '0'];
  if (0 == strncmp(name, "srct", 4)) return &g_fluid.srct[name[4] - '0'];
  if (0 == strcmp(name, "vof")) return &g_interface.vof;
  if (0 == strcmp(name, "ifrcx")) return &g_interface.ifrcx;
  if (0 == strcmp(name, "ifrcy")) return &g_interface.ifrcy;
  if (0 == strcmp(name, "dvof")) return &g_interface.dvof;
  if (0 == strcmp(name, "normal")) return &g_interface.normal;
  if (0 == strcmp(name, "curv")) return &g_interface.curv;
  if (0 == strcmp(name, "flxx")) return &g_interface.flxx;
  if (0 == strcmp(name, "flxy")) return &g_interface.flxy;
  if (0 == strncmp(name, "src", 3) && ('0' == name[3] || '1' == name[3]) && '\0' == name[4]) {
    return &g_interface.src[name[3] - '0'];
  }
  return NULL;
}

/* number of doubles stored for a field (halo cells included) */
long ref_count(const char *name) {
  const array_t *a = lookup(name);
  if (!g_ready || !a) return -1;
  return (long)(a->datasize / sizeof(double));
}

int ref_get(const char *name, double *out) {
  const array_t *a = lookup(name);
  if (!g_ready || !a) return 1;
  memcpy(out, a->data, a->datasize);
  return 0;
}

int ref_set(const char *name, const double *in) {
  array_t *a = lookup(name);
  if (!g_ready || !a) return 1;
  memcpy(a->data, in, a->datasize);
  return 0;
}

int ref_integrate(int nsteps, double *dts) {
  if (!g_ready) return 1;
  for (int n = 0; n < nsteps; n++) {
    double dt = 0.;
    if (0 != integrate(&g_domain, &g_fluid, &g_interface, &dt)) return 1;
    if (dts) dts[n] = dt;
  }
  return 0;
}

/* the individual solver entry points, for per-function comparisons */
int ref_decide_dt(double *dt) { return fluid_decide_dt(&g_domain, &g_fluid, dt); }
int ref_curvature_tensor(void) { return interface_compute_curvature_tensor(&g_domain, &g_interface); }
int ref_force(void) { return interface_compute_force(&g_domain, &g_interface); }
int ref_update_vof(int rkstep, double dt) {
  return interface_update_vof(&g_domain, (size_t)rkstep, dt, &g_fluid, &g_interface);
}
int ref_predict(int rkstep, double dt) {
  return fluid_predict_field(&g_domain, (size_t)rkstep, dt, &g_fluid, &g_interface);
}
int ref_potential(int rkstep, double dt) {
  bool uniform = false;
  domain_check_x_grid_is_uniform(&g_domain, &uniform);
  if (uniform) return fluid_compute_potential_dct(&g_domain, (size_t)rkstep, dt, &g_fluid);
  return fluid_compute_potential_dft(&g_domain, (size_t)rkstep, dt, &g_fluid);
}
int ref_correct(int rkstep, double dt) { return fluid_correct_velocity(&g_domain, (size_t)rkstep, dt, &g_fluid); }
int ref_pressure(int rkstep, double dt) { return fluid_update_pressure(&g_domain, (size_t)rkstep, dt, &g_fluid); }

/* writes the restart set of src/main.c:17-32 (without step/time) */
int ref_save(const char *dirname) {
  if (!g_ready) return 1;
  domain_save(dirname, &g_domain);
  fluid_save(dirname, &g_domain, &g_fluid);
  interface_save(dirname, &g_domain, &g_interface);
  return 0;
}
