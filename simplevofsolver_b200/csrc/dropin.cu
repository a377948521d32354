// dropin.cu -- the reference's solver entry points (include/svof_reference_abi.h)
// on top of the engine of solver.cu.
//
// The reference keeps its solver state in function-local statics initialised
// on first use (src/fluid/compute_potential/dct.c:379-388, predict/ux.c:312-329,
// decide_dt.c:109-119); here the one solver of the process plays that role.
// fluid_init creates it (field memory: CUDA managed, so that the host's
// logging and save code can read array_t.data), interface_init and the first
// fluid_decide_dt / integrate complete its parameters, and every entry point
// leaves the structs' data pointers on the solver's current buffers.
#include <cerrno>
#include <cstddef>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/svof_reference_abi.h"
#include "svof_internal.cuh"

using namespace svof;

// the reference's layouts on x86-64 (LP64); a host compiled against the
// reference's headers must see the same offsets
static_assert(sizeof(array_t) == 32, "array_t layout");
static_assert(sizeof(domain_t) == 112 && offsetof(domain_t, xf) == 72 && offsetof(domain_t, dy) == 104,
              "domain_t layout");
static_assert(sizeof(fluid_t) == 480 && offsetof(fluid_t, Ra) == 448, "fluid_t layout");
static_assert(sizeof(interface_t) == 328 && offsetof(interface_t, tension) == 320, "interface_t layout");
static_assert(sizeof(linear_system_t) == 88 && offsetof(linear_system_t, x1pncl) == 8, "linear_system_t layout");

namespace {

svof_solver_t *g_s = nullptr;
fluid_t *g_fluid = nullptr;
interface_t *g_iface = nullptr;
svof_params_t g_prm{};
bool g_coefs = false;
std::vector<void *> g_extra;  // arrays the device path keeps on chip (dvof, fluxes, src_g)

// index-map halo widths of include/array_macros/** (nadds[dim][lower, upper])
const int NADDS_UX[2][2] = {{0, 1}, {1, 1}};
const int NADDS_CC[2][2] = {{1, 1}, {1, 1}};  // uy, p, psi, t, curv
const int NADDS_SRCX[2][2] = {{-1, 0}, {0, 0}};  // srcux, ifrcx
const int NADDS_SRC[2][2] = {{0, 0}, {0, 0}};    // srcuy, srct, ifrcy, src
const int NADDS_VOF[2][2] = {{1, 1}, {2, 2}};
const int NADDS_DVOF[2][2] = {{0, 1}, {1, 2}};
const int NADDS_NORMAL[2][2] = {{0, 0}, {1, 1}};
const int NADDS_FLXX[2][2] = {{0, 1}, {0, 0}};
const int NADDS_FLXY[2][2] = {{0, 0}, {0, 1}};

int report(const char *msg) {
  fprintf(stderr, "%s\n", msg);
  return 1;
}

int report_engine(const char *where) {
  fprintf(stderr, "%s: %s\n", where, svof_last_error());
  return 1;
}

// config.get_double (src/config.c:14-42)
int get_double(const char *name, double *value) {
  const char *s = getenv(name);
  if (!s) {
    printf("%s not found\n", name);
    return 1;
  }
  errno = 0;
  *value = strtod(s, nullptr);
  if (0 != errno) {
    printf("%s: invalid value as double\n", name);
    return 1;
  }
  return 0;
}

double env_or(const char *name, double dflt) {
  const char *s = getenv(name);
  return s ? strtod(s, nullptr) : dflt;
}

// ---- NPY files (the restart layout of src/array.c:80-206, src/fileio.c) ----
int npy_read(const std::string &dir, const char *name, size_t rows, size_t cols, std::vector<double> &out) {
  const std::string path = dir + (dir.empty() || dir.back() == '/' ? "" : "/") + name + ".npy";
  FILE *fp = fopen(path.c_str(), "rb");
  if (!fp) {
    perror(path.c_str());
    return 1;
  }
  unsigned char pre[12];
  size_t hl = 0;
  int ok = 8 == fread(pre, 1, 8, fp) && 0x93 == pre[0] && 0 == memcmp(pre + 1, "NUMPY", 5);
  if (ok && 1 == pre[6]) {
    ok = 2 == fread(pre + 8, 1, 2, fp);
    hl = (size_t)pre[8] | ((size_t)pre[9] << 8);
  } else if (ok && (2 == pre[6] || 3 == pre[6])) {
    ok = 4 == fread(pre + 8, 1, 4, fp);
    hl = (size_t)pre[8] | ((size_t)pre[9] << 8) | ((size_t)pre[10] << 16) | ((size_t)pre[11] << 24);
  } else {
    ok = 0;
  }
  std::string hdr(hl, '\0');
  ok = ok && hl == fread(&hdr[0], 1, hl, fp);
  char want[96];
  snprintf(want, sizeof(want), "(%zu, %zu)", rows, cols);
  if (!ok || hdr.find("'<f8'") == std::string::npos || hdr.find("False") == std::string::npos ||
      hdr.find(want) == std::string::npos) {
    fclose(fp);
    fprintf(stderr, "%s: expected a C-ordered float64 NPY array of shape %s\n", path.c_str(), want);
    return 1;
  }
  out.resize(rows * cols);
  const size_t n = fread(out.data(), sizeof(double), out.size(), fp);
  fclose(fp);
  if (n != out.size()) {
    fprintf(stderr, "%s: short read\n", path.c_str());
    return 1;
  }
  return 0;
}

int npy_write(const std::string &dir, const char *name, const char *descr, size_t ndim, const size_t *shape,
              const void *data, size_t elem) {
  const std::string path = dir + (dir.empty() || dir.back() == '/' ? "" : "/") + name + ".npy";
  std::string shp = "(";
  size_t n = 1;
  for (size_t d = 0; d < ndim; d++) {
    shp += std::to_string(shape[d]) + (1 == ndim ? "," : (d + 1 < ndim ? ", " : ""));
    n *= shape[d];
  }
  shp += ")";
  std::string dict = std::string("{'descr': '") + descr + "', 'fortran_order': False, 'shape': " + shp + ", }";
  size_t total = 10 + dict.size() + 1;
  dict += std::string((64 - total % 64) % 64, ' ') + "\n";
  FILE *fp = fopen(path.c_str(), "wb");
  if (!fp) {
    perror(path.c_str());
    return 1;
  }
  const unsigned char pre[10] = {0x93, 'N', 'U', 'M', 'P', 'Y', 1, 0, (unsigned char)(dict.size() & 0xff),
                                 (unsigned char)((dict.size() >> 8) & 0xff)};
  int ok = 10 == fwrite(pre, 1, 10, fp) && dict.size() == fwrite(dict.data(), 1, dict.size(), fp) &&
           n == fwrite(data, elem, n, fp);
  fclose(fp);
  return ok ? 0 : 1;
}

// ---- struct plumbing ----
void set_array(array_t *a, const int nadds[2][2], size_t elem, void *data, size_t count_elems) {
  a->size = elem;
  if (!a->nadds) a->nadds = static_cast<int(*)[2]>(calloc(2, 2 * sizeof(int)));
  for (int d = 0; d < 2; d++) {
    a->nadds[d][0] = nadds[d][0];
    a->nadds[d][1] = nadds[d][1];
  }
  a->datasize = count_elems * elem;
  a->data = data;
}

void *extra_zeros(size_t bytes) {
  void *p = nullptr;
  if (cudaSuccess != cudaMallocManaged(&p, bytes ? bytes : 8)) return nullptr;
  memset(p, 0, bytes);
  g_extra.push_back(p);
  return p;
}

double *cur(int field) {
  double *p = nullptr;
  svof_device_field(g_s, field, &p);
  return p;
}

// leaves every struct pointer on the solver's current buffer
void sync_pointers() {
  if (g_fluid) {
    g_fluid->ux.data = cur(SVOF_UX);
    g_fluid->uy.data = cur(SVOF_UY);
    g_fluid->p.data = cur(SVOF_P);
    g_fluid->psi.data = cur(SVOF_PSI);
    g_fluid->t.data = cur(SVOF_T);
    g_fluid->srcux[0].data = cur(SVOF_SRCUX_A);
    g_fluid->srcux[1].data = cur(SVOF_SRCUX_B);
    g_fluid->srcuy[0].data = cur(SVOF_SRCUY_A);
    g_fluid->srcuy[1].data = cur(SVOF_SRCUY_B);
    g_fluid->srct[0].data = cur(SVOF_SRCT_A);
    g_fluid->srct[1].data = cur(SVOF_SRCT_B);
  }
  if (g_iface) {
    g_iface->vof.data = cur(SVOF_VOF);
    g_iface->ifrcx.data = cur(SVOF_IFRCX);
    g_iface->ifrcy.data = cur(SVOF_IFRCY);
    g_iface->normal.data = cur(SVOF_NORMAL);
    g_iface->curv.data = cur(SVOF_CURV);
    g_iface->src[0].data = cur(SVOF_SRC_A);
    g_iface->src[1].data = cur(SVOF_SRC_B);
  }
}

int ensure_coefs() {
  // fluid_decide_dt reads the safety factors on its first call (decide_dt.c:109-119)
  if (g_coefs) return 0;
  if (get_double("coef_dt_adv", &g_prm.coef_dt_adv)) return 1;
  if (get_double("coef_dt_dif", &g_prm.coef_dt_dif)) return 1;
  if (engine_update_params(g_s, &g_prm)) return report_engine("fluid_decide_dt");
  g_coefs = true;
  printf("coefs: (adv) % .3e, (dif) % .3e\n", g_prm.coef_dt_adv, g_prm.coef_dt_dif);
  return 0;
}

int need_solver(const char *where) {
  if (g_s) return 0;
  fprintf(stderr, "%s: fluid_init has not been called\n", where);
  return 1;
}

int load_rows(const char *dir, const char *name, int field, size_t cols) {
  std::vector<double> h;
  if (npy_read(dir, name, g_prm.ny, cols, h)) return 1;
  if (svof_load_interior(g_s, field, h.data(), h.size())) return report_engine(name);
  return 0;
}

int save_rows(const char *dir, const char *name, int field, size_t cols) {
  std::vector<double> h((size_t)g_prm.ny * cols);
  if (svof_store_interior(g_s, field, h.data(), h.size())) return report_engine(name);
  const size_t shape[2] = {(size_t)g_prm.ny, cols};
  return npy_write(dir, name, "<f8", 2, shape, h.data(), sizeof(double));
}

}  // namespace

extern "C" {

// ---------------------------------------------------------------- fluid_solver.h

int fluid_init(const char dirname_ic[], const domain_t *domain, fluid_t *fluid) {
  if (g_s) return report("fluid_init: the solver of this process is already initialised");
  if (domain->mysizes[0] != domain->glsizes[0] || domain->mysizes[1] != domain->glsizes[1])
    return report("fluid_init: the GPU solver runs one process per domain (mysizes must equal glsizes)");
  const int nx = (int)domain->glsizes[0], ny = (int)domain->glsizes[1];
  double Pr = 0., Ra = 0.;
  if (get_double("Pr", &Pr) || get_double("Ra", &Ra)) return 1;
  g_prm = svof_params_t{};
  g_prm.nx = nx;
  g_prm.ny = ny;
  g_prm.lx = domain->lengths[0];
  g_prm.ly = domain->lengths[1];
  g_prm.m_dif = 1. * std::sqrt(Pr) / std::sqrt(Ra);  // src/fluid/init.c:90-93
  g_prm.t_dif = 1. / std::sqrt(Pr) / std::sqrt(Ra);
  g_prm.tension = 0.;                                 // set by interface_init
  g_prm.coef_dt_adv = 1.;                             // set on the first fluid_decide_dt
  g_prm.coef_dt_dif = 1.;
  // src/param/*.c defaults, overridable at run time
  g_prm.add_buoyancy = env_or("SVOF_ADD_BUOYANCY", 1.) != 0.;
  g_prm.uy_xm = env_or("SVOF_UY_XM", 0.);
  g_prm.uy_xp = env_or("SVOF_UY_XP", 0.);
  g_prm.t_xm = env_or("SVOF_T_XM", +0.5);
  g_prm.t_xp = env_or("SVOF_T_XP", -0.5);
  if (engine_create(&g_prm, domain->xf, domain->xc, true, &g_s)) return report_engine("fluid_init");
  // restart fields (src/fluid/init.c:82-88)
  if (load_rows(dirname_ic, "ux", SVOF_UX, nx + 1) || load_rows(dirname_ic, "uy", SVOF_UY, nx + 2) ||
      load_rows(dirname_ic, "p", SVOF_P, nx + 2) || load_rows(dirname_ic, "t", SVOF_T, nx + 2))
    return 1;
  const size_t n_ux = (size_t)(nx + 1) * (ny + 2), n_cc = (size_t)(nx + 2) * (ny + 2);
  const size_t n_srcx = (size_t)(nx - 1) * ny, n_src = (size_t)nx * ny;
  set_array(&fluid->ux, NADDS_UX, sizeof(double), nullptr, n_ux);
  set_array(&fluid->uy, NADDS_CC, sizeof(double), nullptr, n_cc);
  set_array(&fluid->p, NADDS_CC, sizeof(double), nullptr, n_cc);
  set_array(&fluid->psi, NADDS_CC, sizeof(double), nullptr, n_cc);
  set_array(&fluid->t, NADDS_CC, sizeof(double), nullptr, n_cc);
  for (int k = 0; k < 3; k++) {
    set_array(&fluid->srcux[k], NADDS_SRCX, sizeof(double), nullptr, n_srcx);
    set_array(&fluid->srcuy[k], NADDS_SRC, sizeof(double), nullptr, n_src);
    set_array(&fluid->srct[k], NADDS_SRC, sizeof(double), nullptr, n_src);
  }
  // the implicit part of the sources (srcX[rk_g]) stays in registers on the device
  fluid->srcux[2].data = extra_zeros(sizeof(double) * n_srcx);
  fluid->srcuy[2].data = extra_zeros(sizeof(double) * n_src);
  fluid->srct[2].data = extra_zeros(sizeof(double) * n_src);
  fluid->Pr = Pr;
  fluid->Ra = Ra;
  fluid->m_dif = g_prm.m_dif;
  fluid->t_dif = g_prm.t_dif;
  g_fluid = fluid;
  sync_pointers();
  printf("FLUID\n\tRa: % .7e\n\tPr: % .7e\n", fluid->Ra, fluid->Pr);
  printf("\tMomentum    diffusivity: % .7e\n\tTemperature diffusivity: % .7e\n", fluid->m_dif, fluid->t_dif);
  printf("\tdiffusive treatment in x: implicit\n\tdiffusive treatment in y: explicit\n");
  printf("\tsolver: B200 (sm_100a), FP64\n");
  fflush(stdout);
  return 0;
}

int fluid_save(const char dirname[], const domain_t *domain, const fluid_t *fluid) {
  (void)domain;
  if (need_solver("fluid_save")) return 1;
  // src/fluid/save.c:10-28
  npy_write(dirname, "m_dif", "<f8", 0, nullptr, &fluid->m_dif, sizeof(double));
  npy_write(dirname, "t_dif", "<f8", 0, nullptr, &fluid->t_dif, sizeof(double));
  const int nx = g_prm.nx;
  if (save_rows(dirname, "ux", SVOF_UX, nx + 1) || save_rows(dirname, "uy", SVOF_UY, nx + 2) ||
      save_rows(dirname, "p", SVOF_P, nx + 2) || save_rows(dirname, "t", SVOF_T, nx + 2))
    return 1;
  return 0;
}

int fluid_decide_dt(const domain_t *domain, const fluid_t *fluid, double *dt) {
  (void)domain;
  (void)fluid;
  if (need_solver("fluid_decide_dt") || ensure_coefs()) return 1;
  if (svof_fluid_decide_dt(g_s, dt)) return report_engine("fluid_decide_dt");
  return 0;
}

int fluid_predict_field(const domain_t *domain, const size_t rkstep, const double dt, fluid_t *fluid,
                        const interface_t *interface) {
  (void)domain;
  (void)fluid;
  (void)interface;
  if (need_solver("fluid_predict_field")) return 1;
  const int rc = svof_fluid_predict_field(g_s, rkstep, dt);
  sync_pointers();
  return rc ? report_engine("fluid_predict_field") : 0;
}

int fluid_compute_potential_dft(const domain_t *domain, const size_t rkstep, const double dt, fluid_t *fluid) {
  (void)domain;
  (void)fluid;
  if (need_solver("fluid_compute_potential_dft")) return 1;
  const int rc = svof_fluid_compute_potential_dft(g_s, rkstep, dt);
  sync_pointers();
  return rc ? report_engine("fluid_compute_potential_dft") : 0;
}

int fluid_compute_potential_dct(const domain_t *domain, const size_t rkstep, const double dt, fluid_t *fluid) {
  (void)domain;
  (void)fluid;
  if (need_solver("fluid_compute_potential_dct")) return 1;
  const int rc = svof_fluid_compute_potential_dct(g_s, rkstep, dt);
  sync_pointers();
  return rc ? report_engine("fluid_compute_potential_dct") : 0;
}

int fluid_correct_velocity(const domain_t *domain, const size_t rkstep, const double dt, fluid_t *fluid) {
  (void)domain;
  (void)fluid;
  if (need_solver("fluid_correct_velocity")) return 1;
  const int rc = svof_fluid_correct_velocity(g_s, rkstep, dt);
  sync_pointers();
  return rc ? report_engine("fluid_correct_velocity") : 0;
}

int fluid_update_pressure(const domain_t *domain, const size_t rkstep, const double dt, fluid_t *fluid) {
  (void)domain;
  (void)fluid;
  if (need_solver("fluid_update_pressure")) return 1;
  const int rc = svof_fluid_update_pressure(g_s, rkstep, dt);
  sync_pointers();
  return rc ? report_engine("fluid_update_pressure") : 0;
}

static int boundaries(const char *where, int field, array_t *a) {
  if (need_solver(where)) return 1;
  if (!a || !a->data) return report("boundary update of an unallocated array");
  return engine_apply_bc(g_s, field, static_cast<double *>(a->data)) ? report_engine(where) : 0;
}

int fluid_update_boundaries_ux(const domain_t *domain, array_t *ux) {
  (void)domain;
  return boundaries("fluid_update_boundaries_ux", SVOF_UX, ux);
}
int fluid_update_boundaries_uy(const domain_t *domain, array_t *uy) {
  (void)domain;
  return boundaries("fluid_update_boundaries_uy", SVOF_UY, uy);
}
int fluid_update_boundaries_p(const domain_t *domain, array_t *p) {
  (void)domain;
  return boundaries("fluid_update_boundaries_p", SVOF_P, p);
}
int fluid_update_boundaries_psi(const domain_t *domain, array_t *psi) {
  (void)domain;
  return boundaries("fluid_update_boundaries_psi", SVOF_PSI, psi);
}
int fluid_update_boundaries_t(const domain_t *domain, array_t *t) {
  (void)domain;
  return boundaries("fluid_update_boundaries_t", SVOF_T, t);
}

// ---------------------------------------------------------------- interface_solver.h

int interface_init(const char dirname_ic[], const domain_t *domain, interface_t *interface) {
  (void)domain;
  if (need_solver("interface_init")) return 1;
  double We = 0.;
  if (get_double("We", &We)) return 1;
  g_prm.tension = 1. / We;  // src/interface/init.c:66-68
  if (engine_update_params(g_s, &g_prm)) return report_engine("interface_init");
  const int nx = g_prm.nx, ny = g_prm.ny;
  if (load_rows(dirname_ic, "vof", SVOF_VOF, nx + 2)) return 1;
  const size_t n_cc = (size_t)(nx + 2) * (ny + 2);
  set_array(&interface->vof, NADDS_VOF, sizeof(double), nullptr, (size_t)(nx + 2) * (ny + 4));
  set_array(&interface->ifrcx, NADDS_SRCX, sizeof(double), nullptr, (size_t)(nx - 1) * ny);
  set_array(&interface->ifrcy, NADDS_SRC, sizeof(double), nullptr, (size_t)nx * ny);
  set_array(&interface->normal, NADDS_NORMAL, 3 * sizeof(double), nullptr, (size_t)nx * (ny + 2));
  set_array(&interface->curv, NADDS_CC, sizeof(double), nullptr, n_cc);
  for (int k = 0; k < 2; k++) set_array(&interface->src[k], NADDS_SRC, sizeof(double), nullptr, (size_t)nx * ny);
  // corner normals and face fluxes stay in shared memory on the device
  set_array(&interface->dvof, NADDS_DVOF, 2 * sizeof(double),
            extra_zeros(2 * sizeof(double) * (nx + 1) * (ny + 3)), (size_t)(nx + 1) * (ny + 3));
  set_array(&interface->flxx, NADDS_FLXX, sizeof(double), extra_zeros(sizeof(double) * (nx + 1) * ny),
            (size_t)(nx + 1) * ny);
  set_array(&interface->flxy, NADDS_FLXY, sizeof(double), extra_zeros(sizeof(double) * nx * (ny + 1)),
            (size_t)nx * (ny + 1));
  interface->tension = g_prm.tension;
  g_iface = interface;
  sync_pointers();
  printf("INTERFACE\n\tsurface tension: % .7e\n", interface->tension);
  fflush(stdout);
  return 0;
}

int interface_save(const char dirname[], const domain_t *domain, const interface_t *interface) {
  (void)domain;
  if (need_solver("interface_save")) return 1;
  npy_write(dirname, "surface_tension", "<f8", 0, nullptr, &interface->tension, sizeof(double));
  return save_rows(dirname, "vof", SVOF_VOF, g_prm.nx + 2);
}

int interface_compute_curvature_tensor(const domain_t *domain, interface_t *interface) {
  (void)domain;
  (void)interface;
  if (need_solver("interface_compute_curvature_tensor")) return 1;
  const int rc = svof_interface_compute_curvature_tensor(g_s);
  sync_pointers();
  return rc ? report_engine("interface_compute_curvature_tensor") : 0;
}

int interface_compute_force(const domain_t *domain, interface_t *interface) {
  (void)domain;
  (void)interface;
  if (need_solver("interface_compute_force")) return 1;
  const int rc = svof_interface_compute_force(g_s);
  sync_pointers();
  return rc ? report_engine("interface_compute_force") : 0;
}

int interface_update_vof(const domain_t *domain, const size_t rkstep, const double dt, const fluid_t *fluid,
                         interface_t *interface) {
  (void)domain;
  (void)fluid;
  (void)interface;
  if (need_solver("interface_update_vof")) return 1;
  const int rc = svof_interface_update_vof(g_s, rkstep, dt);
  sync_pointers();
  return rc ? report_engine("interface_update_vof") : 0;
}

int interface_update_boundaries_vof(const domain_t *domain, array_t *vof) {
  (void)domain;
  return boundaries("interface_update_boundaries_vof", SVOF_VOF, vof);
}

// ---------------------------------------------------------------- linear_system.h

int linear_system_init(const sdecomp_info_t *info, const bool implicit[NDIMS], const size_t glsizes[NDIMS],
                       linear_system_t *ls) {
  (void)info;
  if (ls->is_initialised) {
    printf("this linear_system object is already initialised\n");
    return 1;
  }
  if (!implicit[0] || implicit[1]) {
    fprintf(stderr, "linear_system_init: the GPU path solves implicit-x, explicit-y systems only\n");
    return 1;
  }
  ls->implicit[0] = implicit[0];
  ls->implicit[1] = implicit[1];
  for (int d = 0; d < NDIMS; d++) {
    ls->x1pncl_mysizes[d] = glsizes[d];
    ls->y1pncl_mysizes[d] = glsizes[d];
  }
  ls->x1pncl = static_cast<double *>(calloc(glsizes[0] * glsizes[1], sizeof(double)));
  ls->y1pncl = nullptr;
  ls->tdm_x = nullptr;
  ls->tdm_y = nullptr;
  ls->transposer_x1_to_y1 = nullptr;
  ls->transposer_y1_to_x1 = nullptr;
  if (!ls->x1pncl) return report("linear_system_init: out of memory");
  ls->is_initialised = true;
  return 0;
}

int linear_system_finalise(linear_system_t *ls) {
  if (!ls || !ls->is_initialised) return 1;
  free(ls->x1pncl);
  free(ls->y1pncl);
  ls->x1pncl = nullptr;
  ls->y1pncl = nullptr;
  ls->is_initialised = false;
  return 0;
}

// ---------------------------------------------------------------- integrate.h

int integrate(const domain_t *domain, fluid_t *fluid, interface_t *interface, double *dt) {
  (void)domain;
  (void)fluid;
  (void)interface;
  if (need_solver("integrate") || ensure_coefs()) return 1;
  const int rc = svof_integrate(g_s, dt);
  sync_pointers();
  return rc ? report_engine("integrate") : 0;
}

}  // extern "C"
