// solver3d.cu -- host engine and C ABI (include/svof3d_b200.h) of the FP64 3D
// path.
//
// Owns the device fields (layouts of tools/define_arrays.py:192-229), the
// grid and line-solver tables, the ping-pong buffers, the line-solve scratch
// and one CUDA stream.  A full step (decide_dt and three Runge-Kutta
// substeps, src/integrate.c:11-68) is captured once per buffer state into a
// CUDA graph and replayed; the only device->host traffic of a step is the
// 8-byte dt.  Tables the reference recomputes on every call (Laplacian
// coefficients, eigenvalues, FFT twiddles) are computed here once, on the
// host, with the restatement's expressions.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <string>
#include <vector>

#include "../../include/svof3d_b200.h"
#include "svof3d_internal.cuh"
#include "stat_internal.cuh"
#include "trace.cuh"
#include "smem_limit.cuh"
#include "fault_hook.cuh"
#include "adjoint3d_internal.cuh"
#include "guard.cuh"

using namespace svof3;

namespace {

thread_local std::string g_err3;

int fail(const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err3 = buf;
  return 1;
}

#define CK(x)                                                                  \
  do {                                                                         \
    cudaError_t e_ = (x);                                                      \
    if (cudaSuccess != e_) return fail("%s: %s", #x, cudaGetErrorString(e_));  \
  } while (0)

#define CK_LAUNCH() CK(cudaGetLastError())

constexpr double kPi = 3.14159265358979323846;   // oracle/svof_fft.c twiddles
constexpr double kGPi = 3.14159265358979324;     // eigenvalues, as src/fluid/compute_potential/dft.c:20
constexpr double RK_A[3] = {32. / 60., 25. / 60., 45. / 60.};
constexpr double RK_B[3] = {0. / 60., -17. / 60., -25. / 60.};

int ilog2_exact(int n) {
  int l = 0;
  while ((1 << l) < n) l++;
  return ((1 << l) == n) ? l : -1;
}

// a device array of n elements of es bytes (8: double, 4: float)
struct DevBuf {
  double *p = nullptr;
  size_t n = 0;
  size_t es = 8;
  template <class T>
  T *as() const {
    return reinterpret_cast<T *>(p);
  }
};

int dalloc(DevBuf &b, size_t n, size_t es = 8) {
  if (svof_fault::next_alloc_fails()) return fail("cudaMalloc: out of memory (injected by SVOF_FAIL_ALLOC)");
  b.n = n;
  b.es = es;
  CK(svof_guard::alloc(reinterpret_cast<void **>(&b.p), es * (n ? n : 1), false));
  CK(cudaMemset(b.p, 0, es * (n ? n : 1)));
  return 0;
}

int upload(DevBuf &b, const std::vector<double> &h) {
  if (dalloc(b, h.size())) return 1;
  CK(cudaMemcpy(b.p, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice));
  return 0;
}

void dfree(DevBuf &b) {
  if (b.p) svof_guard::release(b.p);
  b.p = nullptr;
  b.n = 0;
}

}  // namespace

struct Adjoint3State;  // the differentiation form's buffers (made on first use)
void adjoint3_free(struct svof3d_solver *s);

struct svof3d_solver {
  svof3d_params_t prm{};
  bool mixed = false;  // SVOF3_MIXED or SVOF3_MIXED_DC: FP32 intermediates (see svof3d_b200.h)
  bool dc = false;     // SVOF3_MIXED_DC: FP32 Poisson passes with an FP64 defect correction
  int nx = 0, ny = 0, nz = 0;
  double dy = 0., dz = 0.;
  int log2ny = 0, log2nz = 0;
  cudaStream_t stream = nullptr;
  DevBuf ux[2], uy[2], uz[2], t[2], vof[2];
  DevBuf p, psi, curv, normal, ifrcx, ifrcy, ifrcz;
  DevBuf sux[2], suy[2], suz[2], st[2], svof[2];
  int cur_u = 0, cur_v = 0, sa_f = 0, sa_v = 0;
  DevBuf dxf, dxc, lap_ux, lap_cc, coef;
  double lapy[3] = {0., 0., 0.}, lapz[3] = {0., 0., 0.};
  double lims[4] = {0., 0., 0., 0.};  // explicit diffusive dt limits: m y, m z, t y, t z
  // Poisson
  DevBuf spec, xscratch, twf_y, twb_y, twf_z, twb_z, pl, pu, evy, evz;
  DevBuf twf_y32, twb_y32, twf_z32, twb_z32;  // FP32 twiddles (SVOF3_MIXED_DC)
  // predictor forward-sweep scratch
  DevBuf fw;
  // time step
  double *d_dt = nullptr;
  unsigned long long *d_minbits = nullptr;
  // failure detection: bits set by k3_cfl (a non-finite velocity) and
  // k3_dt_final (a time step that is not a positive finite number), read and
  // cleared by the host at its synchronisations (check_status)
  unsigned *d_status = nullptr;
  // health counters, accumulated until svof3d_health resets them: [0] THINC
  // intercepts whose Newton iteration did not converge, [1] Poisson x lines
  // (other than ky = kz = 0) that met a pivot of magnitude <= DBL_EPSILON
  unsigned long long *d_health = nullptr;
  double *h_dt = nullptr;
  int h_dt_slots = 0;
  DevBuf diag;
  // interfacial-cell worklist of the geometry kernels
  unsigned *d_work = nullptr, *d_nwork = nullptr;
  std::map<int, cudaGraphExec_t> graphs;
  // queued restart-layout copies: a compact staging buffer per field and
  // direction, a copy stream per direction; `filled` marks a buffer written,
  // `drained` a buffer read, so that a reuse waits for the previous copy
  struct IoSlot {
    double *stage = nullptr;
    cudaEvent_t filled = nullptr, drained = nullptr;
    bool pending = false;
  };
  cudaStream_t io_h2d = nullptr, io_d2h = nullptr;
  IoSlot io_in[SVOF3_NFIELDS], io_out[SVOF3_NFIELDS];
  // time-averaged statistics: accumulators (made on the first collection),
  // row-sum scratch (one partial row per z plane, then the result), samples
  DevBuf stat[SVOF3_NSTATS], stat_part;
  size_t stat_num = 0;

  Adjoint3State *adj = nullptr;
  bool adj_f32 = false;  // the adjoint's intermediates in FP32 (svof3d_adjoint_set_precision)
  double adj_tau = -1.;  // gradient floor set by the caller; < 0: the path's default
  // vof buoyancy extension (svof3d_set_gravity; 0 = off)
  double grav_vof = 0., vof_ref = 0.;

  Grid3 grid() const { return Grid3{nx, ny, nz, dy, dz, dxf.p, dxc.p}; }
};

namespace {

int launch_halo_bc(svof3d_solver *s, double *a, int field) {
  const int nx = s->nx;
  int width, nh, kind;
  double lo = 0., hi = 0.;
  switch (field) {
    case SVOF3_UX: width = nx + 1; nh = 1; kind = BC3_ZERO; break;
    case SVOF3_UY: width = nx + 2; nh = 1; kind = BC3_DIRICHLET; lo = s->prm.uy_xm; hi = s->prm.uy_xp; break;
    case SVOF3_UZ: width = nx + 2; nh = 1; kind = BC3_DIRICHLET; lo = s->prm.uz_xm; hi = s->prm.uz_xp; break;
    case SVOF3_T: width = nx + 2; nh = 1; kind = BC3_DIRICHLET; lo = s->prm.t_xm; hi = s->prm.t_xp; break;
    case SVOF3_P: case SVOF3_PSI: width = nx + 2; nh = 1; kind = BC3_NEUMANN; break;
    case SVOF3_VOF: width = nx + 2; nh = 2; kind = BC3_VOF; break;
    default: return fail("no boundary rule for field %d", field);
  }
  const long tot = (long)width * s->ny * s->nz;
  k3_halo_bc<<<(unsigned)((tot + 255) / 256), 256, 0, s->stream>>>(a, width, nh, s->ny, s->nz, kind, lo, hi);
  CK_LAUNCH();
  return 0;
}

// reads and clears the device status word (after the stream's work is
// done): a set bit is reported as a failure of `who`
int check_status(svof3d_solver *s, const char *who) {
  unsigned st = 0;
  CK(cudaMemcpyAsync(&st, s->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  if (0 == st) return 0;
  CK(cudaMemsetAsync(s->d_status, 0, sizeof(unsigned), s->stream));
  CK(cudaStreamSynchronize(s->stream));
  if (st & 1u)
    return fail("%s: the CFL reduction met a non-finite velocity (NaN or Inf): the fields hold non-finite values",
                who);
  return fail("%s: the time step is not a positive finite number", who);
}

int launch_dt(svof3d_solver *s) {
  const dim3 cb(32, 8), cg((s->nx + 31) / 32, (s->ny + 7) / 8, (s->nz + kCflPlanes - 1) / kCflPlanes);
  k3_cfl<<<cg, cb, 0, s->stream>>>(s->ux[s->cur_u].p, s->uy[s->cur_u].p, s->uz[s->cur_u].p, s->d_minbits,
                                        s->d_status, s->grid());
  CK_LAUNCH();
  k3_dt_final<<<1, 1, 0, s->stream>>>(s->d_minbits, s->d_dt, s->prm.coef_dt_adv, s->lims[0], s->lims[1],
                                      s->lims[2], s->lims[3], s->d_status);
  CK_LAUNCH();
  return 0;
}

template <class R>
int launch_geom_t(svof3d_solver *s) {
  CK(interface_geom<R>(s->stream, s->vof[s->cur_v].p, s->normal.as<R>(), s->curv.as<R>(), s->d_work, s->d_nwork,
                       s->grid(), s->d_health));
  return 0;
}
int launch_geom(svof3d_solver *s) { return s->mixed ? launch_geom_t<float>(s) : launch_geom_t<double>(s); }

template <class R>
int launch_force_t(svof3d_solver *s) {
  CK(interface_force<R>(s->stream, s->vof[s->cur_v].p, s->curv.as<R>(), s->ifrcx.as<R>(), s->ifrcy.as<R>(),
                        s->ifrcz.as<R>(), s->prm.tension, s->grid()));
  return 0;
}
int launch_force(svof3d_solver *s) { return s->mixed ? launch_force_t<float>(s) : launch_force_t<double>(s); }

int launch_vof(svof3d_solver *s, int rk) {
  if (0 != rk) s->sa_v ^= 1;
  RK c{RK_A[rk], RK_B[rk], RK_A[rk] + RK_B[rk]};
  const int cv = s->cur_v, cu = s->cur_u;
  if (s->mixed) {
    CK(interface_advect<float>(s->stream, s->vof[cv].p, s->vof[1 - cv].p, s->ux[cu].p, s->uy[cu].p, s->uz[cu].p,
                               s->normal.as<float>(), s->svof[s->sa_v].p, s->svof[1 - s->sa_v].p, s->d_dt, c,
                               rk != 0, s->grid()));
  } else {
    CK(interface_advect<double>(s->stream, s->vof[cv].p, s->vof[1 - cv].p, s->ux[cu].p, s->uy[cu].p, s->uz[cu].p,
                                s->normal.as<double>(), s->svof[s->sa_v].p, s->svof[1 - s->sa_v].p, s->d_dt, c,
                                rk != 0, s->grid()));
  }
  s->cur_v ^= 1;
  return 0;
}

template <class R>
int launch_predict_t(svof3d_solver *s, int rk) {
  Predict3Args<R> a{};
  const int cu = s->cur_u;
  a.ux = s->ux[cu].p;
  a.uy = s->uy[cu].p;
  a.uz = s->uz[cu].p;
  a.t = s->t[cu].p;
  a.p = s->p.p;
  a.ifrcx = s->ifrcx.as<R>();
  a.ifrcy = s->ifrcy.as<R>();
  a.ifrcz = s->ifrcz.as<R>();
  a.ux_new = s->ux[1 - cu].p;
  a.uy_new = s->uy[1 - cu].p;
  a.uz_new = s->uz[1 - cu].p;
  a.t_new = s->t[1 - cu].p;
  DevBuf *srcs[4][2] = {{&s->sux[0], &s->sux[1]}, {&s->suy[0], &s->suy[1]}, {&s->suz[0], &s->suz[1]},
                        {&s->st[0], &s->st[1]}};
  for (int f = 0; f < 4; f++) {
    a.sa[f] = srcs[f][s->sa_f]->as<R>();
    a.sb[f] = srcs[f][1 - s->sa_f]->as<R>();
  }
  a.fw = s->fw.as<R>();
  a.lap_ux = s->lap_ux.p;
  a.lap_cc = s->lap_cc.p;
  a.coef = s->coef.p;
  a.dtp = s->d_dt;
  a.m_dif = s->prm.m_dif;
  a.t_dif = s->prm.t_dif;
  for (int q = 0; q < 3; q++) {
    a.lapy[q] = s->lapy[q];
    a.lapz[q] = s->lapz[q];
  }
  a.rk = RK{RK_A[rk], RK_B[rk], RK_A[rk] + RK_B[rk]};
  a.use_b = rk != 0;
  a.add_buoyancy = s->prm.add_buoyancy;
  a.uy_xm = s->prm.uy_xm;
  a.uy_xp = s->prm.uy_xp;
  a.uz_xm = s->prm.uz_xm;
  a.uz_xp = s->prm.uz_xp;
  a.t_xm = s->prm.t_xm;
  a.t_xp = s->prm.t_xp;
  a.vof = s->vof[s->cur_v].p;  // after this substep's advection
  a.grav_vof = s->grav_vof;
  a.vof_ref = s->vof_ref;
  a.g = s->grid();
  CK(predict_launch<R>(s->stream, a));
  return 0;
}

int launch_predict(svof3d_solver *s, int rk) {
  k3_tdm_coef<<<1, 128, sizeof(double) * 6 * s->nx, s->stream>>>(s->lap_ux.p, s->lap_cc.p, s->d_dt,
                                                                 RK_A[rk] + RK_B[rk], s->prm.m_dif, s->prm.t_dif,
                                                                 s->nx, s->coef.p);
  CK_LAUNCH();
  if (0 != rk) s->sa_f ^= 1;
  const int rc = s->mixed ? launch_predict_t<float>(s, rk) : launch_predict_t<double>(s, rk);
  if (rc) return 1;
  s->cur_u ^= 1;
  return 0;
}

// the Poisson stages; `mark` (may be empty) is called with the kernel kind
// after each launch
using Marker = std::function<int(int)>;

// the defect-corrected form (SVOF3_MIXED_DC): an FP32 pass on b, the FP64
// residual r = b - L psi1, an FP32 pass on r accumulated into psi (b and r in
// the predictor's idle line scratch, the spectrum and the x scratch in their
// FP64 buffers' first halves)
int launch_potential_dc(svof3d_solver *s, int rk, const Marker &mark) {
  const double gam = RK_A[rk] + RK_B[rk];
  const Grid3 g = s->grid();
  auto m = [&](int kind) { return mark ? mark(kind) : 0; };
  const int cu = s->cur_u;
  double *b = s->fw.as<double>(), *r = b + (size_t)s->nx * s->ny * s->nz;
  float *sp = s->spec.as<float>(), *xs = s->xscratch.as<float>();
  for (int pass = 0; pass < 2; pass++) {
    if (0 == pass) {
      CK(pois_fwd_y<float>(s->stream, s->ux[cu].p, s->uy[cu].p, s->uz[cu].p, b, sp, s->twf_y32.as<float>(),
                           s->d_dt, gam, s->log2ny, g));
    } else {
      CK(pois_resid(s->stream, b, s->psi.p, r, s->pl.p, s->pu.p, g));
      CK(pois_fwd_y_array<float>(s->stream, r, sp, s->twf_y32.as<float>(), s->log2ny, g));
    }
    if (m(SVOF3_K_POISSON_FWD)) return 1;
    CK(pois_z<float>(s->stream, sp, s->twf_z32.as<float>(), s->log2nz, g));
    if (m(SVOF3_K_POISSON_Z)) return 1;
    CK(pois_x<float>(s->stream, sp, xs, s->pl.p, s->pu.p, s->evy.p, s->evz.p, g, true, s->d_health + 1));
    if (m(SVOF3_K_POISSON_SOLVE)) return 1;
    CK(pois_z<float>(s->stream, sp, s->twb_z32.as<float>(), s->log2nz, g));
    if (m(SVOF3_K_POISSON_Z)) return 1;
    CK(pois_inv_y<float>(s->stream, sp, s->psi.p, s->twb_y32.as<float>(), s->log2ny, g, 1 == pass));
    if (m(SVOF3_K_POISSON_INV)) return 1;
  }
  return 0;
}

// the Poisson solve, FP64 in the FP64 and mixed paths (one pass)
int launch_potential(svof3d_solver *s, int rk, const Marker &mark = Marker()) {
  if (s->dc) return launch_potential_dc(s, rk, mark);
  const double gam = RK_A[rk] + RK_B[rk];
  const Grid3 g = s->grid();
  auto m = [&](int kind) { return mark ? mark(kind) : 0; };
  const int cu = s->cur_u;
  // (the right-hand side goes through the predictor's line scratch, idle
  // here: 4 nx ny nz elements of 4 or 8 bytes).  The mixed path's y
  // transforms carry two columns per complex line; the FP64 path's follow
  // the restatement's rounding with one real line per transform.
  if (s->mixed) {
    CK(pois_fwd_y_packed(s->stream, s->ux[cu].p, s->uy[cu].p, s->uz[cu].p, s->fw.as<double>(), s->spec.p,
                         s->twf_y.p, s->d_dt, gam, s->log2ny, g));
  } else {
    CK(pois_fwd_y<double>(s->stream, s->ux[cu].p, s->uy[cu].p, s->uz[cu].p, s->fw.as<double>(), s->spec.p,
                          s->twf_y.p, s->d_dt, gam, s->log2ny, g));
  }
  if (m(SVOF3_K_POISSON_FWD)) return 1;
  CK(pois_z<double>(s->stream, s->spec.p, s->twf_z.p, s->log2nz, g));
  if (m(SVOF3_K_POISSON_Z)) return 1;
  CK(pois_x<double>(s->stream, s->spec.p, s->xscratch.p, s->pl.p, s->pu.p, s->evy.p, s->evz.p, g, false,
                    s->d_health + 1));
  if (m(SVOF3_K_POISSON_SOLVE)) return 1;
  CK(pois_z<double>(s->stream, s->spec.p, s->twb_z.p, s->log2nz, g));
  if (m(SVOF3_K_POISSON_Z)) return 1;
  if (s->mixed) CK(pois_inv_y_packed(s->stream, s->spec.p, s->psi.p, s->twb_y.p, s->log2ny, g));
  else CK(pois_inv_y<double>(s->stream, s->spec.p, s->psi.p, s->twb_y.p, s->log2ny, g));
  if (m(SVOF3_K_POISSON_INV)) return 1;
  return 0;
}

int launch_project(svof3d_solver *s, int rk, int do_vel, int do_p) {
  dim3 b(32, 8), gr((s->nx + 31) / 32, (s->ny + 7) / 8, (s->nz + kProjectPlanes - 1) / kProjectPlanes);
  k3_project<<<gr, b, 0, s->stream>>>(s->ux[s->cur_u].p, s->uy[s->cur_u].p, s->uz[s->cur_u].p, s->p.p, s->psi.p,
                                      s->d_dt, RK_A[rk] + RK_B[rk], s->prm.m_dif, s->prm.uy_xm, s->prm.uy_xp,
                                      s->prm.uz_xm, s->prm.uz_xp, do_vel, do_p, s->grid());
  CK_LAUNCH();
  return 0;
}

int launch_step(svof3d_solver *s) {
  if (launch_dt(s)) return 1;
  for (int rk = 0; rk < 3; rk++) {
    if (launch_geom(s) || launch_force(s) || launch_vof(s, rk) || launch_predict(s, rk) ||
        launch_potential(s, rk) || launch_project(s, rk, 1, 1))
      return 1;
  }
  return 0;
}

int state_key(const svof3d_solver *s) { return s->cur_u | (s->cur_v << 1) | (s->sa_f << 2) | (s->sa_v << 3); }

int step_graph(svof3d_solver *s, cudaGraphExec_t *exec) {
  const int key = state_key(s);
  auto it = s->graphs.find(key);
  if (it != s->graphs.end()) {
    *exec = it->second;
    s->cur_u ^= 1;  // three field swaps per step (odd), two source swaps (even)
    s->cur_v ^= 1;
    return 0;
  }
  cudaGraph_t graph;
  CK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
  const int rc = launch_step(s);
  cudaError_t e = cudaStreamEndCapture(s->stream, &graph);
  if (rc) return 1;
  if (cudaSuccess != e) return fail("cudaStreamEndCapture: %s", cudaGetErrorString(e));
  cudaGraphExec_t ge;
  CK(cudaGraphInstantiate(&ge, graph, 0));
  cudaGraphDestroy(graph);
  s->graphs[key] = ge;
  *exec = ge;
  return 0;
}

int field_buf(svof3d_solver *s, int field, DevBuf **b) {
  switch (field) {
    case SVOF3_UX: *b = &s->ux[s->cur_u]; break;
    case SVOF3_UY: *b = &s->uy[s->cur_u]; break;
    case SVOF3_UZ: *b = &s->uz[s->cur_u]; break;
    case SVOF3_T: *b = &s->t[s->cur_u]; break;
    case SVOF3_VOF: *b = &s->vof[s->cur_v]; break;
    case SVOF3_P: *b = &s->p; break;
    case SVOF3_PSI: *b = &s->psi; break;
    case SVOF3_CURV: *b = &s->curv; break;
    case SVOF3_NORMAL: *b = &s->normal; break;
    case SVOF3_IFRCX: *b = &s->ifrcx; break;
    case SVOF3_IFRCY: *b = &s->ifrcy; break;
    case SVOF3_IFRCZ: *b = &s->ifrcz; break;
    case SVOF3_SRCUX_A: *b = &s->sux[s->sa_f]; break;
    case SVOF3_SRCUX_B: *b = &s->sux[1 - s->sa_f]; break;
    case SVOF3_SRCUY_A: *b = &s->suy[s->sa_f]; break;
    case SVOF3_SRCUY_B: *b = &s->suy[1 - s->sa_f]; break;
    case SVOF3_SRCUZ_A: *b = &s->suz[s->sa_f]; break;
    case SVOF3_SRCUZ_B: *b = &s->suz[1 - s->sa_f]; break;
    case SVOF3_SRCT_A: *b = &s->st[s->sa_f]; break;
    case SVOF3_SRCT_B: *b = &s->st[1 - s->sa_f]; break;
    case SVOF3_SRC_A: *b = &s->svof[s->sa_v]; break;
    case SVOF3_SRC_B: *b = &s->svof[1 - s->sa_v]; break;
    default: return fail("unknown field id %d", field);
  }
  return 0;
}

// halo width (y and z) and x width of the restart-layout fields
int interior_layout(const svof3d_solver *s, int field, int *nh, int *width) {
  switch (field) {
    case SVOF3_UX: *nh = 1; *width = s->nx + 1; return 0;
    case SVOF3_UY: case SVOF3_UZ: case SVOF3_P: case SVOF3_T: case SVOF3_PSI: *nh = 1; *width = s->nx + 2; return 0;
    case SVOF3_VOF: *nh = 2; *width = s->nx + 2; return 0;
    default: return fail("field %d has no restart-file layout", field);
  }
}

// staging buffer of `count` doubles and its events, made on first use
int io_slot(svof3d_solver *s, svof3d_solver::IoSlot &q, size_t count) {
  if (!s->io_h2d) CK(cudaStreamCreateWithFlags(&s->io_h2d, cudaStreamNonBlocking));
  if (!s->io_d2h) CK(cudaStreamCreateWithFlags(&s->io_d2h, cudaStreamNonBlocking));
  // the events first and the buffer last, so that a slot with a buffer is
  // complete (a failure leaves the events for the next attempt)
  if (!q.filled) CK(cudaEventCreateWithFlags(&q.filled, cudaEventDisableTiming));
  if (!q.drained) CK(cudaEventCreateWithFlags(&q.drained, cudaEventDisableTiming));
  if (!q.stage) CK(cudaMalloc(&q.stage, sizeof(double) * count));
  return 0;
}

void io_free(svof3d_solver *s) {
  if (s->io_h2d) cudaStreamSynchronize(s->io_h2d);
  if (s->io_d2h) cudaStreamSynchronize(s->io_d2h);
  for (int f = 0; f < SVOF3_NFIELDS; f++) {
    for (svof3d_solver::IoSlot *q : {&s->io_in[f], &s->io_out[f]}) {
      if (q->stage) cudaFree(q->stage);
      if (q->filled) cudaEventDestroy(q->filled);
      if (q->drained) cudaEventDestroy(q->drained);
      *q = svof3d_solver::IoSlot{};
    }
  }
  if (s->io_h2d) cudaStreamDestroy(s->io_h2d);
  if (s->io_d2h) cudaStreamDestroy(s->io_d2h);
  s->io_h2d = s->io_d2h = nullptr;
}

int build_tables(svof3d_solver *s, const double *xf, const double *xc) {
  const int nx = s->nx, ny = s->ny, nz = s->nz;
  std::vector<double> dxf(nx), dxc(nx + 1);
  for (int i = 1; i <= nx; i++) dxf[i - 1] = xf[i] - xf[i - 1];
  for (int i = 1; i <= nx + 1; i++) dxc[i - 1] = xc[i] - xc[i - 1];
  s->dy = s->prm.ly / ny;
  s->dz = s->prm.lz / nz;
  if (upload(s->dxf, dxf) || upload(s->dxc, dxc)) return 1;
  auto DXF = [&](int i) { return dxf[i - 1]; };
  auto DXC = [&](int i) { return dxc[i - 1]; };
  std::vector<double> lux(3 * (nx - 1)), lcc(3 * nx);
  for (int i = 2; i <= nx; i++) {
    const double l = 1. / DXF(i - 1) / DXC(i);
    const double u = 1. / DXF(i) / DXC(i);
    lux[3 * (i - 2) + 0] = l;
    lux[3 * (i - 2) + 1] = -l - u;
    lux[3 * (i - 2) + 2] = u;
  }
  for (int i = 1; i <= nx; i++) {
    const double l = 1. / DXC(i) / DXF(i);
    const double u = 1. / DXC(i + 1) / DXF(i);
    lcc[3 * (i - 1) + 0] = l;
    lcc[3 * (i - 1) + 1] = -l - u;
    lcc[3 * (i - 1) + 2] = u;
  }
  if (upload(s->lap_ux, lux) || upload(s->lap_cc, lcc)) return 1;
  s->lapy[0] = +1. / s->dy / s->dy;
  s->lapy[1] = -2. / s->dy / s->dy;
  s->lapy[2] = +1. / s->dy / s->dy;
  s->lapz[0] = +1. / s->dz / s->dz;
  s->lapz[1] = -2. / s->dz / s->dz;
  s->lapz[2] = +1. / s->dz / s->dz;
  const int ndims = 3;
  const double cd = s->prm.coef_dt_dif;
  s->lims[0] = cd / s->prm.m_dif * 0.5 / ndims * std::pow(s->dy, 2.);
  s->lims[1] = cd / s->prm.m_dif * 0.5 / ndims * std::pow(s->dz, 2.);
  s->lims[2] = cd / s->prm.t_dif * 0.5 / ndims * std::pow(s->dy, 2.);
  s->lims[3] = cd / s->prm.t_dif * 0.5 / ndims * std::pow(s->dz, 2.);
  s->log2ny = ilog2_exact(ny);
  s->log2nz = ilog2_exact(nz);
  if (s->log2ny < 1 || s->log2nz < 1) return fail("svof3d_create: ny and nz must be powers of two (got %d, %d)", ny, nz);
  // (the transforms are compiled for lengths 2 .. 2048)
  if (s->log2ny > 11 || s->log2nz > 11) return fail("svof3d_create: ny and nz at most 2048 (got %d, %d)", ny, nz);
  auto twiddles = [&](int n, DevBuf &f, DevBuf &b) -> int {
    std::vector<double> twf(2 * (n / 2)), twb(2 * (n / 2));
    for (int m = 0; m < n / 2; m++) {
      const double ang = 2.0 * kPi * (double)m / (double)n;
      twf[2 * m] = std::cos(ang);
      twf[2 * m + 1] = -std::sin(ang);
      twb[2 * m] = std::cos(ang);
      twb[2 * m + 1] = std::sin(ang);
    }
    return upload(f, twf) || upload(b, twb);
  };
  if (twiddles(ny, s->twf_y, s->twb_y) || twiddles(nz, s->twf_z, s->twb_z)) return 1;
  if (s->dc) {
    // FP32 copies of the same tables (the FP64 values rounded once)
    auto to32 = [&](const DevBuf &d, DevBuf &f) -> int {
      std::vector<double> h(d.n);
      CK(cudaMemcpy(h.data(), d.p, sizeof(double) * d.n, cudaMemcpyDeviceToHost));
      std::vector<float> hf(h.begin(), h.end());
      if (dalloc(f, d.n, sizeof(float))) return 1;
      CK(cudaMemcpy(f.p, hf.data(), sizeof(float) * d.n, cudaMemcpyHostToDevice));
      return 0;
    };
    if (to32(s->twf_y, s->twf_y32) || to32(s->twb_y, s->twb_y32) || to32(s->twf_z, s->twf_z32) ||
        to32(s->twb_z, s->twb_z32))
      return 1;
  }
  const int nky = ny / 2 + 1;
  std::vector<double> evy(nky), evz(nz), pl(nx), pu(nx);
  for (size_t j = 0; j < (size_t)nky; j++)
    evy[j] = -4. / std::pow(s->prm.ly / ny, 2.) * std::pow(std::sin(kGPi * j / (double)ny), 2.);
  for (size_t k = 0; k < (size_t)nz; k++)
    evz[k] = -4. / std::pow(s->prm.lz / nz, 2.) * std::pow(std::sin(kGPi * k / (double)nz), 2.);
  for (int i = 1; i <= nx; i++) {
    pl[i - 1] = 1. / DXC(i) / DXF(i);
    pu[i - 1] = 1. / DXC(i + 1) / DXF(i);
  }
  if (upload(s->evy, evy) || upload(s->evz, evz) || upload(s->pl, pl) || upload(s->pu, pu)) return 1;
  return 0;
}

}  // namespace

extern "C" {

const char *svof3d_last_error(void) { return g_err3.c_str(); }

int svof3d_destroy(svof3d_solver_t *s) {
  if (!s) return 0;
  if (s->stream) cudaStreamSynchronize(s->stream);
  io_free(s);
  adjoint3_free(s);
  for (auto &kv : s->graphs) cudaGraphExecDestroy(kv.second);
  s->graphs.clear();
  for (int k = 0; k < 2; k++) {
    dfree(s->ux[k]); dfree(s->uy[k]); dfree(s->uz[k]); dfree(s->t[k]); dfree(s->vof[k]);
    dfree(s->sux[k]); dfree(s->suy[k]); dfree(s->suz[k]); dfree(s->st[k]); dfree(s->svof[k]);
  }
  DevBuf *bufs[] = {&s->p, &s->psi, &s->curv, &s->normal, &s->ifrcx, &s->ifrcy, &s->ifrcz, &s->dxf, &s->dxc,
                    &s->lap_ux, &s->lap_cc, &s->coef, &s->spec, &s->xscratch, &s->twf_y, &s->twb_y, &s->twf_z,
                    &s->twb_z, &s->pl, &s->pu, &s->evy, &s->evz, &s->fw, &s->diag, &s->stat_part,
                    &s->twf_y32, &s->twb_y32, &s->twf_z32, &s->twb_z32};
  for (DevBuf *b : bufs) dfree(*b);
  for (DevBuf &b : s->stat) dfree(b);
  if (s->d_dt) cudaFree(s->d_dt);
  if (s->d_minbits) cudaFree(s->d_minbits);
  if (s->d_status) cudaFree(s->d_status);
  if (s->d_health) cudaFree(s->d_health);
  if (s->d_work) cudaFree(s->d_work);
  if (s->d_nwork) cudaFree(s->d_nwork);
  if (s->h_dt) cudaFreeHost(s->h_dt);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
  return 0;
}

int svof3d_create(const svof3d_params_t *prm, const double *xf, const double *xc, svof3d_solver_t **out) {
  if (!prm || !xf || !xc || !out) return fail("svof3d_create: null argument");
  *out = nullptr;
  svof_fault::begin_creation();
  if (prm->nx < 4 || prm->ny < 4 || prm->nz < 4) return fail("svof3d_create: nx, ny and nz must be at least 4");
  if (!(prm->m_dif > 0.) || !(prm->t_dif > 0.)) return fail("svof3d_create: diffusivities must be positive");
  if (prm->ny > 2048 || prm->nz > 2048) return fail("svof3d_create: ny and nz must be at most 2048");
  if ((double)prm->nx * (prm->ny + 4) * (prm->nz + 4) > 4.0e9)
    return fail("svof3d_create: %d x %d x %d cells exceed the 32-bit cell index", prm->nx, prm->ny, prm->nz);
  if (SVOF3_FP64 != prm->precision && SVOF3_MIXED != prm->precision && SVOF3_MIXED_DC != prm->precision)
    return fail("svof3d_create: precision must be SVOF3_FP64, SVOF3_MIXED or SVOF3_MIXED_DC (got %d)",
                prm->precision);
  svof3d_solver *s = new svof3d_solver();
  s->prm = *prm;
  s->mixed = SVOF3_FP64 != prm->precision;
  s->dc = SVOF3_MIXED_DC == prm->precision;
  s->nx = prm->nx;
  s->ny = prm->ny;
  s->nz = prm->nz;
  auto bail = [&]() {
    std::string e = g_err3;
    svof3d_destroy(s);
    g_err3 = e;
    return 1;
  };
  if (cudaSuccess != cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking)) {
    delete s;
    return fail("svof3d_create: no CUDA device available (%s)", cudaGetErrorString(cudaGetLastError()));
  }
  const size_t nx = s->nx, ny = s->ny, nz = s->nz;
  const size_t es = s->mixed ? sizeof(float) : sizeof(double);  // intermediates
  const size_t n_ux = (nx + 1) * (ny + 2) * (nz + 2), n_cc = (nx + 2) * (ny + 2) * (nz + 2);
  const size_t n_vof = (nx + 2) * (ny + 4) * (nz + 4), n_src = nx * ny * nz, n_srcx = (nx - 1) * ny * nz;
  for (int k = 0; k < 2; k++) {
    if (dalloc(s->ux[k], n_ux) || dalloc(s->uy[k], n_cc) || dalloc(s->uz[k], n_cc) || dalloc(s->t[k], n_cc) ||
        dalloc(s->vof[k], n_vof))
      return bail();
    if (dalloc(s->sux[k], n_srcx, es) || dalloc(s->suy[k], n_src, es) || dalloc(s->suz[k], n_src, es) ||
        dalloc(s->st[k], n_src, es) || dalloc(s->svof[k], n_src))
      return bail();
  }
  if (dalloc(s->p, n_cc) || dalloc(s->psi, n_cc) || dalloc(s->curv, n_cc, es) ||
      dalloc(s->normal, 4 * nx * (ny + 2) * (nz + 2), es) || dalloc(s->ifrcx, n_srcx, es) ||
      dalloc(s->ifrcy, n_src, es) || dalloc(s->ifrcz, n_src, es) ||
      dalloc(s->diag, 8 + 5 * (size_t)((nx + 31) / 32) * ((ny + 7) / 8) * ((nz + kDiagPlanes - 1) / kDiagPlanes)))
    return bail();
  if (build_tables(s, xf, xc)) return bail();
  if (dalloc(s->coef, 9 * nx)) return bail();
  const size_t nky = ny / 2 + 1;
  if (dalloc(s->spec, 2 * nx * nky * nz) || dalloc(s->xscratch, nx * nky * nz) ||
      dalloc(s->fw, 4 * nx * ny * nz, es))
    return bail();
  {
    const cudaError_t pe =
        s->dc ? pois_prepare<float>(s->log2ny, s->log2nz) : pois_prepare<double>(s->log2ny, s->log2nz);
    if (cudaSuccess != pe || cudaSuccess != predict_prepare() || cudaSuccess != interface_prepare())
      return fail("cudaFuncSetAttribute(Poisson): %s", cudaGetErrorString(cudaGetLastError())), bail();
    const size_t coef_smem = sizeof(double) * 6 * nx;
    if (coef_smem > 200 * 1024) return fail("svof3d_create: nx too large"), bail();
    if (cudaSuccess != raise_smem_limit(k3_tdm_coef, coef_smem)) return fail("cudaFuncSetAttribute(k3_tdm_coef)"), bail();
  }
  if (cudaSuccess != cudaMalloc(&s->d_dt, sizeof(double))) return fail("cudaMalloc dt"), bail();
  if (cudaSuccess != cudaMalloc(&s->d_work, sizeof(unsigned) * nx * (ny + 2) * (nz + 2)) ||
      cudaSuccess != cudaMalloc(&s->d_nwork, sizeof(unsigned)))
    return fail("cudaMalloc worklist"), bail();
  if (cudaSuccess != cudaMalloc(&s->d_minbits, sizeof(unsigned long long))) return fail("cudaMalloc"), bail();
  if (cudaSuccess != cudaMalloc(&s->d_status, sizeof(unsigned)) ||
      cudaSuccess != cudaMemset(s->d_status, 0, sizeof(unsigned)) ||
      cudaSuccess != cudaMalloc(&s->d_health, 2 * sizeof(unsigned long long)) ||
      cudaSuccess != cudaMemset(s->d_health, 0, 2 * sizeof(unsigned long long)))
    return fail("cudaMalloc status"), bail();
  {
    const double one = 1.;
    unsigned long long bits;
    std::memcpy(&bits, &one, sizeof(bits));
    cudaMemcpy(s->d_minbits, &bits, sizeof(bits), cudaMemcpyHostToDevice);
    cudaMemset(s->d_dt, 0, sizeof(double));
  }
  s->h_dt_slots = 1024;
  if (cudaSuccess != cudaMallocHost(&s->h_dt, sizeof(double) * s->h_dt_slots)) return fail("cudaMallocHost"), bail();
  if (cudaSuccess != cudaDeviceSynchronize())
    return fail("svof3d_create: %s", cudaGetErrorString(cudaGetLastError())), bail();
  *out = s;
  return 0;
}

int svof3d_field_count(const svof3d_solver_t *cs, int field, size_t *count) {
  svof3d_solver *s = const_cast<svof3d_solver *>(cs);
  DevBuf *b;
  if (!s || !count) return fail("null argument");
  if (field_buf(s, field, &b)) return 1;
  *count = b->n;
  return 0;
}

int svof3d_upload_field(svof3d_solver_t *s, int field, const double *host, size_t count) {
  DevBuf *b;
  if (!s || !host) return fail("null argument");
  if (field_buf(s, field, &b)) return 1;
  if (count != b->n) return fail("field %d holds %zu values, got %zu", field, b->n, count);
  if (4 == b->es) {
    std::vector<float> f(host, host + count);
    CK(cudaMemcpyAsync(b->p, f.data(), sizeof(float) * count, cudaMemcpyHostToDevice, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return 0;
  }
  CK(cudaMemcpyAsync(b->p, host, sizeof(double) * count, cudaMemcpyHostToDevice, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return 0;
}

int svof3d_download_field(svof3d_solver_t *s, int field, double *host, size_t count) {
  DevBuf *b;
  if (!s || !host) return fail("null argument");
  if (field_buf(s, field, &b)) return 1;
  if (count != b->n) return fail("field %d holds %zu values, got %zu", field, b->n, count);
  if (4 == b->es) {
    std::vector<float> f(count);
    CK(cudaMemcpyAsync(f.data(), b->p, sizeof(float) * count, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    for (size_t q = 0; q < count; q++) host[q] = (double)f[q];
    return 0;
  }
  CK(cudaMemcpyAsync(host, b->p, sizeof(double) * count, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return 0;
}

int svof3d_device_field(svof3d_solver_t *s, int field, double **dptr) {
  DevBuf *b;
  if (!s || !dptr) return fail("null argument");
  if (field_buf(s, field, &b)) return 1;
  *dptr = b->p;
  return 0;
}

// the restart layout is nz x ny x width; in storage each interior plane k has
// nh halo rows below and above, so the copy is one 2D memcpy of nz planes
int svof3d_load_interior(svof3d_solver_t *s, int field, const double *host, size_t count) {
  SVOF_RANGE();
  int nh, width;
  DevBuf *b;
  if (!s || !host) return fail("null argument");
  if (interior_layout(s, field, &nh, &width) || field_buf(s, field, &b)) return 1;
  const size_t plane = (size_t)width * s->ny;
  if (count != plane * s->nz) return fail("field %d: restart layout holds %zu doubles, got %zu", field,
                                          plane * s->nz, count);
  const size_t spitch = sizeof(double) * plane;
  const size_t dpitch = sizeof(double) * (size_t)width * (s->ny + 2 * nh);
  double *dst = b->p + (size_t)width * (s->ny + 2 * nh) * nh + (size_t)width * nh;
  CK(cudaMemcpy2DAsync(dst, dpitch, host, spitch, spitch, s->nz, cudaMemcpyHostToDevice, s->stream));
  if (launch_halo_bc(s, b->p, field)) return 1;
  CK(cudaStreamSynchronize(s->stream));
  return 0;
}

int svof3d_store_interior(svof3d_solver_t *s, int field, double *host, size_t count) {
  SVOF_RANGE();
  int nh, width;
  DevBuf *b;
  if (!s || !host) return fail("null argument");
  if (interior_layout(s, field, &nh, &width) || field_buf(s, field, &b)) return 1;
  const size_t plane = (size_t)width * s->ny;
  if (count != plane * s->nz) return fail("field %d: restart layout holds %zu doubles, got %zu", field,
                                          plane * s->nz, count);
  const size_t dpitch = sizeof(double) * plane;
  const size_t spitch = sizeof(double) * (size_t)width * (s->ny + 2 * nh);
  const double *src = b->p + (size_t)width * (s->ny + 2 * nh) * nh + (size_t)width * nh;
  CK(cudaMemcpy2DAsync(host, dpitch, src, spitch, dpitch, s->nz, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return 0;
}

// queued load: host -> staging on the copy-in stream (one contiguous copy),
// then staging -> storage and the halo update on the solver's stream, in
// order with the steps queued around it
int svof3d_load_interior_async(svof3d_solver_t *s, int field, const double *host, size_t count) {
  SVOF_RANGE();
  int nh, width;
  DevBuf *b;
  if (!s || !host) return fail("null argument");
  if (interior_layout(s, field, &nh, &width) || field_buf(s, field, &b)) return 1;
  const size_t plane = (size_t)width * s->ny;
  if (count != plane * s->nz) return fail("field %d: restart layout holds %zu doubles, got %zu", field,
                                          plane * s->nz, count);
  svof3d_solver::IoSlot &q = s->io_in[field];
  if (io_slot(s, q, count)) return 1;
  if (q.pending) CK(cudaStreamWaitEvent(s->io_h2d, q.drained, 0));
  CK(cudaMemcpyAsync(q.stage, host, sizeof(double) * count, cudaMemcpyHostToDevice, s->io_h2d));
  CK(cudaEventRecord(q.filled, s->io_h2d));
  CK(cudaStreamWaitEvent(s->stream, q.filled, 0));
  const size_t spitch = sizeof(double) * plane;
  const size_t dpitch = sizeof(double) * (size_t)width * (s->ny + 2 * nh);
  double *dst = b->p + (size_t)width * (s->ny + 2 * nh) * nh + (size_t)width * nh;
  CK(cudaMemcpy2DAsync(dst, dpitch, q.stage, spitch, spitch, s->nz, cudaMemcpyDeviceToDevice, s->stream));
  if (launch_halo_bc(s, b->p, field)) return 1;
  CK(cudaEventRecord(q.drained, s->stream));
  q.pending = true;
  return 0;
}

// queued store: storage -> staging on the solver's stream, then staging ->
// host on the copy-out stream (one contiguous copy)
int svof3d_store_interior_async(svof3d_solver_t *s, int field, double *host, size_t count) {
  SVOF_RANGE();
  int nh, width;
  DevBuf *b;
  if (!s || !host) return fail("null argument");
  if (interior_layout(s, field, &nh, &width) || field_buf(s, field, &b)) return 1;
  const size_t plane = (size_t)width * s->ny;
  if (count != plane * s->nz) return fail("field %d: restart layout holds %zu doubles, got %zu", field,
                                          plane * s->nz, count);
  svof3d_solver::IoSlot &q = s->io_out[field];
  if (io_slot(s, q, count)) return 1;
  if (q.pending) CK(cudaStreamWaitEvent(s->stream, q.drained, 0));
  const size_t dpitch = sizeof(double) * plane;
  const size_t spitch = sizeof(double) * (size_t)width * (s->ny + 2 * nh);
  const double *src = b->p + (size_t)width * (s->ny + 2 * nh) * nh + (size_t)width * nh;
  CK(cudaMemcpy2DAsync(q.stage, dpitch, src, spitch, dpitch, s->nz, cudaMemcpyDeviceToDevice, s->stream));
  CK(cudaEventRecord(q.filled, s->stream));
  CK(cudaStreamWaitEvent(s->io_d2h, q.filled, 0));
  CK(cudaMemcpyAsync(host, q.stage, sizeof(double) * count, cudaMemcpyDeviceToHost, s->io_d2h));
  CK(cudaEventRecord(q.drained, s->io_d2h));
  q.pending = true;
  return 0;
}

int svof3d_io_wait(svof3d_solver_t *s) {
  SVOF_RANGE();
  if (!s) return fail("null argument");
  if (s->io_h2d) CK(cudaStreamSynchronize(s->io_h2d));
  CK(cudaStreamSynchronize(s->stream));
  if (s->io_d2h) CK(cudaStreamSynchronize(s->io_d2h));
  return check_status(s, "svof3d_io_wait");
}

int svof3d_fluid_decide_dt(svof3d_solver_t *s, double *dt) {
  SVOF_RANGE();
  if (!s || !dt) return fail("null argument");
  if (launch_dt(s)) return 1;
  CK(cudaMemcpyAsync(s->h_dt, s->d_dt, sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  *dt = s->h_dt[0];
  return check_status(s, "svof3d_fluid_decide_dt");
}

static int set_dt(svof3d_solver_t *s, double dt) {
  s->h_dt[0] = dt;
  CK(cudaMemcpyAsync(s->d_dt, s->h_dt, sizeof(double), cudaMemcpyHostToDevice, s->stream));
  return 0;
}

static int check_rk(size_t rk) { return rk < 3 ? 0 : fail("rkstep %zu out of range", rk); }

static int finish(svof3d_solver_t *s) {
  CK(cudaStreamSynchronize(s->stream));
  return 0;
}

int svof3d_interface_compute_curvature_tensor(svof3d_solver_t *s) {
  SVOF_RANGE();
  if (!s) return fail("null argument");
  if (launch_geom(s)) return 1;
  return finish(s);
}

int svof3d_interface_compute_force(svof3d_solver_t *s) {
  SVOF_RANGE();
  if (!s) return fail("null argument");
  if (launch_force(s)) return 1;
  return finish(s);
}

int svof3d_interface_update_vof(svof3d_solver_t *s, size_t rk, double dt) {
  SVOF_RANGE();
  if (!s) return fail("null argument");
  if (check_rk(rk) || set_dt(s, dt) || launch_vof(s, (int)rk)) return 1;
  return finish(s);
}

int svof3d_fluid_predict_field(svof3d_solver_t *s, size_t rk, double dt) {
  SVOF_RANGE();
  if (!s) return fail("null argument");
  if (check_rk(rk) || set_dt(s, dt) || launch_predict(s, (int)rk)) return 1;
  return finish(s);
}

int svof3d_fluid_compute_potential_dft(svof3d_solver_t *s, size_t rk, double dt) {
  SVOF_RANGE();
  if (!s) return fail("null argument");
  if (check_rk(rk) || set_dt(s, dt) || launch_potential(s, (int)rk)) return 1;
  return finish(s);
}

int svof3d_fluid_correct_velocity(svof3d_solver_t *s, size_t rk, double dt) {
  SVOF_RANGE();
  if (!s) return fail("null argument");
  if (check_rk(rk) || set_dt(s, dt) || launch_project(s, (int)rk, 1, 0)) return 1;
  return finish(s);
}

int svof3d_fluid_update_pressure(svof3d_solver_t *s, size_t rk, double dt) {
  SVOF_RANGE();
  if (!s) return fail("null argument");
  if (check_rk(rk) || set_dt(s, dt) || launch_project(s, (int)rk, 0, 1)) return 1;
  return finish(s);
}

int svof3d_run(svof3d_solver_t *s, int nsteps, double *dts) {
  SVOF_RANGE();
  if (!s) return fail("null argument");
  if (nsteps < 0) return fail("nsteps must be non-negative");
  for (int n = 0; n < nsteps; n++) {
    cudaGraphExec_t ge;
    if (step_graph(s, &ge)) return 1;
    CK(cudaGraphLaunch(ge, s->stream));
    if (dts) {
      const int slot = n % s->h_dt_slots;
      if (0 == slot && n > 0) {
        CK(cudaStreamSynchronize(s->stream));
        std::memcpy(dts + n - s->h_dt_slots, s->h_dt, sizeof(double) * s->h_dt_slots);
      }
      CK(cudaMemcpyAsync(s->h_dt + slot, s->d_dt, sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    }
  }
  CK(cudaStreamSynchronize(s->stream));
  if (dts && nsteps > 0) {
    const int done = ((nsteps - 1) / s->h_dt_slots) * s->h_dt_slots;
    std::memcpy(dts + done, s->h_dt, sizeof(double) * (nsteps - done));
  }
  return check_status(s, "svof3d_run");
}

int svof3d_enqueue_steps(svof3d_solver_t *s, int nsteps) {
  SVOF_RANGE();
  if (!s) return fail("null argument");
  if (nsteps < 0) return fail("nsteps must be non-negative");
  for (int n = 0; n < nsteps; n++) {
    cudaGraphExec_t ge;
    if (step_graph(s, &ge)) return 1;
    CK(cudaGraphLaunch(ge, s->stream));
    CK(cudaMemcpyAsync(s->h_dt, s->d_dt, sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  }
  return 0;
}

int svof3d_last_dt(svof3d_solver_t *s, double *dt) {
  if (!s || !dt) return fail("null argument");
  CK(cudaStreamSynchronize(s->stream));
  *dt = s->h_dt[0];
  return check_status(s, "svof3d_last_dt");
}

int svof3d_integrate(svof3d_solver_t *s, double *dt) {
  SVOF_RANGE();
  double d = 0.;
  if (svof3d_run(s, 1, &d)) return 1;
  if (dt) *dt = d;
  return 0;
}

int svof3d_profile_step(svof3d_solver_t *s, double *ms, int *launches, int nkinds) {
  SVOF_RANGE();
  if (!s || !ms || !launches || nkinds < SVOF3_NKINDS) return fail("svof3d_profile_step: bad arguments");
  for (int k = 0; k < nkinds; k++) {
    ms[k] = 0.;
    launches[k] = 0;
  }
  std::vector<cudaEvent_t> ev;
  std::vector<int> kind;
  Marker mark = [&](int k) -> int {
    cudaEvent_t e;
    CK(cudaEventCreate(&e));
    CK(cudaEventRecord(e, s->stream));
    ev.push_back(e);
    kind.push_back(k);
    return 0;
  };
  int rc = mark(-1);
  rc = rc || launch_dt(s) || mark(SVOF3_K_DT);
  for (int rk = 0; rk < 3 && !rc; rk++) {
    rc = rc || launch_geom(s) || mark(SVOF3_K_GEOM);
    rc = rc || launch_force(s) || mark(SVOF3_K_FORCE);
    rc = rc || launch_vof(s, rk) || mark(SVOF3_K_VOF);
    rc = rc || launch_predict(s, rk) || mark(SVOF3_K_PREDICT);
    rc = rc || launch_potential(s, rk, mark);
    rc = rc || launch_project(s, rk, 1, 1) || mark(SVOF3_K_PROJECT);
  }
  cudaError_t e = cudaStreamSynchronize(s->stream);
  if (!rc && cudaSuccess == e) {
    for (size_t q = 1; q < ev.size(); q++) {
      float t = 0.f;
      cudaEventElapsedTime(&t, ev[q - 1], ev[q]);
      ms[kind[q]] += t;
      // kernels per kind: predict = coefficients, right-hand sides, line
      // solve; dt = reduction + final; geom = geometry + intercept;
      // poisson_fwd = right-hand side + transform
      const int kq = kind[q];
      launches[kq] += (SVOF3_K_PREDICT == kq) ? 3
                      : ((SVOF3_K_DT == kq || SVOF3_K_GEOM == kq || SVOF3_K_POISSON_FWD == kq) ? 2 : 1);
    }
  }
  for (cudaEvent_t x : ev) cudaEventDestroy(x);
  if (rc) return 1;
  if (cudaSuccess != e) return fail("svof3d_profile_step: %s", cudaGetErrorString(e));
  return 0;
}

int svof3d_diagnostics(svof3d_solver_t *s, double *divmax, double *vofmin, double *vofmax, double *volume) {
  SVOF_RANGE();
  if (!s) return fail("null argument");
  const dim3 db(32, 8), dg((s->nx + 31) / 32, (s->ny + 7) / 8, (s->nz + kDiagPlanes - 1) / kDiagPlanes);
  k3_diag_part<<<dg, db, 0, s->stream>>>(s->ux[s->cur_u].p, s->uy[s->cur_u].p, s->uz[s->cur_u].p,
                                         s->vof[s->cur_v].p, s->diag.p + 8, s->grid());
  CK_LAUNCH();
  k3_diag_final<<<1, kDiagThreads, 0, s->stream>>>(s->diag.p + 8, (long)dg.x * dg.y * dg.z, s->diag.p);
  CK_LAUNCH();
  double h[4];
  CK(cudaMemcpyAsync(h, s->diag.p, sizeof(h), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  if (divmax) *divmax = h[0];
  if (vofmin) *vofmin = h[1];
  if (vofmax) *vofmax = h[2];
  if (volume) *volume = h[3];
  return 0;
}

// x width of a statistics array: faces for ux1 ux2 uxt, cells otherwise
static int stat_width(const svof3d_solver *s, int q) {
  return (SVOF3_STAT_UX1 == q || SVOF3_STAT_UX2 == q || SVOF3_STAT_UXT == q) ? s->nx + 1 : s->nx + 2;
}

int svof3d_statistics_collect(svof3d_solver_t *s) {
  if (!s) return fail("null argument");
  if (!s->stat_part.p) {
    // all accumulators and the row-sum scratch, or none: a failed allocation
    // frees what it made, and the next collection tries again
    DevBuf made[SVOF3_NSTATS + 1];
    cudaError_t e = cudaSuccess;
    for (int q = 0; q <= SVOF3_NSTATS && cudaSuccess == e; q++) {
      made[q].n = q < SVOF3_NSTATS ? (size_t)stat_width(s, q) * s->ny * s->nz : (size_t)(s->nz + 1) * (s->nx + 2);
      e = cudaMalloc(&made[q].p, sizeof(double) * made[q].n);
      if (cudaSuccess == e && q < SVOF3_NSTATS)
        e = cudaMemsetAsync(made[q].p, 0, sizeof(double) * made[q].n, s->stream);
    }
    if (cudaSuccess != e) {
      for (DevBuf &b : made) dfree(b);
      return fail("statistics accumulators: %s", cudaGetErrorString(e));
    }
    for (int q = 0; q < SVOF3_NSTATS; q++) s->stat[q] = made[q];
    s->stat_part = made[SVOF3_NSTATS];
  }
  StatArgs a{s->ux[s->cur_u].p, s->uy[s->cur_u].p, s->uz[s->cur_u].p, s->t[s->cur_u].p,
             s->stat[SVOF3_STAT_UX1].p, s->stat[SVOF3_STAT_UX2].p, s->stat[SVOF3_STAT_UY1].p,
             s->stat[SVOF3_STAT_UY2].p, s->stat[SVOF3_STAT_UZ1].p, s->stat[SVOF3_STAT_UZ2].p,
             s->stat[SVOF3_STAT_T1].p, s->stat[SVOF3_STAT_T2].p, s->stat[SVOF3_STAT_UXT].p,
             s->nx, s->ny, s->nz, 1};
  const dim3 b(32, 8), g((s->nx + 2 + 31) / 32, (s->ny + 7) / 8, s->nz);
  k_stat_collect<<<g, b, 0, s->stream>>>(a);
  CK_LAUNCH();
  s->stat_num += 1;
  return 0;
}

int svof3d_statistics_reset(svof3d_solver_t *s) {
  if (!s) return fail("null argument");
  for (DevBuf &b : s->stat)
    if (b.p) CK(cudaMemsetAsync(b.p, 0, sizeof(double) * b.n, s->stream));
  s->stat_num = 0;
  CK(cudaStreamSynchronize(s->stream));
  return 0;
}

int svof3d_statistics_count(svof3d_solver_t *s, size_t *num) {
  if (!s || !num) return fail("null argument");
  *num = s->stat_num;
  return 0;
}

int svof3d_statistics_reduce(svof3d_solver_t *s, int quantity, double *out, size_t count) {
  if (!s || !out) return fail("null argument");
  if (quantity < 0 || quantity >= SVOF3_NSTATS) return fail("unknown statistics quantity %d", quantity);
  const int w = stat_width(s, quantity);
  if (count != (size_t)w) return fail("statistics quantity %d has %d columns, got %zu", quantity, w, count);
  if (!s->stat_part.p) {
    for (int i = 0; i < w; i++) out[i] = 0.;
    return 0;
  }
  double *part = s->stat_part.p, *res = s->stat_part.p + (size_t)s->nz * w;
  k_stat_reduce_planes<<<dim3((w + 127) / 128, s->nz), 128, 0, s->stream>>>(s->stat[quantity].p, w, s->ny,
                                                                             part);
  CK_LAUNCH();
  k_stat_reduce_final<<<(w + 127) / 128, 128, 0, s->stream>>>(part, w, s->nz, res);
  CK_LAUNCH();
  CK(cudaMemcpyAsync(out, res, sizeof(double) * w, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return 0;
}

int svof3d_statistics_field(svof3d_solver_t *s, int quantity, double *out, size_t count) {
  if (!s || !out) return fail("null argument");
  if (quantity < 0 || quantity >= SVOF3_NSTATS) return fail("unknown statistics quantity %d", quantity);
  const size_t n = (size_t)stat_width(s, quantity) * s->ny * s->nz;
  if (count != n) return fail("statistics quantity %d holds %zu values, got %zu", quantity, n, count);
  if (!s->stat_part.p) {
    for (size_t q = 0; q < n; q++) out[q] = 0.;
    return 0;
  }
  CK(cudaMemcpyAsync(out, s->stat[quantity].p, sizeof(double) * n, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return 0;
}

int svof3d_synchronize(svof3d_solver_t *s) {
  SVOF_RANGE();
  if (!s) return fail("null argument");
  CK(cudaStreamSynchronize(s->stream));
  return check_status(s, "svof3d_synchronize");
}

int svof3d_health(svof3d_solver_t *s, unsigned long long *newton_unconverged, unsigned long long *small_pivots,
                  int reset) {
  SVOF_RANGE();
  if (!s) return fail("null argument");
  unsigned long long h[2] = {0, 0};
  CK(cudaMemcpyAsync(h, s->d_health, sizeof(h), cudaMemcpyDeviceToHost, s->stream));
  if (reset) CK(cudaMemsetAsync(s->d_health, 0, sizeof(h), s->stream));
  CK(cudaStreamSynchronize(s->stream));
  if (newton_unconverged) *newton_unconverged = h[0];
  if (small_pivots) *small_pivots = h[1];
  return check_status(s, "svof3d_health");
}

int svof3d_stream(svof3d_solver_t *s, void **stream) {
  if (!s || !stream) return fail("null argument");
  *stream = (void *)s->stream;
  return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// The differentiation form of the 3D FP64 path (no counterpart in the
// reference), the 2D form (adjoint.cu) carried to the third direction: a
// differentiated run holds the time-step sequence fixed; svof3d_integrate_fixed
// takes one step with a given dt and, when asked, records the primal inputs
// of its three substeps (ux, uy, uz, vof, storage layouts) on a tape in device
// memory; svof3d_adjoint_step maps the adjoint of a step's outputs (ux, uy,
// uz, p, vof) to the adjoint of its inputs in place and accumulates the
// adjoint of the surface-tension coefficient 1/We.  Per substep, in reverse:
// the projection and pressure update, the Poisson solve (a second solve, of
// psi_bar / dxf, by the forward's own transforms and line solves), the
// implicit-x line solves, the momentum right-hand sides, the vof fluxes and
// update, the CSF force, the intercept and normals, the corner gradients
// (k3_adjoint.cu).  The per-function entry points expose the same pieces one
// by one about the solver's current fields.  The temperature is not
// differentiated (add_buoyancy must be 0).  The adjoint computes in FP64 on
// every path: with the mixed paths (FP32 geometry, FP32 sources) it is the
// FP64 step's transpose about the mixed trajectory, its geometry (normals,
// intercepts, curvature) recomputed in FP64 from the taped vof into buffers
// of its own.

struct Adjoint3State {
  // compact: ux faces nz x ny x (nx-1), cells nz x ny x nx
  DevBuf ux, uy, uz, p, vof[2], pend_v[2];
  DevBuf pend_x, pend_y, pend_z, sa_x, sg_x, sa_y, sg_y, sa_z, sg_z, ifx, ify, ifz, kap, m, nrm, sig;
  DevBuf psib, b, psis, gbar, grv, sum;
  DevBuf rxf, rxc;  // 1 / dxf, 1 / dxc
  DevBuf nrm64, curv64;  // FP64 geometry of the mixed paths (storage layouts)
  DevBuf zx, zy, zz;     // the x solve's forward values with FP32 intermediates (FP64)
  bool f32 = false;      // intermediates (sources, forces, curvature, normals, corners) in FP32
  int cv = 0;  // current buffer of vof_bar
  int cp = 0;  // current buffer of the vof source's pending adjoint
  size_t xs_smem = 0;
  double tau = 0.;  // gradient floor (svof3d_adjoint_set_gradient_floor)
  // the adjoint fields and scratch (zeroed by svof3d_adjoint_reset)
  DevBuf *all(int q) {
    DevBuf *l[] = {&ux, &uy, &uz, &p, &vof[0], &vof[1], &pend_v[0], &pend_v[1], &pend_x, &pend_y, &pend_z,
                   &sa_x, &sg_x, &sa_y, &sg_y, &sa_z, &sg_z, &ifx, &ify, &ifz, &kap, &m, &nrm, &sig,
                   &psib, &b, &psis, &gbar, &grv, &sum};
    return q < (int)(sizeof(l) / sizeof(l[0])) ? l[q] : nullptr;
  }
};

void adjoint3_free(svof3d_solver *s) {
  if (!s || !s->adj) return;
  for (int q = 0; DevBuf *b = s->adj->all(q); q++) dfree(*b);
  dfree(s->adj->rxf);
  dfree(s->adj->rxc);
  dfree(s->adj->nrm64);
  dfree(s->adj->curv64);
  dfree(s->adj->zx);
  dfree(s->adj->zy);
  dfree(s->adj->zz);
  delete s->adj;
  s->adj = nullptr;
}

namespace {

// the mixed paths' default gradient floor: their FP32 fluxes leave vof noise
// of order 1e-8 beside the interface, where corners with such tiny gradients
// would make the normals' transposes (I - n n^T) / |g| grow without bound
// from step to step
constexpr double kAdjMixedTau = 1e-5;

int adj3_ensure(svof3d_solver *s) {
  if (s->adj) return 0;
  if (s->prm.add_buoyancy) return fail("the adjoint needs add_buoyancy = 0 (t is not differentiated)");
  const size_t nx = s->nx, ny = s->ny, nz = s->nz;
  if (adj_xsolve_smem((int)nx) > 200 * 1024) return fail("the adjoint's x line solve needs nx <= 7800");
  Adjoint3State *a = new Adjoint3State();
  a->f32 = s->adj_f32;
  const size_t es = a->f32 ? sizeof(float) : sizeof(double);  // the intermediates
  const size_t nc = nx * ny * nz, nf = (nx - 1) * ny * nz, ncc = (nx + 2) * (ny + 2) * (nz + 2);
  bool bad = dalloc(a->ux, nf) || dalloc(a->uy, nc) || dalloc(a->uz, nc) || dalloc(a->p, nc) ||
             dalloc(a->vof[0], nc) || dalloc(a->vof[1], nc) || dalloc(a->pend_v[0], nc) ||
             dalloc(a->pend_v[1], nc) || dalloc(a->pend_x, nf, es) || dalloc(a->pend_y, nc, es) ||
             dalloc(a->pend_z, nc, es) || dalloc(a->sa_x, nf, es) || dalloc(a->sg_x, nf, es) ||
             dalloc(a->sa_y, nc, es) || dalloc(a->sg_y, nc, es) || dalloc(a->sa_z, nc, es) ||
             dalloc(a->sg_z, nc, es) || dalloc(a->ifx, nf, es) || dalloc(a->ify, nc, es) || dalloc(a->ifz, nc, es) ||
             dalloc(a->kap, nc, es) || dalloc(a->m, 3 * nc, es) || dalloc(a->nrm, 4 * nc, es) ||
             dalloc(a->sig, nc) || dalloc(a->psib, nc) || dalloc(a->b, nc) || dalloc(a->psis, ncc) ||
             dalloc(a->gbar, 3 * (nx + 1) * ny * nz, es) || dalloc(a->grv, nc) || dalloc(a->sum, 1);
  if (!bad && a->f32) bad = dalloc(a->zx, nf) || dalloc(a->zy, nc) || dalloc(a->zz, nc);
  if (!bad && s->mixed)
    bad = dalloc(a->nrm64, 4 * nx * (ny + 2) * (nz + 2)) || dalloc(a->curv64, ncc) ||
          (s->dc && cudaSuccess != pois_prepare<double>(s->log2ny, s->log2nz));
  a->xs_smem = adj_xsolve_smem((int)nx);
  // (FP32 intermediates take the floor too: the exact transposes carry values
  // up to ~1e9 at corners of round-off gradients, beyond FP32's resolution)
  a->tau = s->adj_tau >= 0. ? s->adj_tau : ((s->mixed || a->f32) ? kAdjMixedTau : 0.);
  if (!bad && (cudaSuccess != adj3_xsolve_prepare<double>(a->xs_smem) ||
               cudaSuccess != adj3_xsolve_prepare<float>(a->xs_smem)))
    bad = fail("cudaFuncSetAttribute(k3_adj_xsolve)");
  if (!bad) {
    // reciprocal spacings from the device tables
    std::vector<double> h(nx + 1);
    bad = cudaSuccess != cudaMemcpy(h.data(), s->dxf.p, sizeof(double) * nx, cudaMemcpyDeviceToHost);
    for (size_t q = 0; !bad && q < nx; q++) h[q] = 1. / h[q];
    bad = bad || upload(a->rxf, std::vector<double>(h.begin(), h.begin() + nx));
    bad = bad || cudaSuccess != cudaMemcpy(h.data(), s->dxc.p, sizeof(double) * (nx + 1), cudaMemcpyDeviceToHost);
    for (size_t q = 0; !bad && q <= nx; q++) h[q] = 1. / h[q];
    bad = bad || upload(a->rxc, h);
    if (bad && g_err3.empty()) fail("adjoint set-up: spacing tables");
  }
  if (bad) {
    std::string e = g_err3;
    s->adj = a;
    adjoint3_free(s);
    g_err3 = e.empty() ? "adjoint set-up failed" : e;
    return 1;
  }
  s->adj = a;
  return 0;
}

dim3 adj3_cells(const svof3d_solver *s) { return dim3((s->nx + 31) / 32, (s->ny + 7) / 8, s->nz); }

AGrid3 agrid(const svof3d_solver *s) {
  return AGrid3{s->grid(), s->adj->rxf.p, s->adj->rxc.p, 1. / s->dy, 1. / s->dz, s->adj->tau};
}

// the geometry the interface transposes read: the solver's own (FP64 path)
// or, on the mixed paths, an FP64 recomputation from vof into the adjoint's
// buffers (adj3_geometry recomputes it from vof)
double *adj3_normal(svof3d_solver *s) { return s->mixed ? s->adj->nrm64.p : s->normal.p; }
double *adj3_curv(svof3d_solver *s) { return s->mixed ? s->adj->curv64.p : s->curv.p; }
int adj3_geometry(svof3d_solver *s, const double *vof) {
  CK(interface_geom<double>(s->stream, vof, adj3_normal(s), adj3_curv(s), s->d_work, s->d_nwork, s->grid()));
  return 0;
}

int adj3_set_dt(svof3d_solver *s, double dt) {
  k3_adj_set<<<1, 1, 0, s->stream>>>(s->d_dt, dt);
  CK_LAUNCH();
  return 0;
}

// fluid_update_pressure (mode 1) and fluid_correct_velocity (mode 2)
int adj3_project(svof3d_solver *s, int rk, double dt, int mode) {
  Adjoint3State *a = s->adj;
  const double gam = RK_A[rk] + RK_B[rk];
  k3_adj_project<<<adj3_cells(s), dim3(32, 8), 0, s->stream>>>(a->ux.p, a->uy.p, a->uz.p, a->p.p, a->psib.p,
                                                               gam * dt, 0.5 * gam * dt * s->prm.m_dif, mode,
                                                               agrid(s));
  CK_LAUNCH();
  return 0;
}

// fluid_compute_potential_dft: s = the forward solve of psi_bar / dxf, then
// the divergence's transpose of pre_p dxf s (the Poisson operator is dxf^-1
// times a symmetric matrix, so its inverse's transpose is dxf L^-1 dxf^-1)
int adj3_potential(svof3d_solver *s, int rk, double dt) {
  Adjoint3State *a = s->adj;
  const double gam = RK_A[rk] + RK_B[rk];
  const Grid3 g = s->grid();
  k3_adj_scale<<<adj3_cells(s), dim3(32, 8), 0, s->stream>>>(a->psib.p, a->b.p, agrid(s));
  CK_LAUNCH();
  CK(pois_fwd_y_array<double>(s->stream, a->b.p, s->spec.p, s->twf_y.p, s->log2ny, g));
  CK(pois_z<double>(s->stream, s->spec.p, s->twf_z.p, s->log2nz, g));
  CK(pois_x<double>(s->stream, s->spec.p, s->xscratch.p, s->pl.p, s->pu.p, s->evy.p, s->evz.p, g, false));
  CK(pois_z<double>(s->stream, s->spec.p, s->twb_z.p, s->log2nz, g));
  CK(pois_inv_y<double>(s->stream, s->spec.p, a->psis.p, s->twb_y.p, s->log2ny, g, false));
  const double pre_p = 1. / (gam * dt) / (1. * s->ny * s->nz);
  k3_adj_div<<<adj3_cells(s), dim3(32, 8), 0, s->stream>>>(a->ux.p, a->uy.p, a->uz.p, a->psis.p, a->psib.p, pre_p,
                                                           agrid(s));
  CK_LAUNCH();
  return 0;
}

// fluid_predict_field about the primal velocities and the vof after the
// substep's advection (storage layouts); d_dt must hold dt.  S: the
// storage type of the adjoint's intermediates
template <class S>
int adj3_predict_t(svof3d_solver *s, int rk, double dt, const double *ux, const double *uy, const double *uz,
                   const double *vof_post) {
  Adjoint3State *a = s->adj;
  k3_tdm_coef<<<1, 128, sizeof(double) * 6 * s->nx, s->stream>>>(s->lap_ux.p, s->lap_cc.p, s->d_dt,
                                                                 RK_A[rk] + RK_B[rk], s->prm.m_dif, s->prm.t_dif,
                                                                 s->nx, s->coef.p);
  CK_LAUNCH();
  const long lines = (long)s->ny * s->nz;
  // the forward sweep's values: src_g_bar itself (FP64 intermediates) or the FP64 scratch
  double *zx = a->f32 ? a->zx.p : a->sg_x.p, *zy = a->f32 ? a->zy.p : a->sg_y.p;
  double *zz = a->f32 ? a->zz.p : a->sg_z.p;
  CK(adj3_xsolve_launch<S>(s->stream, lines, a->xs_smem, a->ux.p, a->uy.p, a->uz.p, s->coef.p, a->sa_x.as<S>(),
                            a->sg_x.as<S>(), a->sa_y.as<S>(), a->sg_y.as<S>(), a->sa_z.as<S>(), a->sg_z.as<S>(),
                            a->pend_x.as<S>(), a->pend_y.as<S>(), a->pend_z.as<S>(), zx, zy, zz, RK_A[rk] * dt,
                            RK_B[rk] * dt, (RK_A[rk] + RK_B[rk]) * dt, s->grid()));
  Adj3RhsArgs<S> r{};
  r.ux = ux;
  r.uy = uy;
  r.uz = uz;
  r.sa_x = a->sa_x.as<S>();
  r.sg_x = a->sg_x.as<S>();
  r.sa_y = a->sa_y.as<S>();
  r.sg_y = a->sg_y.as<S>();
  r.sa_z = a->sa_z.as<S>();
  r.sg_z = a->sg_z.as<S>();
  r.aux = a->ux.p;
  r.auy = a->uy.p;
  r.auz = a->uz.p;
  r.ap = a->p.p;
  r.aifx = a->ifx.as<S>();
  r.aify = a->ify.as<S>();
  r.aifz = a->ifz.as<S>();
  r.lap_ux = s->lap_ux.p;
  r.lap_cc = s->lap_cc.p;
  r.m_dif = s->prm.m_dif;
  r.ly0 = s->lapy[0];
  r.ly1 = s->lapy[1];
  r.ly2 = s->lapy[2];
  r.lz0 = s->lapz[0];
  r.lz1 = s->lapz[1];
  r.lz2 = s->lapz[2];
  r.grav_vof = s->grav_vof;
  r.vof_ref = s->vof_ref;
  r.vof_post = vof_post;
  r.avof = a->vof[a->cv].p;
  r.agrv = a->grv.p;
  r.ag = agrid(s);
  CK(adj3_rhs_launch<S>(s->stream, r));
  return 0;
}
int adj3_predict(svof3d_solver *s, int rk, double dt, const double *ux, const double *uy, const double *uz,
                 const double *vof_post) {
  return s->adj->f32 ? adj3_predict_t<float>(s, rk, dt, ux, uy, uz, vof_post)
                     : adj3_predict_t<double>(s, rk, dt, ux, uy, uz, vof_post);
}

// interface_update_vof (mode 1), interface_compute_force (2), the intercept
// and normal part of interface_compute_curvature_tensor (4), about the primal
// velocities and vof (storage layouts) and the solver's normal and curv
template <class S>
int adj3_interface_t(svof3d_solver *s, int rk, double dt, int mode, const double *ux, const double *uy,
                     const double *uz, const double *vof) {
  Adjoint3State *a = s->adj;
  Adj3IfaceArgs<S> f{};
  f.ux = ux;
  f.uy = uy;
  f.uz = uz;
  f.vof = vof;
  f.normal = adj3_normal(s);
  f.curv = adj3_curv(s);
  f.avof_in = a->vof[a->cv].p;
  f.avof_out = a->vof[1 - a->cv].p;
  f.pend_in = a->pend_v[a->cp].p;
  f.pend_out = a->pend_v[1 - a->cp].p;
  f.aux = a->ux.p;
  f.auy = a->uy.p;
  f.auz = a->uz.p;
  f.aifx = a->ifx.as<S>();
  f.aify = a->ify.as<S>();
  f.aifz = a->ifz.as<S>();
  f.anrm = a->nrm.as<S>();
  f.am = a->m.as<S>();
  f.akap = a->kap.as<S>();
  f.asig = a->sig.p;
  f.adt = RK_A[rk] * dt;
  f.bdt = RK_B[rk] * dt;
  f.tension = s->prm.tension;
  f.mode = mode;
  f.ag = agrid(s);
  CK(adj3_interface_launch<S>(s->stream, f));
  a->cv ^= 1;
  if (mode & 1) a->cp ^= 1;
  return 0;
}
int adj3_interface(svof3d_solver *s, int rk, double dt, int mode, const double *ux, const double *uy,
                   const double *uz, const double *vof) {
  return s->adj->f32 ? adj3_interface_t<float>(s, rk, dt, mode, ux, uy, uz, vof)
                     : adj3_interface_t<double>(s, rk, dt, mode, ux, uy, uz, vof);
}

// the corner normals and curvature part of interface_compute_curvature_tensor
template <class S>
int adj3_corners_t(svof3d_solver *s, const double *vof) {
  Adjoint3State *a = s->adj;
  CK(adj3_corners_launch<S>(s->stream, vof, a->m.as<S>(), a->kap.as<S>(), a->gbar.as<S>(), a->vof[a->cv].p,
                             agrid(s)));
  return 0;
}
int adj3_corners(svof3d_solver *s, const double *vof) {
  return s->adj->f32 ? adj3_corners_t<float>(s, vof) : adj3_corners_t<double>(s, vof);
}

size_t n_ux3(const svof3d_solver *s) { return (size_t)(s->nx + 1) * (s->ny + 2) * (s->nz + 2); }
size_t n_cc3(const svof3d_solver *s) { return (size_t)(s->nx + 2) * (s->ny + 2) * (s->nz + 2); }
size_t n_vof3(const svof3d_solver *s) { return (size_t)(s->nx + 2) * (s->ny + 4) * (s->nz + 4); }
// one substep's part of a tape: ux, uy, uz, vof; a tape holds three of
// them and the step's final vof
size_t tape_stride3(const svof3d_solver *s) { return n_ux3(s) + 2 * n_cc3(s) + n_vof3(s); }

int adj3_check(svof3d_solver *s) {
  if (!s) return fail("null argument");
  return adj3_ensure(s);
}


}  // namespace

extern "C" {

int svof3d_set_tension(svof3d_solver_t *s, double tension) {
  if (!s) return fail("null argument");
  CK(cudaStreamSynchronize(s->stream));
  s->prm.tension = tension;
  for (auto &kv : s->graphs) cudaGraphExecDestroy(kv.second);
  s->graphs.clear();
  return 0;
}

int svof3d_set_gravity(svof3d_solver_t *s, double grav_vof, double vof_ref) {
  if (!s) return fail("null argument");
  CK(cudaStreamSynchronize(s->stream));
  s->grav_vof = grav_vof;
  s->vof_ref = vof_ref;
  for (auto &kv : s->graphs) cudaGraphExecDestroy(kv.second);
  s->graphs.clear();
  return 0;
}

int svof3d_tape_count(const svof3d_solver_t *s, size_t *count) {
  if (!s || !count) return fail("null argument");
  *count = 3 * tape_stride3(s) + n_vof3(s);
  return 0;
}

int svof3d_integrate_fixed(svof3d_solver_t *s, double dt, double *tape) {
  SVOF_RANGE();
  if (!s) return fail("null argument");
  if (!(dt > 0.)) return fail("svof3d_integrate_fixed: dt must be positive");
  if (adj3_set_dt(s, dt)) return 1;
  const size_t nu = n_ux3(s), nc = n_cc3(s), nv = n_vof3(s), st = tape_stride3(s);
  for (int rk = 0; rk < 3; rk++) {
    if (tape) {
      double *t = tape + rk * st;
      const int cu = s->cur_u;
      CK(cudaMemcpyAsync(t, s->ux[cu].p, sizeof(double) * nu, cudaMemcpyDeviceToDevice, s->stream));
      CK(cudaMemcpyAsync(t + nu, s->uy[cu].p, sizeof(double) * nc, cudaMemcpyDeviceToDevice, s->stream));
      CK(cudaMemcpyAsync(t + nu + nc, s->uz[cu].p, sizeof(double) * nc, cudaMemcpyDeviceToDevice, s->stream));
      CK(cudaMemcpyAsync(t + nu + 2 * nc, s->vof[s->cur_v].p, sizeof(double) * nv, cudaMemcpyDeviceToDevice,
                         s->stream));
    }
    if (launch_geom(s) || launch_force(s) || launch_vof(s, rk) || launch_predict(s, rk) ||
        launch_potential(s, rk) || launch_project(s, rk, 1, 1))
      return 1;
  }
  if (tape)
    CK(cudaMemcpyAsync(tape + 3 * st, s->vof[s->cur_v].p, sizeof(double) * nv, cudaMemcpyDeviceToDevice,
                       s->stream));
  return 0;
}

int svof3d_adjoint_field(svof3d_solver_t *s, int which, double **dptr, size_t *count) {
  if (!s || !dptr) return fail("null argument");
  if (adj3_ensure(s)) return 1;
  Adjoint3State *a = s->adj;
  const size_t nc = (size_t)s->nx * s->ny * s->nz, nf = (size_t)(s->nx - 1) * s->ny * s->nz;
  DevBuf *b = nullptr;
  size_t n = nc;
  switch (which) {
    case SVOF3_ADJ_UX: b = &a->ux; n = nf; break;
    case SVOF3_ADJ_UY: b = &a->uy; break;
    case SVOF3_ADJ_UZ: b = &a->uz; break;
    case SVOF3_ADJ_P: b = &a->p; break;
    case SVOF3_ADJ_VOF: b = &a->vof[a->cv]; break;
    case SVOF3_ADJ_PSI: b = &a->psib; break;
    case SVOF3_ADJ_IFRCX: b = &a->ifx; n = nf; break;
    case SVOF3_ADJ_IFRCY: b = &a->ify; break;
    case SVOF3_ADJ_IFRCZ: b = &a->ifz; break;
    case SVOF3_ADJ_CURV: b = &a->kap; break;
    case SVOF3_ADJ_NORMAL: b = &a->nrm; n = 4 * nc; break;
    case SVOF3_ADJ_SRCUX_A: b = &a->pend_x; n = nf; break;
    case SVOF3_ADJ_SRCUY_A: b = &a->pend_y; break;
    case SVOF3_ADJ_SRCUZ_A: b = &a->pend_z; break;
    case SVOF3_ADJ_SRC_A: b = &a->pend_v[a->cp]; break;
    case SVOF3_ADJ_TENSION: b = &a->sig; break;
    case SVOF3_ADJ_GRAVITY: b = &a->grv; break;
    default: return fail("unknown adjoint field %d", which);
  }
  if (b->es != sizeof(double))
    return fail("svof3d_adjoint_field: field %d holds the FP32 adjoint's intermediates (svof3d_adjoint_set_precision)",
                which);
  *dptr = b->p;
  if (count) *count = n;
  return 0;
}

int svof3d_adjoint_set_gradient_floor(svof3d_solver_t *s, double tau) {
  if (adj3_check(s)) return 1;
  if (!(tau >= 0.)) return fail("svof3d_adjoint_set_gradient_floor: tau must be non-negative");
  s->adj_tau = tau;
  s->adj->tau = tau;
  return 0;
}

int svof3d_adjoint_set_precision(svof3d_solver_t *s, int fp32) {
  if (!s) return fail("null argument");
  const bool f = 0 != fp32;
  if (s->adj && s->adj->f32 != f) {
    // the buffers are made again, in the other type, on the next adjoint call
    CK(cudaStreamSynchronize(s->stream));
    adjoint3_free(s);
  }
  s->adj_f32 = f;
  return 0;
}

int svof3d_adjoint_reset(svof3d_solver_t *s) {
  if (adj3_check(s)) return 1;
  for (int q = 0; DevBuf *b = s->adj->all(q); q++) CK(cudaMemsetAsync(b->p, 0, b->es * b->n, s->stream));
  return 0;
}

int svof3d_adjoint_step(svof3d_solver_t *s, const double *tape, double dt) {
  SVOF_RANGE();
  if (adj3_check(s)) return 1;
  if (!tape) return fail("svof3d_adjoint_step: null tape");
  if (!(dt > 0.)) return fail("svof3d_adjoint_step: dt must be positive");
  Adjoint3State *a = s->adj;
  const size_t nu = n_ux3(s), nc = n_cc3(s), st = tape_stride3(s);
  // no substep follows the last one: its sources' pending adjoints are zero
  DevBuf *pend[] = {&a->pend_x, &a->pend_y, &a->pend_z, &a->pend_v[a->cp]};
  for (DevBuf *b : pend) CK(cudaMemsetAsync(b->p, 0, b->es * b->n, s->stream));
  if (adj3_set_dt(s, dt)) return 1;
  for (int rk = 2; rk >= 0; rk--) {
    const double *ux = tape + rk * st, *uy = ux + nu, *uz = uy + nc, *vof = uz + nc;
    const double *vof_post = tape + (rk + 1) * st + (rk < 2 ? nu + 2 * nc : 0);
    // the substep's geometry (normals, intercepts, curvature) from its vof
    if (adj3_geometry(s, vof)) return 1;
    if (adj3_project(s, rk, dt, 3) || adj3_potential(s, rk, dt) || adj3_predict(s, rk, dt, ux, uy, uz, vof_post) ||
        adj3_interface(s, rk, dt, 7, ux, uy, uz, vof) || adj3_corners(s, vof))
      return 1;
  }
  return 0;
}

#define ADJ3_PRIMAL s->ux[s->cur_u].p, s->uy[s->cur_u].p, s->uz[s->cur_u].p

int svof3d_adjoint_fluid_update_pressure(svof3d_solver_t *s, size_t rk, double dt) {
  SVOF_RANGE();
  if (adj3_check(s) || check_rk(rk)) return 1;
  return adj3_project(s, (int)rk, dt, 1) || finish(s);
}

int svof3d_adjoint_fluid_correct_velocity(svof3d_solver_t *s, size_t rk, double dt) {
  SVOF_RANGE();
  if (adj3_check(s) || check_rk(rk)) return 1;
  return adj3_project(s, (int)rk, dt, 2) || finish(s);
}

int svof3d_adjoint_fluid_compute_potential_dft(svof3d_solver_t *s, size_t rk, double dt) {
  SVOF_RANGE();
  if (adj3_check(s) || check_rk(rk)) return 1;
  return adj3_potential(s, (int)rk, dt) || finish(s);
}

int svof3d_adjoint_fluid_predict_field(svof3d_solver_t *s, size_t rk, double dt) {
  SVOF_RANGE();
  if (adj3_check(s) || check_rk(rk)) return 1;
  return adj3_set_dt(s, dt) || adj3_predict(s, (int)rk, dt, ADJ3_PRIMAL, s->vof[s->cur_v].p) || finish(s);
}

int svof3d_adjoint_interface_update_vof(svof3d_solver_t *s, size_t rk, double dt) {
  SVOF_RANGE();
  if (adj3_check(s) || check_rk(rk)) return 1;
  const double *vof = s->vof[s->cur_v].p;
  return (s->mixed && adj3_geometry(s, vof)) || adj3_interface(s, (int)rk, dt, 1, ADJ3_PRIMAL, vof) || finish(s);
}

int svof3d_adjoint_interface_compute_force(svof3d_solver_t *s) {
  SVOF_RANGE();
  if (adj3_check(s)) return 1;
  const double *vof = s->vof[s->cur_v].p;
  return (s->mixed && adj3_geometry(s, vof)) || adj3_interface(s, 0, 0., 2, ADJ3_PRIMAL, vof) || finish(s);
}

int svof3d_adjoint_interface_compute_curvature_tensor(svof3d_solver_t *s) {
  SVOF_RANGE();
  if (adj3_check(s)) return 1;
  const double *vof = s->vof[s->cur_v].p;
  return (s->mixed && adj3_geometry(s, vof)) || adj3_interface(s, 0, 0., 4, ADJ3_PRIMAL, vof) ||
         adj3_corners(s, vof) || finish(s);
}

#undef ADJ3_PRIMAL

// the deterministic sum of a per-cell accumulator, copied to the host
static int adj3_total(svof3d_solver *s, const DevBuf &b, double *out) {
  Adjoint3State *a = s->adj;
  k3_adj_sum<<<1, 256, 0, s->stream>>>(b.p, (long)b.n, a->sum.p);
  CK_LAUNCH();
  CK(cudaMemcpyAsync(out, a->sum.p, sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return 0;
}

int svof3d_adjoint_tension(svof3d_solver_t *s, double *out) {
  if (adj3_check(s)) return 1;
  if (!out) return fail("null argument");
  return adj3_total(s, s->adj->sig, out);
}

int svof3d_adjoint_gravity(svof3d_solver_t *s, double *out) {
  if (adj3_check(s)) return 1;
  if (!out) return fail("null argument");
  return adj3_total(s, s->adj->grv, out);
}

}  // extern "C"
