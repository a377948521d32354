// solver.cu -- host engine and C ABI (include/svof_b200.h) of the FP64 2D path.
//
// Owns the device fields (reference layouts), the grid and line-solver tables,
// the ping-pong buffers and one CUDA stream.  A full time step
// (src/integrate.c:11-68) is captured once per buffer parity into a CUDA
// graph and replayed; the only device->host traffic of a step is the 8-byte
// dt the reference's integrate() returns.
//
// Tables that the reference recomputes on every call from time-independent
// data (Laplacian coefficients, the Poisson tri-diagonal recurrences, FFT
// twiddles) are computed here once, on the host, with the reference's
// expressions, and uploaded; the values are therefore the ones the
// reference uses.
#include <cmath>
#include <cstdarg>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "guard.cuh"
#include "../../include/svof_b200.h"
#include "svof_internal.cuh"
#include "stat_internal.cuh"
#include "trace.cuh"
#include "smem_limit.cuh"
#include "fault_hook.cuh"
#include "solver_state.cuh"

using namespace svof;

namespace {

constexpr double kPi = 3.14159265358979323846;        // oracle/svof_fft.c
constexpr double kGPi = 3.14159265358979324;          // src/fluid/compute_potential/dct.c:20

int ilog2_exact(int n) {
  int l = 0;
  while ((1 << l) < n) l++;
  return ((1 << l) == n) ? l : -1;
}

// gtsv of src/tdm.c:17-50 on the host (used for the table set-up)
void host_gtsv(int n, const double *l, const double *c, const double *u, double *v, double *q) {
  v[0] = u[0] / c[0];
  q[0] = q[0] / c[0];
  for (int i = 1; i < n - 1; i++) {
    const double val = 1. / (c[i] - l[i] * v[i - 1]);
    v[i] = val * (u[i]);
    q[i] = val * (q[i] - l[i] * q[i - 1]);
  }
  const double val = c[n - 1] - l[n - 1] * v[n - 2];
  if (std::fabs(val) > kDblEpsilon) {
    q[n - 1] = 1. / val * (q[n - 1] - l[n - 1] * q[n - 2]);
  } else {
    q[n - 1] = 0.;
  }
  for (int i = n - 2; i >= 0; i--) q[i] -= v[i] * q[i + 1];
}


}  // namespace


namespace svof {

thread_local std::string g_err;

int fail(const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return 1;
}

// managed: CUDA managed memory, so that a host program holding the pointer
// (the reference's logging and save code read the fields directly) can read it
int dalloc(DevBuf &b, size_t n, bool managed) {
  if (svof_fault::next_alloc_fails()) return fail("cudaMalloc: out of memory (injected by SVOF_FAIL_ALLOC)");
  b.n = n;
  CK(svof_guard::alloc(reinterpret_cast<void **>(&b.p), sizeof(double) * (n ? n : 1), managed));
  CK(cudaMemset(b.p, 0, sizeof(double) * (n ? n : 1)));
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

// ---- launch helpers: each issues the kernels of one reference function ----


int launch_halo_bc(svof_solver *s, double *a, int field) {
  const int nx = s->nx, ny = s->ny;
  int width, nh, kind;
  double lo = 0., hi = 0.;
  switch (field) {
    case SVOF_UX: width = nx + 1; nh = 1; kind = BC_ZERO_UX; break;
    case SVOF_UY: width = nx + 2; nh = 1; kind = BC_DIRICHLET; lo = s->prm.uy_xm; hi = s->prm.uy_xp; break;
    case SVOF_T: width = nx + 2; nh = 1; kind = BC_DIRICHLET; lo = s->prm.t_xm; hi = s->prm.t_xp; break;
    case SVOF_P: case SVOF_PSI: width = nx + 2; nh = 1; kind = BC_NEUMANN; break;
    case SVOF_VOF: width = nx + 2; nh = 2; kind = BC_VOF; break;
    default: return fail("no boundary rule for field %d", field);
  }
  dim3 gr((width + 127) / 128, ny + 2 * nh);
  k_halo_bc<<<gr, 128, 0, s->stream>>>(a, width, nh, ny, kind, lo, hi);
  CK_LAUNCH();
  return 0;
}

// reads and clears the device status word (after the stream's work is
// done): a set bit is reported as a failure of `who`
int check_status(svof_solver *s, const char *who) {
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

int launch_dt(svof_solver *s) {
  const long nf = (long)(s->nx - 1) * s->ny + (long)s->nx * s->ny;
  int blocks = (int)std::min<long>((nf + 255) / 256, 148L * 8);
  CK(launch_k(s->pdl, k_cfl, blocks, 256, 0, s->stream, (const double *)s->ux[s->cur_u].p,
              (const double *)s->uy[s->cur_u].p, s->d_minbits, s->d_status, s->grid()));
  CK(launch_k(s->pdl, k_dt_final, 1, 1, 0, s->stream, s->d_minbits, s->d_dt, s->prm.coef_dt_adv, s->dif_m_y,
              s->dif_t_y, s->d_status));
  return 0;
}

int launch_geom(svof_solver *s) {
  dim3 b(32, 8), gr((s->nx + 31) / 32, (s->ny + 2 + 7) / 8);
  CK(launch_k(s->pdl, k_geom, gr, b, 0, s->stream, (const double *)s->vof[s->cur_v].p, s->normal.p, s->curv.p,
              s->grid()));
  return 0;
}

int launch_force(svof_solver *s, cudaStream_t st) {
  dim3 b(32, 8), gr((s->nx + 31) / 32, (s->ny + 7) / 8);
  CK(launch_k(s->pdl, k_force, gr, b, 0, st ? st : s->stream, (const double *)s->vof[s->cur_v].p,
              (const double *)s->curv.p, s->ifrcx.p, s->ifrcy.p, s->prm.tension, s->grid()));
  return 0;
}

int launch_vof(svof_solver *s, int rk) {
  if (0 != rk) s->sa_v ^= 1;  // reset_srcs, src/interface/update/main.c:28-45
  dim3 b(32, 8), gr((s->nx + 31) / 32, (s->ny + 7) / 8);
  RK c{RK_A[rk], RK_B[rk], RK_A[rk] + RK_B[rk]};
  CK(launch_k(s->pdl, k_vof_advect, gr, b, 0, s->stream, (const double *)s->vof[s->cur_v].p, s->vof[1 - s->cur_v].p,
              (const double *)s->ux[s->cur_u].p, (const double *)s->uy[s->cur_u].p, (const double *)s->normal.p,
              s->svof[s->sa_v].p, (const double *)s->svof[1 - s->sa_v].p, (const double *)s->d_dt, c, rk != 0,
              s->grid()));
  s->cur_v ^= 1;
  return 0;
}

double *coef_table(svof_solver *s, int rk) { return s->coef.p + (size_t)9 * s->nx * rk; }

int launch_coef(svof_solver *s, int rk, cudaStream_t st) {
  Gam3 g{{RK_A[rk] + RK_B[rk], 0., 0.}};
  CK(launch_k(s->pdl, k_tdm_coef, 1, 128, sizeof(double) * 9 * s->nx, st, (const double *)s->lap_ux.p,
              (const double *)s->lap_uy.p, (const double *)s->lap_t.p, (const double *)s->d_dt, g, s->prm.m_dif,
              s->prm.t_dif, s->nx, coef_table(s, rk)));
  return 0;
}

// the three substeps' tables at once (they need only dt), one block each
int launch_coef_all(svof_solver *s, cudaStream_t st) {
  Gam3 g{{RK_A[0] + RK_B[0], RK_A[1] + RK_B[1], RK_A[2] + RK_B[2]}};
  CK(launch_k(s->pdl, k_tdm_coef, 3, 128, sizeof(double) * 9 * s->nx, st, (const double *)s->lap_ux.p,
              (const double *)s->lap_uy.p, (const double *)s->lap_t.p, (const double *)s->d_dt, g, s->prm.m_dif,
              s->prm.t_dif, s->nx, coef_table(s, 0)));
  return 0;
}

// with_coef: launch k_tdm_coef first on the same stream (the step graph
// launches it on the side stream instead)
int launch_predict(svof_solver *s, int rk, bool with_coef) {
  if (with_coef && launch_coef(s, rk, s->stream)) return 1;
  if (0 != rk) s->sa_f ^= 1;  // reset_srcs, src/fluid/predict/main.c:9-29
  PredictArgs a{};
  const int cu = s->cur_u;
  a.ux = s->ux[cu].p;
  a.uy = s->uy[cu].p;
  a.t = s->t[cu].p;
  a.p = s->p.p;
  a.ifrcx = s->ifrcx.p;
  a.ifrcy = s->ifrcy.p;
  a.ux_new = s->ux[1 - cu].p;
  a.uy_new = s->uy[1 - cu].p;
  a.t_new = s->t[1 - cu].p;
  a.sux_a = s->sux[s->sa_f].p;
  a.suy_a = s->suy[s->sa_f].p;
  a.st_a = s->st[s->sa_f].p;
  a.sux_b = s->sux[1 - s->sa_f].p;
  a.suy_b = s->suy[1 - s->sa_f].p;
  a.st_b = s->st[1 - s->sa_f].p;
  a.lap_ux = s->lap_ux.p;
  a.lap_uy = s->lap_uy.p;
  a.lap_t = s->lap_t.p;
  a.coef = coef_table(s, rk);
  a.dtp = s->d_dt;
  a.m_dif = s->prm.m_dif;
  a.t_dif = s->prm.t_dif;
  a.lapy0 = s->lapy[0];
  a.lapy1 = s->lapy[1];
  a.lapy2 = s->lapy[2];
  a.rk = RK{RK_A[rk], RK_B[rk], RK_A[rk] + RK_B[rk]};
  a.use_b = rk != 0;
  a.add_buoyancy = s->prm.add_buoyancy;
  a.uy_xm = s->prm.uy_xm;
  a.uy_xp = s->prm.uy_xp;
  a.t_xm = s->prm.t_xm;
  a.t_xp = s->prm.t_xp;
  a.vof = s->vof[s->cur_v].p;
  a.grav_vof = s->grav_vof;
  a.vof_ref = s->vof_ref;
  a.rows_per_block = s->pred_rows;
  a.g = s->grid();
  if (s->pred_lines) {
    const dim3 tiles((s->nx + 31) / 32, (s->ny + 31) / 32);
    CK(launch_k(s->pdl, k_predict_rhs, tiles, 256, 0, s->stream, a, s->fw.p));
    CK(launch_k(s->pdl, k_predict_xsolve, 3 * ((s->ny + 31) / 32), 32, predict_xsolve_smem(s->nx), s->stream,
                (const double *)coef_table(s, rk), s->fw.p, s->nx, s->ny));
    CK(launch_k(s->pdl, k_predict_update, tiles, 256, 0, s->stream, a, (const double *)s->fw.p));
  } else {
    const int blocks = (s->ny + s->pred_rows - 1) / s->pred_rows;
    CK(launch_k(s->pdl, k_predict, blocks, s->pred_threads, s->pred_smem, s->stream, a));
  }
  s->cur_u ^= 1;
  return 0;
}

int launch_potential(svof_solver *s, int rk, int want_dct) {
  const double gam = RK_A[rk] + RK_B[rk];
  const Grid2 g = s->grid();
  if (want_dct != (int)s->uniform) {
    return fail(want_dct ? "DCT Poisson path needs a uniform x grid" : "DFT path requested on a uniform grid");
  }
  if (s->uniform) {
    const int L = s->log2fft;
    const dim3 rows_grid((s->ny + dct_rows(L) - 1) / dct_rows(L));
    CK(launch_k(s->pdl, dct_fwd_kernel(L), rows_grid, dct_threads(L), dct_smem(L, false), s->stream,
                (const double *)s->ux[s->cur_u].p, (const double *)s->uy[s->cur_u].p, s->spec.p,
                (const double *)s->twf.p, (const double *)s->cs.p, (const double *)s->d_dt, gam, g));
    const int kt = s->ysolve_kt;
    CK(launch_k(s->pdl, k_dct_ysolve, (s->nx + kt - 1) / kt, 128, sizeof(double) * 3 * kt * s->ny, s->stream,
                s->spec.p, s->vt.p, s->rvt.p, s->q1t.p, s->ck.p, s->lastf.p, s->den.p, 1. / s->dy / s->dy, s->nx,
                s->ny, kt));
    CK(launch_k(s->pdl, dct_inv_kernel(L), rows_grid, dct_threads(L), dct_smem(L, true), s->stream,
                (const double *)s->spec.p, s->psi.p, (const double *)s->twb.p, (const double *)s->cs.p, g));
  } else {
    const int cols = s->dft_cols;
    const int blocks = (s->nx + cols - 1) / cols;
    const size_t smem = sizeof(double) * 2 * s->ny * cols;
    const int nky = s->ny / 2 + 1;
    CK(launch_k(s->pdl, k_dft_fwd, blocks, 256, smem, s->stream, s->ux[s->cur_u].p, s->uy[s->cur_u].p, s->spec.p,
                s->twf.p, s->d_dt, gam, s->log2fft, cols, g));
    const int xkt = s->xsolve_kt;
    CK(launch_k(s->pdl, k_dft_xsolve, (nky + xkt - 1) / xkt, 128, sizeof(double) * 4 * xkt * s->nx, s->stream,
                s->spec.p, s->vt.p, s->rvt.p, s->pl.p, s->pu.p, s->evals.p, s->nx, nky, xkt));
    CK(launch_k(s->pdl, k_dft_inv, blocks, 256, smem, s->stream, s->spec.p, s->psi.p, s->twb.p, s->log2fft, cols, g));
  }
  return 0;
}

int launch_project(svof_solver *s, int rk, int do_vel, int do_p) {
  dim3 b(32, 8), gr((s->nx + 31) / 32, (s->ny + 7) / 8);
  CK(launch_k(s->pdl, k_project, gr, b, 0, s->stream, s->ux[s->cur_u].p, s->uy[s->cur_u].p, s->p.p,
              (const double *)s->psi.p, (const double *)s->d_dt, RK_A[rk] + RK_B[rk], s->prm.m_dif, s->prm.uy_xm,
              s->prm.uy_xp, do_vel, do_p, s->grid()));
  return 0;
}

// the kernel sequence of integrate(), src/integrate.c:11-68
int launch_step(svof_solver *s) {
  if (launch_dt(s)) return 1;
  // the three substeps' predictor coefficients need only dt: one launch on a
  // branch of its own, beside the first substep's interface kernels (the
  // serial recurrence takes about as long as they do)
  CK(cudaEventRecord(s->ev_fork[0], s->stream));
  CK(cudaStreamWaitEvent(s->side2, s->ev_fork[0], 0));
  if (launch_coef_all(s, s->side2)) return 1;
  CK(cudaEventRecord(s->ev_coef, s->side2));
  for (int rk = 0; rk < 3; rk++) {
    if (launch_geom(s)) return 1;
    // the CSF force and the vof advection both only need the geometry: the
    // force runs beside the advection, on the side branch
    CK(cudaEventRecord(s->ev_geom[rk], s->stream));
    CK(cudaStreamWaitEvent(s->side, s->ev_geom[rk], 0));
    if (launch_force(s, s->side)) return 1;
    CK(cudaEventRecord(s->ev_join[rk], s->side));
    if (launch_vof(s, rk)) return 1;
    CK(cudaStreamWaitEvent(s->stream, s->ev_join[rk], 0));
    if (0 == rk) CK(cudaStreamWaitEvent(s->stream, s->ev_coef, 0));
    if (launch_predict(s, rk, false)) return 1;
    if (launch_potential(s, rk, s->uniform)) return 1;
    if (launch_project(s, rk, 1, 1)) return 1;
  }
  return 0;
}

int state_key(const svof_solver *s) { return s->cur_u | (s->cur_v << 1) | (s->sa_f << 2) | (s->sa_v << 3); }

int step_graph(svof_solver *s, cudaGraphExec_t *exec) {
  const int key = state_key(s);
  auto it = s->graphs.find(key);
  if (it != s->graphs.end()) {
    *exec = it->second;
    // advance the host-side buffer state as the captured step does: three
    // field swaps per step (odd), two source swaps (even)
    s->cur_u ^= 1;
    s->cur_v ^= 1;
    return 0;
  }
  cudaGraph_t graph;
  CK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
  // launch-bound grids only: at 128^2 and 256^2 cells a step is 3-4 % faster,
  // at 512^2 and above the attribute gains nothing
  s->pdl = (long)s->nx * s->ny <= 256L * 256L;
  const int rc = launch_step(s);
  s->pdl = false;
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

int field_buf(svof_solver *s, int field, DevBuf **b) {
  switch (field) {
    case SVOF_UX: *b = &s->ux[s->cur_u]; break;
    case SVOF_UY: *b = &s->uy[s->cur_u]; break;
    case SVOF_T: *b = &s->t[s->cur_u]; break;
    case SVOF_VOF: *b = &s->vof[s->cur_v]; break;
    case SVOF_P: *b = &s->p; break;
    case SVOF_PSI: *b = &s->psi; break;
    case SVOF_CURV: *b = &s->curv; break;
    case SVOF_NORMAL: *b = &s->normal; break;
    case SVOF_IFRCX: *b = &s->ifrcx; break;
    case SVOF_IFRCY: *b = &s->ifrcy; break;
    case SVOF_SRCUX_A: *b = &s->sux[s->sa_f]; break;
    case SVOF_SRCUX_B: *b = &s->sux[1 - s->sa_f]; break;
    case SVOF_SRCUY_A: *b = &s->suy[s->sa_f]; break;
    case SVOF_SRCUY_B: *b = &s->suy[1 - s->sa_f]; break;
    case SVOF_SRCT_A: *b = &s->st[s->sa_f]; break;
    case SVOF_SRCT_B: *b = &s->st[1 - s->sa_f]; break;
    case SVOF_SRC_A: *b = &s->svof[s->sa_v]; break;
    case SVOF_SRC_B: *b = &s->svof[1 - s->sa_v]; break;
    default: return fail("unknown field id %d", field);
  }
  return 0;
}

// number of halo rows and row width of the restart-file fields
int interior_layout(const svof_solver *s, int field, int *nh, int *width) {
  switch (field) {
    case SVOF_UX: *nh = 1; *width = s->nx + 1; return 0;
    case SVOF_UY: case SVOF_P: case SVOF_T: case SVOF_PSI: *nh = 1; *width = s->nx + 2; return 0;
    case SVOF_VOF: *nh = 2; *width = s->nx + 2; return 0;
    default: return fail("field %d has no restart-file layout", field);
  }
}

int build_tables(svof_solver *s, const double *xf, const double *xc) {
  const int nx = s->nx, ny = s->ny;
  s->xf.assign(xf, xf + nx + 1);
  s->xc.assign(xc, xc + nx + 2);
  // src/domain.c:107-143, :190-192, :75-98
  std::vector<double> dxf(nx), dxc(nx + 1);
  for (int i = 1; i <= nx; i++) dxf[i - 1] = xf[i] - xf[i - 1];
  for (int i = 1; i <= nx + 1; i++) dxc[i - 1] = xc[i] - xc[i - 1];
  s->dxf_h = dxf;
  s->dxc_h = dxc;
  s->dy = s->prm.ly / ny;
  {
    double mn = +1. * 1.7976931348623157e308, mx = -1. * 1.7976931348623157e308;
    for (int i = 0; i < nx; i++) {
      mn = std::fmin(mn, dxf[i]);
      mx = std::fmax(mx, dxf[i]);
    }
    s->uniform = std::fabs(mx - mn) < 1.e-15;
  }
  if (upload(s->dxf, dxf) || upload(s->dxc, dxc)) return 1;
  auto DXF = [&](int i) { return dxf[i - 1]; };
  auto DXC = [&](int i) { return dxc[i - 1]; };
  // Laplacians, src/fluid/predict/{ux,uy,t}.c init_lap
  std::vector<double> lux(3 * (nx - 1)), luy(3 * nx);
  for (int i = 2; i <= nx; i++) {
    const double l = 1. / DXF(i - 1) / DXC(i);
    const double u = 1. / DXF(i) / DXC(i);
    const double c = -l - u;
    lux[3 * (i - 2) + 0] = l;
    lux[3 * (i - 2) + 1] = c;
    lux[3 * (i - 2) + 2] = u;
  }
  for (int i = 1; i <= nx; i++) {
    const double l = 1. / DXC(i) / DXF(i);
    const double u = 1. / DXC(i + 1) / DXF(i);
    const double c = -l - u;
    luy[3 * (i - 1) + 0] = l;
    luy[3 * (i - 1) + 1] = c;
    luy[3 * (i - 1) + 2] = u;
  }
  if (upload(s->lap_ux, lux) || upload(s->lap_uy, luy) || upload(s->lap_t, luy)) return 1;
  s->lapy[0] = +1. / s->dy / s->dy;
  s->lapy[1] = -2. / s->dy / s->dy;
  s->lapy[2] = +1. / s->dy / s->dy;
  // decide_dt_dif y limits, src/fluid/decide_dt.c:73-94
  const int ndims = 2;
  s->dif_m_y = s->prm.coef_dt_dif / s->prm.m_dif * 0.5 / ndims * std::pow(s->dy, 2.);
  s->dif_t_y = s->prm.coef_dt_dif / s->prm.t_dif * 0.5 / ndims * std::pow(s->dy, 2.);
  // FFT twiddles (oracle/svof_fft.c svof_fft_twiddles / svof_dct_twiddles)
  const int nfft = s->uniform ? nx : ny;
  s->log2fft = ilog2_exact(nfft);
  if (s->log2fft < 1) {
    return fail("the %s direction needs a power-of-two size (got %d)", s->uniform ? "x" : "y", nfft);
  }
  {
    std::vector<double> twf(2 * (nfft / 2)), twb(2 * (nfft / 2)), cs(2 * nfft);
    for (int m = 0; m < nfft / 2; m++) {
      const double ang = 2.0 * kPi * (double)m / (double)nfft;
      twf[2 * m] = std::cos(ang);
      twf[2 * m + 1] = -std::sin(ang);
      twb[2 * m] = std::cos(ang);
      twb[2 * m + 1] = std::sin(ang);
    }
    for (int k = 0; k < nfft; k++) {
      const double ang = kPi * (double)k / (2.0 * (double)nfft);
      cs[2 * k] = std::cos(ang);
      cs[2 * k + 1] = std::sin(ang);
    }
    if (upload(s->twf, twf) || upload(s->twb, twb) || upload(s->cs, cs)) return 1;
  }
  if (s->uniform) {
    // src/fluid/compute_potential/dct.c:142-178 and :233-261
    const int n = ny;
    const double lap = 1. / s->dy / s->dy;
    std::vector<double> l(n, lap), u(n, lap), c(n), v(n), q1(n);
    std::vector<double> vt((size_t)n * nx, 0.), rvt((size_t)n * nx, 0.), q1t((size_t)n * nx, 0.), ck(nx),
        den(nx), lastf(nx);
    const double signal_length = 2. * nx;
    const double gridsize = s->prm.lx / nx;
    for (size_t k = 0; k < (size_t)nx; k++) {
      const double ev = -4. / std::pow(gridsize, 2.) * std::pow(std::sin(kGPi * k / signal_length), 2.);
      for (int r = 0; r < n; r++) c[r] = -l[r] - u[r] + ev;
      for (int i = 0; i < n - 1; i++) q1[i] = i == 0 ? -l[i] : i == n - 2 ? -u[i] : 0.;
      host_gtsv(n - 1, l.data(), c.data(), u.data(), v.data(), q1.data());
      for (int i = 0; i < n - 1; i++) {
        vt[(size_t)i * nx + k] = v[i];
        q1t[(size_t)i * nx + k] = q1[i];
      }
      // gtsv's val of the size-(n-1) system, rows 1 .. n-3, and its last row
      for (int i = 1; i < n - 2; i++) rvt[(size_t)i * nx + k] = 1. / (c[i] - l[i] * v[i - 1]);
      {
        const double val = c[n - 2] - l[n - 2] * v[n - 3];
        lastf[k] = std::fabs(val) > kDblEpsilon ? 1. / val : 0.;
      }
      ck[k] = c[0];
      den[k] = c[n - 1] + u[n - 1] * q1[0] + l[n - 1] * q1[n - 2];
    }
    if (upload(s->vt, vt) || upload(s->rvt, rvt) || upload(s->q1t, q1t) || upload(s->ck, ck) ||
        upload(s->den, den) || upload(s->lastf, lastf))
      return 1;
    if (dalloc(s->spec, (size_t)nx * ny)) return 1;
  } else {
    // src/fluid/compute_potential/dft.c:142-198 and :263-291
    const int n = nx, nky = ny / 2 + 1;
    std::vector<double> pl(n), pu(n), ev(nky), c(n), v(n), vt((size_t)n * nky, 0.), rvt((size_t)n * nky, 0.);
    for (int i = 1; i <= n; i++) {
      pl[i - 1] = 1. / DXC(i) / DXF(i);
      pu[i - 1] = 1. / DXC(i + 1) / DXF(i);
    }
    const double signal_length = (double)ny;
    const double gridsize = s->prm.ly / ny;
    for (size_t j = 0; j < (size_t)nky; j++) {
      ev[j] = -4. / std::pow(gridsize, 2.) * std::pow(std::sin(kGPi * j / signal_length), 2.);
    }
    for (int k = 0; k < nky; k++) {
      for (int i = 0; i < n; i++) c[i] = -pl[i] - pu[i] + ev[k];
      c[0] += pl[0];
      c[n - 1] += pu[n - 1];
      v[0] = pu[0] / c[0];
      for (int i = 1; i < n - 1; i++) {
        const double val = 1. / (c[i] - pl[i] * v[i - 1]);
        v[i] = val * (pu[i]);
        rvt[(size_t)i * nky + k] = val;
      }
      for (int i = 0; i < n - 1; i++) vt[(size_t)i * nky + k] = v[i];
    }
    if (upload(s->pl, pl) || upload(s->pu, pu) || upload(s->evals, ev) || upload(s->vt, vt) ||
        upload(s->rvt, rvt))
      return 1;
    if (dalloc(s->spec, 2 * (size_t)nx * nky)) return 1;
  }
  return 0;
}

}  // namespace

// =========================================================================== C ABI
extern "C" {

const char *svof_last_error(void) { return g_err.c_str(); }

int svof_create(const svof_params_t *prm, const double *xf, const double *xc, svof_solver_t **out) {
  return svof::engine_create(prm, xf, xc, false, out);
}

}  // extern "C"

namespace svof {

int engine_create(const svof_params_t *prm, const double *xf, const double *xc, bool managed,
                  svof_solver_t **out) {
  if (!prm || !xf || !xc || !out) return fail("svof_create: null argument");
  *out = nullptr;
  svof_fault::begin_creation();
  if (prm->nx < 4 || prm->ny < 4) return fail("svof_create: nx and ny must be at least 4");
  if (!(prm->m_dif > 0.) || !(prm->t_dif > 0.)) return fail("svof_create: diffusivities must be positive");
  svof_solver *s = new svof_solver();
  s->prm = *prm;
  s->managed = managed;
  const bool mg = managed;
  s->nx = prm->nx;
  s->ny = prm->ny;
  auto bail = [&]() {
    std::string e = g_err;
    svof_destroy(s);
    g_err = e;
    return 1;
  };
  if (cudaSuccess != cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking)) {
    delete s;
    return fail("svof_create: no CUDA device available (%s)", cudaGetErrorString(cudaGetLastError()));
  }
  const int nx = s->nx, ny = s->ny;
  const size_t n_ux = (size_t)(nx + 1) * (ny + 2), n_cc = (size_t)(nx + 2) * (ny + 2);
  const size_t n_vof = (size_t)(nx + 2) * (ny + 4), n_src = (size_t)nx * ny, n_srcx = (size_t)(nx - 1) * ny;
  for (int k = 0; k < 2; k++) {
    if (dalloc(s->ux[k], n_ux, mg) || dalloc(s->uy[k], n_cc, mg) || dalloc(s->t[k], n_cc, mg) ||
        dalloc(s->vof[k], n_vof, mg))
      return bail();
    if (dalloc(s->sux[k], n_srcx, mg) || dalloc(s->suy[k], n_src, mg) || dalloc(s->st[k], n_src, mg) ||
        dalloc(s->svof[k], n_src, mg))
      return bail();
  }
  if (dalloc(s->p, n_cc, mg) || dalloc(s->psi, n_cc, mg) || dalloc(s->curv, n_cc, mg) ||
      dalloc(s->normal, 3 * (size_t)nx * (ny + 2), mg) || dalloc(s->ifrcx, n_srcx, mg) ||
      dalloc(s->ifrcy, n_src, mg) || dalloc(s->diag, 16))
    return bail();
  if (build_tables(s, xf, xc)) return bail();
  if (dalloc(s->coef, 27 * (size_t)nx)) return bail();  // one table per substep
  if (cudaSuccess != cudaStreamCreateWithFlags(&s->side, cudaStreamNonBlocking)) return fail("stream"), bail();
  if (cudaSuccess != cudaStreamCreateWithFlags(&s->side2, cudaStreamNonBlocking)) return fail("stream"), bail();
  if (cudaSuccess != cudaEventCreateWithFlags(&s->ev_coef, cudaEventDisableTiming)) return fail("event"), bail();
  for (int k = 0; k < 3; k++) {
    if (cudaSuccess != cudaEventCreateWithFlags(&s->ev_fork[k], cudaEventDisableTiming) ||
        cudaSuccess != cudaEventCreateWithFlags(&s->ev_geom[k], cudaEventDisableTiming) ||
        cudaSuccess != cudaEventCreateWithFlags(&s->ev_join[k], cudaEventDisableTiming))
      return fail("event"), bail();
  }
  // predict launch shape: R rows per block, enough blocks to cover the SMs,
  // within 200 KB of shared memory
  {
    const long per_row = 3L * (nx + 1);
    const long fixed = 9L * (nx + 1);
    long r = std::max(1, std::min(8, ny / 148));
    while (r > 1 && (fixed + r * per_row) * 8 > 200L * 1024) r--;
    s->pred_rows = (int)r;
    s->pred_threads = (r <= 2) ? 128 : 256;
    s->pred_smem = predict_smem_bytes(nx, s->pred_rows);
    if (s->pred_smem > 200 * 1024) return fail("svof_create: nx = %d too large for the x line solver", nx), bail();
    if (cudaSuccess != raise_smem_limit(k_predict, s->pred_smem))
      return fail("cudaFuncSetAttribute(k_predict): %s", cudaGetErrorString(cudaGetLastError())), bail();
    const size_t coef_smem = sizeof(double) * 9 * nx;
    if (cudaSuccess != raise_smem_limit(k_tdm_coef, coef_smem)) return fail("cudaFuncSetAttribute(k_tdm_coef)"), bail();
    // grids from 512 x 512 cells take the line-streaming predictor: the
    // fused kernel's row tiles leave few lines per SM for its serial sweeps.
    // SVOF_PREDICT_LINES = 0 / 1 forces either form (tests compare them).
    s->pred_lines = (long)nx * ny >= 512L * 512L;
    if (const char *e = std::getenv("SVOF_PREDICT_LINES")) s->pred_lines = (0 != std::atoi(e));
    if (s->pred_lines) {
      if (dalloc(s->fw, 3 * (size_t)nx * 32 * ((ny + 31) / 32))) return bail();
      if (cudaSuccess != raise_smem_limit(k_predict_xsolve, predict_xsolve_smem(nx)))
        return fail("cudaFuncSetAttribute(k_predict_xsolve)"), bail();
    }
  }
  // transforms: rows (DCT) or a tile of columns (DFT) per block
  {
    if (s->uniform && !dct_length_ok(s->log2fft))
      return fail("svof_create: the DCT path takes nx = 4 .. 4096 (got %d)", nx), bail();
    if (s->uniform && cudaSuccess != dct_prepare(s->log2fft))
      return fail("cudaFuncSetAttribute(k_dct_fwd, k_dct_inv)"), bail();
    int cols = 16;
    while (cols > 1 && sizeof(double) * 2 * (size_t)ny * cols > 100 * 1024) cols >>= 1;
    s->dft_cols = cols;
    const size_t dft_smem = sizeof(double) * 2 * (size_t)ny * cols;
    if (!s->uniform && (cudaSuccess != raise_smem_limit(k_dft_fwd, dft_smem) ||
                        cudaSuccess != raise_smem_limit(k_dft_inv, dft_smem)))
      return fail("cudaFuncSetAttribute(k_dft_fwd, k_dft_inv)"), bail();
    if (!s->uniform && sizeof(double) * 2 * (size_t)ny > 200 * 1024)
      return fail("svof_create: FFT length too large for one block"), bail();
  }
  // line solves: lines per block so that there are four blocks per SM where
  // the lines allow (one block's staging overlaps the others' sweeps), within
  // 160 KB of staged shared memory
  auto pick_kt = [](int lines, size_t bytes_per_line) {
    int kt = 32;
    while (kt > 1 && lines / kt < 4 * 148) kt >>= 1;
    while (kt > 1 && bytes_per_line * kt > 160 * 1024) kt >>= 1;
    return kt;
  };
  if (s->uniform) {
    const size_t bpl = sizeof(double) * 3 * (size_t)ny;
    s->ysolve_kt = pick_kt(nx, bpl);
    const size_t sm = bpl * s->ysolve_kt;
    if (sm > 200 * 1024) return fail("svof_create: ny = %d too large for the y line solver", ny), bail();
    if (cudaSuccess != raise_smem_limit(k_dct_ysolve, sm)) return fail("cudaFuncSetAttribute(k_dct_ysolve)"), bail();
  } else {
    const size_t bpl = sizeof(double) * 4 * (size_t)nx;
    s->xsolve_kt = pick_kt(ny / 2 + 1, bpl);
    const size_t sm = bpl * s->xsolve_kt;
    if (sm > 200 * 1024) return fail("svof_create: nx = %d too large for the x line solver", nx), bail();
    if (cudaSuccess != raise_smem_limit(k_dft_xsolve, sm)) return fail("cudaFuncSetAttribute(k_dft_xsolve)"), bail();
  }
  // launch plan checks: every dynamic shared-memory size covers what the
  // kernel indexes, every line solve has a thread per line
  {
    const size_t need_pred = sizeof(double) * (3 * (size_t)s->pred_rows + 9) * (nx + 1);
    if (s->pred_smem < need_pred || s->pred_threads < 3 * s->pred_rows || s->pred_rows < 1)
      return fail("svof_create: inconsistent predictor launch plan"), bail();
    if (s->uniform && (s->ysolve_kt < 1 || s->ysolve_kt > 64 || s->ysolve_kt > 128))
      return fail("svof_create: inconsistent y line-solve launch plan"), bail();
    if (!s->uniform && (s->xsolve_kt < 1 || s->xsolve_kt > 128 || s->dft_cols < 1))
      return fail("svof_create: inconsistent x line-solve launch plan"), bail();
  }
  if (cudaSuccess != cudaMalloc(&s->d_dt, sizeof(double))) return fail("cudaMalloc dt"), bail();
  if (cudaSuccess != cudaMalloc(&s->d_minbits, sizeof(unsigned long long))) return fail("cudaMalloc"), bail();
  if (cudaSuccess != cudaMalloc(&s->d_status, sizeof(unsigned)) ||
      cudaSuccess != cudaMemset(s->d_status, 0, sizeof(unsigned)))
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
  if (cudaSuccess != cudaDeviceSynchronize()) return fail("svof_create: %s", cudaGetErrorString(cudaGetLastError())), bail();
  *out = s;
  return 0;
}

// parameters that the reference reads after allocation (We in interface_init,
// coef_dt_* on the first fluid_decide_dt); the step graphs are rebuilt
int engine_update_params(svof_solver_t *s, const svof_params_t *prm) {
  if (!s || !prm) return fail("null argument");
  if (prm->nx != s->nx || prm->ny != s->ny) return fail("engine_update_params: grid size cannot change");
  CK(cudaStreamSynchronize(s->stream));
  s->prm = *prm;
  const int ndims = 2;
  s->dif_m_y = s->prm.coef_dt_dif / s->prm.m_dif * 0.5 / ndims * std::pow(s->dy, 2.);
  s->dif_t_y = s->prm.coef_dt_dif / s->prm.t_dif * 0.5 / ndims * std::pow(s->dy, 2.);
  for (auto &kv : s->graphs) cudaGraphExecDestroy(kv.second);
  s->graphs.clear();
  return 0;
}

// halo / wall update of one field stored at `ptr` (fluid_update_boundaries_*,
// interface_update_boundaries_vof); waits for completion
int engine_apply_bc(svof_solver_t *s, int field, double *ptr) {
  if (!s || !ptr) return fail("null argument");
  if (launch_halo_bc(s, ptr, field)) return 1;
  CK(cudaStreamSynchronize(s->stream));
  return 0;
}

const svof_params_t *engine_params(const svof_solver_t *s) { return &s->prm; }

}  // namespace svof

extern "C" {

int svof_destroy(svof_solver_t *s) {
  if (!s) return 0;
  if (s->stream) cudaStreamSynchronize(s->stream);
  adjoint_free(s);
  for (auto &kv : s->graphs) cudaGraphExecDestroy(kv.second);
  s->graphs.clear();
  for (int k = 0; k < 2; k++) {
    dfree(s->ux[k]); dfree(s->uy[k]); dfree(s->t[k]); dfree(s->vof[k]);
    dfree(s->sux[k]); dfree(s->suy[k]); dfree(s->st[k]); dfree(s->svof[k]);
  }
  DevBuf *bufs[] = {&s->p, &s->psi, &s->curv, &s->normal, &s->ifrcx, &s->ifrcy, &s->dxf, &s->dxc,
                    &s->lap_ux, &s->lap_uy, &s->lap_t, &s->spec, &s->twf, &s->twb, &s->cs, &s->vt,
                    &s->rvt, &s->q1t, &s->ck, &s->lastf, &s->den, &s->pl, &s->pu, &s->evals, &s->diag,
                    &s->coef, &s->stat_part, &s->fw};
  for (DevBuf *b : bufs) dfree(*b);
  for (DevBuf &b : s->stat) dfree(b);
  if (s->d_dt) cudaFree(s->d_dt);
  if (s->d_minbits) cudaFree(s->d_minbits);
  if (s->d_status) cudaFree(s->d_status);
  if (s->h_dt) cudaFreeHost(s->h_dt);
  for (int k = 0; k < 3; k++) {
    if (s->ev_fork[k]) cudaEventDestroy(s->ev_fork[k]);
    if (s->ev_geom[k]) cudaEventDestroy(s->ev_geom[k]);
    if (s->ev_join[k]) cudaEventDestroy(s->ev_join[k]);
  }
  if (s->ev_coef) cudaEventDestroy(s->ev_coef);
  if (s->side2) cudaStreamDestroy(s->side2);
  if (s->side) cudaStreamDestroy(s->side);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
  return 0;
}

int svof_field_count(const svof_solver_t *cs, int field, size_t *count) {
  svof_solver *s = const_cast<svof_solver *>(cs);
  DevBuf *b;
  if (!s || !count) return fail("null argument");
  if (field_buf(s, field, &b)) return 1;
  *count = b->n;
  return 0;
}

int svof_upload_field(svof_solver_t *s, int field, const double *host, size_t count) {
  DevBuf *b;
  if (!s || !host) return fail("null argument");
  if (field_buf(s, field, &b)) return 1;
  if (count != b->n) return fail("field %d holds %zu doubles, got %zu", field, b->n, count);
  CK(cudaMemcpyAsync(b->p, host, sizeof(double) * count, cudaMemcpyHostToDevice, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return 0;
}

int svof_download_field(svof_solver_t *s, int field, double *host, size_t count) {
  DevBuf *b;
  if (!s || !host) return fail("null argument");
  if (field_buf(s, field, &b)) return 1;
  if (count != b->n) return fail("field %d holds %zu doubles, got %zu", field, b->n, count);
  CK(cudaMemcpyAsync(host, b->p, sizeof(double) * count, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return 0;
}

int svof_device_field(svof_solver_t *s, int field, double **dptr) {
  DevBuf *b;
  if (!s || !dptr) return fail("null argument");
  if (field_buf(s, field, &b)) return 1;
  *dptr = b->p;
  return 0;
}

int svof_load_interior(svof_solver_t *s, int field, const double *host, size_t count) {
  SVOF_RANGE();
  int nh, width;
  DevBuf *b;
  if (!s || !host) return fail("null argument");
  if (interior_layout(s, field, &nh, &width) || field_buf(s, field, &b)) return 1;
  const size_t n = (size_t)width * s->ny;
  if (count != n) return fail("field %d: restart layout holds %zu doubles, got %zu", field, n, count);
  CK(cudaMemcpyAsync(b->p + (size_t)nh * width, host, sizeof(double) * n, cudaMemcpyHostToDevice, s->stream));
  if (launch_halo_bc(s, b->p, field)) return 1;
  CK(cudaStreamSynchronize(s->stream));
  return 0;
}

int svof_store_interior(svof_solver_t *s, int field, double *host, size_t count) {
  SVOF_RANGE();
  int nh, width;
  DevBuf *b;
  if (!s || !host) return fail("null argument");
  if (interior_layout(s, field, &nh, &width) || field_buf(s, field, &b)) return 1;
  const size_t n = (size_t)width * s->ny;
  if (count != n) return fail("field %d: restart layout holds %zu doubles, got %zu", field, n, count);
  CK(cudaMemcpyAsync(host, b->p + (size_t)nh * width, sizeof(double) * n, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return 0;
}

int svof_x_grid_is_uniform(const svof_solver_t *s, int *u) {
  if (!s || !u) return fail("null argument");
  *u = s->uniform ? 1 : 0;
  return 0;
}

int svof_fluid_decide_dt(svof_solver_t *s, double *dt) {
  SVOF_RANGE();
  if (!s || !dt) return fail("null argument");
  if (launch_dt(s)) return 1;
  CK(cudaMemcpyAsync(s->h_dt, s->d_dt, sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  *dt = s->h_dt[0];
  return check_status(s, "svof_fluid_decide_dt");
}

static int set_dt(svof_solver_t *s, double dt) {
  s->h_dt[0] = dt;
  CK(cudaMemcpyAsync(s->d_dt, s->h_dt, sizeof(double), cudaMemcpyHostToDevice, s->stream));
  return 0;
}

static int check_rk(size_t rkstep) { return rkstep < 3 ? 0 : fail("rkstep %zu out of range", rkstep); }

static int finish(svof_solver_t *s) {
  CK(cudaStreamSynchronize(s->stream));
  return 0;
}

int svof_interface_compute_curvature_tensor(svof_solver_t *s) {
  SVOF_RANGE();
  if (!s) return fail("null argument");
  if (launch_geom(s)) return 1;
  return finish(s);
}

int svof_interface_compute_force(svof_solver_t *s) {
  SVOF_RANGE();
  if (!s) return fail("null argument");
  if (launch_force(s)) return 1;
  return finish(s);
}

int svof_interface_update_vof(svof_solver_t *s, size_t rk, double dt) {
  SVOF_RANGE();
  if (!s) return fail("null argument");
  if (check_rk(rk) || set_dt(s, dt) || launch_vof(s, (int)rk)) return 1;
  return finish(s);
}

int svof_fluid_predict_field(svof_solver_t *s, size_t rk, double dt) {
  SVOF_RANGE();
  if (!s) return fail("null argument");
  if (check_rk(rk) || set_dt(s, dt) || launch_predict(s, (int)rk)) return 1;
  return finish(s);
}

int svof_fluid_compute_potential_dct(svof_solver_t *s, size_t rk, double dt) {
  SVOF_RANGE();
  if (!s) return fail("null argument");
  if (check_rk(rk) || set_dt(s, dt) || launch_potential(s, (int)rk, 1)) return 1;
  return finish(s);
}

int svof_fluid_compute_potential_dft(svof_solver_t *s, size_t rk, double dt) {
  SVOF_RANGE();
  if (!s) return fail("null argument");
  if (check_rk(rk) || set_dt(s, dt) || launch_potential(s, (int)rk, 0)) return 1;
  return finish(s);
}

int svof_fluid_correct_velocity(svof_solver_t *s, size_t rk, double dt) {
  SVOF_RANGE();
  if (!s) return fail("null argument");
  if (check_rk(rk) || set_dt(s, dt) || launch_project(s, (int)rk, 1, 0)) return 1;
  return finish(s);
}

int svof_fluid_update_pressure(svof_solver_t *s, size_t rk, double dt) {
  SVOF_RANGE();
  if (!s) return fail("null argument");
  if (check_rk(rk) || set_dt(s, dt) || launch_project(s, (int)rk, 0, 1)) return 1;
  return finish(s);
}

int svof_run(svof_solver_t *s, int nsteps, double *dts) {
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
  return check_status(s, "svof_run");
}

int svof_enqueue_steps(svof_solver_t *s, int nsteps) {
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

int svof_last_dt(svof_solver_t *s, double *dt) {
  if (!s || !dt) return fail("null argument");
  CK(cudaStreamSynchronize(s->stream));
  *dt = s->h_dt[0];
  return check_status(s, "svof_last_dt");
}

int svof_integrate(svof_solver_t *s, double *dt) {
  SVOF_RANGE();
  double d = 0.;
  if (svof_run(s, 1, &d)) return 1;
  if (dt) *dt = d;
  return 0;
}

// one time step launched kernel by kernel (no graph) with CUDA events between
// the launches; ms[k] and launches[k] accumulate per kernel kind k (see
// svof_b200.h).  Advances the solution exactly as svof_integrate does.
int svof_profile_step(svof_solver_t *s, double *ms, int *launches, int nkinds) {
  SVOF_RANGE();
  if (!s || !ms || !launches || nkinds < SVOF_NKINDS) return fail("svof_profile_step: bad arguments");
  for (int k = 0; k < nkinds; k++) {
    ms[k] = 0.;
    launches[k] = 0;
  }
  std::vector<cudaEvent_t> ev;
  std::vector<int> kind;
  auto mark = [&](int k) -> int {
    cudaEvent_t e;
    CK(cudaEventCreate(&e));
    CK(cudaEventRecord(e, s->stream));
    ev.push_back(e);
    kind.push_back(k);
    return 0;
  };
  int rc = mark(-1);
  rc = rc || launch_dt(s) || mark(SVOF_K_DT);
  for (int rk = 0; rk < 3 && !rc; rk++) {
    rc = rc || launch_geom(s) || mark(SVOF_K_GEOM);
    rc = rc || launch_force(s) || mark(SVOF_K_FORCE);
    rc = rc || launch_vof(s, rk) || mark(SVOF_K_VOF);
    rc = rc || launch_predict(s, rk) || mark(SVOF_K_PREDICT);
    if (!rc) {
      const double gam = RK_A[rk] + RK_B[rk];
      const Grid2 g = s->grid();
      if (s->uniform) {
        const int L = s->log2fft;
        const dim3 rows_grid((s->ny + dct_rows(L) - 1) / dct_rows(L));
        dct_fwd_kernel(L)<<<rows_grid, dct_threads(L), dct_smem(L, false), s->stream>>>(
            s->ux[s->cur_u].p, s->uy[s->cur_u].p, s->spec.p, s->twf.p, s->cs.p, s->d_dt, gam, g);
        rc = rc || mark(SVOF_K_POISSON_FWD);
        const int kt = s->ysolve_kt;
        k_dct_ysolve<<<(s->nx + kt - 1) / kt, 128, sizeof(double) * 3 * kt * s->ny, s->stream>>>(
            s->spec.p, s->vt.p, s->rvt.p, s->q1t.p, s->ck.p, s->lastf.p, s->den.p, 1. / s->dy / s->dy, s->nx,
            s->ny, kt);
        rc = rc || mark(SVOF_K_POISSON_SOLVE);
        dct_inv_kernel(L)<<<rows_grid, dct_threads(L), dct_smem(L, true), s->stream>>>(s->spec.p, s->psi.p, s->twb.p,
                                                                                     s->cs.p, g);
        rc = rc || mark(SVOF_K_POISSON_INV);
      } else {
        const int cols = s->dft_cols;
        const int blocks = (s->nx + cols - 1) / cols;
        const size_t smem = sizeof(double) * 2 * s->ny * cols;
        const int nky = s->ny / 2 + 1;
        k_dft_fwd<<<blocks, 256, smem, s->stream>>>(s->ux[s->cur_u].p, s->uy[s->cur_u].p, s->spec.p, s->twf.p,
                                                    s->d_dt, gam, s->log2fft, cols, g);
        rc = rc || mark(SVOF_K_POISSON_FWD);
        const int xkt = s->xsolve_kt;
        k_dft_xsolve<<<(nky + xkt - 1) / xkt, 128, sizeof(double) * 4 * xkt * s->nx, s->stream>>>(
            s->spec.p, s->vt.p, s->rvt.p, s->pl.p, s->pu.p, s->evals.p, s->nx, nky, xkt);
        rc = rc || mark(SVOF_K_POISSON_SOLVE);
        k_dft_inv<<<blocks, 256, smem, s->stream>>>(s->spec.p, s->psi.p, s->twb.p, s->log2fft, cols, g);
        rc = rc || mark(SVOF_K_POISSON_INV);
      }
      rc = rc || (cudaSuccess != cudaGetLastError());
    }
    rc = rc || launch_project(s, rk, 1, 1) || mark(SVOF_K_PROJECT);
  }
  cudaError_t e = cudaStreamSynchronize(s->stream);
  if (!rc && cudaSuccess == e) {
    for (size_t q = 1; q < ev.size(); q++) {
      float t = 0.f;
      cudaEventElapsedTime(&t, ev[q - 1], ev[q]);
      ms[kind[q]] += t;
      launches[kind[q]] += SVOF_K_DT == kind[q] ? 2 : (SVOF_K_PREDICT == kind[q] ? (s->pred_lines ? 4 : 2) : 1);
    }
  }
  for (cudaEvent_t x : ev) cudaEventDestroy(x);
  if (rc) return 1;
  if (cudaSuccess != e) return fail("svof_profile_step: %s", cudaGetErrorString(e));
  return 0;
}

int svof_diagnostics(svof_solver_t *s, double *divmax, double *vofmin, double *vofmax, double *vofmean) {
  SVOF_RANGE();
  if (!s) return fail("null argument");
  k_diag<<<1, 1024, 0, s->stream>>>(s->ux[s->cur_u].p, s->uy[s->cur_u].p, s->vof[s->cur_v].p, s->diag.p,
                                    s->grid());
  CK_LAUNCH();
  double h[5];
  CK(cudaMemcpyAsync(h, s->diag.p, sizeof(h), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  if (divmax) *divmax = h[0];
  if (vofmin) *vofmin = h[1];
  if (vofmax) *vofmax = h[2];
  if (vofmean) *vofmean = h[3] / h[4];
  return 0;
}

int svof_logging_quantities(svof_solver_t *s, double *out, int nout) {
  if (!s || !out || nout < 9) return fail("svof_logging_quantities: bad arguments (nout must be >= 9)");
  k_logging<<<1, 1024, 0, s->stream>>>(s->ux[s->cur_u].p, s->uy[s->cur_u].p, s->t[s->cur_u].p, s->prm.m_dif,
                                       s->prm.t_dif, s->prm.ly, s->diag.p, s->grid());
  CK_LAUNCH();
  CK(cudaMemcpyAsync(out, s->diag.p, 9 * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return 0;
}

// x width of a statistics array (array_macros/statistics/ux1.h .. uxt.h)
static int stat_width(const svof_solver *s, int q) {
  return (SVOF_STAT_UX1 == q || SVOF_STAT_UX2 == q || SVOF_STAT_UXT == q) ? s->nx + 1 : s->nx + 2;
}

int svof_statistics_collect(svof_solver_t *s) {
  if (!s) return fail("null argument");
  if (!s->stat_part.p) {
    // all accumulators and the row-sum scratch, or none: a failed allocation
    // frees what it made, and the next collection tries again
    DevBuf made[SVOF_NSTATS + 1];
    cudaError_t e = cudaSuccess;
    for (int q = 0; q <= SVOF_NSTATS && cudaSuccess == e; q++) {
      made[q].n = q < SVOF_NSTATS ? (size_t)stat_width(s, q) * s->ny : 2 * (size_t)(s->nx + 2);
      e = cudaMalloc(&made[q].p, sizeof(double) * made[q].n);
      if (cudaSuccess == e && q < SVOF_NSTATS)
        e = cudaMemsetAsync(made[q].p, 0, sizeof(double) * made[q].n, s->stream);
    }
    if (cudaSuccess != e) {
      for (DevBuf &b : made) dfree(b);
      return fail("statistics accumulators: %s", cudaGetErrorString(e));
    }
    for (int q = 0; q < SVOF_NSTATS; q++) s->stat[q] = made[q];
    s->stat_part = made[SVOF_NSTATS];
  }
  StatArgs a{s->ux[s->cur_u].p, s->uy[s->cur_u].p, nullptr, s->t[s->cur_u].p,
             s->stat[SVOF_STAT_UX1].p, s->stat[SVOF_STAT_UX2].p, s->stat[SVOF_STAT_UY1].p,
             s->stat[SVOF_STAT_UY2].p, nullptr, nullptr, s->stat[SVOF_STAT_T1].p, s->stat[SVOF_STAT_T2].p,
             s->stat[SVOF_STAT_UXT].p, s->nx, s->ny, 1, 0};
  const dim3 b(32, 8), g((s->nx + 2 + 31) / 32, (s->ny + 7) / 8, 1);
  k_stat_collect<<<g, b, 0, s->stream>>>(a);
  CK_LAUNCH();
  s->stat_num += 1;
  return 0;
}

int svof_statistics_reset(svof_solver_t *s) {
  if (!s) return fail("null argument");
  for (DevBuf &b : s->stat)
    if (b.p) CK(cudaMemsetAsync(b.p, 0, sizeof(double) * b.n, s->stream));
  s->stat_num = 0;
  CK(cudaStreamSynchronize(s->stream));
  return 0;
}

int svof_statistics_count(svof_solver_t *s, size_t *num) {
  if (!s || !num) return fail("null argument");
  *num = s->stat_num;
  return 0;
}

int svof_statistics_reduce(svof_solver_t *s, int quantity, double *out, size_t count) {
  if (!s || !out) return fail("null argument");
  if (quantity < 0 || quantity >= SVOF_NSTATS) return fail("unknown statistics quantity %d", quantity);
  const int w = stat_width(s, quantity);
  if (count != (size_t)w) return fail("statistics quantity %d has %d columns, got %zu", quantity, w, count);
  if (!s->stat_part.p) {
    for (int i = 0; i < w; i++) out[i] = 0.;
    return 0;
  }
  double *part = s->stat_part.p, *res = s->stat_part.p + w;
  k_stat_reduce_planes<<<dim3((w + 127) / 128, 1), 128, 0, s->stream>>>(s->stat[quantity].p, w, s->ny, part);
  CK_LAUNCH();
  k_stat_reduce_final<<<(w + 127) / 128, 128, 0, s->stream>>>(part, w, 1, res);
  CK_LAUNCH();
  CK(cudaMemcpyAsync(out, res, sizeof(double) * w, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return 0;
}

int svof_statistics_field(svof_solver_t *s, int quantity, double *out, size_t count) {
  if (!s || !out) return fail("null argument");
  if (quantity < 0 || quantity >= SVOF_NSTATS) return fail("unknown statistics quantity %d", quantity);
  const size_t n = (size_t)stat_width(s, quantity) * s->ny;
  if (count != n) return fail("statistics quantity %d holds %zu values, got %zu", quantity, n, count);
  if (!s->stat_part.p) {
    for (size_t q = 0; q < n; q++) out[q] = 0.;
    return 0;
  }
  CK(cudaMemcpyAsync(out, s->stat[quantity].p, sizeof(double) * n, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return 0;
}

int svof_synchronize(svof_solver_t *s) {
  SVOF_RANGE();
  if (!s) return fail("null argument");
  CK(cudaStreamSynchronize(s->stream));
  return check_status(s, "svof_synchronize");
}

int svof_stream(svof_solver_t *s, void **stream) {
  if (!s || !stream) return fail("null argument");
  *stream = (void *)s->stream;
  return 0;
}

}  // extern "C"
