// adjoint.cu -- the differentiation form of the 2D FP64 path (C ABI in
// include/svof_b200.h; no counterpart in the reference).
//
// A differentiated run holds the time-step sequence fixed: svof_integrate_fixed
// takes one step with a given dt and, when asked, records the primal inputs of
// its three substeps (ux, uy, vof, storage layouts) and its final vof on a
// tape in device memory.  svof_adjoint_step maps the adjoint of a step's
// outputs (ux, uy, p, vof) to the adjoint of its inputs in place, and
// accumulates the adjoints of the surface-tension coefficient 1/We and of the
// vof buoyancy coefficient; per substep, in reverse: the projection and
// pressure update, the Poisson solve (a second solve with the x grid's metric
// weights), the implicit-x line solves, the momentum right-hand sides, the
// vof fluxes and update, the CSF force, the intercept
// and normals (k_adjoint.cu).  The per-function entry points expose the same
// pieces one by one, each reading the primal state from the solver's current
// fields, for tests and for callers that drive the reference's functions
// themselves.  The temperature is not differentiated (the adjoint requires
// add_buoyancy == 0, so that u and vof do not depend on t).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>

#include "../../include/svof_b200.h"
#include "adjoint_internal.cuh"
#include "trace.cuh"
#include "smem_limit.cuh"
#include "solver_state.cuh"

namespace svof {

struct AdjointState {
  // adjoint fields (compact: ux faces [ny][nx-1], cells [ny][nx])
  DevBuf ux, uy, p, vof[2], pend_v[2];
  DevBuf pend_x, pend_y, sa_x, sg_x, sa_y, sg_y, ifx, ify, kap, m, nrm, sig, grv, psib, psis, sum;
  int cv = 0;  // current buffer of vof_bar
  int cp = 0;  // current buffer of the vof source's pending adjoint
  int xs_rows = 1;
  size_t xs_smem = 0;
};

namespace {

int adj_ensure(svof_solver *s) {
  if (s->adj) return 0;
  if (s->prm.add_buoyancy) return fail("the adjoint needs add_buoyancy = 0 (t is not differentiated)");
  const int nx = s->nx, ny = s->ny;
  if (sizeof(double) * 2 * (size_t)nx > 200 * 1024) return fail("the adjoint's x line solve needs nx <= 12800");
  AdjointState *a = new AdjointState();
  const size_t nc = (size_t)nx * ny, nf = (size_t)(nx - 1) * ny;
  const size_t ncc = (size_t)(nx + 2) * (ny + 2);
  bool bad = dalloc(a->ux, nf) || dalloc(a->uy, nc) || dalloc(a->p, nc) || dalloc(a->vof[0], nc) ||
             dalloc(a->vof[1], nc) || dalloc(a->pend_v[0], nc) || dalloc(a->pend_v[1], nc) ||
             dalloc(a->pend_x, nf) || dalloc(a->pend_y, nc) || dalloc(a->sa_x, nf) || dalloc(a->sg_x, nf) ||
             dalloc(a->sa_y, nc) || dalloc(a->sg_y, nc) || dalloc(a->ifx, nf) || dalloc(a->ify, nc) ||
             dalloc(a->kap, nc) || dalloc(a->m, 2 * nc) || dalloc(a->nrm, 3 * nc) || dalloc(a->sig, nc) ||
             dalloc(a->grv, nc) || dalloc(a->psib, nc) || dalloc(a->psis, ncc) || dalloc(a->sum, 1);
  // transposed line solves: R rows per block so that the blocks cover the SMs,
  // within 160 KB of staged rows
  int r = std::max(1, std::min(8, ny / 148));
  while (r > 1 && sizeof(double) * 2 * (size_t)r * nx > 160 * 1024) r--;

  a->xs_rows = r;
  a->xs_smem = sizeof(double) * 2 * (size_t)r * nx;
  if (!bad && cudaSuccess != raise_smem_limit(k_adj_xsolve, a->xs_smem)) bad = true;
  // the forward transforms on an array right-hand side share the forward's shapes
  if (!bad && s->uniform && cudaSuccess != dct_prepare(s->log2fft)) bad = true;
  if (!bad && !s->uniform &&
      cudaSuccess != raise_smem_limit(k_dft_fwd_rhs, sizeof(double) * 2 * (size_t)ny * s->dft_cols))
    bad = true;
  if (bad) {
    std::string e = g_err;
    DevBuf *bufs[] = {&a->ux, &a->uy, &a->p, &a->vof[0], &a->vof[1], &a->pend_v[0], &a->pend_v[1],
                      &a->pend_x, &a->pend_y, &a->sa_x, &a->sg_x, &a->sa_y, &a->sg_y, &a->ifx, &a->ify,
                      &a->kap, &a->m, &a->nrm, &a->sig, &a->grv, &a->psib, &a->psis, &a->sum};
    for (DevBuf *b : bufs) dfree(*b);
    delete a;
    g_err = e.empty() ? "adjoint set-up failed" : e;
    return 1;
  }
  s->adj = a;
  return 0;
}

dim3 cell_grid(const svof_solver *s) { return dim3((s->nx + 31) / 32, (s->ny + 7) / 8); }

// dt in stream order (no host staging)
int adj_set_dt(svof_solver *s, double dt) {
  k_adj_set<<<1, 1, 0, s->stream>>>(s->d_dt, dt);
  CK_LAUNCH();
  return 0;
}

// fluid_update_pressure (mode 1) and fluid_correct_velocity (mode 2)
int adj_project(svof_solver *s, int rk, double dt, int mode) {
  AdjointState *a = s->adj;
  const double gam = RK_A[rk] + RK_B[rk];
  k_adj_project<<<cell_grid(s), dim3(32, 8), 0, s->stream>>>(a->ux.p, a->uy.p, a->p.p, a->psib.p, gam * dt,
                                                             0.5 * gam * dt * s->prm.m_dif, mode, s->grid());
  CK_LAUNCH();
  return 0;
}

// fluid_compute_potential_{dct,dft}: the solve of psi_bar / dxf, then the
// divergence's transpose
int adj_potential(svof_solver *s, int rk, double dt) {
  AdjointState *a = s->adj;
  const double gam = RK_A[rk] + RK_B[rk];
  const Grid2 g = s->grid();
  double pre_p;
  if (s->uniform) {
    const int L = s->log2fft;
    const dim3 rows_grid((s->ny + dct_rows(L) - 1) / dct_rows(L));
    dct_fwd_rhs_kernel(L)<<<rows_grid, dct_threads(L), dct_smem(L, false), s->stream>>>(a->psib.p, s->spec.p, s->twf.p,
                                                                                    s->cs.p, g);
    CK_LAUNCH();
    const int kt = s->ysolve_kt;
    k_dct_ysolve<<<(s->nx + kt - 1) / kt, 128, sizeof(double) * 3 * kt * s->ny, s->stream>>>(
        s->spec.p, s->vt.p, s->rvt.p, s->q1t.p, s->ck.p, s->lastf.p, s->den.p, 1. / s->dy / s->dy, s->nx, s->ny,
        kt);
    CK_LAUNCH();
    dct_inv_kernel(L)<<<rows_grid, dct_threads(L), dct_smem(L, true), s->stream>>>(s->spec.p, a->psis.p, s->twb.p,
                                                                                 s->cs.p, g);
    CK_LAUNCH();
    pre_p = 1. / (gam * dt) / (2. * s->nx);
  } else {
    const int cols = s->dft_cols;
    const int blocks = (s->nx + cols - 1) / cols;
    const size_t smem = sizeof(double) * 2 * s->ny * cols;
    const int nky = s->ny / 2 + 1;
    k_dft_fwd_rhs<<<blocks, 256, smem, s->stream>>>(a->psib.p, s->spec.p, s->twf.p, s->log2fft, cols, g);
    CK_LAUNCH();
    const int xkt = s->xsolve_kt;
    k_dft_xsolve<<<(nky + xkt - 1) / xkt, 128, sizeof(double) * 4 * xkt * s->nx, s->stream>>>(
        s->spec.p, s->vt.p, s->rvt.p, s->pl.p, s->pu.p, s->evals.p, s->nx, nky, xkt);
    CK_LAUNCH();
    k_dft_inv<<<blocks, 256, smem, s->stream>>>(s->spec.p, a->psis.p, s->twb.p, s->log2fft, cols, g);
    CK_LAUNCH();
    pre_p = 1. / (gam * dt) / (1. * s->ny);
  }
  k_adj_div<<<cell_grid(s), dim3(32, 8), 0, s->stream>>>(a->ux.p, a->uy.p, a->psis.p, a->psib.p, pre_p, g);
  CK_LAUNCH();
  return 0;
}

// fluid_predict_field about the primal velocities ux, uy and the vof after
// the substep's advection (storage layouts); d_dt must hold dt
int adj_predict(svof_solver *s, int rk, double dt, const double *ux, const double *uy, const double *vof_post) {
  AdjointState *a = s->adj;
  if (launch_coef(s, rk, s->stream)) return 1;
  const int R = a->xs_rows;
  k_adj_xsolve<<<(s->ny + R - 1) / R, 128, a->xs_smem, s->stream>>>(
      a->ux.p, a->uy.p, coef_table(s, rk), a->sa_x.p, a->sg_x.p, a->sa_y.p, a->sg_y.p, a->pend_x.p, a->pend_y.p,
      RK_A[rk] * dt, RK_B[rk] * dt, (RK_A[rk] + RK_B[rk]) * dt, R, s->grid());
  CK_LAUNCH();
  AdjRhsArgs r{};
  r.ux = ux;
  r.uy = uy;
  r.sa_x = a->sa_x.p;
  r.sg_x = a->sg_x.p;
  r.sa_y = a->sa_y.p;
  r.sg_y = a->sg_y.p;
  r.aux = a->ux.p;
  r.auy = a->uy.p;
  r.ap = a->p.p;
  r.avof = a->vof[a->cv].p;
  r.aifx = a->ifx.p;
  r.aify = a->ify.p;
  r.lap_ux = s->lap_ux.p;
  r.lap_uy = s->lap_uy.p;
  r.m_dif = s->prm.m_dif;
  r.lapy0 = s->lapy[0];
  r.lapy1 = s->lapy[1];
  r.lapy2 = s->lapy[2];
  r.grav_vof = s->grav_vof;
  r.vof_ref = s->vof_ref;
  r.vof_post = vof_post;
  r.agrv = a->grv.p;
  r.g = s->grid();
  k_adj_rhs<<<cell_grid(s), dim3(32, 8), 0, s->stream>>>(r);
  CK_LAUNCH();
  return 0;
}

// interface_update_vof (mode 1), interface_compute_force (2), the intercept
// and normal part of interface_compute_curvature_tensor (4), about the primal
// ux, uy, vof (storage layouts) and the solver's normal and curv
int adj_interface(svof_solver *s, int rk, double dt, int mode, const double *ux, const double *uy,
                  const double *vof) {
  AdjointState *a = s->adj;
  AdjIfaceArgs f{};
  f.ux = ux;
  f.uy = uy;
  f.vof = vof;
  f.normal = s->normal.p;
  f.curv = s->curv.p;
  f.avof_in = a->vof[a->cv].p;
  f.avof_out = a->vof[1 - a->cv].p;
  f.pend_in = a->pend_v[a->cp].p;
  f.pend_out = a->pend_v[1 - a->cp].p;
  f.aux = a->ux.p;
  f.auy = a->uy.p;
  f.aifx = a->ifx.p;
  f.aify = a->ify.p;
  f.anrm = a->nrm.p;
  f.am = a->m.p;
  f.akap = a->kap.p;
  f.asig = a->sig.p;
  f.adt = RK_A[rk] * dt;
  f.bdt = RK_B[rk] * dt;
  f.tension = s->prm.tension;
  f.mode = mode;
  f.g = s->grid();
  k_adj_interface<<<cell_grid(s), dim3(32, 8), 0, s->stream>>>(f);
  CK_LAUNCH();
  a->cv ^= 1;
  if (mode & 1) a->cp ^= 1;
  return 0;
}

// the corner normals and curvature part of interface_compute_curvature_tensor
int adj_corners(svof_solver *s, const double *vof) {
  AdjointState *a = s->adj;
  k_adj_corners<<<dim3((s->nx + CBX - 1) / CBX, (s->ny + CBY - 1) / CBY), dim3(CBX, CBY), 0, s->stream>>>(
      vof, a->m.p, a->kap.p, a->vof[a->cv].p, s->grid());
  CK_LAUNCH();
  return 0;
}

size_t vof_count(const svof_solver *s) { return (size_t)(s->nx + 2) * (s->ny + 4); }

// one substep's part of a tape: ux, uy, vof; the tape holds three of them and
// the step's final vof
size_t tape_stride(const svof_solver *s) {
  const size_t n_ux = (size_t)(s->nx + 1) * (s->ny + 2), n_cc = (size_t)(s->nx + 2) * (s->ny + 2);
  return n_ux + n_cc + vof_count(s);
}

int check_prim(svof_solver *s) {
  if (!s) return fail("null argument");
  return adj_ensure(s);
}

int sync(svof_solver *s) {
  CK(cudaStreamSynchronize(s->stream));
  return 0;
}

}  // namespace

}  // namespace svof

using namespace svof;

extern "C" {

int svof_set_gravity(svof_solver_t *s, double grav_vof, double vof_ref) {
  if (!s) return fail("null argument");
  CK(cudaStreamSynchronize(s->stream));
  s->grav_vof = grav_vof;
  s->vof_ref = vof_ref;
  for (auto &kv : s->graphs) cudaGraphExecDestroy(kv.second);
  s->graphs.clear();
  return 0;
}

int svof_set_params(svof_solver_t *s, const svof_params_t *prm) {
  if (!s || !prm) return fail("null argument");
  if (prm->add_buoyancy != s->prm.add_buoyancy && s->adj) return fail("svof_set_params: add_buoyancy is fixed once the adjoint is in use");
  return engine_update_params(s, prm);
}

int svof_tape_count(const svof_solver_t *s, size_t *count) {
  if (!s || !count) return fail("null argument");
  *count = 3 * tape_stride(s) + vof_count(s);
  return 0;
}

int svof_integrate_fixed(svof_solver_t *s, double dt, double *tape) {
  SVOF_RANGE();
  if (!s) return fail("null argument");
  if (!(dt > 0.)) return fail("svof_integrate_fixed: dt must be positive");
  if (adj_set_dt(s, dt)) return 1;
  const size_t n_ux = (size_t)(s->nx + 1) * (s->ny + 2), n_cc = (size_t)(s->nx + 2) * (s->ny + 2);
  const size_t n_vof = (size_t)(s->nx + 2) * (s->ny + 4), st = tape_stride(s);
  for (int rk = 0; rk < 3; rk++) {
    if (tape) {
      double *t = tape + rk * st;
      CK(cudaMemcpyAsync(t, s->ux[s->cur_u].p, sizeof(double) * n_ux, cudaMemcpyDeviceToDevice, s->stream));
      CK(cudaMemcpyAsync(t + n_ux, s->uy[s->cur_u].p, sizeof(double) * n_cc, cudaMemcpyDeviceToDevice, s->stream));
      CK(cudaMemcpyAsync(t + n_ux + n_cc, s->vof[s->cur_v].p, sizeof(double) * n_vof, cudaMemcpyDeviceToDevice,
                         s->stream));
    }
    if (launch_coef(s, rk, s->stream) || launch_geom(s) || launch_force(s) || launch_vof(s, rk) ||
        launch_predict(s, rk, false) || launch_potential(s, rk, s->uniform) || launch_project(s, rk, 1, 1))
      return 1;
  }
  if (tape)
    CK(cudaMemcpyAsync(tape + 3 * st, s->vof[s->cur_v].p, sizeof(double) * n_vof, cudaMemcpyDeviceToDevice,
                       s->stream));
  return 0;
}

int svof_adjoint_field(svof_solver_t *s, int which, double **dptr, size_t *count) {
  if (!s || !dptr) return fail("null argument");
  if (adj_ensure(s)) return 1;
  AdjointState *a = s->adj;
  const size_t nc = (size_t)s->nx * s->ny, nf = (size_t)(s->nx - 1) * s->ny;
  DevBuf *b = nullptr;
  size_t n = nc;
  switch (which) {
    case SVOF_ADJ_UX: b = &a->ux; n = nf; break;
    case SVOF_ADJ_UY: b = &a->uy; break;
    case SVOF_ADJ_P: b = &a->p; break;
    case SVOF_ADJ_VOF: b = &a->vof[a->cv]; break;
    case SVOF_ADJ_PSI: b = &a->psib; break;
    case SVOF_ADJ_IFRCX: b = &a->ifx; n = nf; break;
    case SVOF_ADJ_IFRCY: b = &a->ify; break;
    case SVOF_ADJ_CURV: b = &a->kap; break;
    case SVOF_ADJ_NORMAL: b = &a->nrm; n = 3 * nc; break;
    case SVOF_ADJ_SRCUX_A: b = &a->pend_x; n = nf; break;
    case SVOF_ADJ_SRCUY_A: b = &a->pend_y; break;
    case SVOF_ADJ_SRC_A: b = &a->pend_v[a->cp]; break;
    case SVOF_ADJ_TENSION: b = &a->sig; break;
    case SVOF_ADJ_GRAVITY: b = &a->grv; break;
    default: return fail("unknown adjoint field %d", which);
  }
  *dptr = b->p;
  if (count) *count = n;
  return 0;
}

int svof_adjoint_reset(svof_solver_t *s) {
  if (check_prim(s)) return 1;
  AdjointState *a = s->adj;
  DevBuf *bufs[] = {&a->ux, &a->uy, &a->p, &a->vof[0], &a->vof[1], &a->pend_v[0], &a->pend_v[1],
                    &a->pend_x, &a->pend_y, &a->sa_x, &a->sg_x, &a->sa_y, &a->sg_y, &a->ifx, &a->ify,
                    &a->kap, &a->m, &a->nrm, &a->sig, &a->grv, &a->psib, &a->psis};
  for (DevBuf *b : bufs) CK(cudaMemsetAsync(b->p, 0, sizeof(double) * b->n, s->stream));
  return 0;
}

int svof_adjoint_step(svof_solver_t *s, const double *tape, double dt) {
  SVOF_RANGE();
  if (check_prim(s)) return 1;
  if (!tape) return fail("svof_adjoint_step: null tape");
  if (!(dt > 0.)) return fail("svof_adjoint_step: dt must be positive");
  AdjointState *a = s->adj;
  const size_t n_ux = (size_t)(s->nx + 1) * (s->ny + 2), n_cc = (size_t)(s->nx + 2) * (s->ny + 2);
  const size_t st = tape_stride(s);
  // no substep follows the last one: its sources' pending adjoints are zero
  CK(cudaMemsetAsync(a->pend_x.p, 0, sizeof(double) * a->pend_x.n, s->stream));
  CK(cudaMemsetAsync(a->pend_y.p, 0, sizeof(double) * a->pend_y.n, s->stream));
  CK(cudaMemsetAsync(a->pend_v[a->cp].p, 0, sizeof(double) * a->pend_v[a->cp].n, s->stream));
  if (adj_set_dt(s, dt)) return 1;
  for (int rk = 2; rk >= 0; rk--) {
    const double *ux = tape + rk * st, *uy = ux + n_ux, *vof = uy + n_cc;
    const double *vof_post = tape + (rk + 1) * st + (rk < 2 ? n_ux + n_cc : 0);
    // the substep's geometry from its vof (normals, intercepts, curvature)
    k_geom<<<dim3((s->nx + 31) / 32, (s->ny + 2 + 7) / 8), dim3(32, 8), 0, s->stream>>>(vof, s->normal.p,
                                                                                         s->curv.p, s->grid());
    CK_LAUNCH();
    if (adj_project(s, rk, dt, 3) || adj_potential(s, rk, dt) || adj_predict(s, rk, dt, ux, uy, vof_post) ||
        adj_interface(s, rk, dt, 7, ux, uy, vof) || adj_corners(s, vof))
      return 1;
  }
  return 0;
}

int svof_adjoint_fluid_update_pressure(svof_solver_t *s, size_t rk, double dt) {
  SVOF_RANGE();
  if (check_prim(s)) return 1;
  if (rk > 2) return fail("rkstep out of range");
  return adj_project(s, (int)rk, dt, 1) || sync(s);
}

int svof_adjoint_fluid_correct_velocity(svof_solver_t *s, size_t rk, double dt) {
  SVOF_RANGE();
  if (check_prim(s)) return 1;
  if (rk > 2) return fail("rkstep out of range");
  return adj_project(s, (int)rk, dt, 2) || sync(s);
}

int svof_adjoint_fluid_compute_potential(svof_solver_t *s, size_t rk, double dt) {
  SVOF_RANGE();
  if (check_prim(s)) return 1;
  if (rk > 2) return fail("rkstep out of range");
  return adj_potential(s, (int)rk, dt) || sync(s);
}

int svof_adjoint_fluid_predict_field(svof_solver_t *s, size_t rk, double dt) {
  SVOF_RANGE();
  if (check_prim(s)) return 1;
  if (rk > 2) return fail("rkstep out of range");
  return adj_set_dt(s, dt) ||
         adj_predict(s, (int)rk, dt, s->ux[s->cur_u].p, s->uy[s->cur_u].p, s->vof[s->cur_v].p) || sync(s);
}

int svof_adjoint_interface_update_vof(svof_solver_t *s, size_t rk, double dt) {
  SVOF_RANGE();
  if (check_prim(s)) return 1;
  if (rk > 2) return fail("rkstep out of range");
  return adj_interface(s, (int)rk, dt, 1, s->ux[s->cur_u].p, s->uy[s->cur_u].p, s->vof[s->cur_v].p) || sync(s);
}

int svof_adjoint_interface_compute_force(svof_solver_t *s) {
  SVOF_RANGE();
  if (check_prim(s)) return 1;
  return adj_interface(s, 0, 0., 2, s->ux[s->cur_u].p, s->uy[s->cur_u].p, s->vof[s->cur_v].p) || sync(s);
}

int svof_adjoint_interface_compute_curvature_tensor(svof_solver_t *s) {
  SVOF_RANGE();
  if (check_prim(s)) return 1;
  const double *vof = s->vof[s->cur_v].p;
  return adj_interface(s, 0, 0., 4, s->ux[s->cur_u].p, s->uy[s->cur_u].p, vof) || adj_corners(s, vof) || sync(s);
}

// the deterministic sum of a per-cell accumulator, copied to the host
static int adj_total(svof_solver *s, const DevBuf &b, double *out) {
  AdjointState *a = s->adj;
  k_adj_sum<<<1, 256, 0, s->stream>>>(b.p, (long)b.n, a->sum.p);
  CK_LAUNCH();
  CK(cudaMemcpyAsync(out, a->sum.p, sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return 0;
}

int svof_adjoint_tension(svof_solver_t *s, double *out) {
  if (check_prim(s)) return 1;
  if (!out) return fail("null argument");
  return adj_total(s, s->adj->sig, out);
}

int svof_adjoint_gravity(svof_solver_t *s, double *out) {
  if (check_prim(s)) return 1;
  if (!out) return fail("null argument");
  return adj_total(s, s->adj->grv, out);
}

}  // extern "C"

namespace svof {

// frees the adjoint's buffers (svof_destroy)
void adjoint_free(svof_solver *s) {
  if (!s || !s->adj) return;
  AdjointState *a = s->adj;
  DevBuf *bufs[] = {&a->ux, &a->uy, &a->p, &a->vof[0], &a->vof[1], &a->pend_v[0], &a->pend_v[1],
                    &a->pend_x, &a->pend_y, &a->sa_x, &a->sg_x, &a->sa_y, &a->sg_y, &a->ifx, &a->ify,
                    &a->kap, &a->m, &a->nrm, &a->sig, &a->grv, &a->psib, &a->psis, &a->sum};
  for (DevBuf *b : bufs) dfree(*b);
  delete a;
  s->adj = nullptr;
}

}  // namespace svof
