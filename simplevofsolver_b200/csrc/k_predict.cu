// k_predict.cu -- fused momentum / scalar predictor of the FP64 2D path.
//
// One block owns R consecutive rows j.  Phase 1 evaluates, for every cell of
// its rows, the right-hand sides of ux, uy and t exactly as
// src/fluid/predict/{ux,uy,t}.c (compute_rhs_* with the explicit parts
// accumulated into src_a and the x-implicit diffusion and pressure gradient
// into src_g), stores src_a for the next substep and keeps the increment
// delta = dt (alpha src_a + beta src_b + gamma src_g) in shared memory.
// Phase 2 solves the implicit-x systems (1 - gamma dt nu / 2 Lx) delta' =
// delta with the Thomas recurrence of src/tdm.c:17-50, one line (field, row)
// per thread.  Phase 3 writes u + delta' into the other buffer of the
// ping-pong pair together with the halo rows and wall values that
// fluid_update_boundaries_{ux,uy,t} assign.
#include "svof_internal.cuh"

namespace svof {

// increments [3][R][nx+1] and the substep's Thomas coefficients [9][nx+1]
size_t predict_smem_bytes(int nx, int R) {
  return sizeof(double) * ((size_t)3 * R * (nx + 1) + (size_t)9 * (nx + 1));
}

// Thomas coefficients of the three implicit-x systems of one substep
// (solve_in_x of src/fluid/predict/{ux,uy,t}.c and gtsv, src/tdm.c:17-50):
// they depend on dt and the substep only, so one thread per field computes
// them once and every line solve reads them.  Layout per field f at
// coef + 3 f nx:  L[i] = tdm_l[i];  R[0] = tdm_c[0], R[i] = 1 / (c_i - l_i
// v_{i-1}) for 0 < i < n-1, R[n-1] = 1 / (c - l v) of the last row or 0 when
// the reference zeroes that row;  V[i] = v_i.
__global__ void k_tdm_coef(const double *__restrict__ lap_ux, const double *__restrict__ lap_uy,
                           const double *__restrict__ lap_t, const double *__restrict__ dtp, double gam,
                           double m_dif, double t_dif, int nx, double *__restrict__ coef) {
  pdl_enter();
  // the Laplacian tables are staged in shared memory first: the recurrence
  // below then waits on arithmetic only
  extern __shared__ double slap[];  // [3][3 nx]
  for (int w = threadIdx.x; w < 3 * nx; w += blockDim.x) {
    slap[w] = (w < 3 * (nx - 1)) ? lap_ux[w] : 0.;
    slap[3 * nx + w] = lap_uy[w];
    slap[6 * nx + w] = lap_t[w];
  }
  __syncthreads();
  const int f = threadIdx.x;
  if (f >= 3) return;
  const double *lap = slap + 3 * nx * f;
  const double dif = (2 == f) ? t_dif : m_dif;
  const int n = (0 == f) ? nx - 1 : nx;
  double *L = coef + (size_t)(3 * f + 0) * nx;
  double *R = coef + (size_t)(3 * f + 1) * nx;
  double *V = coef + (size_t)(3 * f + 2) * nx;
  const double dt = *dtp;
  const double pf = 0.5 * gam * dt * dif;  // ux.c:330-332
  const double c0 = 1. - pf * lap[1];
  double v = (-pf * lap[2]) / c0;
  L[0] = -pf * lap[0];
  R[0] = c0;
  V[0] = v;
  for (int i = 1; i < n - 1; i++) {
    const double l = -pf * lap[3 * i + 0];
    const double c = 1. - pf * lap[3 * i + 1];
    const double u = -pf * lap[3 * i + 2];
    const double val = 1. / (c - l * v);
    v = val * (u);
    L[i] = l;
    R[i] = val;
    V[i] = v;
  }
  {
    const double l = -pf * lap[3 * (n - 1) + 0];
    const double c = 1. - pf * lap[3 * (n - 1) + 1];
    const double val = c - l * v;
    L[n - 1] = l;
    R[n - 1] = fabs(val) > kDblEpsilon ? 1. / val : 0.;
  }
}

__global__ void __launch_bounds__(256) k_predict(PredictArgs a) {
  pdl_enter();
  extern __shared__ double sm[];
  const Grid2 g = a.g;
  const int nx = g.nx, ny = g.ny, R = a.rows_per_block;
  const int ld = nx + 1;
  double *sd = sm;                  // [3][R][ld] increments
  double *sc = sm + 3 * R * ld;     // [9][ld] Thomas coefficients (L, R, V of ux, uy, t)
  const int j0 = 1 + blockIdx.x * R;
  const int nrows = min(R, ny - j0 + 1);
  const double dt = *a.dtp;
  const double ca = a.rk.a * dt, cb = a.rk.b * dt, cg = a.rk.g * dt;
  const double dy = g.dy;
  const double *ux = a.ux, *uy = a.uy, *p = a.p, *t = a.t;
  const int tid = threadIdx.x;

  for (int w = tid; w < 9 * nx; w += blockDim.x) sc[(w / nx) * ld + (w % nx)] = a.coef[w];

  // ---------------- phase 1: right-hand sides and increments
  for (int w = tid; w < nrows * nx; w += blockDim.x) {
    const int jj = w / nx;
    const int i = 1 + w % nx;
    const int j = j0 + jj;
    const double dxf_i = g.dxf[i - 1];
    // ---- ux at (i, j), i in [2, nx]: compute_rhs_ux, ux.c:218-249
    if (i >= 2) {
      const double dxc_i = g.dxc[i - 1];
      const double uxm = ux[ix_ux(nx, i - 1, j)], uxc = ux[ix_ux(nx, i, j)], uxp = ux[ix_ux(nx, i + 1, j)];
      const double uxs = ux[ix_ux(nx, i, j - 1)], uxn = ux[ix_ux(nx, i, j + 1)];
      double sa = 0., sg = 0.;
      {  // advection_x, ux.c:71-92
        const double ux_l = +0.5 * uxm + 0.5 * uxc;
        const double ux_u = +0.5 * uxc + 0.5 * uxp;
        const double l = +0.5 / dxc_i * ux_l;
        const double u = -0.5 / dxc_i * ux_u;
        const double c = -l - u;
        sa += +l * uxm + c * uxc + u * uxp;
      }
      {  // advection_y, ux.c:94-120
        const double w_xm = 0.5 * g.dxf[i - 2] / dxc_i;
        const double w_xp = 0.5 * dxf_i / dxc_i;
        const double uy_l = w_xm * uy[ix_cc(nx, i - 1, j)] + w_xp * uy[ix_cc(nx, i, j)];
        const double uy_u = w_xm * uy[ix_cc(nx, i - 1, j + 1)] + w_xp * uy[ix_cc(nx, i, j + 1)];
        const double l = +0.5 / dy * uy_l;
        const double u = -0.5 / dy * uy_u;
        const double c = -l - u;
        sa += +l * uxs + c * uxc + u * uxn;
      }
      {  // diffusion_x (implicit, src_g), ux.c:123-141
        const double *lx = a.lap_ux + 3 * (i - 2);
        sg += a.m_dif * (+lx[0] * uxm + lx[1] * uxc + lx[2] * uxp);
      }
      // diffusion_y (explicit, src_a), ux.c:143-161
      sa += a.m_dif * (+a.lapy0 * uxs + a.lapy1 * uxc + a.lapy2 * uxn);
      // pressure (src_g), ux.c:164-179
      sg -= 1. / dxc_i * (-p[ix_cc(nx, i - 1, j)] + p[ix_cc(nx, i, j)]);
      // buoyancy, ux.c:181-197
      if (a.add_buoyancy) sa += +0.5 * t[ix_cc(nx, i - 1, j)] + 0.5 * t[ix_cc(nx, i, j)];
      // surface, ux.c:199-210
      sa += a.ifrcx[ix_srcx(nx, i, j)];
      a.sux_a[ix_srcx(nx, i, j)] = sa;
      const double sb = a.use_b ? cb * a.sux_b[ix_srcx(nx, i, j)] : 0.;
      sd[(0 * R + jj) * ld + (i - 2)] = +ca * sa + sb + cg * sg;
    }
    // ---- uy at (i, j): compute_rhs_uy, uy.c:195-221
    {
      const double uym = uy[ix_cc(nx, i - 1, j)], uyc = uy[ix_cc(nx, i, j)], uyp = uy[ix_cc(nx, i + 1, j)];
      const double uys = uy[ix_cc(nx, i, j - 1)], uyn = uy[ix_cc(nx, i, j + 1)];
      double sa = 0., sg = 0.;
      {  // advection_x, uy.c:70-92
        const double ux_l = +0.5 * ux[ix_ux(nx, i, j - 1)] + 0.5 * ux[ix_ux(nx, i, j)];
        const double ux_u = +0.5 * ux[ix_ux(nx, i + 1, j - 1)] + 0.5 * ux[ix_ux(nx, i + 1, j)];
        const double l = +0.5 / dxf_i * ux_l;
        const double u = -0.5 / dxf_i * ux_u;
        const double c = -l - u;
        sa += +l * uym + c * uyc + u * uyp;
      }
      {  // advection_y, uy.c:94-115
        const double uy_l = +0.5 * uys + 0.5 * uyc;
        const double uy_u = +0.5 * uyc + 0.5 * uyn;
        const double l = +0.5 / dy * uy_l;
        const double u = -0.5 / dy * uy_u;
        const double c = -l - u;
        sa += +l * uys + c * uyc + u * uyn;
      }
      {  // diffusion_x (src_g), uy.c:118-136
        const double *lx = a.lap_uy + 3 * (i - 1);
        sg += a.m_dif * (+lx[0] * uym + lx[1] * uyc + lx[2] * uyp);
      }
      // diffusion_y (src_a), uy.c:138-156
      sa += a.m_dif * (+a.lapy0 * uys + a.lapy1 * uyc + a.lapy2 * uyn);
      // pressure (src_g), uy.c:159-174
      sg -= 1. / dy * (-p[ix_cc(nx, i, j - 1)] + p[ix_cc(nx, i, j)]);
      // surface, uy.c:176-187
      sa += a.ifrcy[ix_src(nx, i, j)];
      // extension: buoyancy of the volume fraction (not in the reference)
      if (0. != a.grav_vof) {
        sa += a.grav_vof * (0.5 * a.vof[ix_vof(nx, i, j - 1)] + 0.5 * a.vof[ix_vof(nx, i, j)] - a.vof_ref);
      }
      a.suy_a[ix_src(nx, i, j)] = sa;
      const double sb = a.use_b ? cb * a.suy_b[ix_src(nx, i, j)] : 0.;
      sd[(1 * R + jj) * ld + (i - 1)] = +ca * sa + sb + cg * sg;
    }
    // ---- t at (i, j): compute_rhs_t, t.c:160-182
    {
      const double tm = t[ix_cc(nx, i - 1, j)], tc = t[ix_cc(nx, i, j)], tp = t[ix_cc(nx, i + 1, j)];
      const double ts = t[ix_cc(nx, i, j - 1)], tn = t[ix_cc(nx, i, j + 1)];
      double sa = 0., sg = 0.;
      {  // advection_x, t.c:68-89
        const double l = +0.5 / dxf_i * ux[ix_ux(nx, i, j)];
        const double u = -0.5 / dxf_i * ux[ix_ux(nx, i + 1, j)];
        const double c = -l - u;
        sa += +l * tm + c * tc + u * tp;
      }
      {  // advection_y, t.c:91-112
        const double l = +0.5 / dy * uy[ix_cc(nx, i, j)];
        const double u = -0.5 / dy * uy[ix_cc(nx, i, j + 1)];
        const double c = -l - u;
        sa += +l * ts + c * tc + u * tn;
      }
      {  // diffusion_x (src_g), t.c:115-133
        const double *lx = a.lap_t + 3 * (i - 1);
        sg += a.t_dif * (+lx[0] * tm + lx[1] * tc + lx[2] * tp);
      }
      // diffusion_y (src_a), t.c:135-153
      sa += a.t_dif * (+a.lapy0 * ts + a.lapy1 * tc + a.lapy2 * tn);
      a.st_a[ix_src(nx, i, j)] = sa;
      const double sb = a.use_b ? cb * a.st_b[ix_src(nx, i, j)] : 0.;
      sd[(2 * R + jj) * ld + (i - 1)] = +ca * sa + sb + cg * sg;
    }
  }
  __syncthreads();

  // ---------------- phase 2: Thomas sweeps (gtsv, src/tdm.c:17-50) with the
  // coefficients of k_tdm_coef
  const bool line = tid < 3 * nrows;
  if (line) {
    const int f = tid / nrows;
    const int jj = tid % nrows;
    const int n = (0 == f) ? nx - 1 : nx;
    double *q = sd + (f * R + jj) * ld;
    const double *L = sc + (3 * f + 0) * ld;
    const double *Rv = sc + (3 * f + 1) * ld;
    const double *V = sc + (3 * f + 2) * ld;
    double qprev = q[0] / Rv[0];
    q[0] = qprev;
#pragma unroll 4
    for (int i = 1; i < n - 1; i++) {
      qprev = Rv[i] * (q[i] - L[i] * qprev);
      q[i] = qprev;
    }
    {
      const double rl = Rv[n - 1];
      q[n - 1] = (0. != rl) ? rl * (q[n - 1] - L[n - 1] * qprev) : 0.;
    }
    double qn = q[n - 1];
#pragma unroll 4
    for (int i = n - 2; i >= 0; i--) {
      qn = q[i] - V[i] * qn;
      q[i] = qn;
    }
  }
  __syncthreads();

  // ---------------- phase 3: u + delta', halo rows and walls
  for (int w = tid; w < nrows * (nx + 2); w += blockDim.x) {
    const int r = w / (nx + 2);
    const int c = w % (nx + 2);
    const int j = j0 + r;
    const bool to_top = (1 == j), to_bottom = (ny == j);  // halo copies j -> ny+1, j -> 0
    // uy and t: storage column c is i = c
    {
      double nuy, nt, huy, ht;
      if (0 == c || nx + 1 == c) {
        huy = a.uy[ix_cc(nx, c, j)];  // value before the wall assignment
        ht = a.t[ix_cc(nx, c, j)];
        nuy = (0 == c) ? a.uy_xm : a.uy_xp;
        nt = (0 == c) ? a.t_xm : a.t_xp;
      } else {
        nuy = a.uy[ix_cc(nx, c, j)] + sd[(1 * R + r) * ld + (c - 1)];
        nt = a.t[ix_cc(nx, c, j)] + sd[(2 * R + r) * ld + (c - 1)];
        huy = nuy;
        ht = nt;
      }
      a.uy_new[ix_cc(nx, c, j)] = nuy;
      a.t_new[ix_cc(nx, c, j)] = nt;
      if (to_top) {
        a.uy_new[ix_cc(nx, c, ny + 1)] = huy;
        a.t_new[ix_cc(nx, c, ny + 1)] = ht;
      }
      if (to_bottom) {
        a.uy_new[ix_cc(nx, c, 0)] = huy;
        a.t_new[ix_cc(nx, c, 0)] = ht;
      }
    }
    // ux: storage column c in [0, nx] is i = c + 1
    if (c <= nx) {
      const int i = c + 1;
      double nux, hux;
      if (1 == i || nx + 1 == i) {
        hux = a.ux[ix_ux(nx, i, j)];
        nux = 0.;
      } else {
        nux = a.ux[ix_ux(nx, i, j)] + sd[(0 * R + r) * ld + (i - 2)];
        hux = nux;
      }
      a.ux_new[ix_ux(nx, i, j)] = nux;
      if (to_top) a.ux_new[ix_ux(nx, i, ny + 1)] = hux;
      if (to_bottom) a.ux_new[ix_ux(nx, i, 0)] = hux;
    }
  }
}

}  // namespace svof
