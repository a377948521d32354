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
#include <cuda_pipeline.h>

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
                           const double *__restrict__ lap_t, const double *__restrict__ dtp, Gam3 gams,
                           double m_dif, double t_dif, int nx, double *__restrict__ coef_all) {
  pdl_enter();
  // block b: the table of gamma = gams.g[b] at coef_all + 9 nx b
  const double gam = gams.g[blockIdx.x];
  double *coef = coef_all + (size_t)9 * nx * blockIdx.x;
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

// right-hand sides of ux (i >= 2), uy and t at cell (i, j), exactly as
// compute_rhs_{ux,uy,t} (src/fluid/predict/{ux,uy,t}.c): src_a is stored for
// the next substep, the increments dt (alpha src_a + beta src_b + gamma src_g)
// go to d[0..2] (d[0] only for i >= 2)
__device__ __forceinline__ void predict_rhs_cell(const PredictArgs &a, int i, int j, double ca, double cb,
                                                 double cg, double *d) {
  const Grid2 &g = a.g;
  const int nx = g.nx;
  const double dy = g.dy;
  const double *ux = a.ux, *uy = a.uy, *p = a.p, *t = a.t;
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
      d[0] = +ca * sa + sb + cg * sg;
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
      d[1] = +ca * sa + sb + cg * sg;
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
      d[2] = +ca * sa + sb + cg * sg;
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
  const int tid = threadIdx.x;

  for (int w = tid; w < 9 * nx; w += blockDim.x) sc[(w / nx) * ld + (w % nx)] = a.coef[w];

  // ---------------- phase 1: right-hand sides and increments
  for (int w = tid; w < nrows * nx; w += blockDim.x) {
    const int jj = w / nx;
    const int i = 1 + w % nx;
    const int j = j0 + jj;
    double d[3];
    predict_rhs_cell(a, i, j, ca, cb, cg, d);
    if (i >= 2) sd[(0 * R + jj) * ld + (i - 2)] = d[0];
    sd[(1 * R + jj) * ld + (i - 1)] = d[1];
    sd[(2 * R + jj) * ld + (i - 1)] = d[2];
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

// ---------------------------------------------------------------------------
// Line-streaming form for large grids: the fused kernel above keeps whole
// rows in shared memory, so a block holds few rows and its Thomas phase runs
// few lines per SM (the serial recurrence then sets the time).  Here the
// right-hand sides of a 32 x 32 tile go to a line array, one warp per field
// and 32 lines sweeps it (forward and backward) from a ring of shared-memory
// chunks that cp.async fills ahead, and a tiled pass writes u + delta', the
// halo rows and the walls.  The arithmetic (predict_rhs_cell, the sweeps with
// the k_tdm_coef table, u + delta') is the fused kernel's, so the results are
// identical.
//
// Line array layout: lines in blocks of 32, fw[((f * nb + jb) * nx + p) * 32
// + l] for field f (0 ux: p = i - 2; 1 uy, 2 t: p = i - 1), row j = 32 jb + l
// + 1, nb = ceil(ny / 32): the 32 lines of a block are contiguous at every
// position, so a chunk of positions is one contiguous run.
__device__ __forceinline__ size_t fw_ix(int nx, int ny, int f, int p, int j) {
  const int nb = (ny + 31) >> 5, jb = (j - 1) >> 5, l = (j - 1) & 31;
  return (((size_t)f * nb + jb) * nx + p) * 32 + l;
}

constexpr int PT = 32;  // tile edge of the right-hand-side and update passes

__global__ void __launch_bounds__(256, 3) k_predict_rhs(PredictArgs a, double *__restrict__ fw) {
  pdl_enter();
  __shared__ double sd[3][PT][PT + 1];  // [f][i - i0][j - j0]
  const Grid2 g = a.g;
  const int nx = g.nx, ny = g.ny;
  const int i0 = 1 + blockIdx.x * PT, j0 = 1 + blockIdx.y * PT;
  const double dt = *a.dtp;
  const double ca = a.rk.a * dt, cb = a.rk.b * dt, cg = a.rk.g * dt;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  // the thread's four cells unrolled, so that their loads overlap
#pragma unroll
  for (int r = ty; r < PT; r += 8) {
    const int i = i0 + tx, j = j0 + r;
    if (i <= nx && j <= ny) {
      double d[3];
      predict_rhs_cell(a, i, j, ca, cb, cg, d);
      sd[0][tx][r] = d[0];
      sd[1][tx][r] = d[1];
      sd[2][tx][r] = d[2];
    }
  }
  __syncthreads();
  // transposed store: lanes along j (one contiguous 256-byte run)
  for (int c = ty; c < PT; c += 8) {
    const int i = i0 + c, j = j0 + tx;
    if (i > nx || j > ny) continue;
    if (i >= 2) fw[fw_ix(nx, ny, 0, i - 2, j)] = sd[0][c][tx];
    fw[fw_ix(nx, ny, 1, i - 1, j)] = sd[1][c][tx];
    fw[fw_ix(nx, ny, 2, i - 1, j)] = sd[2][c][tx];
  }
}

// one warp per (field, block of 32 lines); chunks of XC positions in a ring
// of XS shared-memory slots; the substep's coefficients of the field in
// shared memory.  Dynamic shared memory: (XS * XC * 32 + 3 nx) doubles.
constexpr int XC = 64, XS = 4, XB = 16;

__global__ void __launch_bounds__(32) k_predict_xsolve(const double *__restrict__ coef, double *__restrict__ fw,
                                                      int nx, int ny) {
  pdl_enter();
  extern __shared__ double sm[];
  double *ring = sm;                         // [XS][XC][32]
  double *sL = sm + (size_t)XS * XC * 32;    // [nx] L, then R, then V, at even offsets
  const int nxp = (nx + 1) & ~1;
  double *sR = sL + nxp, *sV = sR + nxp;
  const int nb = (ny + 31) >> 5;
  const int f = blockIdx.x / nb, jb = blockIdx.x % nb;
  const int l = threadIdx.x;  // line 32 jb + l + 1 (lanes past ny sweep zeros)
  const int n = (0 == f) ? nx - 1 : nx;
  for (int w = l; w < nx; w += 32) {
    sL[w] = coef[(size_t)(3 * f + 0) * nx + w];
    sR[w] = coef[(size_t)(3 * f + 1) * nx + w];
    sV[w] = coef[(size_t)(3 * f + 2) * nx + w];
  }
  double *base = fw + ((size_t)f * nb + jb) * nx * 32;  // position p at base + 32 p
  const int nch = (n + XC - 1) / XC;
  // chunk c (positions c XC .. ) into slot s: 16-byte copies, 32 lanes.
  // Results go from registers straight to the line array (each lane its own
  // 8-byte column of a 256-byte row); the slot is only read.
  auto load = [&](int c, int slot) {
    const int p0 = c * XC, m = min(XC, n - p0);
    const double *src = base + (size_t)p0 * 32;
    double *dst = ring + (size_t)slot * XC * 32;
#pragma unroll 8
    for (int e = 2 * l; e < m * 32; e += 64) __pipeline_memcpy_async(dst + e, src + e, 16);
    __pipeline_commit();
  };
  __syncwarp();
  // ------------------------------------------------------------ forward
  for (int c = 0; c < XS - 1; c++) {
    if (c < nch) load(c, c % XS);
    else __pipeline_commit();
  }
  double qprev = 0.;
  for (int c = 0; c < nch; c++) {
    if (c + XS - 1 < nch) load(c + XS - 1, (c + XS - 1) % XS);
    else __pipeline_commit();
    __pipeline_wait_prior(XS - 1);
    __syncwarp();
    const double *q = ring + (size_t)(c % XS) * XC * 32 + l;
    const int p0 = c * XC, m = min(XC, n - p0);
    double *gq = base + (size_t)p0 * 32 + l;
    // batches of XB positions: the batch's loads are issued ahead of the
    // dependent chain, which then runs on registers.  A full batch inside
    // the line (neither its first nor its last position) runs the bare
    // recurrence with no per-position tests: the warp runs nearly alone on
    // its SM, so every issued instruction counts.  Same expression, same
    // order, same results as the general path below.
    for (int s0 = 0; s0 < m; s0 += XB) {
      const int mb = min(XB, m - s0);
      const int pb = p0 + s0;
      if (XB == mb && pb > 0 && pb + XB < n) {
        // pb is a multiple of XB: the coefficient pairs are 16-byte aligned
        double xv[XB], lv[XB], rv[XB];
        const double2 *l2 = reinterpret_cast<const double2 *>(sL + pb);
        const double2 *r2 = reinterpret_cast<const double2 *>(sR + pb);
#pragma unroll
        for (int k = 0; k < XB / 2; k++) {
          const double2 a = l2[k], b = r2[k];
          lv[2 * k] = a.x;
          lv[2 * k + 1] = a.y;
          rv[2 * k] = b.x;
          rv[2 * k + 1] = b.y;
        }
#pragma unroll
        for (int k = 0; k < XB; k++) xv[k] = q[(s0 + k) * 32];
#pragma unroll
        for (int k = 0; k < XB; k++) {
          qprev = rv[k] * (xv[k] - lv[k] * qprev);
          xv[k] = qprev;
        }
#pragma unroll
        for (int k = 0; k < XB; k++) gq[(s0 + k) * 32] = xv[k];
        continue;
      }
      double xv[XB], lv[XB], rv[XB];
#pragma unroll
      for (int k = 0; k < XB; k++) {
        if (k < mb) {
          xv[k] = q[(s0 + k) * 32];
          lv[k] = sL[p0 + s0 + k];
          rv[k] = sR[p0 + s0 + k];
        }
      }
#pragma unroll
      for (int k = 0; k < XB; k++) {
        if (k < mb) {
          const int p = p0 + s0 + k;
          if (0 == p) {
            qprev = xv[k] / rv[k];
          } else if (p < n - 1) {
            qprev = rv[k] * (xv[k] - lv[k] * qprev);
          } else {
            qprev = (0. != rv[k]) ? rv[k] * (xv[k] - lv[k] * qprev) : 0.;
          }
          xv[k] = qprev;
        }
      }
#pragma unroll
      for (int k = 0; k < XB; k++)
        if (k < mb) gq[(s0 + k) * 32] = xv[k];
    }
    // every lane done reading the slot (the next load refills it) and its
    // stores ordered before the other lanes' later copies of them
    __syncwarp();
  }
  __pipeline_wait_prior(0);
  __syncwarp();
  // ------------------------------------------------------------ backward
  // (the forward's stores are visible to the warp's later copies)
  __threadfence_block();
  for (int c = 0; c < XS - 1; c++) {
    if (c < nch) load(nch - 1 - c, c % XS);
    else __pipeline_commit();
  }
  double qn = qprev;  // q[n - 1]
  for (int it = 0; it < nch; it++) {
    const int c = nch - 1 - it;
    if (it + XS - 1 < nch) load(nch - 1 - (it + XS - 1), (it + XS - 1) % XS);
    else __pipeline_commit();
    __pipeline_wait_prior(XS - 1);
    __syncwarp();
    const double *q = ring + (size_t)(it % XS) * XC * 32 + l;
    const int p0 = c * XC, m = min(XC, n - p0);
    double *gq = base + (size_t)p0 * 32 + l;
    // batches from the top of the chunk down, loads ahead of the chain; a
    // full batch below the last row runs the bare recurrence
    for (int s1 = m; s1 > 0; s1 -= XB) {
      const int mb = min(XB, s1);  // positions s1 - 1 .. s1 - mb
      const int pt = p0 + s1 - 1;  // the batch's top position
      if (XB == mb && pt < n - 1) {
        double xv[XB], vv[XB];
#pragma unroll
        for (int k = 0; k < XB; k++) {
          xv[k] = q[(s1 - 1 - k) * 32];
          vv[k] = sV[pt - k];
        }
#pragma unroll
        for (int k = 0; k < XB; k++) {
          qn = xv[k] - vv[k] * qn;
          xv[k] = qn;
        }
#pragma unroll
        for (int k = 0; k < XB; k++) gq[(s1 - 1 - k) * 32] = xv[k];
        continue;
      }
      double xv[XB], vv[XB];
#pragma unroll
      for (int k = 0; k < XB; k++) {
        if (k < mb) {
          xv[k] = q[(s1 - 1 - k) * 32];
          vv[k] = sV[p0 + s1 - 1 - k];
        }
      }
#pragma unroll
      for (int k = 0; k < XB; k++) {
        if (k < mb) {
          const int p = p0 + s1 - 1 - k;
          if (p != n - 1) {  // the last row keeps its forward value
            qn = xv[k] - vv[k] * qn;
            xv[k] = qn;
          }
        }
      }
#pragma unroll
      for (int k = 0; k < XB; k++)
        if (k < mb) gq[(s1 - 1 - k) * 32] = xv[k];
    }
    __syncwarp();
  }
}

// u + delta' of a 32 x 32 tile (delta' read transposed through shared
// memory), halo rows and walls as fluid_update_boundaries_{ux,uy,t}
__global__ void __launch_bounds__(256) k_predict_update(PredictArgs a, const double *__restrict__ fw) {
  pdl_enter();
  __shared__ double sd[3][PT][PT + 1];  // [f][i - i0][j - j0]
  const Grid2 g = a.g;
  const int nx = g.nx, ny = g.ny;
  const int i0 = 1 + blockIdx.x * PT, j0 = 1 + blockIdx.y * PT;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  for (int c = ty; c < PT; c += 8) {
    const int i = i0 + c, j = j0 + tx;
    if (i > nx || j > ny) continue;
    sd[0][c][tx] = (i >= 2) ? fw[fw_ix(nx, ny, 0, i - 2, j)] : 0.;
    sd[1][c][tx] = fw[fw_ix(nx, ny, 1, i - 1, j)];
    sd[2][c][tx] = fw[fw_ix(nx, ny, 2, i - 1, j)];
  }
  __syncthreads();
  for (int r = ty; r < PT; r += 8) {
    const int j = j0 + r;
    if (j > ny) continue;
    const bool to_top = (1 == j), to_bottom = (ny == j);
    // storage columns of this tile: interior i = i0 + tx, plus the walls
    // handled by the tiles at the two x ends
    const int i = i0 + tx;
    if (i <= nx) {
      const double nuy = a.uy[ix_cc(nx, i, j)] + sd[1][tx][r];
      const double nt = a.t[ix_cc(nx, i, j)] + sd[2][tx][r];
      a.uy_new[ix_cc(nx, i, j)] = nuy;
      a.t_new[ix_cc(nx, i, j)] = nt;
      if (to_top) {
        a.uy_new[ix_cc(nx, i, ny + 1)] = nuy;
        a.t_new[ix_cc(nx, i, ny + 1)] = nt;
      }
      if (to_bottom) {
        a.uy_new[ix_cc(nx, i, 0)] = nuy;
        a.t_new[ix_cc(nx, i, 0)] = nt;
      }
      if (i >= 2) {
        const double nux = a.ux[ix_ux(nx, i, j)] + sd[0][tx][r];
        a.ux_new[ix_ux(nx, i, j)] = nux;
        if (to_top) a.ux_new[ix_ux(nx, i, ny + 1)] = nux;
        if (to_bottom) a.ux_new[ix_ux(nx, i, 0)] = nux;
      }
    }
    // walls: uy, t at i = 0 and nx + 1, ux at i = 1 and nx + 1; the halo rows
    // take the value before the wall assignment
    const bool left = (1 == i0) && (0 == tx), right = (i0 + PT > nx) && (0 == tx);
    for (int side = 0; side < 2; side++) {
      if (!(side ? right : left)) continue;
      const int c = side ? nx + 1 : 0;
      const double huy = a.uy[ix_cc(nx, c, j)], ht = a.t[ix_cc(nx, c, j)];
      a.uy_new[ix_cc(nx, c, j)] = side ? a.uy_xp : a.uy_xm;
      a.t_new[ix_cc(nx, c, j)] = side ? a.t_xp : a.t_xm;
      if (to_top) {
        a.uy_new[ix_cc(nx, c, ny + 1)] = huy;
        a.t_new[ix_cc(nx, c, ny + 1)] = ht;
      }
      if (to_bottom) {
        a.uy_new[ix_cc(nx, c, 0)] = huy;
        a.t_new[ix_cc(nx, c, 0)] = ht;
      }
      const int iu = side ? nx + 1 : 1;
      const double hux = a.ux[ix_ux(nx, iu, j)];
      a.ux_new[ix_ux(nx, iu, j)] = 0.;
      if (to_top) a.ux_new[ix_ux(nx, iu, ny + 1)] = hux;
      if (to_bottom) a.ux_new[ix_ux(nx, iu, 0)] = hux;
    }
  }
}

}  // namespace svof
