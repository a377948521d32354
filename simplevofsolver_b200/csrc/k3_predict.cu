// k3_predict.cu -- momentum / scalar predictor of the FP64 3D path.
//
// ux, uy, uz and t each take dt (alpha src_a + beta src_b + gamma src_g),
// solve (1 - gamma dt nu / 2 Lx) delta' = delta along x, and update
// u += delta' (src/fluid/predict/{ux,uy,t}.c in 2D, carried to z by the
// restatement oracle/svof_oracle3d.c).  The x lines are short and many
// (ny nz of them), and the Thomas recurrence is serial along a line, so a
// block owns 32 lines and walks them in 32-cell x-chunks:
//
//   forward, chunk by chunk: all 256 threads evaluate the four right-hand
//     sides of a 32 x 32 tile (x coalesced), store src_a, and keep the
//     increments in shared memory; warps 0..3 (one field each, one line per
//     lane) continue the forward Thomas recurrence through the chunk with the
//     carry in a register; the swept chunk goes to a scratch array.
//   backward, chunk by chunk in reverse: the tile comes back, warps 0..3 run
//     the back substitution, all threads write u + delta' into the other
//     buffer of the ping-pong pair together with the halo images.
//   walls: the x wall values of the four fields and their halo images.
//
// The Thomas coefficients depend on the substep only and come from
// k3_tdm_coef (three distinct systems: ux, uy/uz, t).  The arithmetic keeps
// the restatement's association, so the result matches it bit for bit.
#include "svof3d_internal.cuh"

namespace svof3 {

// Layout per system s at coef + 3 s nx:  L[i] = tdm_l[i];  R[0] = tdm_c[0],
// R[i] = 1 / (c_i - l_i v_{i-1}) for 0 < i < n-1, R[n-1] = 1 / (c - l v) of
// the last row or 0 when that row is zeroed (src/tdm.c:17-50);  V[i] = v_i.
__global__ void k3_tdm_coef(const double *__restrict__ lap_ux, const double *__restrict__ lap_cc,
                            const double *__restrict__ dtp, double gam, double m_dif, double t_dif, int nx,
                            double *__restrict__ coef) {
  extern __shared__ double slap[];  // [2][3 nx]
  for (int w = threadIdx.x; w < 3 * nx; w += blockDim.x) {
    slap[w] = (w < 3 * (nx - 1)) ? lap_ux[w] : 0.;
    slap[3 * nx + w] = lap_cc[w];
  }
  __syncthreads();
  const int f = threadIdx.x;
  if (f >= 3) return;
  const double *lap = slap + ((0 == f) ? 0 : 3 * nx);
  const double dif = (2 == f) ? t_dif : m_dif;
  const int n = (0 == f) ? nx - 1 : nx;
  double *L = coef + (size_t)(3 * f + 0) * nx;
  double *R = coef + (size_t)(3 * f + 1) * nx;
  double *V = coef + (size_t)(3 * f + 2) * nx;
  const double dt = *dtp;
  const double pf = 0.5 * gam * dt * dif;
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

// Right-hand sides of one thread's cell: uy, uz and t at cell i and ux at the
// face i + 1 (do_ux: i < nx).  The explicit part goes to sa[f], the
// x-implicit diffusion and the pressure gradient to sg[f], in the
// restatement's order (advection x, y, z; diffusion x, y, z; pressure;
// buoyancy; surface).  All stencil values are loaded before any arithmetic,
// so that the ~50 loads of a cell are in flight together.
// Field order: 0 ux, 1 uy, 2 uz, 3 t.
template <class R>
__device__ __forceinline__ void rhs4(const Predict3Args<R> &a, const Grid3 &g, int i, int j, int k, bool do_ux,
                                     double *sa, double *sg) {
  const double *ux = a.ux, *uy = a.uy, *uz = a.uz, *t = a.t, *p = a.p;
  // ---- loads
  const double u00 = ldg(ux + ix_ux(g, i, j, k)), u10 = ldg(ux + ix_ux(g, i + 1, j, k));
  const double u0s = ldg(ux + ix_ux(g, i, j - 1, k)), u1s = ldg(ux + ix_ux(g, i + 1, j - 1, k));
  const double u0b = ldg(ux + ix_ux(g, i, j, k - 1)), u1b = ldg(ux + ix_ux(g, i + 1, j, k - 1));
  const double vc = ldg(uy + ix_cc(g, i, j, k)), vxm = ldg(uy + ix_cc(g, i - 1, j, k));
  const double vxp = ldg(uy + ix_cc(g, i + 1, j, k));
  const double vs = ldg(uy + ix_cc(g, i, j - 1, k)), vn = ldg(uy + ix_cc(g, i, j + 1, k));
  const double vb = ldg(uy + ix_cc(g, i, j, k - 1)), vt = ldg(uy + ix_cc(g, i, j, k + 1));
  const double vnb = ldg(uy + ix_cc(g, i, j + 1, k - 1));
  const double wc = ldg(uz + ix_cc(g, i, j, k)), wxm = ldg(uz + ix_cc(g, i - 1, j, k));
  const double wxp = ldg(uz + ix_cc(g, i + 1, j, k));
  const double ws = ldg(uz + ix_cc(g, i, j - 1, k)), wn = ldg(uz + ix_cc(g, i, j + 1, k));
  const double wb = ldg(uz + ix_cc(g, i, j, k - 1)), wt = ldg(uz + ix_cc(g, i, j, k + 1));
  const double wst = ldg(uz + ix_cc(g, i, j - 1, k + 1));
  const double tc = ldg(t + ix_cc(g, i, j, k)), txm = ldg(t + ix_cc(g, i - 1, j, k));
  const double txp = ldg(t + ix_cc(g, i + 1, j, k));
  const double ts = ldg(t + ix_cc(g, i, j - 1, k)), tn = ldg(t + ix_cc(g, i, j + 1, k));
  const double tb = ldg(t + ix_cc(g, i, j, k - 1)), tt = ldg(t + ix_cc(g, i, j, k + 1));
  const double pc = ldg(p + ix_cc(g, i, j, k)), ps = ldg(p + ix_cc(g, i, j - 1, k));
  const double pb = ldg(p + ix_cc(g, i, j, k - 1));
  const double ify = ldg(a.ifrcy + ix_src(g, i, j, k)), ifz = ldg(a.ifrcz + ix_src(g, i, j, k));
  const double dxf_i = ldg(g.dxf + i - 1);
  const double lc0 = ldg(a.lap_cc + 3 * (i - 1) + 0), lc1 = ldg(a.lap_cc + 3 * (i - 1) + 1);
  const double lc2 = ldg(a.lap_cc + 3 * (i - 1) + 2);
  double u20 = 0., u1n = 0., u1t = 0., v1n = 0., w1t = 0., pxp = 0., ifx = 0., dxf_i1 = 1., dxc_i1 = 1.;
  double lu0 = 0., lu1 = 0., lu2 = 0.;
  if (do_ux) {
    u20 = ldg(ux + ix_ux(g, i + 2, j, k));
    u1n = ldg(ux + ix_ux(g, i + 1, j + 1, k));
    u1t = ldg(ux + ix_ux(g, i + 1, j, k + 1));
    v1n = ldg(uy + ix_cc(g, i + 1, j + 1, k));
    w1t = ldg(uz + ix_cc(g, i + 1, j, k + 1));
    pxp = ldg(p + ix_cc(g, i + 1, j, k));
    ifx = ldg(a.ifrcx + ix_srcx(g, i + 1, j, k));
    dxf_i1 = ldg(g.dxf + i);
    dxc_i1 = ldg(g.dxc + i);
    lu0 = ldg(a.lap_ux + 3 * (i - 1) + 0);
    lu1 = ldg(a.lap_ux + 3 * (i - 1) + 1);
    lu2 = ldg(a.lap_ux + 3 * (i - 1) + 2);
  }
  const double md = a.m_dif, td = a.t_dif, dy = g.dy, dz = g.dz;
  const double *ly = a.lapy, *lz = a.lapz;
  // ---- ux at the face iu = i + 1: xm = UX(iu-1), xc = UX(iu), xp = UX(iu+1)
  if (do_ux) {
    const double xm = u00, xc = u10, xp = u20, ys = u1s, yn = u1n, zs = u1b, zn = u1t;
    const double dxc = dxc_i1;
    double ra = 0., rg = 0.;
    {
      const double ul = +0.5 * xm + 0.5 * xc, uu = +0.5 * xc + 0.5 * xp;
      const double l = +0.5 / dxc * ul, u = -0.5 / dxc * uu, cc = -l - u;
      ra += +l * xm + cc * xc + u * xp;
    }
    const double w_xm = 0.5 * dxf_i / dxc, w_xp = 0.5 * dxf_i1 / dxc;
    {
      const double ul = w_xm * vc + w_xp * vxp;
      const double uu = w_xm * vn + w_xp * v1n;
      const double l = +0.5 / dy * ul, u = -0.5 / dy * uu, cc = -l - u;
      ra += +l * ys + cc * xc + u * yn;
    }
    {
      const double ul = w_xm * wc + w_xp * wxp;
      const double uu = w_xm * wt + w_xp * w1t;
      const double l = +0.5 / dz * ul, u = -0.5 / dz * uu, cc = -l - u;
      ra += +l * zs + cc * xc + u * zn;
    }
    rg += md * (+lu0 * xm + lu1 * xc + lu2 * xp);
    ra += md * (+ly[0] * ys + ly[1] * xc + ly[2] * yn);
    ra += md * (+lz[0] * zs + lz[1] * xc + lz[2] * zn);
    rg -= 1. / dxc * (-pc + pxp);
    if (a.add_buoyancy) ra += +0.5 * tc + 0.5 * txp;
    ra += ifx;
    sa[0] = ra;
    sg[0] = rg;
  }
  const double dxf = dxf_i;
  // ---- uy at cell i
  {
    const double xm = vxm, xc = vc, xp = vxp, ys = vs, yn = vn, zs = vb, zn = vt;
    double ra = 0., rg = 0.;
    {
      const double ul = +0.5 * u0s + 0.5 * u00;
      const double uu = +0.5 * u1s + 0.5 * u10;
      const double l = +0.5 / dxf * ul, u = -0.5 / dxf * uu, cc = -l - u;
      ra += +l * xm + cc * xc + u * xp;
    }
    {
      const double ul = +0.5 * ys + 0.5 * xc, uu = +0.5 * xc + 0.5 * yn;
      const double l = +0.5 / dy * ul, u = -0.5 / dy * uu, cc = -l - u;
      ra += +l * ys + cc * xc + u * yn;
    }
    {
      const double ul = +0.5 * ws + 0.5 * wc;
      const double uu = +0.5 * wst + 0.5 * wt;
      const double l = +0.5 / dz * ul, u = -0.5 / dz * uu, cc = -l - u;
      ra += +l * zs + cc * xc + u * zn;
    }
    rg += md * (+lc0 * xm + lc1 * xc + lc2 * xp);
    ra += md * (+ly[0] * ys + ly[1] * xc + ly[2] * yn);
    ra += md * (+lz[0] * zs + lz[1] * xc + lz[2] * zn);
    rg -= 1. / dy * (-ps + pc);
    ra += ify;
    sa[1] = ra;
    sg[1] = rg;
  }
  // ---- uz at cell i
  {
    const double xm = wxm, xc = wc, xp = wxp, ys = ws, yn = wn, zs = wb, zn = wt;
    double ra = 0., rg = 0.;
    {
      const double ul = +0.5 * u0b + 0.5 * u00;
      const double uu = +0.5 * u1b + 0.5 * u10;
      const double l = +0.5 / dxf * ul, u = -0.5 / dxf * uu, cc = -l - u;
      ra += +l * xm + cc * xc + u * xp;
    }
    {
      const double ul = +0.5 * vb + 0.5 * vc;
      const double uu = +0.5 * vnb + 0.5 * vn;
      const double l = +0.5 / dy * ul, u = -0.5 / dy * uu, cc = -l - u;
      ra += +l * ys + cc * xc + u * yn;
    }
    {
      const double ul = +0.5 * zs + 0.5 * xc, uu = +0.5 * xc + 0.5 * zn;
      const double l = +0.5 / dz * ul, u = -0.5 / dz * uu, cc = -l - u;
      ra += +l * zs + cc * xc + u * zn;
    }
    rg += md * (+lc0 * xm + lc1 * xc + lc2 * xp);
    ra += md * (+ly[0] * ys + ly[1] * xc + ly[2] * yn);
    ra += md * (+lz[0] * zs + lz[1] * xc + lz[2] * zn);
    rg -= 1. / dz * (-pb + pc);
    ra += ifz;
    sa[2] = ra;
    sg[2] = rg;
  }
  // ---- t at cell i
  {
    const double xm = txm, xc = tc, xp = txp, ys = ts, yn = tn, zs = tb, zn = tt;
    double ra = 0., rg = 0.;
    {
      const double l = +0.5 / dxf * u00, u = -0.5 / dxf * u10, cc = -l - u;
      ra += +l * xm + cc * xc + u * xp;
    }
    {
      const double l = +0.5 / dy * vc, u = -0.5 / dy * vn, cc = -l - u;
      ra += +l * ys + cc * xc + u * yn;
    }
    {
      const double l = +0.5 / dz * wc, u = -0.5 / dz * wt, cc = -l - u;
      ra += +l * zs + cc * xc + u * zn;
    }
    rg += td * (+lc0 * xm + lc1 * xc + lc2 * xp);
    ra += td * (+ly[0] * ys + ly[1] * xc + ly[2] * yn);
    ra += td * (+lz[0] * zs + lz[1] * xc + lz[2] * zn);
    sa[3] = ra;
    sg[3] = rg;
  }
}

constexpr int PL = kPredLines, PC = kPredChunk;

template <class R>
__global__ void __launch_bounds__(256, 2) k3_predict(Predict3Args<R> a) {
  __shared__ double sd[4][PL][PC + 1];  // the four fields' increments of one tile
  __shared__ double sco[9][PC];         // L, R, V of the three systems, one chunk
  const Grid3 g = a.g;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const long nlines = (long)ny * nz;
  const long l0 = (long)blockIdx.x * PL;
  const int tid = threadIdx.x;
  const int tx = tid & 31, ty = tid >> 5;
  const int nchunks = (nx + PC - 1) / PC;
  const double dt = ldg(a.dtp);
  const double ca = a.rk.a * dt, cb = a.rk.b * dt, cg = a.rk.g * dt;
  // the sweeping warps: warp f < 4 owns field f, lane = line of the block
  const int f = ty;
  const bool sweeper = f < 4 && (l0 + tx < nlines);
  const int set = (0 == f) ? 0 : (3 == f ? 2 : 1);
  const int nf = (0 == f) ? nx - 1 : nx;
  const size_t fstride = (size_t)nlines * nx;  // scratch per field
  double carry = 0.;

  // ------------------------------------------------------------ forward
  for (int c = 0; c < nchunks; c++) {
    const int p0 = c * PC;
    for (int w = tid; w < 9 * PC; w += 256) {
      const int r = w / PC, q = w - r * PC;
      sco[r][q] = (p0 + q < nx) ? ldg(a.coef + (size_t)r * nx + p0 + q) : 0.;
    }
#pragma unroll 1
    for (int m = 0; m < 4; m++) {
      const int ll = ty + 8 * m;
      const long l = l0 + ll;
      if (l >= nlines) continue;
      const int j = 1 + (int)(l % ny), k = 1 + (int)(l / ny);
      const int p = p0 + tx;
      if (p >= nx) continue;
      // cell i = p + 1 for uy, uz, t (line position p) and face i + 1 for ux
      // (line position p of the ux system, which has nx - 1 unknowns)
      const int i = p + 1;
      const bool do_ux = p < nx - 1;
      double sa[4], sg[4];
      rhs4(a, g, i, j, k, do_ux, sa, sg);
      if (do_ux) {
        const long is = ix_srcx(g, i + 1, j, k);
        a.sa[0][is] = R(sa[0]);
        const double sb = a.use_b ? cb * ldg(a.sb[0] + is) : 0.;
        sd[0][ll][tx] = +ca * sa[0] + sb + cg * sg[0];
      }
      const long is = ix_src(g, i, j, k);
#pragma unroll
      for (int q = 1; q < 4; q++) {
        a.sa[q][is] = R(sa[q]);
        const double sb = a.use_b ? cb * ldg(a.sb[q] + is) : 0.;
        sd[q][ll][tx] = +ca * sa[q] + sb + cg * sg[q];
      }
    }
    __syncthreads();
    if (sweeper) {
      double *q = sd[f][tx];
      const double *L = sco[3 * set], *R = sco[3 * set + 1];
      const int smax = min(PC, nf - p0);
#pragma unroll 4
      for (int s = 0; s < smax; s++) {
        const int pp = p0 + s;
        const double x = q[s];
        if (0 == pp) {
          carry = x / R[s];
        } else if (pp < nf - 1) {
          carry = R[s] * (x - L[s] * carry);
        } else {
          carry = (0. != R[s]) ? R[s] * (x - L[s] * carry) : 0.;
        }
        q[s] = carry;
      }
    }
    __syncthreads();
#pragma unroll 1
    for (int m = 0; m < 4; m++) {
      const int ll = ty + 8 * m;
      const long l = l0 + ll;
      const int p = p0 + tx;
      if (l >= nlines || p >= nx) continue;
      R *fw = a.fw + (size_t)l * nx + p;
      if (p < nx - 1) fw[0] = R(sd[0][ll][tx]);
      fw[fstride] = R(sd[1][ll][tx]);
      fw[2 * fstride] = R(sd[2][ll][tx]);
      fw[3 * fstride] = R(sd[3][ll][tx]);
    }
    __syncthreads();
  }

  // ------------------------------------------------------------ backward
  double nxt = 0.;
  for (int c = nchunks - 1; c >= 0; c--) {
    const int p0 = c * PC;
    for (int w = tid; w < 3 * PC; w += 256) {
      const int r = w / PC, q = w - r * PC;
      sco[3 * r + 2][q] = (p0 + q < nx) ? ldg(a.coef + (size_t)(3 * r + 2) * nx + p0 + q) : 0.;
    }
#pragma unroll 1
    for (int m = 0; m < 4; m++) {
      const int ll = ty + 8 * m;
      const long l = l0 + ll;
      const int p = p0 + tx;
      if (l >= nlines || p >= nx) continue;
      const R *fw = a.fw + (size_t)l * nx + p;
      sd[0][ll][tx] = (p < nx - 1) ? fw[0] : 0.;
      sd[1][ll][tx] = fw[fstride];
      sd[2][ll][tx] = fw[2 * fstride];
      sd[3][ll][tx] = fw[3 * fstride];
    }
    __syncthreads();
    if (sweeper) {
      double *q = sd[f][tx];
      const double *V = sco[3 * set + 2];
      const int smax = min(PC, nf - p0);
#pragma unroll 4
      for (int s = smax - 1; s >= 0; s--) {
        const int pp = p0 + s;
        if (nf - 1 == pp) {
          nxt = q[s];
        } else {
          nxt = q[s] - V[s] * nxt;
          q[s] = nxt;
        }
      }
    }
    __syncthreads();
#pragma unroll 1
    for (int m = 0; m < 4; m++) {
      const int ll = ty + 8 * m;
      const long l = l0 + ll;
      const int p = p0 + tx;
      if (l >= nlines || p >= nx) continue;
      const int j = 1 + (int)(l % ny), k = 1 + (int)(l / ny);
      if (p < nx - 1) {
        const int i = p + 2;
        const double v = ldg(a.ux + ix_ux(g, i, j, k)) + sd[0][ll][tx];
        for_images(j, k, ny, nz, true, [&](int jj, int kk) { a.ux_new[ix_ux(g, i, jj, kk)] = v; });
      }
      {
        const int i = p + 1;
        const long ic = ix_cc(g, i, j, k);
        const double vy = ldg(a.uy + ic) + sd[1][ll][tx];
        const double vz = ldg(a.uz + ic) + sd[2][ll][tx];
        const double vt = ldg(a.t + ic) + sd[3][ll][tx];
        for_images(j, k, ny, nz, true, [&](int jj, int kk) {
          const long o = ix_cc(g, i, jj, kk);
          a.uy_new[o] = vy;
          a.uz_new[o] = vz;
          a.t_new[o] = vt;
        });
      }
    }
    __syncthreads();
  }

  // ------------------------------------------------------------ walls
  // each interior row's wall cell takes its wall value; its halo images take
  // the value it held before (halo copy before the wall assignment)
  for (int w = tid; w < 2 * PL; w += 256) {
    const int ll = w % PL, side = w / PL;
    const long l = l0 + ll;
    if (l >= nlines) continue;
    const int j = 1 + (int)(l % ny), k = 1 + (int)(l / ny);
    {
      const int i = side ? nx + 1 : 1;
      const double old = ldg(a.ux + ix_ux(g, i, j, k));
      a.ux_new[ix_ux(g, i, j, k)] = 0.;
      for_images(j, k, ny, nz, false, [&](int jj, int kk) { a.ux_new[ix_ux(g, i, jj, kk)] = old; });
    }
    {
      const int i = side ? nx + 1 : 0;
      const long ic = ix_cc(g, i, j, k);
      const double oy = ldg(a.uy + ic), oz = ldg(a.uz + ic), ot = ldg(a.t + ic);
      a.uy_new[ic] = side ? a.uy_xp : a.uy_xm;
      a.uz_new[ic] = side ? a.uz_xp : a.uz_xm;
      a.t_new[ic] = side ? a.t_xp : a.t_xm;
      for_images(j, k, ny, nz, false, [&](int jj, int kk) {
        const long o = ix_cc(g, i, jj, kk);
        a.uy_new[o] = oy;
        a.uz_new[o] = oz;
        a.t_new[o] = ot;
      });
    }
  }
}

template <class R>
cudaError_t predict_launch(cudaStream_t st, const Predict3Args<R> &a) {
  const long nlines = (long)a.g.ny * a.g.nz;
  k3_predict<R><<<(unsigned)((nlines + PL - 1) / PL), 256, 0, st>>>(a);
  return cudaGetLastError();
}
template cudaError_t predict_launch<double>(cudaStream_t, const Predict3Args<double> &);
template cudaError_t predict_launch<float>(cudaStream_t, const Predict3Args<float> &);

}  // namespace svof3
