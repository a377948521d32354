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

// right-hand sides at (i, j, k): the explicit part into sa, the x-implicit
// diffusion and the pressure gradient into sg, in the restatement's order
// (advection x, y, z; diffusion x, y, z; pressure; buoyancy; surface)
__device__ __forceinline__ void rhs_ux(const Predict3Args &a, const Grid3 &g, int i, int j, int k, double &sa,
                                       double &sg) {
  const double *ux = a.ux, *uy = a.uy, *uz = a.uz;
  const double dxc = ldg(g.dxc + i - 1), dxf = ldg(g.dxf + i - 1);
  const double xm = ldg(ux + ix_ux(g, i - 1, j, k)), xc = ldg(ux + ix_ux(g, i, j, k)), xp = ldg(ux + ix_ux(g, i + 1, j, k));
  const double ys = ldg(ux + ix_ux(g, i, j - 1, k)), yn = ldg(ux + ix_ux(g, i, j + 1, k));
  const double zs = ldg(ux + ix_ux(g, i, j, k - 1)), zn = ldg(ux + ix_ux(g, i, j, k + 1));
  sa = 0.;
  sg = 0.;
  {
    const double ul = +0.5 * xm + 0.5 * xc, uu = +0.5 * xc + 0.5 * xp;
    const double l = +0.5 / dxc * ul, u = -0.5 / dxc * uu, cc = -l - u;
    sa += +l * xm + cc * xc + u * xp;
  }
  const double w_xm = 0.5 * ldg(g.dxf + i - 2) / dxc, w_xp = 0.5 * dxf / dxc;
  {
    const double ul = w_xm * ldg(uy + ix_cc(g, i - 1, j, k)) + w_xp * ldg(uy + ix_cc(g, i, j, k));
    const double uu = w_xm * ldg(uy + ix_cc(g, i - 1, j + 1, k)) + w_xp * ldg(uy + ix_cc(g, i, j + 1, k));
    const double l = +0.5 / g.dy * ul, u = -0.5 / g.dy * uu, cc = -l - u;
    sa += +l * ys + cc * xc + u * yn;
  }
  {
    const double ul = w_xm * ldg(uz + ix_cc(g, i - 1, j, k)) + w_xp * ldg(uz + ix_cc(g, i, j, k));
    const double uu = w_xm * ldg(uz + ix_cc(g, i - 1, j, k + 1)) + w_xp * ldg(uz + ix_cc(g, i, j, k + 1));
    const double l = +0.5 / g.dz * ul, u = -0.5 / g.dz * uu, cc = -l - u;
    sa += +l * zs + cc * xc + u * zn;
  }
  const double *lx = a.lap_ux + 3 * (i - 2);
  sg += a.m_dif * (+ldg(lx + 0) * xm + ldg(lx + 1) * xc + ldg(lx + 2) * xp);
  sa += a.m_dif * (+a.lapy[0] * ys + a.lapy[1] * xc + a.lapy[2] * yn);
  sa += a.m_dif * (+a.lapz[0] * zs + a.lapz[1] * xc + a.lapz[2] * zn);
  sg -= 1. / dxc * (-ldg(a.p + ix_cc(g, i - 1, j, k)) + ldg(a.p + ix_cc(g, i, j, k)));
  if (a.add_buoyancy) sa += +0.5 * ldg(a.t + ix_cc(g, i - 1, j, k)) + 0.5 * ldg(a.t + ix_cc(g, i, j, k));
  sa += ldg(a.ifrcx + ix_srcx(g, i, j, k));
}

__device__ __forceinline__ void rhs_uy(const Predict3Args &a, const Grid3 &g, int i, int j, int k, double &sa,
                                       double &sg) {
  const double *ux = a.ux, *uy = a.uy, *uz = a.uz;
  const double dxf = ldg(g.dxf + i - 1);
  const double xm = ldg(uy + ix_cc(g, i - 1, j, k)), xc = ldg(uy + ix_cc(g, i, j, k)), xp = ldg(uy + ix_cc(g, i + 1, j, k));
  const double ys = ldg(uy + ix_cc(g, i, j - 1, k)), yn = ldg(uy + ix_cc(g, i, j + 1, k));
  const double zs = ldg(uy + ix_cc(g, i, j, k - 1)), zn = ldg(uy + ix_cc(g, i, j, k + 1));
  sa = 0.;
  sg = 0.;
  {
    const double ul = +0.5 * ldg(ux + ix_ux(g, i, j - 1, k)) + 0.5 * ldg(ux + ix_ux(g, i, j, k));
    const double uu = +0.5 * ldg(ux + ix_ux(g, i + 1, j - 1, k)) + 0.5 * ldg(ux + ix_ux(g, i + 1, j, k));
    const double l = +0.5 / dxf * ul, u = -0.5 / dxf * uu, cc = -l - u;
    sa += +l * xm + cc * xc + u * xp;
  }
  {
    const double ul = +0.5 * ys + 0.5 * xc, uu = +0.5 * xc + 0.5 * yn;
    const double l = +0.5 / g.dy * ul, u = -0.5 / g.dy * uu, cc = -l - u;
    sa += +l * ys + cc * xc + u * yn;
  }
  {
    const double ul = +0.5 * ldg(uz + ix_cc(g, i, j - 1, k)) + 0.5 * ldg(uz + ix_cc(g, i, j, k));
    const double uu = +0.5 * ldg(uz + ix_cc(g, i, j - 1, k + 1)) + 0.5 * ldg(uz + ix_cc(g, i, j, k + 1));
    const double l = +0.5 / g.dz * ul, u = -0.5 / g.dz * uu, cc = -l - u;
    sa += +l * zs + cc * xc + u * zn;
  }
  const double *lx = a.lap_cc + 3 * (i - 1);
  sg += a.m_dif * (+ldg(lx + 0) * xm + ldg(lx + 1) * xc + ldg(lx + 2) * xp);
  sa += a.m_dif * (+a.lapy[0] * ys + a.lapy[1] * xc + a.lapy[2] * yn);
  sa += a.m_dif * (+a.lapz[0] * zs + a.lapz[1] * xc + a.lapz[2] * zn);
  sg -= 1. / g.dy * (-ldg(a.p + ix_cc(g, i, j - 1, k)) + ldg(a.p + ix_cc(g, i, j, k)));
  sa += ldg(a.ifrcy + ix_src(g, i, j, k));
}

__device__ __forceinline__ void rhs_uz(const Predict3Args &a, const Grid3 &g, int i, int j, int k, double &sa,
                                       double &sg) {
  const double *ux = a.ux, *uy = a.uy, *uz = a.uz;
  const double dxf = ldg(g.dxf + i - 1);
  const double xm = ldg(uz + ix_cc(g, i - 1, j, k)), xc = ldg(uz + ix_cc(g, i, j, k)), xp = ldg(uz + ix_cc(g, i + 1, j, k));
  const double ys = ldg(uz + ix_cc(g, i, j - 1, k)), yn = ldg(uz + ix_cc(g, i, j + 1, k));
  const double zs = ldg(uz + ix_cc(g, i, j, k - 1)), zn = ldg(uz + ix_cc(g, i, j, k + 1));
  sa = 0.;
  sg = 0.;
  {
    const double ul = +0.5 * ldg(ux + ix_ux(g, i, j, k - 1)) + 0.5 * ldg(ux + ix_ux(g, i, j, k));
    const double uu = +0.5 * ldg(ux + ix_ux(g, i + 1, j, k - 1)) + 0.5 * ldg(ux + ix_ux(g, i + 1, j, k));
    const double l = +0.5 / dxf * ul, u = -0.5 / dxf * uu, cc = -l - u;
    sa += +l * xm + cc * xc + u * xp;
  }
  {
    const double ul = +0.5 * ldg(uy + ix_cc(g, i, j, k - 1)) + 0.5 * ldg(uy + ix_cc(g, i, j, k));
    const double uu = +0.5 * ldg(uy + ix_cc(g, i, j + 1, k - 1)) + 0.5 * ldg(uy + ix_cc(g, i, j + 1, k));
    const double l = +0.5 / g.dy * ul, u = -0.5 / g.dy * uu, cc = -l - u;
    sa += +l * ys + cc * xc + u * yn;
  }
  {
    const double ul = +0.5 * zs + 0.5 * xc, uu = +0.5 * xc + 0.5 * zn;
    const double l = +0.5 / g.dz * ul, u = -0.5 / g.dz * uu, cc = -l - u;
    sa += +l * zs + cc * xc + u * zn;
  }
  const double *lx = a.lap_cc + 3 * (i - 1);
  sg += a.m_dif * (+ldg(lx + 0) * xm + ldg(lx + 1) * xc + ldg(lx + 2) * xp);
  sa += a.m_dif * (+a.lapy[0] * ys + a.lapy[1] * xc + a.lapy[2] * yn);
  sa += a.m_dif * (+a.lapz[0] * zs + a.lapz[1] * xc + a.lapz[2] * zn);
  sg -= 1. / g.dz * (-ldg(a.p + ix_cc(g, i, j, k - 1)) + ldg(a.p + ix_cc(g, i, j, k)));
  sa += ldg(a.ifrcz + ix_src(g, i, j, k));
}

__device__ __forceinline__ void rhs_t(const Predict3Args &a, const Grid3 &g, int i, int j, int k, double &sa,
                                      double &sg) {
  const double *ux = a.ux, *uy = a.uy, *uz = a.uz, *t = a.t;
  const double dxf = ldg(g.dxf + i - 1);
  const double xm = ldg(t + ix_cc(g, i - 1, j, k)), xc = ldg(t + ix_cc(g, i, j, k)), xp = ldg(t + ix_cc(g, i + 1, j, k));
  const double ys = ldg(t + ix_cc(g, i, j - 1, k)), yn = ldg(t + ix_cc(g, i, j + 1, k));
  const double zs = ldg(t + ix_cc(g, i, j, k - 1)), zn = ldg(t + ix_cc(g, i, j, k + 1));
  sa = 0.;
  sg = 0.;
  {
    const double l = +0.5 / dxf * ldg(ux + ix_ux(g, i, j, k)), u = -0.5 / dxf * ldg(ux + ix_ux(g, i + 1, j, k)), cc = -l - u;
    sa += +l * xm + cc * xc + u * xp;
  }
  {
    const double l = +0.5 / g.dy * ldg(uy + ix_cc(g, i, j, k)), u = -0.5 / g.dy * ldg(uy + ix_cc(g, i, j + 1, k));
    const double cc = -l - u;
    sa += +l * ys + cc * xc + u * yn;
  }
  {
    const double l = +0.5 / g.dz * ldg(uz + ix_cc(g, i, j, k)), u = -0.5 / g.dz * ldg(uz + ix_cc(g, i, j, k + 1));
    const double cc = -l - u;
    sa += +l * zs + cc * xc + u * zn;
  }
  const double *lx = a.lap_cc + 3 * (i - 1);
  sg += a.t_dif * (+ldg(lx + 0) * xm + ldg(lx + 1) * xc + ldg(lx + 2) * xp);
  sa += a.t_dif * (+a.lapy[0] * ys + a.lapy[1] * xc + a.lapy[2] * yn);
  sa += a.t_dif * (+a.lapz[0] * zs + a.lapz[1] * xc + a.lapz[2] * zn);
}

constexpr int PL = kPredLines, PC = kPredChunk;

__global__ void __launch_bounds__(256) k3_predict(Predict3Args a) {
  __shared__ double sd[4][PL][PC + 1];  // the four fields' increments of one tile
  __shared__ double sco[9][PC];         // L, R, V of the three systems, one chunk
  const Grid3 g = a.g;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const long nlines = (long)ny * nz;
  const long l0 = (long)blockIdx.x * PL;
  const int tid = threadIdx.x;
  const int tx = tid & 31, ty = tid >> 5;
  const int nchunks = (nx + PC - 1) / PC;
  const double dt = *a.dtp;
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
      if (p < nx - 1) {
        const int i = p + 2;
        double sa, sg;
        rhs_ux(a, g, i, j, k, sa, sg);
        const long is = ix_srcx(g, i, j, k);
        a.sa[0][is] = sa;
        const double sb = a.use_b ? cb * ldg(a.sb[0] + is) : 0.;
        sd[0][ll][tx] = +ca * sa + sb + cg * sg;
      }
      if (p < nx) {
        const int i = p + 1;
        const long is = ix_src(g, i, j, k);
        double sa, sg;
        rhs_uy(a, g, i, j, k, sa, sg);
        a.sa[1][is] = sa;
        double sb = a.use_b ? cb * ldg(a.sb[1] + is) : 0.;
        sd[1][ll][tx] = +ca * sa + sb + cg * sg;
        rhs_uz(a, g, i, j, k, sa, sg);
        a.sa[2][is] = sa;
        sb = a.use_b ? cb * ldg(a.sb[2] + is) : 0.;
        sd[2][ll][tx] = +ca * sa + sb + cg * sg;
        rhs_t(a, g, i, j, k, sa, sg);
        a.sa[3][is] = sa;
        sb = a.use_b ? cb * ldg(a.sb[3] + is) : 0.;
        sd[3][ll][tx] = +ca * sa + sb + cg * sg;
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
      double *fw = a.fw + (size_t)l * nx + p;
      if (p < nx - 1) fw[0] = sd[0][ll][tx];
      fw[fstride] = sd[1][ll][tx];
      fw[2 * fstride] = sd[2][ll][tx];
      fw[3 * fstride] = sd[3][ll][tx];
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
      const double *fw = a.fw + (size_t)l * nx + p;
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

}  // namespace svof3
