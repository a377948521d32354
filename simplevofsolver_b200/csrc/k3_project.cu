// k3_project.cu -- projection, pressure update, time step and diagnostics of
// the FP64 3D path.
//
//   k3_project   u -= gamma dt grad psi (x, y, z) and p += psi - gamma dt nu / 2
//                Lx psi, in place, with halo images and walls
//                (src/fluid/correct_velocity/*.c, src/fluid/update_pressure.c
//                in 2D, carried to z by oracle/svof_oracle3d.c)
//   k3_cfl       min over faces of dx / (|u| + 1e-8) (src/fluid/decide_dt.c:28-64)
//   k3_dt_final  safety factor and the explicit y and z diffusion limits
//   k3_diag      max |div u|, vof min / max, compensated volume sum
#include "svof3d_internal.cuh"

namespace svof3 {

// one thread per interior (i, j) and kProjectPlanes planes k; the threads at
// i = 1 and i = nx also own the wall cells of their rows.  The planes go in
// pairs, every load of a pair issued before its first store; psi at k - 1 is
// the previous plane's centre value.  A wall cell's old value is read only
// where the cell has halo images to take it (rows j = 1, ny or planes
// k = 1, nz).
__global__ void __launch_bounds__(256, 3) k3_project(double *__restrict__ ux, double *__restrict__ uy,
                                                  double *__restrict__ uz, double *__restrict__ p,
                                                  const double *__restrict__ psi, const double *__restrict__ dtp,
                                                  double gam, double m_dif, double uy_xm, double uy_xp,
                                                  double uz_xm, double uz_xp, int do_vel, int do_p, Grid3 g) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  if (i > nx || j > ny) return;
  const int k0 = 1 + blockIdx.z * kProjectPlanes;
  if (k0 > nz) return;
  const double dt = ldg(dtp);
  // quotients the restatement evaluates per cell, once per thread (same values)
  const double pv = gam * dt, pp = 0.5 * gam * dt * m_dif;
  const double dxc_m = ldg(g.dxc + i - 1);
  const double cvx = pv / dxc_m, cvy = pv / g.dy, cvz = pv / g.dz;
  const double cpx = pp / ldg(g.dxf + i - 1);
  const double dxc_p = (do_p) ? ldg(g.dxc + i) : 1.;
  const bool wall = (1 == i || nx == i);
  const int iwu = (1 == i) ? 1 : nx + 1;  // the wall face of ux
  const int iw = (1 == i) ? 0 : nx + 1;   // the wall cell of the others
  double pzm_next = do_vel ? ldg(psi + ix_cc(g, i, j, k0 - 1)) : 0.;
  constexpr int B = 2;
#pragma unroll
  for (int kb = 0; kb < kProjectPlanes; kb += B) {
    double psc[B], pxm[B], pym[B], pxp[B], u0[B], v0[B], w0[B], p0[B];
    // ---- loads
#pragma unroll
    for (int h = 0; h < B; h++) {
      const int k = k0 + kb + h;
      if (k > nz) break;
      const long ic = ix_cc(g, i, j, k);
      psc[h] = ldg(psi + ic);
      pxm[h] = ldg(psi + ix_cc(g, i - 1, j, k));
      if (do_vel) {
        pym[h] = ldg(psi + ix_cc(g, i, j - 1, k));
        u0[h] = ux[ix_ux(g, i, j, k)];
        v0[h] = uy[ic];
        w0[h] = uz[ic];
      }
      if (do_p) {
        pxp[h] = ldg(psi + ix_cc(g, i + 1, j, k));
        p0[h] = p[ic];
      }
    }
    // ---- updates
#pragma unroll
    for (int h = 0; h < B; h++) {
      const int k = k0 + kb + h;
      if (k > nz) break;
      const double pzm = pzm_next;
      pzm_next = psc[h];
      if (do_vel) {
        if (i >= 2) {
          double v = u0[h];
          v -= cvx * (+psc[h] - pxm[h]);
          for_images(j, k, ny, nz, true, [&](int jj, int kk) { ux[ix_ux(g, i, jj, kk)] = v; });
        }
        double vy = v0[h];
        vy -= cvy * (+psc[h] - pym[h]);
        for_images(j, k, ny, nz, true, [&](int jj, int kk) { uy[ix_cc(g, i, jj, kk)] = vy; });
        double vz = w0[h];
        vz -= cvz * (+psc[h] - pzm);
        for_images(j, k, ny, nz, true, [&](int jj, int kk) { uz[ix_cc(g, i, jj, kk)] = vz; });
        if (wall) {
          const bool img = (1 == j || ny == j || 1 == k || nz == k);
          const long o = ix_cc(g, iw, j, k);
          double old = 0., oy = 0., oz = 0.;
          if (img) {
            old = ux[ix_ux(g, iwu, j, k)];
            oy = uy[o];
            oz = uz[o];
          }
          ux[ix_ux(g, iwu, j, k)] = 0.;
          for_images(j, k, ny, nz, false, [&](int jj, int kk) { ux[ix_ux(g, iwu, jj, kk)] = old; });
          uy[o] = (1 == i) ? uy_xm : uy_xp;
          uz[o] = (1 == i) ? uz_xm : uz_xp;
          for_images(j, k, ny, nz, false, [&](int jj, int kk) {
            uy[ix_cc(g, iw, jj, kk)] = oy;
            uz[ix_cc(g, iw, jj, kk)] = oz;
          });
        }
      }
      if (do_p) {
        double v = p0[h];
        v += psc[h];
        const double dm = (-pxm[h] + psc[h]) / dxc_m;
        const double dp = (-psc[h] + pxp[h]) / dxc_p;
        v -= cpx * (-dm + dp);
        for_images(j, k, ny, nz, true, [&](int jj, int kk) { p[ix_cc(g, i, jj, kk)] = v; });
        if (wall) {
          const bool img = (1 == j || ny == j || 1 == k || nz == k);
          const double old = img ? p[ix_cc(g, iw, j, k)] : 0.;
          p[ix_cc(g, iw, j, k)] = v;
          for_images(j, k, ny, nz, false, [&](int jj, int kk) { p[ix_cc(g, iw, jj, kk)] = old; });
        }
      }
    }
  }
}

__device__ __forceinline__ unsigned long long warp_min_u64(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
    v = w < v ? w : v;
  }
  return v;
}

// one thread per interior (i, j) and kCflPlanes planes k: the ux face i in
// [2, nx], the uy and the uz faces of each cell.  The candidate d / (|u| +
// 1e-8) decreases with |u|, and rounded addition and division are monotone,
// so the thread's minimum over its faces of a kind is the quotient of its
// maximum |u| (NaN velocities are skipped by fmax, as by the fmin of the
// per-face form): three divisions a thread instead of three a cell.  All
// candidates are positive, so the minimum of their IEEE bit patterns as
// unsigned integers is the bit pattern of the minimum.
__global__ void __launch_bounds__(256) k3_cfl(const double *__restrict__ ux, const double *__restrict__ uy,
                                              const double *__restrict__ uz, unsigned long long *__restrict__ minbits,
                                              Grid3 g) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  const int k0 = 1 + blockIdx.z * kCflPlanes;
  const double small = 1.e-8;
  unsigned long long best = 0x7ff0000000000000ull;
  if (i <= nx && j <= ny) {
    double vy[kCflPlanes], vz[kCflPlanes], vx[kCflPlanes];
#pragma unroll
    for (int h = 0; h < kCflPlanes; h++) {
      const int k = min(k0 + h, nz);
      vy[h] = ldg(uy + ix_cc(g, i, j, k));
      vz[h] = ldg(uz + ix_cc(g, i, j, k));
      vx[h] = (i >= 2) ? ldg(ux + ix_ux(g, i, j, k)) : 0.;
    }
    double my = -1., mz = -1., mx = -1.;
#pragma unroll
    for (int h = 0; h < kCflPlanes; h++) {
      if (k0 + h > nz) break;
      my = fmax(my, fabs(vy[h]));
      mz = fmax(mz, fabs(vz[h]));
      if (i >= 2) mx = fmax(mx, fabs(vx[h]));
    }
    double cand = __longlong_as_double(0x7ff0000000000000ll);
    if (my >= 0.) cand = fmin(cand, g.dy / (my + small));
    if (mz >= 0.) cand = fmin(cand, g.dz / (mz + small));
    if (mx >= 0.) cand = fmin(cand, ldg(g.dxc + i - 1) / (mx + small));
    best = (unsigned long long)__double_as_longlong(cand);
  }
  best = warp_min_u64(best);
  __shared__ unsigned long long sbest[8];
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
  const int lane = tid & 31, warp = tid >> 5;
  if (0 == lane) sbest[warp] = best;
  __syncthreads();
  if (0 == warp) {
    best = lane < 8 ? sbest[lane] : 0x7ff0000000000000ull;
    best = warp_min_u64(best);
    if (0 == lane) atomicMin(minbits, best);
  }
}

// dt = min(coef_adv min(1, advective minimum), the four explicit diffusive
// limits); resets the accumulator to the bit pattern of 1.0
__global__ void k3_dt_final(unsigned long long *minbits, double *dt, double coef_adv, double l0, double l1,
                            double l2, double l3) {
  double dta = fmin(1., __longlong_as_double((long long)*minbits));
  dta *= coef_adv;
  double r = dta;
  r = fmin(r, l0);
  r = fmin(r, l1);
  r = fmin(r, l2);
  r = fmin(r, l3);
  *dt = r;
  *minbits = (unsigned long long)__double_as_longlong(1.);
}

__device__ __forceinline__ void two_sum_acc(double &s, double &c, double x) {
  const double t = s + x;
  const double bp = t - s;
  const double err = (s - (t - bp)) + (x - bp);
  s = t;
  c += err;
}

// out = {max |div u|, vof min, vof max, sum vof dx dy dz}; one block of
// kDiagThreads threads, deterministic order
constexpr int kDiagThreads = 512;

__global__ void __launch_bounds__(kDiagThreads) k3_diag(const double *__restrict__ ux, const double *__restrict__ uy, const double *__restrict__ uz,
                        const double *__restrict__ vof, double *__restrict__ out, Grid3 g) {
  const int nx = g.nx, ny = g.ny;
  const long ncell = (long)nx * ny * g.nz;
  double dmax = 0., vmin = 1., vmax = 0., s0 = 0., c0 = 0.;
  for (long w = threadIdx.x; w < ncell; w += blockDim.x) {
    const int i = 1 + (int)(w % nx);
    const long r = w / nx;
    const int j = 1 + (int)(r % ny), k = 1 + (int)(r / ny);
    const double dx = g.dxf[i - 1];
    const double div = +(ux[ix_ux(g, i + 1, j, k)] - ux[ix_ux(g, i, j, k)]) / dx +
                       (uy[ix_cc(g, i, j + 1, k)] - uy[ix_cc(g, i, j, k)]) / g.dy +
                       (uz[ix_cc(g, i, j, k + 1)] - uz[ix_cc(g, i, j, k)]) / g.dz;
    dmax = fmax(dmax, fabs(div));
    const double lv = vof[ix_vof(g, i, j, k)];
    vmin = fmin(vmin, lv);
    vmax = fmax(vmax, lv);
    two_sum_acc(s0, c0, lv * (dx * g.dy * g.dz));
  }
  __shared__ double red[4][kDiagThreads];
  red[0][threadIdx.x] = dmax;
  red[1][threadIdx.x] = vmin;
  red[2][threadIdx.x] = vmax;
  red[3][threadIdx.x] = s0 + c0;
  __syncthreads();
  if (0 == threadIdx.x) {
    double a = 0., b = 1., c = 0., ss = 0., cc = 0.;
    for (int t = 0; t < (int)blockDim.x; t++) {
      a = fmax(a, red[0][t]);
      b = fmin(b, red[1][t]);
      c = fmax(c, red[2][t]);
      two_sum_acc(ss, cc, red[3][t]);
    }
    out[0] = a;
    out[1] = b;
    out[2] = c;
    out[3] = ss + cc;
  }
}

}  // namespace svof3
