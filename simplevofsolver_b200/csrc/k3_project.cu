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

// one thread per interior cell; the threads at i = 1 and i = nx also own the
// wall cells of their row
__global__ void __launch_bounds__(256) k3_project(double *__restrict__ ux, double *__restrict__ uy,
                                                  double *__restrict__ uz, double *__restrict__ p,
                                                  const double *__restrict__ psi, const double *__restrict__ dtp,
                                                  double gam, double m_dif, double uy_xm, double uy_xp,
                                                  double uz_xm, double uz_xp, int do_vel, int do_p, Grid3 g) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  if (i > nx || j > ny) return;
  const double dt = ldg(dtp);
  // quotients the restatement evaluates per cell, once per thread (same values)
  const double pv = gam * dt, pp = 0.5 * gam * dt * m_dif;
  const double cvx = pv / ldg(g.dxc + i - 1), cvy = pv / g.dy, cvz = pv / g.dz;
  const double cpx = pp / ldg(g.dxf + i - 1);
#pragma unroll 2
  for (int kz = 0; kz < kProjectPlanes; kz++) {
  const int k = 1 + blockIdx.z * kProjectPlanes + kz;
  if (k > nz) break;
  const double psc = ldg(psi + ix_cc(g, i, j, k));
  const bool wall = (1 == i || nx == i);
  if (do_vel) {
    const double pxm = ldg(psi + ix_cc(g, i - 1, j, k));
    const double pym = ldg(psi + ix_cc(g, i, j - 1, k));
    const double pzm = ldg(psi + ix_cc(g, i, j, k - 1));
    const long iu = ix_ux(g, i, j, k), ic = ix_cc(g, i, j, k);
    const double ux0 = ux[iu], uy0 = uy[ic], uz0 = uz[ic];
    // ux
    if (i >= 2) {
      double v = ux0;
      v -= cvx * (+psc - pxm);
      for_images(j, k, ny, nz, true, [&](int jj, int kk) { ux[ix_ux(g, i, jj, kk)] = v; });
    }
    double vy = uy0;
    vy -= cvy * (+psc - pym);
    for_images(j, k, ny, nz, true, [&](int jj, int kk) { uy[ix_cc(g, i, jj, kk)] = vy; });
    double vz = uz0;
    vz -= cvz * (+psc - pzm);
    for_images(j, k, ny, nz, true, [&](int jj, int kk) { uz[ix_cc(g, i, jj, kk)] = vz; });
    if (wall) {
      const int iwu = (1 == i) ? 1 : nx + 1;
      const double old = ux[ix_ux(g, iwu, j, k)];
      ux[ix_ux(g, iwu, j, k)] = 0.;
      for_images(j, k, ny, nz, false, [&](int jj, int kk) { ux[ix_ux(g, iwu, jj, kk)] = old; });
      const int iw = (1 == i) ? 0 : nx + 1;
      const long o = ix_cc(g, iw, j, k);
      const double oy = uy[o], oz = uz[o];
      uy[o] = (1 == i) ? uy_xm : uy_xp;
      uz[o] = (1 == i) ? uz_xm : uz_xp;
      for_images(j, k, ny, nz, false, [&](int jj, int kk) {
        uy[ix_cc(g, iw, jj, kk)] = oy;
        uz[ix_cc(g, iw, jj, kk)] = oz;
      });
    }
  }
  if (do_p) {
    const double pxm = ldg(psi + ix_cc(g, i - 1, j, k));
    const double pxp = ldg(psi + ix_cc(g, i + 1, j, k));
    double v = p[ix_cc(g, i, j, k)];
    v += psc;
    const double dm = (-pxm + psc) / ldg(g.dxc + i - 1);
    const double dp = (-psc + pxp) / ldg(g.dxc + i);
    v -= cpx * (-dm + dp);
    for_images(j, k, ny, nz, true, [&](int jj, int kk) { p[ix_cc(g, i, jj, kk)] = v; });
    if (wall) {
      const int iw = (1 == i) ? 0 : nx + 1;
      const double old = p[ix_cc(g, iw, j, k)];
      p[ix_cc(g, iw, j, k)] = v;
      for_images(j, k, ny, nz, false, [&](int jj, int kk) { p[ix_cc(g, iw, jj, kk)] = old; });
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

// grid-stride over the ux faces i in [2, nx], the uy and the uz faces of the
// interior cells.  All candidates are positive, so the minimum of their IEEE
// bit patterns as unsigned integers is the bit pattern of the minimum.
__global__ void k3_cfl(const double *__restrict__ ux, const double *__restrict__ uy, const double *__restrict__ uz,
                       unsigned long long *__restrict__ minbits, Grid3 g) {
  const int nx = g.nx, ny = g.ny;
  const double small = 1.e-8;
  unsigned long long best = 0x7ff0000000000000ull;
  const long ncell = (long)nx * ny * g.nz;
  const long stride = (long)gridDim.x * blockDim.x;
  for (long w = (long)blockIdx.x * blockDim.x + threadIdx.x; w < ncell; w += stride) {
    const int i = 1 + (int)(w % nx);
    const long r = w / nx;
    const int j = 1 + (int)(r % ny), k = 1 + (int)(r / ny);
    double cand = g.dy / (fabs(uy[ix_cc(g, i, j, k)]) + small);
    const double cz = g.dz / (fabs(uz[ix_cc(g, i, j, k)]) + small);
    cand = fmin(cand, cz);
    if (i >= 2) cand = fmin(cand, g.dxc[i - 1] / (fabs(ux[ix_ux(g, i, j, k)]) + small));
    const unsigned long long b = (unsigned long long)__double_as_longlong(cand);
    best = b < best ? b : best;
  }
  best = warp_min_u64(best);
  __shared__ unsigned long long sbest[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (0 == lane) sbest[warp] = best;
  __syncthreads();
  if (0 == warp) {
    best = lane < (int)(blockDim.x >> 5) ? sbest[lane] : 0x7ff0000000000000ull;
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
