// k3_project.cu -- projection, pressure update, time step and diagnostics of
// the FP64 3D path.
//
//   k3_project   u -= gamma dt grad psi (x, y, z) and p += psi - gamma dt nu / 2
//                Lx psi, in place, with halo images and walls
//                (src/fluid/correct_velocity/*.c, src/fluid/update_pressure.c
//                in 2D, carried to z by oracle/svof_oracle3d.c)
//   k3_cfl       min over faces of dx / (|u| + 1e-8) (src/fluid/decide_dt.c:28-64)
//   k3_dt_final  safety factor and the explicit y and z diffusion limits
//   k3_diag_part / k3_diag_final  max |div u|, vof min / max and the
//                compensated volume sum, in two deterministic stages
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
// unsigned integers is the bit pattern of the minimum.  A non-finite
// velocity (NaN or Inf) sets bit 0 of *status for the host to report.
__global__ void __launch_bounds__(256) k3_cfl(const double *__restrict__ ux, const double *__restrict__ uy,
                                              const double *__restrict__ uz, unsigned long long *__restrict__ minbits,
                                              unsigned *__restrict__ status, Grid3 g) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  const int k0 = 1 + blockIdx.z * kCflPlanes;
  const double small = 1.e-8;
  unsigned long long best = 0x7ff0000000000000ull;
  bool bad = false;
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
      bad |= !(fabs(vy[h]) <= kDblMax && fabs(vz[h]) <= kDblMax && fabs(vx[h]) <= kDblMax);
    }
    double cand = __longlong_as_double(0x7ff0000000000000ll);
    if (my >= 0.) cand = fmin(cand, g.dy / (my + small));
    if (mz >= 0.) cand = fmin(cand, g.dz / (mz + small));
    if (mx >= 0.) cand = fmin(cand, ldg(g.dxc + i - 1) / (mx + small));
    best = (unsigned long long)__double_as_longlong(cand);
  }
  if (__any_sync(0xffffffffu, bad) && 0 == ((threadIdx.x + blockDim.x * threadIdx.y) & 31)) atomicOr(status, 1u);
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
// limits); resets the accumulator to the bit pattern of 1.0; a time step
// that is not a positive finite number sets bit 1 of *status
__global__ void k3_dt_final(unsigned long long *minbits, double *dt, double coef_adv, double l0, double l1,
                            double l2, double l3, unsigned *status) {
  double dta = fmin(1., __longlong_as_double((long long)*minbits));
  dta *= coef_adv;
  double r = dta;
  r = fmin(r, l0);
  r = fmin(r, l1);
  r = fmin(r, l2);
  r = fmin(r, l3);
  *dt = r;
  if (!(r > 0. && r <= kDblMax)) atomicOr(status, 2u);
  *minbits = (unsigned long long)__double_as_longlong(1.);
}

__device__ __forceinline__ void two_sum_acc(double &s, double &c, double x) {
  const double t = s + x;
  const double bp = t - s;
  const double err = (s - (t - bp)) + (x - bp);
  s = t;
  c += err;
}

// compensated pair (s, c) += (s2, c2): s2 added exactly (TwoSum), the
// correction terms summed
__device__ __forceinline__ void comp_add(double &s, double &c, double s2, double c2) {
  two_sum_acc(s, c, s2);
  c += c2;
}

// the five partial values of a thread set, reduced over a warp by a fixed
// xor-butterfly (the same order on every run)
struct DiagPart {
  double dmax, vmin, vmax, s, c;
};
__device__ __forceinline__ void warp_reduce_diag(DiagPart &d) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    d.dmax = fmax(d.dmax, __shfl_xor_sync(0xffffffffu, d.dmax, o));
    d.vmin = fmin(d.vmin, __shfl_xor_sync(0xffffffffu, d.vmin, o));
    d.vmax = fmax(d.vmax, __shfl_xor_sync(0xffffffffu, d.vmax, o));
    const double s2 = __shfl_xor_sync(0xffffffffu, d.s, o), c2 = __shfl_xor_sync(0xffffffffu, d.c, o);
    comp_add(d.s, d.c, s2, c2);
  }
}

// stage 1: one thread per interior (i, j) and kDiagPlanes planes (uz at
// k + 1 carried to the next plane); each block of 32 x 8 threads writes its
// partial {max |div u|, vof min, vof max, volume sum, its correction} to
// part[5 b]
__global__ void __launch_bounds__(256) k3_diag_part(const double *__restrict__ ux, const double *__restrict__ uy,
                                                    const double *__restrict__ uz, const double *__restrict__ vof,
                                                    double *__restrict__ part, Grid3 g) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  const int k0 = 1 + blockIdx.z * kDiagPlanes;
  DiagPart d{0., 1., 0., 0., 0.};
  if (i <= nx && j <= ny && k0 <= nz) {
    const double dx = ldg(g.dxf + i - 1);
    const double cell = dx * g.dy * g.dz;
    double uzk = ldg(uz + ix_cc(g, i, j, k0));
#pragma unroll 4
    for (int h = 0; h < kDiagPlanes; h++) {
      const int k = k0 + h;
      if (k > nz) break;
      const double x0 = ldg(ux + ix_ux(g, i, j, k)), x1 = ldg(ux + ix_ux(g, i + 1, j, k));
      const double y0 = ldg(uy + ix_cc(g, i, j, k)), y1 = ldg(uy + ix_cc(g, i, j + 1, k));
      const double zp = ldg(uz + ix_cc(g, i, j, k + 1));
      const double lv = ldg(vof + ix_vof(g, i, j, k));
      const double div = +(x1 - x0) / dx + (y1 - y0) / g.dy + (zp - uzk) / g.dz;
      uzk = zp;
      d.dmax = fmax(d.dmax, fabs(div));
      d.vmin = fmin(d.vmin, lv);
      d.vmax = fmax(d.vmax, lv);
      two_sum_acc(d.s, d.c, lv * cell);
    }
  }
  warp_reduce_diag(d);
  __shared__ DiagPart sp[8];
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
  const int lane = tid & 31, warp = tid >> 5;
  if (0 == lane) sp[warp] = d;
  __syncthreads();
  if (0 == tid) {
    DiagPart r = sp[0];
    for (int w = 1; w < 8; w++) {
      r.dmax = fmax(r.dmax, sp[w].dmax);
      r.vmin = fmin(r.vmin, sp[w].vmin);
      r.vmax = fmax(r.vmax, sp[w].vmax);
      comp_add(r.s, r.c, sp[w].s, sp[w].c);
    }
    double *o = part + 5 * (size_t)(blockIdx.x + gridDim.x * (blockIdx.y + (size_t)gridDim.y * blockIdx.z));
    o[0] = r.dmax;
    o[1] = r.vmin;
    o[2] = r.vmax;
    o[3] = r.s;
    o[4] = r.c;
  }
}

// stage 2: one block of kDiagThreads threads folds the nparts partials in a
// fixed order into out = {max |div u|, vof min, vof max, sum vof dx dy dz}
__global__ void __launch_bounds__(kDiagThreads) k3_diag_final(const double *__restrict__ part, long nparts,
                                                               double *__restrict__ out) {
  DiagPart d{0., 1., 0., 0., 0.};
  for (long b = threadIdx.x; b < nparts; b += kDiagThreads) {
    const double *o = part + 5 * b;
    d.dmax = fmax(d.dmax, o[0]);
    d.vmin = fmin(d.vmin, o[1]);
    d.vmax = fmax(d.vmax, o[2]);
    comp_add(d.s, d.c, o[3], o[4]);
  }
  warp_reduce_diag(d);
  __shared__ DiagPart sp[kDiagThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (0 == lane) sp[warp] = d;
  __syncthreads();
  if (0 == threadIdx.x) {
    DiagPart r = sp[0];
    for (int w = 1; w < kDiagThreads / 32; w++) {
      r.dmax = fmax(r.dmax, sp[w].dmax);
      r.vmin = fmin(r.vmin, sp[w].vmin);
      r.vmax = fmax(r.vmax, sp[w].vmax);
      comp_add(r.s, r.c, sp[w].s, sp[w].c);
    }
    out[0] = r.dmax;
    out[1] = r.vmin;
    out[2] = r.vmax;
    out[3] = r.s + r.c;
  }
}

}  // namespace svof3
