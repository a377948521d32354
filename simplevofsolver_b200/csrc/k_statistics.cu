// Time-averaged statistics on the device: the accumulation of
// src/statistics.c:117-204 (collect_mean_ux, collect_mean_uy, collect_mean_t,
// collect_uxt) and the row sums of its reduce_and_write
// (src/statistics.c:232-281), for the 2D and the 3D solver.
//
// Compiled with -fmad=false like every kernel here, so 0.5 * t(i-1) +
// 0.5 * t(i) and ux * t_ round as the reference's C does.  The reference adds
// pow(x, 1.) and pow(x, 2.); pow(x, 1.) is x, and the squares here are the
// correctly rounded products x * x (glibc's pow(x, 2.) is within one unit in
// the last place of them).
#include "stat_internal.cuh"

__global__ void __launch_bounds__(256) k_stat_collect(StatArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;  // 0 .. nx+1
  const int j = blockIdx.y * blockDim.y + threadIdx.y;  // interior row j+1
  const int k = blockIdx.z;                             // interior plane k+1
  if (i > a.nx + 1 || j >= a.ny) return;
  const int wx = a.nx + 1, wc = a.nx + 2;
  const long row = (long)k * a.ny + j;                         // statistics row
  const long srow = (long)(k + a.zh) * (a.ny + 2) + (j + 1);  // storage row
  const double *tr = a.t + srow * wc;
  const double vy = a.uy[srow * wc + i];
  const double vt = tr[i];
  const long qc = row * wc + i;
  a.uy1[qc] = a.uy1[qc] + vy;
  a.uy2[qc] = a.uy2[qc] + vy * vy;
  if (a.uz) {
    const double vz = a.uz[srow * wc + i];
    a.uz1[qc] = a.uz1[qc] + vz;
    a.uz2[qc] = a.uz2[qc] + vz * vz;
  }
  a.t1[qc] = a.t1[qc] + vt;
  a.t2[qc] = a.t2[qc] + vt * vt;
  if (i <= a.nx) {
    // face i+1 of the reference's 1-based ux index, between cells i and i+1
    const double vx = a.ux[srow * wx + i];
    const double t_ = 0.5 * tr[i] + 0.5 * tr[i + 1];
    const long qx = row * wx + i;
    a.ux1[qx] = a.ux1[qx] + vx;
    a.ux2[qx] = a.ux2[qx] + vx * vx;
    a.uxt[qx] = a.uxt[qx] + vx * t_;
  }
}

// one thread per column and plane; loads eight rows ahead, adds in row order
__global__ void __launch_bounds__(128) k_stat_reduce_planes(const double *__restrict__ acc, int w, int ny,
                                                            double *__restrict__ part) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = blockIdx.y;
  if (i >= w) return;
  const double *p = acc + (long)k * ny * w + i;
  double s = 0.;
  int j = 0;
  for (; j + 8 <= ny; j += 8) {
    double v[8];
#pragma unroll
    for (int q = 0; q < 8; q++) v[q] = p[(long)(j + q) * w];
#pragma unroll
    for (int q = 0; q < 8; q++) s += v[q];
  }
  for (; j < ny; j++) s += p[(long)j * w];
  part[(long)k * w + i] = s;
}

__global__ void __launch_bounds__(128) k_stat_reduce_final(const double *__restrict__ part, int w, int nz,
                                                           double *__restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= w) return;
  double s = 0.;
  for (int k = 0; k < nz; k++) s += part[(long)k * w + i];
  out[i] = s;
}
