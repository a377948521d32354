// Device kernels of the time-averaged statistics (src/statistics.c), shared
// by the 2D and the 3D solver.  A 2D field is one z plane (nz = 1, no z halo).
#pragma once

// one sample: every accumulator += its quantity over the interior rows
// (j = 1 .. ny, k = 1 .. nz), x ghost cells included.  Statistics arrays
// hold rows in (k, j) order without halo, widths nx+1 (ux1 ux2 uxt) and
// nx+2 (the others).  uz, uz1 and uz2 are null in 2D.
struct StatArgs {
  const double *ux, *uy, *uz, *t;
  double *ux1, *ux2, *uy1, *uy2, *uz1, *uz2, *t1, *t2, *uxt;
  int nx, ny, nz;
  int zh;  // z halo rows of the field storage: 1 in 3D, 0 in 2D
};

__global__ void k_stat_collect(StatArgs a);
// part[k][i] = sum over j = 0 .. ny-1, in order from zero, of acc[k][j][i]
__global__ void k_stat_reduce_planes(const double *__restrict__ acc, int w, int ny, double *__restrict__ part);
// out[i] = sum over k = 0 .. nz-1, in order from zero, of part[k][i]
__global__ void k_stat_reduce_final(const double *__restrict__ part, int w, int nz, double *__restrict__ out);
