// qas_hall.cuh -- Hall term of the 1D Hall driver on sm_100a: HMHD1D::hall_
// (1D/SERIAL/h-shock/hmhd1d_solve.cpp:138-264) and HMHD1D::haldt
// (1D/SERIAL/h-shock/hmhd1d_class.cpp:3-13), without electron inertia (de = 0).
//
// One hall_(dt) call: ut = u, then per SSP-RK stage
//   k_hvel     Hall velocity h = -(di/ro) rot B at every cell, its ghosts filled as a gather
//              with the momentum flags (hallv + bound(pv,3,&dnxs[1]));
//   k_hlr      nonlinear face interpolation of ro, hx, hy, hz, by, bz, en (mhd_lr_single);
//   k_hflux    Lax-Friedrichs Hall flux of by, bz, en (calc_flux_hall_lf, common/mhd_flux.c:784-813)
//              with the speed |h_n| + vphix |B_n / ro|;
//   k_hupdate  RK update of by, bz, en (mhd_updt1d);
// then the state's ghost fill (k_bound).  The arrays reused here: dv[0..2] = hx, hy, hz (1D has
// no shock detector), vl/vr = face states, f[0][5..7] = fluxes.
#pragma once

#include "qas_kernels.cuh"

namespace qas {

// hx, hy, hz of HMHD1D::hallv at cell i, rotc (common/common_interp.h:39-43) on the state's B
__device__ __forceinline__ void hall_vel(const View &v, int i, double di, double idx, double h[3])
{
  const double *bx = v.u[4], *by = v.u[5], *bz = v.u[6];
  const double fac = di / v.u[0][i];
  h[0] = 0.0;
  h[1] = -fac * (0.5 * ((bx[i + 0] - bx[i - 0]) * 0.0 - (bz[i + 1] - bz[i - 1]) * idx));
  h[2] = -fac * (0.5 * ((by[i + 1] - by[i - 1]) * idx - (bx[i + 0] - bx[i - 0]) * 0.0));
}

// haldt's maximum over the interior: max(1, |hx| + vphix |bx/ro|), into *bits (atomic max of
// the bit patterns of non-negative doubles); *bits must hold the bits of 1.0 before
__global__ void k_hall_vmax(View v, double vphix, unsigned long long *bits)
{
  if (v.ctl->done) return;
  const int i = GH + blockIdx.x * blockDim.x + threadIdx.x;
  double best = 1.0;
  if (i < v.g.nx - GH) {
    const double vt = fabs(0.0) + vphix * fabs(v.u[4][i] / v.u[0][i]);  // hx = 0 in hallv
    if (vt > best) best = vt;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double other = __shfl_xor_sync(0xffffffffu, best, o);
    best = (other > best) ? other : best;
  }
  if ((threadIdx.x & 31) == 0) atomicMax(bits, (unsigned long long)__double_as_longlong(best));
}

__global__ void k_hvel(View v, double di, double idx)
{
  if (v.ctl->done) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= v.g.nx) return;
  double h[3], nv[3];
  bool any = false;
#pragma unroll
  for (int f = 0; f < 3; f++) {
    const int src = map_src(v.maps, 3, f, 0, i);
    if (src != i) {  // a ghost: the fill copies the computed value at its source, times the factor
      hall_vel(v, src, di, idx, h);
      nv[f] = map_fac(v.maps, 3, f, 0, i) * h[f];
    } else {
      if (!any) hall_vel(v, i, di, idx, h);
      any = true;
      nv[f] = h[f];
    }
  }
#pragma unroll
  for (int f = 0; f < 3; f++) v.dv[f][i] = nv[f];
}

template <int ODR>
__global__ void k_hlr(View v)
{
  if (v.ctl->done) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < 2 || i >= v.g.nx - 2) return;
  const double *q[7] = {v.u[0], v.dv[0], v.dv[1], v.dv[2], v.u[5], v.u[6], v.u[7]};
#pragma unroll
  for (int m = 0; m < 7; m++) {
    const double s5[5] = {q[m][i - 2], q[m][i - 1], q[m][i], q[m][i + 1], q[m][i + 2]};
    double fl, fr;
    nl_lr<ODR>(s5, fl, fr);
    v.vl[m][i] = fl;  // left state at face i+1/2
    v.vr[m][i] = fr;  // right state at face i-1/2
  }
}

__global__ void k_hflux(View v, double vphix)
{
  if (v.ctl->done) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < 3 || i >= v.g.nx - 2) return;
  double L[7], R[7];
#pragma unroll
  for (int m = 0; m < 7; m++) {
    L[m] = v.vl[m][i - 1];
    R[m] = v.vr[m][i];
  }
  const double bnf = v.u[4][i];
  const double bnc = 0.5 * (bnf + bnf);
  const double rn = qmin(L[0], R[0]);
  double smax = 0.0;
  smax += qmax(fabs(L[1]), fabs(R[1]));
  smax += vphix * fabs(bnc / rn);
  const double pml = 0.5 * (bnc * bnc + L[4] * L[4] + L[5] * L[5]);
  const double vbl = L[1] * bnc + L[2] * L[4] + L[3] * L[5];
  const double pmr = 0.5 * (bnc * bnc + R[4] * R[4] + R[5] * R[5]);
  const double vbr = R[1] * bnc + R[2] * R[4] + R[3] * R[5];
  const double fbtl = L[4] * L[1] - bnc * L[2];
  const double fbul = L[5] * L[1] - bnc * L[3];
  const double fenl = 2.0 * pml * L[1] - bnc * vbl;
  const double fbtr = R[4] * R[1] - bnc * R[2];
  const double fbur = R[5] * R[1] - bnc * R[3];
  const double fenr = 2.0 * pmr * R[1] - bnc * vbr;
  v.f[0][5][i] = 0.5 * (fbtl + fbtr - smax * (R[4] - L[4]));
  v.f[0][6][i] = 0.5 * (fbul + fbur - smax * (R[5] - L[5]));
  v.f[0][7][i] = 0.5 * (fenl + fenr - smax * (pmr - pml));
}

template <int ODR>
__global__ void k_hupdate(View v, double dtdx, double c0, double c1)
{
  if (v.ctl->done) return;
  const int i = GH + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= v.g.nx - GH) return;
  double nv[3];
#pragma unroll
  for (int q = 0; q < 3; q++) {
    const int m = 5 + q;
    nv[q] = rk_combine(v.u[m][i], v.u0[m][i], -dtdx * d4<ODR>(v.f[0][m], i, 1), c0, c1);
  }
#pragma unroll
  for (int q = 0; q < 3; q++) v.u[5 + q][i] = nv[q];
}

}  // namespace qas
