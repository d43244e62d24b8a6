// qas_hall.cuh -- Hall term of the 1D Hall driver on sm_100a: HMHD1D::hall_
// (1D/SERIAL/h-shock/hmhd1d_solve.cpp:138-264) and HMHD1D::haldt
// (1D/SERIAL/h-shock/hmhd1d_class.cpp:3-13).
//
// With an electron inertia length de != 0, the by/bz fluxes of hall_ and of the 1D ideal
// step get HMHD1D::crcte (hmhd1d_solve.cpp:275-300): Enew solves (1 - de^2 d2/dx2) Enew = Eorg by
// the reference's conjugate-gradient loop (eorg2enew_cg, :326-403) in one CTA -- the vector
// updates in parallel, every sum (numer, denom, anorm, anormf) by one thread in index order, as
// the reference accumulates them -- so the iterates and the stop test are bit-identical.
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

// bc1d (common/common_func.c:34-58) of one array with any flag (others leave the ghosts alone);
// threads 0..GH-1 fill one lower and one upper ghost each, sources are interior cells
__device__ __forceinline__ void bc1d_any(double *f, int nx, int dn, int t)
{
  if (t >= GH) return;
  if (dn == 0) {
    f[t] = f[nx - 2 * GH + t];
    f[nx - 1 - t] = f[2 * GH - 1 - t];
  } else if (dn == 1 || dn == -1) {
    f[t] = dn * f[2 * GH - 1 - t];
    f[nx - 1 - t] = dn * f[nx - 2 * GH + t];
  } else if (dn == 2 || dn == -2) {
    f[t] = 0.25 * (2 + dn) * f[GH];
    f[nx - 1 - t] = 0.25 * (2 + dn) * f[nx - 1 - GH];
  }
}

// df2[ODR-1] (common/common_interp.h:27-35)
template <int ODR>
__device__ __forceinline__ double d2f(const double *f, int i)
{
  if (ODR >= 3) return (-(f[i + 2] + f[i - 2]) + 16.0 * (f[i + 1] + f[i - 1]) - 30.0 * f[i]) / 12.0;
  return (f[i + 1] + f[i - 1]) - 2.0 * f[i];
}

// crcte of one flux pair, one CTA: fbt = the by or bz flux, fen = the energy flux, bt = by or bz,
// dn = the flag product, fac = de^2/dx^2; eorg, enew, rk, pk, ap = scratch arrays of nx doubles
template <int ODR>
__global__ void __launch_bounds__(1024) k_crcte(View v, double *fbt, double *fen, const double *bt, int dn,
                                                double fac, double *eorg, double *enew, double *rk, double *pk,
                                                double *ap)
{
  if (v.ctl->done) return;
  const int nx = v.g.nx, t = threadIdx.x, nt = blockDim.x;
  const double one = 1.0, eps = 1e-8;
  __shared__ double s_numer, s_anormf, s_coef, s_coef2;
  __shared__ int s_go;
  for (int i = t; i < nx; i += nt) eorg[i] = enew[i] = fbt[i];
  __syncthreads();
  bc1d_any(enew, nx, dn, t);
  __syncthreads();
  for (int i = GH + t; i < nx - GH; i += nt) {
    const double r = one * eorg[i] - (one * enew[i] - fac * d2f<ODR>(enew, i));
    rk[i] = r;
    pk[i] = r;
  }
  __syncthreads();
  if (t == 0) {
    double numer = 0.0, anormf = 0.0;
    for (int i = GH; i < nx - GH; i++) {
      numer += rk[i] * rk[i];
      anormf += fabs(rk[i]);
    }
    s_numer = numer;
    s_anormf = anormf;
  }
  __syncthreads();
  int cnt = 0;  // thread 0's copy decides
  const int cmax = nx;
  for (;;) {
    bc1d_any(pk, nx, dn, t);
    __syncthreads();
    for (int i = GH + t; i < nx - GH; i += nt) ap[i] = (one * pk[i] - fac * d2f<ODR>(pk, i));
    __syncthreads();
    if (t == 0) {
      double denom = 0.0;
      for (int i = GH; i < nx - GH; i++) denom += pk[i] * ap[i];
      s_coef = (denom == 0) ? 0 : s_numer / denom;
    }
    __syncthreads();
    const double coef = s_coef;
    for (int i = GH + t; i < nx - GH; i += nt) {
      enew[i] += coef * pk[i];
      rk[i] -= coef * ap[i];
    }
    __syncthreads();
    if (t == 0) {
      double anorm = 0.0, numer = 0.0;
      for (int i = GH; i < nx - GH; i++) anorm += fabs(rk[i]);
      const double denom = s_numer;
      for (int i = GH; i < nx - GH; i++) numer += rk[i] * rk[i];
      s_numer = numer;
      s_coef2 = (denom == 0) ? 0 : numer / denom;
      s_go = (anorm > eps * s_anormf) && (++cnt < cmax);
    }
    __syncthreads();
    const double coef2 = s_coef2;
    for (int i = GH + t; i < nx - GH; i += nt) pk[i] = rk[i] + coef2 * pk[i];
    __syncthreads();
    if (!s_go) break;
  }
  bc1d_any(enew, nx, dn, t);
  __syncthreads();
  for (int i = 1 + t; i < nx; i += nt) {
    const double dd = enew[i] - eorg[i];
    const double bb = 0.5 * (bt[i - 1] + bt[i]);
    fbt[i] = enew[i];
    fen[i] += dd * bb;
  }
}

}  // namespace qas
