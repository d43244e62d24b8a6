// qas_dissip.cuh -- visco-resistive update of the 2D and 3D drivers on sm_100a:
// DMHD2D::dsptv (2D/SERIAL/MRX/dmhd2d_solve.cpp:3-151) and DMHD3D::dsptv
// (3D/MPI/MRX/dmhd3d_solve.cpp:3-179) with uniform nu, eta, sub-cycled as in
// DMHD2D::exec_ (2D/SERIAL/MRX/dmhd2d_class.cpp:19-26) and DMHD3D::exec_
// (3D/MPI/MRX/dmhd3d_class.cpp:20-28).
#pragma once

#include "qas_kernels.cuh"

namespace qas {

// Extra device control for the sub-cycles: ncmax and dt/ncmax of the current step.
struct DCtl {
  int ncmax;
  int pad;
  double sdt;      // dt/ncmax
  double sdtd[3];  // sdt*idx, sdt*idy, sdt*idz (dtdx = dt*idx as in dsptv)
};

// setdc + ncmax = 1 + (int)(2*(dcmax*dt)/(dr*dr))
__global__ void k_dsub_setup(View v, DCtl *dc, double dcmax, double dr, double idx, double idy, int cap,
                             double idz = 0.0)
{
  if (v.ctl->done) return;
  const double dt = v.ctl->dt;
  int ncmax = 0;
  if (dcmax > 1e-15) ncmax = 1 + (int)(2 * (dcmax * dt) / (dr * dr));
  if (ncmax > cap) {
    atomicOr(&v.ctl->err, 4);
    ncmax = cap;
  }
  dc->ncmax = ncmax;
  dc->sdt = ncmax > 0 ? dt / ncmax : 0.0;
  dc->sdtd[0] = dc->sdt * idx;
  dc->sdtd[1] = dc->sdt * idy;
  dc->sdtd[2] = dc->sdt * idz;
}

// host-supplied dt for one dsptv(dt) call
__global__ void k_dsub_fixed(View v, DCtl *dc, double dt, double idx, double idy, double idz)
{
  dc->ncmax = 1;
  dc->sdt = dt;
  dc->sdtd[0] = dt * idx;
  dc->sdtd[1] = dt * idy;
  dc->sdtd[2] = dt * idz;
}

#define QAS_DSUB_GUARD()                        \
  if (v.ctl->done || nc >= dc->ncmax) return;

// velocity at every cell (vlcty, common/mhd_class.hpp:59-65)
__global__ void k_dvel(View v, const DCtl *dc, int nc)
{
  QAS_DSUB_GUARD();
  QAS_CELL_INDEX();
  const long long c = cidx(v.g, i, j, k);
  const double iro = 1.0 / v.u[0][c];
  v.vx[c] = v.u[1][c] * iro;
  v.vy[c] = v.u[2][c] * iro;
  v.vz[c] = v.u[3][c] * iro;
}

// eta*J on the CT edges, mhd_ct_eres (common/mhd_func.c:78-106): in 2D with zoffset = 0 and
// idz = 0 (dmhd2d_solve.cpp:46-54), in 3D with the real z stencils (dmhd3d_solve.cpp:48-57)
template <int ODR>
__global__ void k_eres(View v, const DCtl *dc, int nc, double eta0, double idx, double idy, double idz3 = 0.0)
{
  QAS_DSUB_GUARD();
  QAS_CELL_INDEX();
  const Geo &g = v.g;
  if (i < 2 || i >= g.nx - 1 || j < 2 || j >= g.ny - 1) return;
  if (g.dim == 3 && (k < 2 || k >= g.nz - 1)) return;
  const long long c = cidx(g, i, j, k);
  const long long sy = g.s[1];
  const double *bx = v.u[4], *by = v.u[5], *bz = v.u[6];
  double dbxz, dbyz, idz;
  if (g.dim == 3) {
    const long long sz = g.s[2];
    idz = idz3;
    dbxz = dfc<ODR>(bx[c - 2 * sz], bx[c - sz], bx[c], bx[c + sz]);
    dbyz = dfc<ODR>(by[c - 2 * sz], by[c - sz], by[c], by[c + sz]);
  } else {
    // derivatives along the absent z axis see four equal values
    idz = 0.0;
    dbxz = dfc<ODR>(bx[c], bx[c], bx[c], bx[c]);
    dbyz = dfc<ODR>(by[c], by[c], by[c], by[c]);
  }
  const double jx = dfc<ODR>(bz[c - 2 * sy], bz[c - sy], bz[c], bz[c + sy]) * idy - dbyz * idz;
  const double jy = dbxz * idz - dfc<ODR>(bz[c - 2], bz[c - 1], bz[c], bz[c + 1]) * idx;
  const double jz = dfc<ODR>(by[c - 2], by[c - 1], by[c], by[c + 1]) * idx -
                    dfc<ODR>(bx[c - 2 * sy], bx[c - sy], bx[c], bx[c + sy]) * idy;
  if (v.eta) {  // per-cell resistivity averaged to the edges (mhd_func.c:103-105)
    const double *et = v.eta;
    const long long xo = 1, yo = sy, zo = g.dim == 3 ? g.s[2] : 0;
    v.ex[c] = 0.25 * (et[c - yo - zo] + et[c - zo] + et[c - yo] + et[c]) * jx;
    v.ey[c] = 0.25 * (et[c - zo - xo] + et[c - xo] + et[c - zo] + et[c]) * jy;
    v.ez[c] = 0.25 * (et[c - xo - yo] + et[c - yo] + et[c - xo] + et[c]) * jz;
    return;
  }
  const double e = eta0;
  v.ex[c] = 0.25 * (e + e + e + e) * jx;
  v.ey[c] = 0.25 * (e + e + e + e) * jy;
  v.ez[c] = 0.25 * (e + e + e + e) * jz;
}

// viscous face flux at i-1/2 along stride xo with transverse strides yo, zo (0 for the
// absent axis), calc_flux_viscous (common/mhd_flux.c:700-752); returns fmx, fmy, fmz, fen.
template <int ODR>
__device__ __forceinline__ void visc_flux(const double *vx, const double *vy, const double *vz, long long c,
                                          double rnu, double idx, double idy, double idz, long long xo, long long yo,
                                          long long zo, double &fmx, double &fmy, double &fmz, double &fen)
{
  const double c2 = 2. / 3., c4 = 4. / 3.;
  double a[4], b[4], d[4];
#pragma unroll
  for (int m = 0; m < 4; m++) {
    a[m] = vx[c + (m - 2) * xo];
    b[m] = vy[c + (m - 2) * xo];
    d[m] = vz[c + (m - 2) * xo];
  }
  const double vx0 = fcen<ODR>(a[0], a[1], a[2], a[3]);
  const double vy0 = fcen<ODR>(b[0], b[1], b[2], b[3]);
  const double vz0 = fcen<ODR>(d[0], d[1], d[2], d[3]);
  const double dvxdx = dfc<ODR>(a[0], a[1], a[2], a[3]) * idx;
  const double dvydx = dfc<ODR>(b[0], b[1], b[2], b[3]) * idx;
  const double dvzdx = dfc<ODR>(d[0], d[1], d[2], d[3]) * idx;
  double t[4];
#pragma unroll
  for (int m = 0; m < 4; m++) t[m] = 0.5 * (vx[c + (m - 2) * xo + yo] - vx[c + (m - 2) * xo - yo]);
  const double dvxdy = fcen<ODR>(t[0], t[1], t[2], t[3]) * idy;
#pragma unroll
  for (int m = 0; m < 4; m++) t[m] = 0.5 * (vy[c + (m - 2) * xo + yo] - vy[c + (m - 2) * xo - yo]);
  const double dvydy = fcen<ODR>(t[0], t[1], t[2], t[3]) * idy;
#pragma unroll
  for (int m = 0; m < 4; m++) t[m] = 0.5 * (vx[c + (m - 2) * xo + zo] - vx[c + (m - 2) * xo - zo]);
  const double dvxdz = fcen<ODR>(t[0], t[1], t[2], t[3]) * idz;
#pragma unroll
  for (int m = 0; m < 4; m++) t[m] = 0.5 * (vz[c + (m - 2) * xo + zo] - vz[c + (m - 2) * xo - zo]);
  const double dvzdz = fcen<ODR>(t[0], t[1], t[2], t[3]) * idz;
  fmx = -rnu * (c4 * dvxdx - c2 * (dvydy + dvzdz));
  fmy = -rnu * (dvydx + dvxdy);
  fmz = -rnu * (dvzdx + dvxdz);
  fen = fmx * vx0 + fmy * vy0 + fmz * vz0;
}

// resistive face flux, calc_flux_resistive (common/mhd_flux.c:754-782): B pair (by,bz) with
// offsets yo (of by) and zo (of bz), E pair (ey averaged over zo, ez over yo).
template <int ODR>
__device__ __forceinline__ void resist_flux(const double *by, const double *bz, const double *ey, const double *ez,
                                            long long c, long long xo, long long yo, long long zo, double &fby,
                                            double &fbz, double &fen)
{
  const double ey0 = 0.5 * (ey[c] + ey[c + zo]);
  const double ez0 = 0.5 * (ez[c] + ez[c + yo]);
  double byi[4], bzi[4];
#pragma unroll
  for (int m = 0; m < 4; m++) {
    const long long p = c + (m - 2) * xo;
    byi[m] = 0.5 * (by[p] + by[p + yo]);
    bzi[m] = 0.5 * (bz[p] + bz[p + zo]);
  }
  const double by0 = fcen<ODR>(byi[0], byi[1], byi[2], byi[3]);
  const double bz0 = fcen<ODR>(bzi[0], bzi[1], bzi[2], bzi[3]);
  fby = -ez0;
  fbz = +ey0;
  fen = ey0 * bz0 - ez0 * by0;
}

template <int ODR>
__global__ void k_dflux(View v, const DCtl *dc, int nc, double nu0, double idx, double idy, double idz3 = 0.0)
{
  QAS_DSUB_GUARD();
  QAS_CELL_INDEX();
  const Geo &g = v.g;
  if (i < 2 || i >= g.nx - 1 || j < 2 || j >= g.ny - 1) return;
  const bool d3 = g.dim == 3;
  if (d3 && (k < 2 || k >= g.nz - 1)) return;
  const long long c = cidx(g, i, j, k);
  const long long sy = g.s[1];
  const long long sz = d3 ? g.s[2] : 0;  // the absent axis has offset 0 and idz 0 in 2D
  const double idz = d3 ? idz3 : 0.0;
  const double *ro = v.u[0];
  double fmx, fmy, fmz, fenv, fby, fbz, fenr;
  // x face (dmhd2d_solve.cpp:70-82, dmhd3d_solve.cpp:72-84)
  const double *nua = v.nu;  // per-cell viscosity, or the uniform nu0
  double rnu = nua ? 0.5 * (ro[c - 1] * nua[c - 1] + ro[c] * nua[c]) : 0.5 * (ro[c - 1] * nu0 + ro[c] * nu0);
  visc_flux<ODR>(v.vx, v.vy, v.vz, c, rnu, idx, idy, idz, 1, sy, sz, fmx, fmy, fmz, fenv);
  resist_flux<ODR>(v.u[5], v.u[6], v.ey, v.ez, c, 1, sy, sz, fby, fbz, fenr);
  v.f[0][0][c] = 0.0 + 0.0;
  v.f[0][1][c] = fmx + 0.0;
  v.f[0][2][c] = fmy + 0.0;
  v.f[0][3][c] = fmz + 0.0;
  v.f[0][5][c] = 0.0 + fby;
  v.f[0][6][c] = 0.0 + fbz;
  v.f[0][7][c] = fenv + fenr;
  // y face (dmhd2d_solve.cpp:83-94, dmhd3d_solve.cpp:86-97)
  rnu = nua ? 0.5 * (ro[c - sy] * nua[c - sy] + ro[c] * nua[c]) : 0.5 * (ro[c - sy] * nu0 + ro[c] * nu0);
  visc_flux<ODR>(v.vy, v.vz, v.vx, c, rnu, idy, idz, idx, sy, sz, 1, fmx, fmy, fmz, fenv);
  resist_flux<ODR>(v.u[6], v.u[4], v.ez, v.ex, c, sy, sz, 1, fby, fbz, fenr);
  v.f[1][0][c] = 0.0 + 0.0;
  v.f[1][2][c] = fmx + 0.0;
  v.f[1][3][c] = fmy + 0.0;
  v.f[1][1][c] = fmz + 0.0;
  v.f[1][6][c] = 0.0 + fby;
  v.f[1][4][c] = 0.0 + fbz;
  v.f[1][7][c] = fenv + fenr;
  if (d3) {  // z face (dmhd3d_solve.cpp:99-110)
    rnu = nua ? 0.5 * (ro[c - sz] * nua[c - sz] + ro[c] * nua[c]) : 0.5 * (ro[c - sz] * nu0 + ro[c] * nu0);
    visc_flux<ODR>(v.vz, v.vx, v.vy, c, rnu, idz, idx, idy, sz, 1, sy, fmx, fmy, fmz, fenv);
    resist_flux<ODR>(v.u[4], v.u[5], v.ex, v.ey, c, sz, 1, sy, fby, fbz, fenr);
    v.f[2][0][c] = 0.0 + 0.0;
    v.f[2][3][c] = fmx + 0.0;
    v.f[2][1][c] = fmy + 0.0;
    v.f[2][2][c] = fmz + 0.0;
    v.f[2][4][c] = 0.0 + fby;
    v.f[2][5][c] = 0.0 + fbz;
    v.f[2][7][c] = fenv + fenr;
  }
}

// RK update of the 2D dsptv (dmhd2d_solve.cpp:107-146)
template <int ODR>
__device__ __forceinline__ void dupdate2(const View &v, const DCtl *dc, int i, int j, double c0, double c1)
{
  const Geo &g = v.g;
  const long long c = cidx(g, i, j, 0);
  const long long sy = g.s[1];
  const double dtdx = dc->sdtd[0], dtdy = dc->sdtd[1];
  const bool ci = i < g.nx - GH, cj = j < g.ny - GH;
  // all new values before the first store (see update_body)
  const int cen[6] = {0, 1, 2, 3, 6, 7};
  double nv[6], nbx = 0.0, nby = 0.0;
  if (ci && cj) {
#pragma unroll
    for (int q = 0; q < 6; q++) {
      const int m = cen[q];
      const double du0 = d4<ODR>(v.f[0][m], c, 1);
      const double du1 = d4<ODR>(v.f[1][m], c, sy);
      nv[q] = rk_combine(v.u[m][c], v.u0[m][c], (-dtdx * du0 - dtdy * du1), c0, c1);
    }
  }
  if (cj) {
    const double du = d4<ODR>(v.ez, c, sy);
    nbx = rk_combine(v.u[4][c], v.u0[4][c], -(+dtdy) * du, c0, c1);
  }
  if (ci) {
    const double du = d4<ODR>(v.ez, c, 1);
    nby = rk_combine(v.u[5][c], v.u0[5][c], -(-dtdx) * du, c0, c1);
  }
  if (ci && cj) {
#pragma unroll
    for (int q = 0; q < 6; q++) v.u[cen[q]][c] = nv[q];
  }
  if (cj) v.u[4][c] = nbx;
  if (ci) v.u[5][c] = nby;
}

// RK update of the 3D dsptv (dmhd3d_solve.cpp:114-167): mhd_updt3d on ro,mx,my,mz,en over the
// interior, mhd_updt3d_ctb on bx (one extra face along x), by (along y) and bz (along z)
template <int ODR>
__device__ __forceinline__ void dupdate3(const View &v, const DCtl *dc, int i, int j, int k, double c0, double c1)
{
  const Geo &g = v.g;
  const long long c = cidx(g, i, j, k);
  const long long sy = g.s[1], sz = g.s[2];
  const double dtdx = dc->sdtd[0], dtdy = dc->sdtd[1], dtdz = dc->sdtd[2];
  const bool ci = i < g.nx - GH, cj = j < g.ny - GH, ck = k < g.nz - GH;
  const int cen[5] = {0, 1, 2, 3, 7};
  double nv[5], nb[3] = {0.0, 0.0, 0.0};
  if (ci && cj && ck) {
#pragma unroll
    for (int q = 0; q < 5; q++) {
      const int m = cen[q];
      const double du0 = d4<ODR>(v.f[0][m], c, 1);
      const double du1 = d4<ODR>(v.f[1][m], c, sy);
      const double du2 = d4<ODR>(v.f[2][m], c, sz);
      nv[q] = rk_combine(v.u[m][c], v.u0[m][c], (-dtdx * du0 - dtdy * du1 - dtdz * du2), c0, c1);
    }
  }
  if (cj && ck) {
    const double du0 = +d4<ODR>(v.ez, c, sy);
    const double du1 = -d4<ODR>(v.ey, c, sz);
    nb[0] = rk_combine(v.u[4][c], v.u0[4][c], -dtdy * du0 - dtdz * du1, c0, c1);
  }
  if (ci && ck) {
    const double du0 = +d4<ODR>(v.ex, c, sz);
    const double du1 = -d4<ODR>(v.ez, c, 1);
    nb[1] = rk_combine(v.u[5][c], v.u0[5][c], -dtdz * du0 - dtdx * du1, c0, c1);
  }
  if (ci && cj) {
    const double du0 = +d4<ODR>(v.ey, c, 1);
    const double du1 = -d4<ODR>(v.ex, c, sy);
    nb[2] = rk_combine(v.u[6][c], v.u0[6][c], -dtdx * du0 - dtdy * du1, c0, c1);
  }
  if (ci && cj && ck) {
#pragma unroll
    for (int q = 0; q < 5; q++) v.u[cen[q]][c] = nv[q];
  }
  if (cj && ck) v.u[4][c] = nb[0];
  if (ci && ck) v.u[5][c] = nb[1];
  if (ci && cj) v.u[6][c] = nb[2];
}

template <int ODR>
__global__ void k_dupdate(View v, const DCtl *dc, int nc, double c0, double c1)
{
  QAS_DSUB_GUARD();
  const Geo &g = v.g;
  const int i = GH + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = GH + blockIdx.y * blockDim.y + threadIdx.y;
  const int kt = blockIdx.z * blockDim.z + threadIdx.z;
  if (i > g.nx - GH || j > g.ny - GH) return;
  if (g.dim == 3) {
    const int k = GH + kt;
    if (k > g.nz - GH) return;
    dupdate3<ODR>(v, dc, i, j, k, c0, c1);
  } else {
    if (kt > 0) return;
    dupdate2<ODR>(v, dc, i, j, c0, c1);
  }
}

__global__ void k_dbound(View v, const DCtl *dc, int nc)
{
  QAS_DSUB_GUARD();
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= shell_cells(v.g)) return;
  int i, j, k;
  shell_cell(v.g, t, i, j, k);
  bound_body(v, i, j, k);
}

// ut = u at the start of each dsptv call
__global__ void k_dcopy(View v, const DCtl *dc, int nc)
{
  QAS_DSUB_GUARD();
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= v.g.nd) return;
#pragma unroll
  for (int m = 0; m < 8; m++) v.u0[m][c] = v.u[m][c];
}

}  // namespace qas
