// qas_kernels.cuh -- kernels of one SSP-RK stage of the qasMHD step on sm_100a.
//
// Data layout in HBM (one pool per context): structure-of-arrays FP64, one
// array per field in the reference's ghost-padded order ss = nx*(ny*k+j)+i,
// so host<->device copies are single memcpys.  Per stage:
//   k_prim      cell-centre B (with its ghost fill folded in as a gather) and
//               primitives for every cell                     (mhd2d_solve.cpp:51-89)
//   k_dv        shock detector dv with its ghost fill         (:105-125)  MLAU/LHLLD only
//   k_lr        characteristic WCNS face states of each cell + CUCT induction states
//   k_flux      Riemann flux per face, central/upwind split of the induction flux
//   k_emf       corner EMFs with the CUCT weight computed in place
//   k_update    SSP-RK combine of the cell-centred fields and the CT update of B
//   k_bound     ghost fill of the state as a gather over precomputed per-axis maps
#pragma once

#include "qas_device.cuh"

// Resident-block caps of the memory-bound kernels (0: no launch bound, the compiler's choice).
// Measured on B200 (OT 1024^2 / KH 160^3 per launch): k_update at 16 blocks (32 registers, a
// few spills) 0.0887 -> 0.0804 ms / 0.383 -> 0.328 ms, k_prim at 16 0.125 -> 0.113 ms in 3D;
// k_emf is slower capped (0.230 -> 0.250 ms at 12), so it keeps the compiler's choice.
#ifndef QAS_PRIM_MINB
#define QAS_PRIM_MINB 16
#endif
#ifndef QAS_EMF_MINB
#define QAS_EMF_MINB 0
#endif
#ifndef QAS_UPDATE_MINB
#define QAS_UPDATE_MINB 16
#endif
#if QAS_PRIM_MINB > 0
#define QAS_PRIM_BOUNDS __launch_bounds__(128, QAS_PRIM_MINB)
#else
#define QAS_PRIM_BOUNDS
#endif
#if QAS_EMF_MINB > 0
#define QAS_EMF_BOUNDS __launch_bounds__(128, QAS_EMF_MINB)
#else
#define QAS_EMF_BOUNDS
#endif
#if QAS_UPDATE_MINB > 0
#define QAS_UPDATE_BOUNDS __launch_bounds__(128, QAS_UPDATE_MINB)
#else
#define QAS_UPDATE_BOUNDS
#endif

namespace qas {

constexpr int GH = 4;  // ghost cells per side

struct Geo {
  int dim, nx, ny, nz;
  long long nd;
  long long s[3];  // strides of x, y, z
  int n[3];        // extents incl. ghosts
};

// Device control block of the exec_ loop (dt, tim, n kept on the device).
struct Ctl {
  double dt;
  double tim;
  double tmax;
  double dtd[3];                 // dt/dx, dt/dy, dt/dz of the current step
  unsigned long long vmax_bits;  // setdt reduction (positive doubles order like their bits)
  int n, nmax, done, first;
  int err;                       // latched device error bits
  int pad;
};

// Ghost-fill maps: for group G (0 state, 1 cell-centre B, 2 dv), field m, axis a and
// index i along that axis: the source index and factor after all fill passes of that
// axis (built on the host by replaying the reference's passes symbolically).
struct Maps {
  const int *src;
  const double *fac;
  int nmax;
};

struct View {
  Geo g;
  int rmn, odr, rk, ctw;
  double gam;
  double dx, dy, dz;
  double *u[8];    // state ro,mx,my,mz,bx,by,bz,en
  double *u0[8];   // state at the start of the step (ut)
  double *vx, *vy, *vz, *pr, *cx, *cy, *cz;
  double *dv[3];
  double *vl[7], *vr[7];  // face states of each cell along the current axis
  double *ql[2], *qr[2];  // induction-flux states
  double *f[3][8];        // face fluxes per direction
  double *fc[3][2];       // central parts of the induction fluxes per direction
  double *ex, *ey, *ez;
  Ctl *ctl;
  Maps maps;
  double dr;  // min cell size, the dr of setdt
  // gravity drivers (2D/SERIAL/RTI, 3D/MPI/RTI): potential phi_g per cell, or null; and
  // (2-gam)/(gam-1) of their boundary energy rule
  const double *phi;
  double gfac;
  // per-cell viscosity / resistivity of the dissipative drivers (the API's nu/eta), or null
  // for the uniform nu0/eta0 of the run options
  const double *nu, *eta;
  int recon;  // face-value reconstruction: 0 characteristic (mhd_m/a_reconst), 1 primitive (mhd_reconst),
              // 2 Athena-type characteristic (mhd_c_reconst)
};

__device__ __forceinline__ long long cidx(const Geo &g, int i, int j, int k)
{
  return (long long)g.nx * ((long long)g.ny * k + j) + i;
}

__device__ __forceinline__ int map_src(const Maps &m, int G, int f, int a, int i)
{
  return m.src[((G * 8 + f) * 3 + a) * m.nmax + i];
}
__device__ __forceinline__ double map_fac(const Maps &m, int G, int f, int a, int i)
{
  return m.fac[((G * 8 + f) * 3 + a) * m.nmax + i];
}

// source cell and factor of (i,j,k) for group G / field f
__device__ __forceinline__ void gather_src(const View &v, int G, int f, int i, int j, int k, int &si, int &sj, int &sk,
                                           double &fac)
{
  si = map_src(v.maps, G, f, 0, i);
  fac = map_fac(v.maps, G, f, 0, i);
  sj = j;
  sk = k;
  if (v.g.dim >= 2) {
    sj = map_src(v.maps, G, f, 1, j);
    fac = fac * map_fac(v.maps, G, f, 1, j);
  }
  if (v.g.dim >= 3) {
    sk = map_src(v.maps, G, f, 2, k);
    fac = fac * map_fac(v.maps, G, f, 2, k);
  }
}

// cell of this thread: blocks tile the grid in x, y and z (tile = blockDim)
#define QAS_CELL_INDEX()                                              \
  const int i = blockIdx.x * blockDim.x + threadIdx.x;                \
  const int j = blockIdx.y * blockDim.y + threadIdx.y;                \
  const int k = blockIdx.z * blockDim.z + threadIdx.z;                \
  if (i >= v.g.nx || j >= v.g.ny || k >= v.g.nz) return;

// a cell no ghost-fill pass writes: every per-axis map is the identity with factor 1 there,
// so the gather reduces to the cell itself (1.0*x == x bit for bit)
__device__ __forceinline__ bool interior_cell(const Geo &g, int i, int j, int k)
{
  return i >= GH && i < g.nx - GH && (g.dim < 2 || (j >= GH && j < g.ny - GH)) &&
         (g.dim < 3 || (k >= GH && k < g.nz - GH));
}

// ---------------------------------------------------------------------------
// primitives + cell-centre B (prmtv, bcell/bb2cc + bound(cx,cy,cz))
// ---------------------------------------------------------------------------
// WB: store the gravity drivers' rounded energy back (the stage's prmtv); false for a read-only
// evaluation of the primitives (qas_primitives)
template <int ODR, bool WB = true>
__device__ __forceinline__ void prim_body(const View &v, int i, int j, int k)
{
  const Geo &g = v.g;
  const long long c = cidx(g, i, j, k);
  double cx, cy, cz;
  if (g.dim == 1) {
    cx = v.u[4][c];
    cy = v.u[5][c];
    cz = v.u[6][c];
  } else if (interior_cell(g, i, j, k)) {
    const double *bx = v.u[4], *by = v.u[5];
    const long long sy = g.s[1];
    cx = fcen<ODR>(bx[c - 1], bx[c], bx[c + 1], bx[c + 2]);
    cy = fcen<ODR>(by[c - sy], by[c], by[c + sy], by[c + 2 * sy]);
    if (g.dim == 3) {
      const double *bz = v.u[6];
      const long long sz = g.s[2];
      cz = fcen<ODR>(bz[c - sz], bz[c], bz[c + sz], bz[c + 2 * sz]);
    } else {
      cz = v.u[6][c];
    }
  } else {
    int si, sj, sk;
    double fac;
    gather_src(v, 1, 0, i, j, k, si, sj, sk, fac);
    long long s = cidx(g, si, sj, sk);
    const double *bx = v.u[4];
    cx = fac * fcen<ODR>(bx[s - 1], bx[s], bx[s + 1], bx[s + 2]);
    gather_src(v, 1, 1, i, j, k, si, sj, sk, fac);
    s = cidx(g, si, sj, sk);
    const double *by = v.u[5];
    const long long sy = g.s[1];
    cy = fac * fcen<ODR>(by[s - sy], by[s], by[s + sy], by[s + 2 * sy]);
    if (g.dim == 3) {
      gather_src(v, 1, 2, i, j, k, si, sj, sk, fac);
      s = cidx(g, si, sj, sk);
      const double *bz = v.u[6];
      const long long sz = g.s[2];
      cz = fac * fcen<ODR>(bz[s - sz], bz[s], bz[s + sz], bz[s + 2 * sz]);
    } else {
      cz = v.u[6][c];
    }
  }
  const double ro = v.u[0][c];
  // gravity drivers: en -= ro*phi; prmtv; en += ro*phi, which leaves en rounded in place
  // (2D/SERIAL/RTI/mhd2d_solve.cpp:85-88, 3D/MPI/RTI/mhd3d_solve.cpp:95-97)
  double en = v.u[7][c];
  if (v.phi) en = en - ro * v.phi[c];
  const double iro = 1.0 / ro;
  const double vx = v.u[1][c] * iro;
  const double vy = v.u[2][c] * iro;
  const double vz = v.u[3][c] * iro;
  const double v2 = vx * vx + vy * vy + vz * vz;
  const double b2 = cx * cx + cy * cy + cz * cz;
  const double pr = (v.gam - 1) * (en - 0.5 * (ro * v2 + b2));
  if (WB && v.phi) v.u[7][c] = en + ro * v.phi[c];
  v.vx[c] = vx;
  v.vy[c] = vy;
  v.vz[c] = vz;
  v.pr[c] = pr;
  v.cx[c] = cx;
  v.cy[c] = cy;
  v.cz[c] = cz;
  // latch a device error for a broken interior state (results are not altered)
  bool interior = i >= GH && i < g.nx - GH && (g.dim < 2 || (j >= GH && j < g.ny - GH)) &&
                  (g.dim < 3 || (k >= GH && k < g.nz - GH));
  if (interior && !(ro > 0.0 && pr > 0.0 && isfinite(vx) && isfinite(vy) && isfinite(vz))) atomicOr(&v.ctl->err, 1);
}
template <int ODR>
__global__ void QAS_PRIM_BOUNDS k_prim(View v)
{
  if (v.ctl->done) return;
  QAS_CELL_INDEX();
  prim_body<ODR>(v, i, j, k);
}
// the primitives of the current state without touching it (no stop-flag guard)
template <int ODR>
__global__ void k_prim_eval(View v)
{
  QAS_CELL_INDEX();
  prim_body<ODR, false>(v, i, j, k);
}

// ---------------------------------------------------------------------------
// shock detector dv (mhd2d_solve.cpp:105-125, mhd3d_solve.cpp:138-164)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void dv_body(const View &v, int i, int j, int k)
{
  const Geo &g = v.g;
  const long long c = cidx(g, i, j, k);
  const double *vel[3] = {v.vx, v.vy, v.vz};
  if (interior_cell(g, i, j, k)) {
#pragma unroll
    for (int a = 0; a < 3; a++) {
      if (a >= g.dim) break;
      const long long st = g.s[a];
      const double *p = vel[a];
      v.dv[a][c] = qmin((p[c + st] - p[c]), (p[c] - p[c - st]));
    }
    return;
  }
#pragma unroll
  for (int a = 0; a < 3; a++) {
    if (a >= g.dim) break;
    int si, sj, sk;
    double fac;
    gather_src(v, 2, a, i, j, k, si, sj, sk, fac);
    const long long s = cidx(g, si, sj, sk);
    const long long st = g.s[a];
    const double *p = vel[a];
    const double raw = qmin((p[s + st] - p[s]), (p[s] - p[s - st]));
    v.dv[a][c] = fac * raw;
  }
}
__global__ void k_dv(View v)
{
  if (v.ctl->done) return;
  QAS_CELL_INDEX();
  dv_body(v, i, j, k);
}

// ---------------------------------------------------------------------------
// face states of each cell along axis A (mhd_lrstate + mhd_lr_fb)
// ---------------------------------------------------------------------------
// 6 resident blocks (80 registers, 52 B spilled to L1): 0.498 -> 0.478 ms per launch at KH 160^3,
// unchanged in 2D; 5 blocks (96 registers) and 4 (118) are slower
#ifndef QAS_LR_MINB
#define QAS_LR_MINB 6
#endif

// stencil accessor of k_lr: field f of (ro, vn, vb, vc, cb, cc, pr) along axis A at point m
// (0..4) of cell c; the field pointers are read from the kernel's View parameter at each use,
// so no pointer stays live in registers
template <int A>
struct LrStencil {
  const View &v;
  long long c, s;
  __device__ __forceinline__ const double *field(int f) const
  {
    constexpr int B = (A + 1) % 3, C = (A + 2) % 3;
    switch (f) {
      case 0: return v.u[0];
      case 1: return A == 0 ? v.vx : (A == 1 ? v.vy : v.vz);
      case 2: return B == 0 ? v.vx : (B == 1 ? v.vy : v.vz);
      case 3: return C == 0 ? v.vx : (C == 1 ? v.vy : v.vz);
      case 4: return B == 0 ? v.cx : (B == 1 ? v.cy : v.cz);
      case 5: return C == 0 ? v.cx : (C == 1 ? v.cy : v.cz);
      default: return v.pr;
    }
  }
  __device__ __forceinline__ double operator()(int f, int m) const { return __ldg(field(f) + c + (m - 2) * s); }
  // plain load, for reads issued after the face-state stores (kept in order behind them)
  __device__ __forceinline__ double late(int f, int m) const { return field(f)[c + (m - 2) * s]; }
};

// PR: the face-value form, 0 characteristic (mhd_m/a_reconst), 1 primitive (mhd_reconst), 2
// Athena-type characteristic (mhd_c_reconst), -1 chosen at run time by v.recon (the forms whose
// instances may differ per launch); the default kernels take it as a template argument so the
// characteristic code is compiled without the other branches
template <int ODR, int A, int PR = -1, class ST>
__device__ __forceinline__ void lr_cell(const View &v, long long c, long long s, const ST &st, double cnc)
{
  double vl[7], vr[7];
  if (PR == 1 || (PR < 0 && v.recon == 1))
    face_states_prim<ODR>(st, vl, vr);
  else if (PR == 2 || (PR < 0 && v.recon == 2))
    face_states_athena<ODR>(st, cnc, v.gam, vl, vr);
  else
    face_states_grouped<ODR>(st, cnc, v.gam, vl, vr);
#pragma unroll
  for (int m = 0; m < 7; m++) {
    v.vl[m][c] = vl[m];
    v.vr[m][c] = vr[m];
  }
  if (v.g.dim >= 2) {
    // the induction states are read after the face states are stored (keeps their loads from
    // being hoisted over the reconstruction, which would raise register pressure)
    asm volatile("" ::: "memory");
    const double *bnf = v.u[4 + A];
    const double bfl = bnf[c + s], bfr = bnf[c];
    // transverse component t0 = B axis (used in 3D; in 2D along x), t1 = C axis (3D; 2D along y)
#pragma unroll
    for (int t = 0; t < 2; t++) {
      if (v.g.dim == 2 && ((A == 0 && t == 1) || (A == 1 && t == 0))) continue;
      double prod[5], vts[5];
#pragma unroll
      for (int m = 0; m < 5; m++) {
        prod[m] = st.late(4 + t, m) * st.late(1, m);  // bt * vn
        vts[m] = st.late(2 + t, m);                   // vt
      }
      double fl0, fr0, fl1, fr1;
      lin_lr<ODR>(prod, fl0, fr0);
      lin_lr<ODR>(vts, fl1, fr1);
      v.ql[t][c] = fl0 - bfl * fl1;
      v.qr[t][c] = fr0 - bfr * fr1;
    }
  }
}

template <int ODR, int A, int PR = -1>
__device__ __forceinline__ void lr_body(const View &v, int i, int j, int k)
{
  const Geo &g = v.g;
  const int pos = A == 0 ? i : (A == 1 ? j : k);
  const int n = g.n[A];
  if (pos < 2 || pos >= n - 2) return;
  const long long c = cidx(g, i, j, k);
  const long long s = g.s[A];
  const double *cn = A == 0 ? v.cx : (A == 1 ? v.cy : v.cz);
  const LrStencil<A> st{v, c, s};
  lr_cell<ODR, A, PR>(v, c, s, st, cn[c]);
}
template <int ODR, int A, int PR = 0>
__global__ void __launch_bounds__(128, QAS_LR_MINB) k_lr(View v)
{
  if (v.ctl->done) return;
  QAS_CELL_INDEX();
  lr_body<ODR, A, PR>(v, i, j, k);
}

// ---------------------------------------------------------------------------
// Riemann flux per face along axis A (mhd2d_solve.cpp:172-199 and 3D analogues)
// ---------------------------------------------------------------------------
// Stores one face's fluxes as the solver finishes them: F[0..3] to the mass and momentum fluxes
// (normal component at 1+A), F[4] / F[5] minus the central part of the induction flux (also
// stored, fc), F[6] plus the work of gravity.  The central parts come from the induction states
// of the two cells: loaded here (LOADQ, the split form) or handed over in registers (fused).
template <int A, bool LOADQ>
struct FaceSink {
  const View &v;
  long long f, s;
  double ql0, qr0, ql1, qr1;  // induction states when !LOADQ
  double f0;
  __device__ __forceinline__ double central(int t)
  {
    const double l = LOADQ ? v.ql[t][f - s] : (t == 0 ? ql0 : ql1);
    const double r = LOADQ ? v.qr[t][f] : (t == 0 ? qr0 : qr1);
    const double fc = 0.5 * (l + r);
    v.fc[A][t][f] = fc;
    return fc;
  }
  __device__ __forceinline__ void operator()(int m, double x)
  {
    constexpr int B = (A + 1) % 3, C = (A + 2) % 3;
    const int dim = v.g.dim;
    switch (m) {
      case 0:
        v.f[A][0][f] = x;
        f0 = x;
        break;
      case 1: v.f[A][1 + A][f] = x; break;
      case 2: v.f[A][1 + B][f] = x; break;
      case 3: v.f[A][1 + C][f] = x; break;
      case 4: v.f[A][4 + B][f] = (dim == 3 || (dim == 2 && A == 0)) ? x - central(0) : x; break;
      case 5: v.f[A][4 + C][f] = (dim == 3 || (dim == 2 && A == 1)) ? x - central(1) : x; break;
      default:
        // work done by gravity (2D/SERIAL/RTI/mhd2d_solve.cpp:197, :305; 3D/MPI/RTI/mhd3d_solve.cpp:247, :412, :577)
        v.f[A][7][f] = v.phi ? x + f0 * 0.5 * (v.phi[f - s] + v.phi[f]) : x;
        break;
    }
  }
};

template <int RMN, int A>
__device__ __forceinline__ void flux_body(const View &v, int i, int j, int k)
{
  const Geo &g = v.g;
  const int pos = A == 0 ? i : (A == 1 ? j : k);
  const int n = g.n[A];
  if (pos < 3 || pos >= n - 2) return;
  const long long f = cidx(g, i, j, k);
  const long long s = g.s[A];
  constexpr int B = (A + 1) % 3, C = (A + 2) % 3;
  double L[7], R[7];
#pragma unroll
  for (int m = 0; m < 7; m++) {
    L[m] = v.vl[m][f - s];
    R[m] = v.vr[m][f];
  }
  const double bnf = v.u[4 + A][f];
  const double bn = 0.5 * (bnf + bnf);
  double dv0 = 0.0, dv1 = 0.0;
  if (RMN >= 2) {
    const double *vn = A == 0 ? v.vx : (A == 1 ? v.vy : v.vz);
    dv0 = vn[f] - vn[f - s];
    if (g.dim == 2) {
      const double *dt = v.dv[A == 0 ? 1 : 0];
      dv1 = qmin(dt[f - s], dt[f]);
    } else if (g.dim == 3) {
      const double *d1 = v.dv[B], *d2 = v.dv[C];
      dv1 = qmin(qmin(d1[f - s], d1[f]), qmin(d2[f - s], d2[f]));
    }
  }
  riemann_out<RMN>(L, R, bn, v.gam, dv0, dv1, FaceSink<A, true>{v, f, s, 0.0, 0.0, 0.0, 0.0, 0.0});
}
// resident-block caps of the flux kernel per solver, measured on B200 per launch: Roe at 4
// (128 registers, from 162) 0.0906 -> 0.0782 ms (KH 2D 1024^2); HLLD at 8 (64 registers, a
// few spills) 0.0525 -> 0.0501 ms (OT 1024^2); LHLLD at 8 0.181 -> 0.152 ms (KH 3D 128^3)
#ifndef QAS_FLUX_ROE_MINB
#define QAS_FLUX_ROE_MINB 4
#endif
#ifndef QAS_FLUX_HLLD_MINB
#define QAS_FLUX_HLLD_MINB 8
#endif
#ifndef QAS_FLUX_LHLLD_MINB
#define QAS_FLUX_LHLLD_MINB 8
#endif
#define QAS_FLUX_MINB_OF(RMN) ((RMN) == 0 ? QAS_FLUX_ROE_MINB : ((RMN) == 1 ? QAS_FLUX_HLLD_MINB : QAS_FLUX_LHLLD_MINB))
template <int RMN, int A>
__global__ void __launch_bounds__(128, QAS_FLUX_MINB_OF(RMN)) k_flux(View v)
{
  if (v.ctl->done) return;
  QAS_CELL_INDEX();
  flux_body<RMN, A>(v, i, j, k);
}
// MLAU's flux (the largest of the four) is latency-bound at the ~124 registers the compiler
// picks without a bound; capping it for QAS_FLUX_MLAU_MINB resident blocks trades a few spills
// for occupancy (measured on B200, KH 256^3: 1.43 ms -> 1.32 / 1.27 ms per launch at 5 / 6 blocks)
#ifndef QAS_FLUX_MLAU_MINB
#define QAS_FLUX_MLAU_MINB 6
#endif
template <int A>
__global__ void __launch_bounds__(128, QAS_FLUX_MLAU_MINB) k_flux_mlau(View v)
{
  if (v.ctl->done) return;
  QAS_CELL_INDEX();
  flux_body<3, A>(v, i, j, k);
}

// ---------------------------------------------------------------------------
// Fused face sweep along axis A: characteristic face states of every cell and
// the Riemann flux of every face in one kernel, so the face states never go
// through HBM.
//  * x faces: the cells pos in [2, nx-2) of all rows form one flattened
//    sequence; warp w takes cells [31w, 31w+32) of it, and each lane hands its
//    cell's right-face state to the next lane with a shuffle (31 faces per warp,
//    every lane busy whatever the row length).
//  * y / z faces: one thread per column (x fastest, then the other transverse
//    axis, flattened), marching along A over a segment of faces; the previous
//    cell's right-face state waits in a shared-memory slot of the thread, not in
//    registers, so the reconstruction and the Riemann solver do not hold it live.
// Resident-block caps per Riemann solver: the reconstruction's 6 (80 registers),
// Roe's 4 (its flux needs 128).  PR: 0 the characteristic or primitive reconstruction by
// v.recon (the default scheme), -1 also the Athena-type form, whose code raises the kernels'
// register pressure (spills 156 -> 712 B).  Built for 4th-order interpolation (the other orders
// take the two-kernel form).
// ---------------------------------------------------------------------------
#ifndef QAS_SWEEP_MINB
#define QAS_SWEEP_MINB 6
#endif
#ifndef QAS_SWEEP_ROE_MINB
#define QAS_SWEEP_ROE_MINB 4
#endif
#define QAS_SWEEP_MINB_OF(RMN) ((RMN) == 0 ? QAS_SWEEP_ROE_MINB : QAS_SWEEP_MINB)

// PR: 0 the characteristic or primitive form by v.recon, -1 any of the three
template <int ODR, int A, int PR>
__device__ __forceinline__ void cell_states(const View &v, long long c, double vl[7], double vr[7], double ql[2],
                                            double qr[2])
{
  const Geo &g = v.g;
  const long long s = g.s[A];
  constexpr int B = (A + 1) % 3, C = (A + 2) % 3;
  const double *vn = A == 0 ? v.vx : (A == 1 ? v.vy : v.vz);
  const double *vb = B == 0 ? v.vx : (B == 1 ? v.vy : v.vz);
  const double *vc = C == 0 ? v.vx : (C == 1 ? v.vy : v.vz);
  const double *cn = A == 0 ? v.cx : (A == 1 ? v.cy : v.cz);
  const double *cb = B == 0 ? v.cx : (B == 1 ? v.cy : v.cz);
  const double *ccp = C == 0 ? v.cx : (C == 1 ? v.cy : v.cz);
  const LrStencil<A> st{v, c, s};
  if (PR <= 0 && v.recon == 1)
    face_states_prim<ODR>(st, vl, vr);
  else if (PR < 0 && v.recon == 2)
    face_states_athena<ODR>(st, __ldg(cn + c), v.gam, vl, vr);
  else
    face_states_grouped<ODR>(st, __ldg(cn + c), v.gam, vl, vr);
  if (g.dim >= 2) {
    const double *bnf = v.u[4 + A];
    const double bfl = __ldg(bnf + c + s), bfr = __ldg(bnf + c);
#pragma unroll
    for (int t = 0; t < 2; t++) {
      if (g.dim == 2 && ((A == 0 && t == 1) || (A == 1 && t == 0))) continue;
      const double *vt = t == 0 ? vb : vc;
      const double *bt = t == 0 ? cb : ccp;
      double prod[5], vts[5];
#pragma unroll
      for (int m = 0; m < 5; m++) {
        const long long p = c + (m - 2) * s;
        prod[m] = __ldg(bt + p) * __ldg(vn + p);
        vts[m] = __ldg(vt + p);
      }
      double fl0, fr0, fl1, fr1;
      lin_lr<ODR>(prod, fl0, fr0);
      lin_lr<ODR>(vts, fl1, fr1);
      ql[t] = fl0 - bfl * fl1;
      qr[t] = fr0 - bfr * fr1;
    }
  }
}

// flux at face f from the left cell's right-face state L/QL and this cell's left-face state R/QR
template <int RMN, int A>
__device__ __forceinline__ void face_flux(const View &v, long long f, const double L[7], const double R[7],
                                          const double QL[2], const double QR[2])
{
  const Geo &g = v.g;
  const long long s = g.s[A];
  constexpr int B = (A + 1) % 3, C = (A + 2) % 3;
  const double bnf = __ldg(v.u[4 + A] + f);
  const double bn = 0.5 * (bnf + bnf);
  double dv0 = 0.0, dv1 = 0.0;
  if (RMN >= 2) {
    const double *vn = A == 0 ? v.vx : (A == 1 ? v.vy : v.vz);
    dv0 = __ldg(vn + f) - __ldg(vn + f - s);
    if (g.dim == 2) {
      const double *dt = v.dv[A == 0 ? 1 : 0];
      dv1 = qmin(__ldg(dt + f - s), __ldg(dt + f));
    } else if (g.dim == 3) {
      const double *d1 = v.dv[B], *d2 = v.dv[C];
      dv1 = qmin(qmin(__ldg(d1 + f - s), __ldg(d1 + f)), qmin(__ldg(d2 + f - s), __ldg(d2 + f)));
    }
  }
  riemann_out<RMN>(L, R, bn, v.gam, dv0, dv1, FaceSink<A, false>{v, f, s, QL[0], QR[0], QL[1], QR[1], 0.0});
}

// one lane of an x-sweep warp: the face states of cell (i, j, k) (a valid cell even for a lane
// past the end, have_cell false, so that the warp stays converged), the hand-off of the right-face
// state to the next lane, and the flux at the cell's left face when the previous lane holds the
// cell to its left (i >= 3)
template <int ODR, int RMN, int PR>
__device__ __forceinline__ void sweep_x_cell(const View &v, int i, int j, int k, int lane, bool have_cell)
{
  const long long c = cidx(v.g, i, j, k);
  double vl[7], vr[7], ql[2] = {0.0, 0.0}, qr[2] = {0.0, 0.0};
  cell_states<ODR, 0, PR>(v, c, vl, vr, ql, qr);
  double L[7], QL[2];
#pragma unroll
  for (int m = 0; m < 7; m++) L[m] = __shfl_up_sync(0xffffffffu, vl[m], 1);
  QL[0] = __shfl_up_sync(0xffffffffu, ql[0], 1);
  QL[1] = __shfl_up_sync(0xffffffffu, ql[1], 1);
  if (lane >= 1 && have_cell && i >= 3) face_flux<RMN, 0>(v, c, L, vr, QL, qr);
}

// x sweep: 4 warps per block, 31 faces per warp over the flattened cells of all rows
template <int ODR, int RMN, int PR>
__global__ void __launch_bounds__(128, QAS_SWEEP_MINB_OF(RMN)) k_sweep_x(View v, long long nwarps)
{
  if (v.ctl->done) return;
  const Geo &g = v.g;
  const int lane = threadIdx.x & 31;
  const long long w = (long long)blockIdx.x * 4 + (threadIdx.x >> 5);
  if (w >= nwarps) return;  // the whole warp leaves together
  const long long ncell = g.nx - 4;
  const long long total = ncell * g.ny * g.nz;
  long long t = w * 31 + lane;
  const bool have_cell = t < total;
  if (!have_cell) t = total - 1;  // a valid cell, computed and discarded (keeps the warp converged)
  const long long row = t / ncell;
  const int i = 2 + (int)(t - row * ncell);
  const long long c = cidx(g, i, (int)(row % g.ny), (int)(row / g.ny));
  double vl[7], vr[7], ql[2] = {0.0, 0.0}, qr[2] = {0.0, 0.0};
  cell_states<ODR, 0, PR>(v, c, vl, vr, ql, qr);
  double L[7], QL[2];
#pragma unroll
  for (int m = 0; m < 7; m++) L[m] = __shfl_up_sync(0xffffffffu, vl[m], 1);
  QL[0] = __shfl_up_sync(0xffffffffu, ql[0], 1);
  QL[1] = __shfl_up_sync(0xffffffffu, ql[1], 1);
  // lane-1 holds cell i-1 of the same row exactly when i >= 3
  if (lane >= 1 && have_cell && i >= 3) face_flux<RMN, 0>(v, c, L, vr, QL, qr);
}

// one column of a y / z sweep: the faces p in [p0, p1) along A of the column through (i, o)
// (o = k for the y sweep, j for the z sweep), from the cell before p0 on; the previous cell's
// right-face state waits in the thread's shared-memory slot carry[.][tid]
template <int ODR, int RMN, int A, int PR>
__device__ __forceinline__ void sweep_column(const View &v, int i, int o, int p0, int p1, double (*carry)[128], int tid)
{
  const Geo &g = v.g;
  const long long s = g.s[A];
  long long c = A == 1 ? cidx(g, i, p0 - 1, o) : cidx(g, i, o, p0 - 1);
  {
    double vl[7], vr[7], ql[2] = {0.0, 0.0}, qr[2] = {0.0, 0.0};
    cell_states<ODR, A, PR>(v, c, vl, vr, ql, qr);
#pragma unroll
    for (int m = 0; m < 7; m++) carry[m][tid] = vl[m];
    carry[7][tid] = ql[0];
    carry[8][tid] = ql[1];
  }
  for (int p = p0; p < p1; p++) {
    c += s;
    double vl[7], vr[7], ql[2] = {0.0, 0.0}, qr[2] = {0.0, 0.0};
    cell_states<ODR, A, PR>(v, c, vl, vr, ql, qr);
    double L[7], QL[2];
#pragma unroll
    for (int m = 0; m < 7; m++) {
      L[m] = carry[m][tid];
      carry[m][tid] = vl[m];
    }
    QL[0] = carry[7][tid];
    QL[1] = carry[8][tid];
    carry[7][tid] = ql[0];
    carry[8][tid] = ql[1];
    face_flux<RMN, A>(v, c, L, vr, QL, qr);
  }
}

// y / z sweep: one thread per column, marching over `seg` faces along A
template <int ODR, int RMN, int A, int PR>
__global__ void __launch_bounds__(128, QAS_SWEEP_MINB_OF(RMN)) k_sweep_m(View v, int seg)
{
  if (v.ctl->done) return;
  const Geo &g = v.g;
  __shared__ double carry[9][128];  // previous cell's right-face state and induction state, per thread
  const int tid = threadIdx.x;
  const int no = A == 1 ? g.nz : g.ny;  // extent of the other transverse axis
  const long long col = (long long)blockIdx.x * 128 + tid;
  if (col >= (long long)g.nx * no) return;  // no barrier below: threads leave freely
  const int i = (int)(col % g.nx), o = (int)(col / g.nx);
  const int p0 = 3 + blockIdx.y * seg;
  const int p1 = min(p0 + seg, g.n[A] - 2);
  const long long s = g.s[A];
  long long c = A == 1 ? cidx(g, i, p0 - 1, o) : cidx(g, i, o, p0 - 1);
  {
    double vl[7], vr[7], ql[2] = {0.0, 0.0}, qr[2] = {0.0, 0.0};
    cell_states<ODR, A, PR>(v, c, vl, vr, ql, qr);
#pragma unroll
    for (int m = 0; m < 7; m++) carry[m][tid] = vl[m];
    carry[7][tid] = ql[0];
    carry[8][tid] = ql[1];
  }
  for (int p = p0; p < p1; p++) {
    c += s;
    double vl[7], vr[7], ql[2] = {0.0, 0.0}, qr[2] = {0.0, 0.0};
    cell_states<ODR, A, PR>(v, c, vl, vr, ql, qr);
    double L[7], QL[2];
#pragma unroll
    for (int m = 0; m < 7; m++) {
      L[m] = carry[m][tid];
      carry[m][tid] = vl[m];
    }
    QL[0] = carry[7][tid];
    QL[1] = carry[8][tid];
    carry[7][tid] = ql[0];
    carry[8][tid] = ql[1];
    face_flux<RMN, A>(v, c, L, vr, QL, qr);
  }
}

// ---------------------------------------------------------------------------
// corner EMFs (mhd2d_solve.cpp:201-232, :308-339; mhd3d_solve.cpp:259-328,
// :423-492, :587-656) with the CUCT weight (mhd_func.c:56-76) computed here.
// ---------------------------------------------------------------------------
template <int ODR>
__device__ __forceinline__ double emf_term(const double *up, const double *cen, long long c, long long s, double sgn,
                                           double wgt)
{
  double a[5], b[5];
#pragma unroll
  for (int m = 0; m < 5; m++) {
    a[m] = up[c + (m - 3) * s];
    b[m] = up[c + (m - 2) * s];
  }
  const double l0 = lin_left<ODR>(a), r0 = lin_right<ODR>(b);
#pragma unroll
  for (int m = 0; m < 5; m++) {
    a[m] = cen[c + (m - 3) * s];
    b[m] = cen[c + (m - 2) * s];
  }
  const double l1 = lin_left<ODR>(a), r1 = lin_right<ODR>(b);
  return sgn * ((l0 + r0) + wgt * (l1 + r1));
}

__device__ __forceinline__ double cuct_at(const View &v, const double *va, const double *vb, const double *ba,
                                          const double *bb, long long c, long long oa, long long ob)
{
  if (!v.ctw) return 0.5;
  const double *ro = v.u[0];
  return cuct_weight(ro[c - oa - ob], ro[c - ob], ro[c - oa], ro[c], va[c - oa - ob], va[c - ob], va[c - oa], va[c],
                     vb[c - oa - ob], vb[c - ob], vb[c - oa], vb[c], ba[c - ob], ba[c], bb[c - oa], bb[c]);
}

template <int ODR>
__device__ __forceinline__ void emf_body(const View &v, int i, int j, int k)
{
  const Geo &g = v.g;
  const long long c = cidx(g, i, j, k);
  const long long sx = 1, sy = g.s[1], sz = g.s[2];
  const bool ii = i >= 3 && i < g.nx - 2, jj = j >= 3 && j < g.ny - 2;
  if (g.dim == 2) {
    if (ii && jj) {
      const double ct = cuct_at(v, v.vx, v.vy, v.u[4], v.u[5], c, sx, sy);
      double ez = 0.0;
      ez += emf_term<ODR>(v.f[0][5], v.fc[0][0], c, sy, -0.5, (1.0 - ct));
      ez += emf_term<ODR>(v.f[1][4], v.fc[1][1], c, sx, +0.5, ct);
      v.ez[c] = ez;
    }
    return;
  }
  const bool kk = k >= 3 && k < g.nz - 2;
  if (ii && jj) {
    const double ct0 = cuct_at(v, v.vx, v.vy, v.u[4], v.u[5], c, sx, sy);
    double ez = 0.0;
    ez += emf_term<ODR>(v.f[0][5], v.fc[0][0], c, sy, -0.5, (1.0 - ct0));
    ez += emf_term<ODR>(v.f[1][4], v.fc[1][1], c, sx, +0.5, ct0);
    v.ez[c] = ez;
  }
  if (ii && kk) {
    const double ct2 = cuct_at(v, v.vz, v.vx, v.u[6], v.u[4], c, sz, sx);
    double ey = 0.0;
    ey += emf_term<ODR>(v.f[0][6], v.fc[0][1], c, sz, +0.5, ct2);
    ey += emf_term<ODR>(v.f[2][4], v.fc[2][0], c, sx, -0.5, (1.0 - ct2));
    v.ey[c] = ey;
  }
  if (jj && kk) {
    const double ct1 = cuct_at(v, v.vy, v.vz, v.u[5], v.u[6], c, sy, sz);
    double ex = 0.0;
    ex += emf_term<ODR>(v.f[1][6], v.fc[1][0], c, sz, -0.5, (1.0 - ct1));
    ex += emf_term<ODR>(v.f[2][5], v.fc[2][1], c, sy, +0.5, ct1);
    v.ex[c] = ex;
  }
}
template <int ODR>
__global__ void QAS_EMF_BOUNDS k_emf(View v)
{
  if (v.ctl->done) return;
  QAS_CELL_INDEX();
  emf_body<ODR>(v, i, j, k);
}

// ---------------------------------------------------------------------------
// SSP-RK combine + CT update (mhd_updt1d/2d/3d, mhd_updt2d_ctb/3d_ctb:
// common/mhd_func.c:207-325)
// ---------------------------------------------------------------------------
template <int ODR>
__device__ __forceinline__ double d4(const double *p, long long c, long long s)
{
  return dfc<ODR>(p[c - s], p[c], p[c + s], p[c + 2 * s]);
}

// update cell (i,j,k), i in [GH, nx-GH] etc.: the extra face of the staggered fields included.
// The stage input is read from uin (default: the state v.u itself, updated in place)
template <int ODR>
__device__ __forceinline__ void update_body(const View &v, int i, int j, int k, double c0, double c1,
                                            double *const *uin = nullptr)
{
  double *const *const ui = uin ? uin : v.u;
  const Geo &g = v.g;
  const long long c = cidx(g, i, j, k);
  const double dtdx = v.ctl->dtd[0], dtdy = v.ctl->dtd[1], dtdz = v.ctl->dtd[2];
  const bool ci = i < g.nx - GH;
  const bool cj = g.dim < 2 || j < g.ny - GH;
  const bool ck = g.dim < 3 || k < g.nz - GH;
  const long long sy = g.s[1], sz = g.s[2];
  // every new value is formed before the first store (the compiler cannot prove that the
  // state and flux arrays do not alias, and interleaved stores would serialise the loads)
  double nv[8];
  bool wr[8];
#pragma unroll
  for (int m = 0; m < 8; m++) wr[m] = false;
  if (ci && cj && ck) {
#pragma unroll
    for (int m = 0; m < 8; m++) {
      if (m == 4) continue;
      if (g.dim >= 2 && m == 5) continue;
      if (g.dim >= 3 && m == 6) continue;
      double du;
      const double du0 = d4<ODR>(v.f[0][m], c, 1);
      if (g.dim == 1) {
        du = -dtdx * du0;
      } else {
        const double du1 = d4<ODR>(v.f[1][m], c, sy);
        if (g.dim == 2) {
          du = (-dtdx * du0 - dtdy * du1);
        } else {
          const double du2 = d4<ODR>(v.f[2][m], c, sz);
          du = (-dtdx * du0 - dtdy * du1 - dtdz * du2);
        }
      }
      nv[m] = rk_combine(ui[m][c], v.u0[m][c], du, c0, c1);
      wr[m] = true;
    }
    if (v.phi) {
      // work done by gravity on the momentum, with the updated density (2D/SERIAL/RTI/
      // mhd2d_solve.cpp:361-362, 3D/MPI/RTI/mhd3d_solve.cpp:679-681)
      const double *ph = v.phi;
      nv[1] = nv[1] + -c1 * nv[0] * 0.5 * (ph[c + 1] - ph[c - 1]) * dtdx;
      nv[2] = nv[2] + -c1 * nv[0] * 0.5 * (ph[c + sy] - ph[c - sy]) * dtdy;
      if (g.dim == 3) nv[3] = nv[3] + -c1 * nv[0] * 0.5 * (ph[c + sz] - ph[c - sz]) * dtdz;
    }
  }
  if (g.dim == 2) {
    if (cj) {  // bx on i in [GH, nx-GH]
      const double du = d4<ODR>(v.ez, c, sy);
      nv[4] = rk_combine(ui[4][c], v.u0[4][c], -(+dtdy) * du, c0, c1);
      wr[4] = true;
    }
    if (ci && j <= g.ny - GH) {  // by on j in [GH, ny-GH]
      const double du = d4<ODR>(v.ez, c, 1);
      nv[5] = rk_combine(ui[5][c], v.u0[5][c], -(-dtdx) * du, c0, c1);
      wr[5] = true;
    }
  } else if (g.dim == 3) {
    if (ck && cj) {
      const double du0 = +d4<ODR>(v.ez, c, sy);
      const double du1 = -d4<ODR>(v.ey, c, sz);
      nv[4] = rk_combine(ui[4][c], v.u0[4][c], -dtdy * du0 - dtdz * du1, c0, c1);
      wr[4] = true;
    }
    if (ck && ci) {
      const double du0 = +d4<ODR>(v.ex, c, sz);
      const double du1 = -d4<ODR>(v.ez, c, 1);
      nv[5] = rk_combine(ui[5][c], v.u0[5][c], -dtdz * du0 - dtdx * du1, c0, c1);
      wr[5] = true;
    }
    if (cj && ci) {
      const double du0 = +d4<ODR>(v.ey, c, 1);
      const double du1 = -d4<ODR>(v.ex, c, sy);
      nv[6] = rk_combine(ui[6][c], v.u0[6][c], -dtdx * du0 - dtdy * du1, c0, c1);
      wr[6] = true;
    }
  }
#pragma unroll
  for (int m = 0; m < 8; m++)
    if (wr[m]) v.u[m][c] = nv[m];
}

// offset of the update launch: threads start at the first interior cell
__device__ __forceinline__ bool update_cell(const Geo &g, int ti, int tj, int tk, int &i, int &j, int &k)
{
  i = GH + ti;
  j = (g.dim >= 2 ? GH : 0) + tj;
  k = (g.dim >= 3 ? GH : 0) + tk;
  if (i > g.nx - GH) return false;
  if (g.dim >= 2 && j > g.ny - GH) return false;
  if (g.dim >= 3 && k > g.nz - GH) return false;
  if (g.dim < 2 && j > 0) return false;
  if (g.dim < 3 && k > 0) return false;
  return true;
}

template <int ODR>
__global__ void QAS_UPDATE_BOUNDS k_update(View v, double c0, double c1)
{
  if (v.ctl->done) return;
  int i, j, k;
  if (!update_cell(v.g, blockIdx.x * blockDim.x + threadIdx.x, blockIdx.y * blockDim.y + threadIdx.y,
                   blockIdx.z * blockDim.z + threadIdx.z, i, j, k))
    return;
  update_body<ODR>(v, i, j, k, c0, c1);
}

// ---------------------------------------------------------------------------
// ghost fill of the state (bound()), launched over the ghost shell only: the
// cells with an index in [0,GH) or [n-GH,n) along some active axis
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ long long shell_cells(const Geo &g)
{
  const long long ix = g.nx - 2 * GH;
  if (g.dim == 1) return 2 * GH;
  if (g.dim == 2) return (long long)g.nx * g.ny - ix * (g.ny - 2 * GH);
  return (long long)g.nx * g.ny * g.nz - ix * (g.ny - 2 * GH) * (g.nz - 2 * GH);
}

__device__ __forceinline__ void shell_cell(const Geo &g, long long t, int &i, int &j, int &k)
{
  k = 0;
  j = 0;
  if (g.dim == 1) {
    i = t < GH ? (int)t : g.nx - 2 * GH + (int)t;
    return;
  }
  if (g.dim == 3) {
    const long long plane = (long long)g.nx * g.ny;
    if (t < 2 * GH * plane) {
      const int kid = (int)(t / plane);
      k = kid < GH ? kid : g.nz - 2 * GH + kid;
      const long long r = t - kid * plane;
      j = (int)(r / g.nx);
      i = (int)(r - (long long)j * g.nx);
      return;
    }
    t -= 2 * GH * plane;
    const long long s2 = plane - (long long)(g.nx - 2 * GH) * (g.ny - 2 * GH);
    const int kk = (int)(t / s2);
    k = GH + kk;
    t -= kk * s2;
  }
  if (t < 2 * GH * (long long)g.nx) {
    const int jid = (int)(t / g.nx);
    j = jid < GH ? jid : g.ny - 2 * GH + jid;
    i = (int)(t - (long long)jid * g.nx);
    return;
  }
  t -= 2 * GH * (long long)g.nx;
  j = GH + (int)(t / (2 * GH));
  const int col = (int)(t % (2 * GH));
  i = col < GH ? col : g.nx - 2 * GH + col;
}

__device__ __forceinline__ void bound_body(const View &v, int i, int j, int k)
{
  const Geo &g = v.g;
  const long long c = cidx(g, i, j, k);
  // sources are never written by the fill, so all values are gathered before any store
  double nv[8];
  bool wr[8];
#pragma unroll
  for (int m = 0; m < 8; m++) {
    int si, sj, sk;
    double fac;
    gather_src(v, 0, m, i, j, k, si, sj, sk, fac);
    wr[m] = si != i || sj != j || sk != k;
    nv[m] = wr[m] ? fac * v.u[m][cidx(g, si, sj, sk)] : 0.0;
  }
  if (v.phi && g.dim >= 2) {
    // gravity drivers: the energy of the ghost layers of the last axis from the filled first /
    // last interior layer (2D/SERIAL/RTI/mhd2d_class.cpp:10-32, 3D/MPI/RTI/mhd3d_class.cpp:14-40)
    const int h = g.dim == 3 ? k : j, n = g.dim == 3 ? g.nz : g.ny;
    if (h < GH || h >= n - GH) {
      const int hb = h < GH ? GH : n - GH - 1;
      const int bj = g.dim == 3 ? j : hb, bk = g.dim == 3 ? hb : k;
      int si, sj, sk;
      double fr, fe;
      gather_src(v, 0, 0, i, bj, bk, si, sj, sk, fr);
      const double ro_b = fr * v.u[0][cidx(g, si, sj, sk)];
      gather_src(v, 0, 7, i, bj, bk, si, sj, sk, fe);
      const double en_b = fe * v.u[7][cidx(g, si, sj, sk)];
      const long long b = cidx(g, i, bj, bk);
      nv[7] = en_b - v.gfac * ro_b * (v.phi[c] - v.phi[b]);
      wr[7] = true;
    }
  }
#pragma unroll
  for (int m = 0; m < 8; m++)
    if (wr[m]) v.u[m][c] = nv[m];
}

__global__ void k_bound(View v)
{
  if (v.ctl->done) return;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= shell_cells(v.g)) return;
  int i, j, k;
  shell_cell(v.g, t, i, j, k);
  bound_body(v, i, j, k);
}

// ---------------------------------------------------------------------------
// exec_ loop control and setdt
// ---------------------------------------------------------------------------
// begin of a loop iteration: the while() test of exec_, tim += dt, dt/dx
__device__ __forceinline__ void begin_body(const View &v, int check_tim)
{
  Ctl *c = v.ctl;
  if (c->done) return;
  const bool go = check_tim ? (c->n < c->nmax && c->tim < c->tmax) : (c->n < c->nmax);
  if (!go) {
    c->done = 1;
    return;
  }
  c->n += 1;
  c->tim += c->dt;
  c->dtd[0] = c->dt / v.dx;
  c->dtd[1] = v.g.dim >= 2 ? c->dt / v.dy : 0.0;
  c->dtd[2] = v.g.dim >= 3 ? c->dt / v.dz : 0.0;
}
__global__ void k_begin_step(View v, int check_tim) { begin_body(v, check_tim); }

// dt/dx etc. for a host-supplied dt (qas_step)
__global__ void k_set_dt(View v, double dt)
{
  Ctl *c = v.ctl;
  c->dt = dt;
  c->dtd[0] = dt / v.dx;
  c->dtd[1] = v.g.dim >= 2 ? dt / v.dy : 0.0;
  c->dtd[2] = v.g.dim >= 3 ? dt / v.dz : 0.0;
}

__global__ void k_vmax_reset(View v)
{
  if (v.ctl->done) return;
  v.ctl->vmax_bits = (unsigned long long)__double_as_longlong(1.0);
}

// |v| + c_f at interior cell (i,j,k) with B from the 2nd-order face average (setdt)
__device__ __forceinline__ double vmax_cell(const View &v, int i, int j, int k)
{
  const Geo &g = v.g;
  const long long c = cidx(g, i, j, k);
    double cx, cy, cz;
    if (g.dim == 1) {
      cx = v.u[4][c];
      cy = v.u[5][c];
      cz = v.u[6][c];
    } else {
      cx = 0.5 * (v.u[4][c] + v.u[4][c + 1]);
      cy = 0.5 * (v.u[5][c] + v.u[5][c + g.s[1]]);
      cz = g.dim == 3 ? 0.5 * (v.u[6][c] + v.u[6][c + g.s[2]]) : v.u[6][c];
    }
    const double ro = v.u[0][c];
    const double iro = 1.0 / ro;
    const double vx = v.u[1][c] * iro, vy = v.u[2][c] * iro, vz = v.u[3][c] * iro;
    const double v2 = vx * vx + vy * vy + vz * vz;
    const double b2 = cx * cx + cy * cy + cz * cz;
    // gravity drivers' setdt: the same en -= ro*phi; prmtv; en += ro*phi on the interior
    // (2D/SERIAL/RTI/mhd2d_class.cpp:46-48, 3D/MPI/RTI/mhd3d_class.cpp:56-58)
    double en = v.u[7][c];
    if (v.phi) en = en - ro * v.phi[c];
    const double pr = (v.gam - 1) * (en - 0.5 * (ro * v2 + b2));
    if (v.phi) v.u[7][c] = en + ro * v.phi[c];
    const double vf = sqrt((v.gam * pr + (cx * cx + cy * cy + cz * cz)) / ro);
    double vt;
    if (g.dim == 1)
      vt = fabs(vx) + vf;
    else if (g.dim == 2)
      vt = sqrt(vx * vx + vy * vy) + vf;
    else
      vt = sqrt(vx * vx + vy * vy + vz * vz) + vf;
    return vt;
}

// max over the interior of |v| + c_f with B from the 2nd-order face average
// (mhd2d_class.cpp:17-26); NaN never wins, as with `if (vtmp > vmax)`.
__global__ void k_vmax(View v)
{
  if (v.ctl->done) return;
  const Geo &g = v.g;
  const int i = GH + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = (g.dim >= 2 ? GH : 0) + blockIdx.y;
  const int k = (g.dim >= 3 ? GH : 0) + blockIdx.z;
  double best = 1.0;
  if (i < g.nx - GH) {
    const double vt = vmax_cell(v, i, j, k);
    if (vt > best) best = vt;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double other = __shfl_xor_sync(0xffffffffu, best, o);
    best = (other > best) ? other : best;
  }
  __shared__ double red[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) red[wid] = best;
  __syncthreads();
  if (wid == 0) {
    best = (lane < (int)(blockDim.x >> 5)) ? red[lane] : 1.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double other = __shfl_xor_sync(0xffffffffu, best, o);
      best = (other > best) ? other : best;
    }
    if (lane == 0) atomicMax(&v.ctl->vmax_bits, (unsigned long long)__double_as_longlong(best));
  }
}

// dt = cfl*dr/vmax; on the first call also exec_'s nmax (mhd2d_class.cpp:27-32,
// mhd1d_class.cpp:146-151)
__device__ __forceinline__ void setdt_body(const View &v, double cfl, double dr, int rule, double dtrec, int nout)
{
  Ctl *c = v.ctl;
  if (c->done) return;
  const double vmax = __longlong_as_double((long long)c->vmax_bits);
  c->dt = cfl * dr / vmax;
  if (c->first) {
    if (rule == 2) {
      const int nrec = (int)(dtrec / c->dt + 0.5);
      c->nmax = nrec * nout;
    } else if (rule == 1) {
      c->nmax = (int)(c->tmax / c->dt + 0.5);
    }
    c->first = 0;
  }
}
__global__ void k_setdt(View v, double cfl, double dr, int rule, double dtrec, int nout)
{
  setdt_body(v, cfl, dr, rule, dtrec, nout);
}

// |div B| with df1[ODR-1] over the interior; max by bit pattern of non-negative doubles
template <int ODR>
__global__ void k_divb(View v, unsigned long long *out)
{
  const Geo &g = v.g;
  const int i = GH + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = (g.dim >= 2 ? GH : 0) + blockIdx.y;
  const int k = (g.dim >= 3 ? GH : 0) + blockIdx.z;
  double d = 0.0;
  if (i < g.nx - GH && g.dim >= 2) {
    const long long c = cidx(g, i, j, k);
    double s = d4<ODR>(v.u[4], c, 1) / v.dx + d4<ODR>(v.u[5], c, g.s[1]) / v.dy;
    if (g.dim == 3) s += d4<ODR>(v.u[6], c, g.s[2]) / v.dz;
    d = fabs(s);
    if (!(d == d)) d = __longlong_as_double(0x7ff0000000000000LL);  // NaN reports as +inf
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double other = __shfl_xor_sync(0xffffffffu, d, o);
    d = (other > d) ? other : d;
  }
  if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(d));
}

// FP64 throughput probe: 8 independent DFMA chains per thread (2 flops each)
__global__ void k_fp64_peak(double *out, int iters, double a, double b)
{
  double x0 = threadIdx.x * 1e-9, x1 = x0 + 1.0, x2 = x0 + 2.0, x3 = x0 + 3.0;
  double x4 = x0 + 4.0, x5 = x0 + 5.0, x6 = x0 + 6.0, x7 = x0 + 7.0;
  for (int it = 0; it < iters; it++) {
    x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
    x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
  }
  const double r = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
  if (r == 12345.0) out[0] = r;  // keeps the chains live
}

}  // namespace qas
