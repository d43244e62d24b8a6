// qas_adjoint_kernels.cuh -- reverse (adjoint) kernels of one 2D SSP-RK stage:
// the ideal stage with characteristic WCNS4 reconstruction, the Roe flux, CUCT
// corner EMFs and the CT update (mhd2d_solve.cpp:3-400), and the resistive
// stage of dsptv (dmhd2d_solve.cpp:3-151) with uniform eta and nu = 0.
//
// Every kernel is a gather: a thread owns one output cell and sums the
// contributions of the forward outputs that read it, in a fixed order, so the
// gradient is deterministic (no atomics).  Forward intermediates come from a
// per-stage tape written by the forward kernels themselves (stage input state,
// primitives, face states, central induction fluxes).
//
// Reverse of one ideal stage (forward: prim, lr+flux per axis, emf, update, bound):
//   k_a_update   bound^T (as a gather over the inverse ghost maps) and the RK
//                combine: w = masked output adjoint, ai = c1 w, a0 += c0 w
//   k_a_emf      corner EMF adjoint from the CT update of bx, by; CUCT weight adjoint
//   k_a_flux<A>  face-flux adjoint (update + EMF), Roe VJP -> face-state adjoints
//   k_a_lr<A>    characteristic reconstruction VJP -> per-stencil-slot adjoints
//   k_a_prim     gather of the slots, CUCT inputs, primitive -> conservative
//   k_a_cb       cell-centre B (4th-order face average + its ghost fill)^T -> bx, by
#pragma once

#include "qas_adjoint.cuh"
#include "qas_kernels.cuh"

namespace qas {

// Inverse ghost-fill maps: for group G, field f, axis a and index s, the indices i
// whose fill source is s (s itself first when s is a fixed point), with factors.
struct InvMaps {
  const int *cnt;
  const int *idx;
  const double *fac;
  int nmax, kmax;
  int lo[2][2], hi[2][2];  // per group and axis: indices whose inverse map is the identity for every field
};

// One reverse stage.  Tape arrays are read-only; adjoint arrays as documented.
struct AView {
  Geo g;
  double gam;
  int ctw;
  InvMaps im;
  // tape of the stage
  const double *u[8];  // stage input state
  const double *vx, *vy, *vz, *pr, *cx, *cy, *cz;
  const double *vl[2][7], *vr[2][7];  // face states per axis
  const double *fcx, *fcy;            // central induction fluxes fc[0][0], fc[1][1]
  // adjoints
  const double *ao[8];  // of the stage output
  double *ai[8];        // of the stage input (written)
  double *a0[8];        // of u0 (accumulated)
  double *w[8];         // masked output adjoint after bound^T
  double *ez, *ct, *ctb;
  double *avl[7], *avr[7], *aql, *aqr;
  double *gs;     // per-axis stencil-slot adjoints: gs[(A*36 + v*5 + m)*ast + c], v*5+m < 35, 35: bn
  double *acx, *acy;
  double *eb;     // per-cell eta adjoint accumulator
  long long ast;  // array stride (doubles)
  double c0, c1, dtdx, dtdy;
};

#define QAS_ADJ_CELL(g)                                 \
  const int i = blockIdx.x * blockDim.x + threadIdx.x; \
  const int j = blockIdx.y * blockDim.y + threadIdx.y; \
  if (i >= (g).nx || j >= (g).ny) return;              \
  const long long c = (long long)(g).nx * j + i;

// Sum over the fill preimage of cell (i,j): the transpose of the ghost fill of group G /
// field f applied to array a (0 at cells that the fill writes).  A 2D preimage has at most
// ADJ_KMAX indices per axis (the index itself plus the 4 ghosts of an open boundary), checked
// on the host; the entries are loaded unconditionally (an unused entry points at the cell
// itself) so that all loads of a boundary cell are in flight together.
#define ADJ_KMAX 5
__device__ __forceinline__ void preimage(const InvMaps &im, int G, int f, int ax, int i, int ii[ADJ_KMAX],
                                         double fa[ADJ_KMAX])
{
  const int e = ((G * 8 + f) * 3 + ax) * im.nmax + i;
  const int n = im.cnt[e];
#pragma unroll
  for (int q = 0; q < ADJ_KMAX; q++) {
    const bool ok = q < n;
    ii[q] = ok ? im.idx[e * im.kmax + q] : i;
    fa[q] = ok ? im.fac[e * im.kmax + q] : 0.0;
  }
}
__device__ __forceinline__ double bound_t(const InvMaps &im, const Geo &g, int G, int f, const double *a, int i, int j)
{
  if (i >= im.lo[G][0] && i < im.hi[G][0] && j >= im.lo[G][1] && j < im.hi[G][1]) return a[(long long)g.nx * j + i];
  int ix[ADJ_KMAX], jy[ADJ_KMAX];
  double fx[ADJ_KMAX], fy[ADJ_KMAX];
  preimage(im, G, f, 0, i, ix, fx);
  preimage(im, G, f, 1, j, jy, fy);
  double s = 0.0;
#pragma unroll
  for (int qy = 0; qy < ADJ_KMAX; qy++)
#pragma unroll
    for (int qx = 0; qx < ADJ_KMAX; qx++) {
      const double v = a[(long long)g.nx * jy[qy] + ix[qx]];
      const double w = fx[qx] * fy[qy];
      s += (w != 0.0) ? w * v : 0.0;
    }
  return s;
}
__device__ __forceinline__ double bound_t2(const InvMaps &im, const Geo &g, int G, int f, const double *a,
                                           const double *b, int i, int j)
{
  if (i >= im.lo[G][0] && i < im.hi[G][0] && j >= im.lo[G][1] && j < im.hi[G][1]) {
    const long long p = (long long)g.nx * j + i;
    return a[p] + b[p];
  }
  int ix[ADJ_KMAX], jy[ADJ_KMAX];
  double fx[ADJ_KMAX], fy[ADJ_KMAX];
  preimage(im, G, f, 0, i, ix, fx);
  preimage(im, G, f, 1, j, jy, fy);
  double s = 0.0;
#pragma unroll
  for (int qy = 0; qy < ADJ_KMAX; qy++)
#pragma unroll
    for (int qx = 0; qx < ADJ_KMAX; qx++) {
      const long long p = (long long)g.nx * jy[qy] + ix[qx];
      const double v = a[p] + b[p];
      const double w = fx[qx] * fy[qy];
      s += (w != 0.0) ? w * v : 0.0;
    }
  return s;
}

// transpose of d4 = dfc<4>(p[c-s], p[c], p[c+s], p[c+2s]) applied to a cell array:
// the adjoint of the face value at e from the cells whose divergence reads it
__device__ __forceinline__ double d4_t(const double *w, long long e, long long s)
{
  return (1.0 / 24.0) * w[e + s] - (27.0 / 24.0) * w[e] + (27.0 / 24.0) * w[e - s] - (1.0 / 24.0) * w[e - 2 * s];
}

// 4th-order linear face interpolation (cal_flr_4th) of the EMF: lin_left over
// points e-3s..e+s plus lin_right over e-2s..e+2s; weight of point e+d*s, d=-3..2
__device__ __forceinline__ double emf_kernel(int d)
{
  const double k[6] = {9.0, -67.0, 378.0, 378.0, -67.0, 9.0};
  return 0.003125 * k[d + 3];
}

// update region of field m at (i,j) (mhd_updt2d / mhd_updt2d_ctb)
__device__ __forceinline__ bool upd_region(const Geo &g, int m, int i, int j)
{
  const bool ci = i >= GH && i < g.nx - GH, cj = j >= GH && j < g.ny - GH;
  if (m == 4) return cj && i >= GH && i <= g.nx - GH;
  if (m == 5) return ci && j >= GH && j <= g.ny - GH;
  return ci && cj;
}

// ---------------------------------------------------------------------------
// bound^T + RK combine^T
// ---------------------------------------------------------------------------
// (every kernel below issues all of its loads before its first store: the arrays are
// distinct but the compiler cannot prove it, and interleaving would serialise the loads)
__global__ void k_a_update(AView a)
{
  QAS_ADJ_CELL(a.g);
  double w[8], o[8];
#pragma unroll
  for (int m = 0; m < 8; m++) w[m] = upd_region(a.g, m, i, j) ? bound_t(a.im, a.g, 0, m, a.ao[m], i, j) : 0.0;
#pragma unroll
  for (int m = 0; m < 8; m++) o[m] = a.a0[m][c];
#pragma unroll
  for (int m = 0; m < 8; m++) {
    a.w[m][c] = w[m];
    a.ai[m][c] = a.c1 * w[m];
    a.a0[m][c] = o[m] + a.c0 * w[m];
  }
}

// out = bound^T(x + y): the step-start fill (ideal) or the sub-cycle-start fill
// followed by the copy u0 = u (dsptv)
__global__ void k_a_fold(AView a)
{
  QAS_ADJ_CELL(a.g);
  double r[8];
#pragma unroll
  for (int m = 0; m < 8; m++) r[m] = bound_t2(a.im, a.g, 0, m, a.ao[m], a.a0[m], i, j);
#pragma unroll
  for (int m = 0; m < 8; m++) a.ai[m][c] = r[m];
}

// ---------------------------------------------------------------------------
// corner EMF adjoint and CUCT weight (emf_body, cuct_weight)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cuct_inputs(const AView &a, long long e, double in[16])
{
  const long long oa = 1, ob = a.g.s[1];
  const double *ro = a.u[0];
  in[0] = ro[e - oa - ob];
  in[1] = ro[e - ob];
  in[2] = ro[e - oa];
  in[3] = ro[e];
  in[4] = a.vx[e - oa - ob];
  in[5] = a.vx[e - ob];
  in[6] = a.vx[e - oa];
  in[7] = a.vx[e];
  in[8] = a.vy[e - oa - ob];
  in[9] = a.vy[e - ob];
  in[10] = a.vy[e - oa];
  in[11] = a.vy[e];
  in[12] = a.u[4][e - ob];
  in[13] = a.u[4][e];
  in[14] = a.u[5][e - oa];
  in[15] = a.u[5][e];
}

__device__ __forceinline__ bool corner_in(const Geo &g, int i, int j)
{
  return i >= 3 && i < g.nx - 2 && j >= 3 && j < g.ny - 2;
}

__global__ void k_a_emf(AView a)
{
  QAS_ADJ_CELL(a.g);
  const Geo &g = a.g;
  if (!corner_in(g, i, j)) {
    a.ez[c] = 0.0;
    a.ct[c] = 0.0;
    a.ctb[c] = 0.0;
    return;
  }
  const long long sy = g.s[1];
  const double ezb = a.c1 * (-a.dtdy * d4_t(a.w[4], c, sy) + a.dtdx * d4_t(a.w[5], c, 1));
  a.ez[c] = ezb;
  if (!a.ctw) {
    a.ct[c] = 0.5;
    a.ctb[c] = 0.0;
    return;
  }
  double in[16];
  cuct_inputs(a, c, in);
  a.ct[c] = cuct_weight(in[0], in[1], in[2], in[3], in[4], in[5], in[6], in[7], in[8], in[9], in[10], in[11], in[12],
                        in[13], in[14], in[15]);
  double fa[5], fb[5], fa2[5], fb2[5];
#pragma unroll
  for (int m = 0; m < 5; m++) {
    fa[m] = a.fcx[c + (m - 3) * sy];
    fb[m] = a.fcx[c + (m - 2) * sy];
    fa2[m] = a.fcy[c + (m - 3)];
    fb2[m] = a.fcy[c + (m - 2)];
  }
  const double s1 = (lin_left<4>(fa) + lin_right<4>(fb)) + (lin_left<4>(fa2) + lin_right<4>(fb2));
  a.ctb[c] = 0.5 * s1 * ezb;
}

// ---------------------------------------------------------------------------
// face flux adjoint + Roe VJP along axis A
// ---------------------------------------------------------------------------
template <int A>
__device__ __forceinline__ void a_flux_cell(const AView &a, int i, int j, long long c)
{
  const Geo &g = a.g;
  const int pos = A == 0 ? i : j;
  const int n = g.n[A];
  const long long s = g.s[A];
  const bool in = pos >= 3 && pos < n - 2;
  if (!in) {
#pragma unroll
    for (int m = 0; m < 7; m++) {
      a.avr[m][c] = 0.0;
      if (pos >= 1) a.avl[m][c - s] = 0.0;
    }
    a.aqr[c] = 0.0;
    if (pos >= 1) a.aql[c - s] = 0.0;
    return;
  }
  const double fac = -a.c1 * (A == 0 ? a.dtdx : a.dtdy);
  double Fb[7];
  // conservative field of each Roe component (flux_body's store order)
  constexpr int mB = A == 0 ? 2 : 3, mC = A == 0 ? 3 : 1;
  Fb[0] = fac * d4_t(a.w[0], c, s);
  Fb[1] = fac * d4_t(a.w[1 + A], c, s);
  Fb[2] = fac * d4_t(a.w[mB], c, s);
  Fb[3] = fac * d4_t(a.w[mC], c, s);
  Fb[6] = fac * d4_t(a.w[7], c, s);
  // transverse induction flux: the EMF reads it (and the central part) along the other axis
  const long long so = A == 0 ? g.s[1] : 1;
  const int po = A == 0 ? j : i, no = A == 0 ? g.ny : g.nx;
  const double sg = A == 0 ? -0.5 : 0.5;
  double eup = 0.0, ecen = 0.0;
#pragma unroll
  for (int d = -3; d <= 2; d++) {
    if (po - d < 0 || po - d >= no) continue;
    const long long e = c - d * so;
    const double k = emf_kernel(d) * sg * a.ez[e];
    eup += k;
    ecen += k * (A == 0 ? (1.0 - a.ct[e]) : a.ct[e]);
  }
  if (A == 0) {
    Fb[4] = eup;                       // f[0][5] = F4 - fc
    Fb[5] = fac * d4_t(a.w[6], c, s);  // f[0][6] = F5
  } else {
    Fb[4] = fac * d4_t(a.w[6], c, s);  // f[1][6] = F4
    Fb[5] = eup;                       // f[1][4] = F5 - fc
  }
  const double fcb = ecen - eup;
  double L[7], R[7], gL[7], gR[7];
#pragma unroll
  for (int m = 0; m < 7; m++) {
    L[m] = a.vl[A][m][c - s];
    R[m] = a.vr[A][m][c];
    gL[m] = 0.0;
    gR[m] = 0.0;
  }
  const double bnf = a.u[4 + A][c];
  const double bn = 0.5 * (bnf + bnf);
  double gbn = 0.0;
  const double ob = a.ai[4 + A][c];
  flux_roe_vjp(L, R, bn, a.gam, Fb, gL, gR, gbn);
#pragma unroll
  for (int m = 0; m < 7; m++) {
    a.avl[m][c - s] = gL[m];
    a.avr[m][c] = gR[m];
  }
  a.ai[4 + A][c] = ob + gbn;
  a.aql[c - s] = 0.5 * fcb;
  a.aqr[c] = 0.5 * fcb;
}

// ---------------------------------------------------------------------------
// characteristic reconstruction VJP along axis A -> stencil-slot adjoints
// ---------------------------------------------------------------------------
template <int A>
__device__ __forceinline__ void a_lr_cell(const AView &a, int i, int j, long long c)
{
  const Geo &g = a.g;
  const int pos = A == 0 ? i : j;
  const int n = g.n[A];
  const long long s = g.s[A];
  // stencil fields of this axis: ro, vn, vb, vc, cb, cc, pr; cn; vt/bt of the 2D induction state
  const double *vn = A == 0 ? a.vx : a.vy;
  const double *vb = A == 0 ? a.vy : a.vz;
  const double *vc = A == 0 ? a.vz : a.vx;
  const double *cb = A == 0 ? a.cy : a.cz;
  const double *cc = A == 0 ? a.cz : a.cx;
  const double *cn = A == 0 ? a.cx : a.cy;
  const double *vt = A == 0 ? vb : vc;
  const bool in = pos >= 2 && pos < n - 2;
  // normal-face B of the induction states: bfr = b[c] for this cell, bfl = b[c] for cell c-s
  double badd = 0.0;
  {
    if (in) {
      double f[5];
#pragma unroll
      for (int m = 0; m < 5; m++) f[m] = vt[c + (m - 2) * s];
      badd += -lin_right<4>(f) * a.aqr[c];
    }
    if (pos - 1 >= 2 && pos - 1 < n - 2) {
      double f[5];
#pragma unroll
      for (int m = 0; m < 5; m++) f[m] = vt[c - s + (m - 2) * s];
      badd += -lin_left<4>(f) * a.aql[c - s];
    }
  }
  double *gsA = a.gs + (long long)A * 36 * a.ast;
  if (!in) {
    const double ob = a.ai[4 + A][c];
#pragma unroll
    for (int q = 0; q < 36; q++) gsA[q * a.ast + c] = 0.0;
    a.ai[4 + A][c] = ob + badd;
    return;
  }
  double q[7][5], gq[7][5];
#pragma unroll
  for (int m = 0; m < 5; m++) {
    const long long p = c + (m - 2) * s;
    q[0][m] = a.u[0][p];
    q[1][m] = vn[p];
    q[2][m] = vb[p];
    q[3][m] = vc[p];
    q[4][m] = cb[p];
    q[5][m] = cc[p];
    q[6][m] = a.pr[p];
#pragma unroll
    for (int v = 0; v < 7; v++) gq[v][m] = 0.0;
  }
  double gvl[7], gvr[7];
#pragma unroll
  for (int m = 0; m < 7; m++) {
    gvl[m] = a.avl[m][c];
    gvr[m] = a.avr[m][c];
  }
  double gbn = 0.0;
  const double ob = a.ai[4 + A][c];
  face_states_vjp(q, cn[c], a.gam, gvl, gvr, gq, gbn);
  // induction states ql = L(bt*vn) - bfl L(vt), qr = R(bt*vn) - bfr R(vt)
  {
    const double gl = a.aql[c], gr = a.aqr[c];
    const double bfl = a.u[4 + A][c + s], bfr = a.u[4 + A][c];
    double gprod[5] = {0, 0, 0, 0, 0}, gvt[5] = {0, 0, 0, 0, 0};
    lin4_vjp(gl, gr, gprod);
    lin4_vjp(-bfl * gl, -bfr * gr, gvt);
    constexpr int sb = A == 0 ? 4 : 5, sv = A == 0 ? 2 : 3;
#pragma unroll
    for (int m = 0; m < 5; m++) {
      gq[sb][m] += gprod[m] * q[1][m];
      gq[1][m] += gprod[m] * q[sb][m];
      gq[sv][m] += gvt[m];
    }
  }
#pragma unroll
  for (int v = 0; v < 7; v++)
#pragma unroll
    for (int m = 0; m < 5; m++) gsA[(v * 5 + m) * a.ast + c] = gq[v][m];
  gsA[35 * a.ast + c] = gbn;
  a.ai[4 + A][c] = ob + badd;
}

// The two heavy reverse kernels run persistent: a grid of (SMs x resident blocks) walks
// 128-cell strips along x, so the last wave is never a few stray blocks (at 256^2 the
// tiled launch needed 3 waves of which the last held 2 blocks).
#define QAS_ADJ_STRIPS(body)                                                        \
  const long long ncell = (long long)a.g.nx * a.g.ny;                              \
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < ncell;  \
       t += (long long)gridDim.x * blockDim.x) {                                    \
    const int i = (int)(t % a.g.nx), j = (int)(t / a.g.nx);                         \
    body;                                                                           \
  }

template <int A>
__global__ void __launch_bounds__(128) k_a_flux(AView a)
{
  QAS_ADJ_STRIPS(a_flux_cell<A>(a, i, j, t));
}

template <int A>
__global__ void __launch_bounds__(128) k_a_lr(AView a)
{
  QAS_ADJ_STRIPS(a_lr_cell<A>(a, i, j, t));
}

// ---------------------------------------------------------------------------
// primitives^T: gather the slots of both axes and the CUCT inputs, then
// prmtv^T (vx = mx/ro, pr = (gam-1)(en - (ro v^2 + b^2)/2))
// ---------------------------------------------------------------------------
__global__ void k_a_prim(AView a)
{
  QAS_ADJ_CELL(a.g);
  const Geo &g = a.g;
  const long long sy = g.s[1];
  double rob = 0, vxb = 0, vyb = 0, vzb = 0, prb = 0, cxb = 0, cyb = 0, czb = 0, bxb = 0, byb = 0;
  // axis 0: slots ro, vx, vy, vz, cy, cz, pr; axis 1: ro, vy, vz, vx, cz, cx, pr
#pragma unroll
  for (int m = 0; m < 5; m++) {
    const int ic = i - (m - 2);
    if (ic >= 0 && ic < g.nx) {
      const long long cc = c - (m - 2);
      const double *G0 = a.gs;
      rob += G0[(0 * 5 + m) * a.ast + cc];
      vxb += G0[(1 * 5 + m) * a.ast + cc];
      vyb += G0[(2 * 5 + m) * a.ast + cc];
      vzb += G0[(3 * 5 + m) * a.ast + cc];
      cyb += G0[(4 * 5 + m) * a.ast + cc];
      czb += G0[(5 * 5 + m) * a.ast + cc];
      prb += G0[(6 * 5 + m) * a.ast + cc];
    }
    const int jc = j - (m - 2);
    if (jc >= 0 && jc < g.ny) {
      const long long cc = c - (m - 2) * sy;
      const double *G1 = a.gs + 36 * a.ast;
      rob += G1[(0 * 5 + m) * a.ast + cc];
      vyb += G1[(1 * 5 + m) * a.ast + cc];
      vzb += G1[(2 * 5 + m) * a.ast + cc];
      vxb += G1[(3 * 5 + m) * a.ast + cc];
      czb += G1[(4 * 5 + m) * a.ast + cc];
      cxb += G1[(5 * 5 + m) * a.ast + cc];
      prb += G1[(6 * 5 + m) * a.ast + cc];
    }
  }
  cxb += a.gs[35 * a.ast + c];
  cyb += a.gs[(36 + 35) * a.ast + c];
  if (a.ctw) {
    // corners e = c (slot 3), c+1 (slot 2), c+sy (slot 1), c+1+sy (slot 0)
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int di = (q == 1 || q == 3) ? 1 : 0, dj = (q >= 2) ? 1 : 0;
      if (!corner_in(g, i + di, j + dj)) continue;
      const long long e = c + di + dj * sy;
      const double gct = a.ctb[e];
      double in[16], gi[16];
      cuct_inputs(a, e, in);
#pragma unroll
      for (int k = 0; k < 16; k++) gi[k] = 0.0;
      cuct_weight_vjp(in, gct, gi);
      const int slot = 3 - di - 2 * dj;
      rob += gi[slot];
      vxb += gi[4 + slot];
      vyb += gi[8 + slot];
      if (di == 0) bxb += gi[dj ? 12 : 13];  // ba1 = bx[e - sy], ba3 = bx[e]
      if (dj == 0) byb += gi[di ? 14 : 15];  // bb2 = by[e - 1], bb3 = by[e]
    }
  }
  const double ro = a.u[0][c];
  const double iro = 1.0 / ro;
  const double vx = a.vx[c], vy = a.vy[c], vz = a.vz[c];
  const double cx = a.cx[c], cy = a.cy[c], cz = a.cz[c];
  const double gm1 = a.gam - 1;
  const double v2 = vx * vx + vy * vy + vz * vz;
  const double enb = gm1 * prb;
  rob += -gm1 * 0.5 * v2 * prb;
  vxb += -gm1 * ro * vx * prb;
  vyb += -gm1 * ro * vy * prb;
  vzb += -gm1 * ro * vz * prb;
  cxb += -gm1 * cx * prb;
  cyb += -gm1 * cy * prb;
  czb += -gm1 * cz * prb;
  const double irob = a.u[1][c] * vxb + a.u[2][c] * vyb + a.u[3][c] * vzb;
  rob += -iro * iro * irob;
  double o[8];
#pragma unroll
  for (int m = 0; m < 8; m++) o[m] = a.ai[m][c];
  a.ai[0][c] = o[0] + rob;
  a.ai[1][c] = o[1] + iro * vxb;
  a.ai[2][c] = o[2] + iro * vyb;
  a.ai[3][c] = o[3] + iro * vzb;
  a.ai[4][c] = o[4] + bxb;
  a.ai[5][c] = o[5] + byb;
  a.ai[6][c] = o[6] + czb;
  a.ai[7][c] = o[7] + enb;
  a.acx[c] = cxb;
  a.acy[c] = cyb;
}

// cell-centre B^T: cx(c) = fac * fcen(bx[s-1..s+2]) at the fill source s of c
__global__ void k_a_cb(AView a)
{
  QAS_ADJ_CELL(a.g);
  const Geo &g = a.g;
  const double w[4] = {-0.0625, 0.5625, 0.5625, -0.0625};  // fcen<4> weights of s-1, s, s+1, s+2
  double bxb = 0.0, byb = 0.0;
#pragma unroll
  for (int m = 0; m < 4; m++) {
    // bx[i] is point m of source s = i + 1 - m
    const int si = i + 1 - m;
    if (si >= 0 && si < g.nx) bxb += w[m] * bound_t(a.im, g, 1, 0, a.acx, si, j);
    const int sj = j + 1 - m;
    if (sj >= 0 && sj < g.ny) byb += w[m] * bound_t(a.im, g, 1, 1, a.acy, i, sj);
  }
  const double ox = a.ai[4][c], oy = a.ai[5][c];
  a.ai[4][c] = ox + bxb;
  a.ai[5][c] = oy + byb;
}

// ---------------------------------------------------------------------------
// resistive stage of dsptv (nu = 0): E = eta J at the CT edges (mhd_ct_eres),
// resistive face fluxes (calc_flux_resistive), CT update of bx, by, flux update
// of bz, en.  Dissipative kernels share k_a_update / k_a_fold.
// Scratch use: avl[0..3] = flux adjoints (x bz, x en, y bz, y en), avl[4..6] = J adjoint,
// avr[0..2] = the forward E.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool dflux_in(const Geo &g, int i, int j)
{
  return i >= 2 && i < g.nx - 1 && j >= 2 && j < g.ny - 1;
}

__global__ void k_d_flux(AView a)
{
  QAS_ADJ_CELL(a.g);
  const Geo &g = a.g;
  if (!dflux_in(g, i, j)) {
#pragma unroll
    for (int q = 0; q < 4; q++) a.avl[q][c] = 0.0;
    return;
  }
  const long long sy = g.s[1];
  const double fx = -a.c1 * a.dtdx, fy = -a.c1 * a.dtdy;
  a.avl[0][c] = fx * d4_t(a.w[6], c, 1);
  a.avl[1][c] = fx * d4_t(a.w[7], c, 1);
  a.avl[2][c] = fy * d4_t(a.w[6], c, sy);
  a.avl[3][c] = fy * d4_t(a.w[7], c, sy);
}

// current density at cell c (mhd_ct_eres with idz = 0)
__device__ __forceinline__ void cur_j(const AView &a, long long c, double idx, double idy, double &jx, double &jy,
                                      double &jz)
{
  const long long sy = a.g.s[1];
  const double *bx = a.u[4], *by = a.u[5], *bz = a.u[6];
  const double idz = 0.0;
  const double dbxz = dfc<4>(bx[c], bx[c], bx[c], bx[c]);
  const double dbyz = dfc<4>(by[c], by[c], by[c], by[c]);
  jx = dfc<4>(bz[c - 2 * sy], bz[c - sy], bz[c], bz[c + sy]) * idy - dbyz * idz;
  jy = dbxz * idz - dfc<4>(bz[c - 2], bz[c - 1], bz[c], bz[c + 1]) * idx;
  jz = dfc<4>(by[c - 2], by[c - 1], by[c], by[c + 1]) * idx - dfc<4>(bx[c - 2 * sy], bx[c - sy], bx[c], bx[c + sy]) * idy;
}

// face-centred averages of the resistive energy flux
__device__ __forceinline__ double by0_xface(const AView &a, long long f)
{
  const long long sy = a.g.s[1];
  const double *by = a.u[5];
  double b[4];
#pragma unroll
  for (int m = 0; m < 4; m++) {
    const long long p = f + (m - 2);
    b[m] = 0.5 * (by[p] + by[p + sy]);
  }
  return fcen<4>(b[0], b[1], b[2], b[3]);
}
__device__ __forceinline__ double bz0_xface(const AView &a, long long f)
{
  const double *bz = a.u[6];
  return fcen<4>(bz[f - 2], bz[f - 1], bz[f], bz[f + 1]);
}
__device__ __forceinline__ double bx0_yface(const AView &a, long long f)
{
  const long long sy = a.g.s[1];
  const double *bx = a.u[4];
  double b[4];
#pragma unroll
  for (int m = 0; m < 4; m++) {
    const long long p = f + (m - 2) * sy;
    b[m] = 0.5 * (bx[p] + bx[p + 1]);
  }
  return fcen<4>(b[0], b[1], b[2], b[3]);
}
__device__ __forceinline__ double bz0_yface(const AView &a, long long f)
{
  const long long sy = a.g.s[1];
  const double *bz = a.u[6];
  return fcen<4>(bz[f - 2 * sy], bz[f - sy], bz[f], bz[f + sy]);
}

__global__ void k_d_emf(AView a, double eta, double idx, double idy)
{
  QAS_ADJ_CELL(a.g);
  const Geo &g = a.g;
  if (!dflux_in(g, i, j)) {
#pragma unroll
    for (int q = 4; q < 7; q++) a.avl[q][c] = 0.0;
#pragma unroll
    for (int q = 0; q < 3; q++) a.avr[q][c] = 0.0;  // E is not formed outside the eres range
    return;
  }
  const long long sy = g.s[1];
  // CT update of bx, by
  double ezb = a.c1 * (-a.dtdy * d4_t(a.w[4], c, sy) + a.dtdx * d4_t(a.w[5], c, 1));
  // x-face energy flux at c and c-sy: -0.5 (ez[f] + ez[f+sy]) by0
  ezb += -0.5 * by0_xface(a, c) * a.avl[1][c];
  if (dflux_in(g, i, j - 1)) ezb += -0.5 * by0_xface(a, c - sy) * a.avl[1][c - sy];
  // y-face energy flux at c and c-1: +0.5 (ez[f] + ez[f+1]) bx0
  ezb += 0.5 * bx0_yface(a, c) * a.avl[3][c];
  if (dflux_in(g, i - 1, j)) ezb += 0.5 * bx0_yface(a, c - 1) * a.avl[3][c - 1];
  // ey: x-face bz flux and energy flux
  const double eyb = a.avl[0][c] + bz0_xface(a, c) * a.avl[1][c];
  // ex: y-face bz flux (-ex) and energy flux (-ex bz0)
  const double exb = -a.avl[2][c] - bz0_yface(a, c) * a.avl[3][c];
  const double e4 = 0.25 * (eta + eta + eta + eta);
  double jx, jy, jz;
  cur_j(a, c, idx, idy, jx, jy, jz);
  const double oeb = a.eb[c];
  a.avl[4][c] = e4 * exb;
  a.avl[5][c] = e4 * eyb;
  a.avl[6][c] = e4 * ezb;
  a.eb[c] = oeb + (jx * exb + jy * eyb + jz * ezb);
  // the forward E of this cell (mhd_ct_eres), for k_d_b
  a.avr[0][c] = e4 * jx;
  a.avr[1][c] = e4 * jy;
  a.avr[2][c] = e4 * jz;
}

__global__ void k_d_b(AView a, double eta, double idx, double idy)
{
  QAS_ADJ_CELL(a.g);
  const Geo &g = a.g;
  const long long sy = g.s[1];
  const double dw[4] = {1.0 / 24.0, -27.0 / 24.0, 27.0 / 24.0, -1.0 / 24.0};  // dfc<4> weights of fm, f0, f1, f2
  const double cw[4] = {-0.0625, 0.5625, 0.5625, -0.0625};                     // fcen<4> weights
  const double *jxb = a.avl[4], *jyb = a.avl[5], *jzb = a.avl[6];
  double bxb = 0.0, byb = 0.0, bzb = 0.0;
  // J^T: point m of the stencil at cell c is c + (m-2) s for m = 0..3
#pragma unroll
  for (int m = 0; m < 4; m++) {
    // along y: cell c' = c - (m-2) sy
    const int jc = j - (m - 2);
    if (jc >= 0 && jc < g.ny && dflux_in(g, i, jc)) {
      const long long cc = c - (m - 2) * sy;
      bzb += idy * dw[m] * jxb[cc];
      bxb += -idy * dw[m] * jzb[cc];
    }
    const int ic = i - (m - 2);
    if (ic >= 0 && ic < g.nx && dflux_in(g, ic, j)) {
      const long long cc = c - (m - 2);
      bzb += -idx * dw[m] * jyb[cc];
      byb += idx * dw[m] * jzb[cc];
    }
  }
  // energy fluxes: x face f: ey[f] bz0 - 0.5 (ez[f] + ez[f+sy]) by0
  //                y face f: 0.5 (ez[f] + ez[f+1]) bx0 - ex[f] bz0
  // (E from k_d_emf: zero outside the eres range, as the forward never reads it there
  //  for a face whose flux adjoint is non-zero)
  const double *ex = a.avr[0], *ey = a.avr[1], *ez = a.avr[2];
#pragma unroll
  for (int m = 0; m < 4; m++) {
    // bz[c] is point m of the x face f = c - (m-2)
    {
      const int fi = i - (m - 2);
      if (fi >= 0 && fi < g.nx && dflux_in(g, fi, j)) {
        const long long f = c - (m - 2);
        bzb += ey[f] * cw[m] * a.avl[1][f];
      }
    }
    // by[c] is point m of x face f = c - (m-2) (as p) and of f = c - sy - (m-2) (as p + sy)
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int fi = i - (m - 2), fj = j - h;
      if (fi >= 0 && fi < g.nx && fj >= 0 && dflux_in(g, fi, fj)) {
        const long long f = c - (m - 2) - h * sy;
        const double ez0 = 0.5 * (ez[f] + ez[f + sy]);
        byb += -ez0 * 0.5 * cw[m] * a.avl[1][f];
      }
    }
    // bx[c] is point m of y face f = c - (m-2) sy (as p) and of f = c - 1 - (m-2) sy (as p + 1)
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int fi = i - h, fj = j - (m - 2);
      if (fj >= 0 && fj < g.ny && fi >= 0 && dflux_in(g, fi, fj)) {
        const long long f = c - (m - 2) * sy - h;
        const double ey0 = 0.5 * (ez[f] + ez[f + 1]);
        bxb += ey0 * 0.5 * cw[m] * a.avl[3][f];
      }
    }
    // bz[c] is point m of y face f = c - (m-2) sy
    {
      const int fj = j - (m - 2);
      if (fj >= 0 && fj < g.ny && dflux_in(g, i, fj)) {
        const long long f = c - (m - 2) * sy;
        bzb += -ex[f] * cw[m] * a.avl[3][f];
      }
    }
  }
  const double ox = a.ai[4][c], oy = a.ai[5][c], oz = a.ai[6][c];
  a.ai[4][c] = ox + bxb;
  a.ai[5][c] = oy + byb;
  a.ai[6][c] = oz + bzb;
}

// deterministic sum of the per-cell eta adjoint (one block)
__global__ void k_a_sum(const double *x, long long n, double *out)
{
  __shared__ double sh[1024];
  double s = 0.0;
  for (long long k = threadIdx.x; k < n; k += blockDim.x) s += x[k];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sh[0];
}

}  // namespace qas
