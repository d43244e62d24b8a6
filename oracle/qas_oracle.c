/*
 * qas_oracle.c -- plain-C restatement of qasMHD's ideal-MHD step.
 *
 * TEST INFRASTRUCTURE (the checker).  Only tests/, __graft_entry__.smoke() and
 * the CPU-baseline leg of bench.py load this library; the product never does.
 *
 * Parity is pinned: tests/test_oracle_pins.py checks this restatement
 * bit-for-bit against the reference's own code built from its sources
 * (oracle/_ref, oracle/Makefile) and against the committed golden fixtures
 * made from it (tests/golden/make_golden.py).
 *
 * Every arithmetic expression keeps the reference's evaluation order and
 * constants, because bit-identical IEEE results need the identical operation
 * sequence; compiled with -ffp-contract=off.  Loop organisation, data layout
 * (SoA fluxes, per-direction central-flux buffers) and the ghost-fill passes
 * are our own.  Each function names the reference lines it restates.
 */
#include "qas_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NM 8
#define GH 4

typedef void (*lr_fn)(const double *f, double *fl, double *fr);
typedef double (*pt_fn)(const double *f);
typedef void (*flux_fn)(const double *L, const double *R, double bnc, double gamma,
                        const double *dv, double *F);

/* ------------------------------------------------------------------------ */
/* generic helpers: common/common_func.h:4-31                                */
/* ------------------------------------------------------------------------ */
static inline double qmax(double a, double b) { return (a >= b) ? a : b; }
static inline double qmin(double a, double b) { return (a >= b) ? b : a; }
static inline double qminmod(double a, double b) { return +qmin(qmax(a, b), 0.0) + qmax(qmin(a, b), 0.0); }
static inline double qminmod3(double a, double b, double c)
{
  return +qmin(qmax(qmax(a, b), c), 0.0) + qmax(qmin(qmin(a, b), c), 0.0);
}
static inline void rk_combine(double *f1, double f0, double df, double c0, double c1)
{
  *f1 = c0 * f0 + c1 * ((*f1) + df);
}

/* ------------------------------------------------------------------------ */
/* face/centre stencils: common/common_interp.h:6-24                         */
/* ------------------------------------------------------------------------ */
static double fcen2(const double *f) { return (0.5 * (f[0] + f[1])); }
static double fcen4(const double *f) { return (0.0625 * (9.0 * (f[0] + f[1]) - (f[-1] + f[2]))); }
static double dfc2(const double *f) { return (f[1] - f[0]); }
static double dfc4(const double *f) { return ((27.0 * (f[1] - f[0]) - (f[2] - f[-1])) / 24.0); }

/* linear and nonlinear face interpolations: common/common_interp.c:7-150 */
static void flr1(const double *f, double *fl, double *fr) { *fl = f[0]; *fr = f[0]; }
static void flr2(const double *f, double *fl, double *fr)
{
  *fl = (-f[-1] + 5.0 * f[0] + 2.0 * f[+1]) / 6.0;
  *fr = (-f[+1] + 5.0 * f[0] + 2.0 * f[-1]) / 6.0;
}
static void flr3(const double *f, double *fl, double *fr)
{
  *fl = 0.125 * (-f[-1] + 6.0 * f[0] + 3.0 * f[+1]);
  *fr = 0.125 * (-f[+1] + 6.0 * f[0] + 3.0 * f[-1]);
}
static void flr4(const double *f, double *fl, double *fr)
{
  *fl = 0.003125 * (9.0 * f[-2] - 56.0 * f[-1] + 234.0 * f[0] + 144.0 * f[+1] - 11.0 * f[+2]);
  *fr = 0.003125 * (9.0 * f[+2] - 56.0 * f[+1] + 234.0 * f[0] + 144.0 * f[-1] - 11.0 * f[-2]);
}
static void muscl_mm(const double *f, double *fl, double *fr)
{
  double d = 0.5 * qminmod(f[0] - f[-1], f[+1] - f[0]);
  *fl = f[0] + d;
  *fr = f[0] - d;
}
static void muscl_mc(const double *f, double *fl, double *fr)
{
  double alpha = 2.0;
  double d = 0.5 * qminmod(alpha * qminmod(f[0] - f[-1], f[+1] - f[0]), 0.5 * (f[+1] - f[-1]));
  *fl = f[0] + d;
  *fr = f[0] - d;
}
static void muscl_vl(const double *f, double *fl, double *fr)
{
  double a = f[0] - f[-1], b = f[+1] - f[0];
  double ab = a * b;
  double d = (ab > 0) ? (ab / (a + b)) : 0;
  *fl = f[0] + d;
  *fr = f[0] - d;
}
static void muscl_kr(const double *f, double *fl, double *fr)
{
  double d1 = 2.0 * (f[0] - f[-1]);
  double d2 = 2.0 * (f[+1] - f[0]);
  double dl = 0.5 * qminmod3(d1, d2, (0.5 * d1 + d2) / 3.0);
  double dr = 0.5 * qminmod3(d1, d2, (d1 + 0.5 * d2) / 3.0);
  *fl = f[0] + dl;
  *fr = f[0] - dr;
}
static void wcns3(const double *f, double *fl, double *fr)
{
  double is0, is1, w0, w1, c1, tau;
  const double eps = 1e-40;
  c1 = f[-1] - f[0];
  is0 = c1 * c1;
  c1 = f[+1] - f[0];
  is1 = c1 * c1;
  tau = f[+1] - 2.0 * f[0] + f[-1];
  tau = tau * tau;
  is0 = (1.0 + tau / (is0 + eps));
  is1 = (1.0 + tau / (is1 + eps));
  w0 = 0.25 * is0;
  w1 = 0.75 * is1;
  w0 /= (w0 + w1);
  w1 = 1.0 - w0;
  *fl = 0.5 * (w0 * (-f[-1] + 3.0 * f[0]) + w1 * (f[0] + f[+1]));
  w0 = 0.75 * is0;
  w1 = 0.25 * is1;
  w0 /= (w0 + w1);
  w1 = 1.0 - w0;
  *fr = 0.5 * (w1 * (-f[+1] + 3.0 * f[0]) + w0 * (f[0] + f[-1]));
}
static void wcns4(const double *f, double *fl, double *fr)
{
  double s0, s1, s2, w0, w1, w2, c1, c2, dn;
  const double eps = 1e-40;
  c1 = f[-2] - 4.0 * f[-1] + 3.0 * f[0];
  c2 = f[-2] - 2.0 * f[-1] + f[0];
  s0 = (13. / 12.) * c2 * c2 + 0.25 * c1 * c1;
  c1 = f[-1] - f[+1];
  c2 = f[-1] - 2.0 * f[0] + f[+1];
  s1 = (13. / 12.) * c2 * c2 + 0.25 * c1 * c1;
  c1 = f[+2] - 4.0 * f[+1] + 3.0 * f[0];
  c2 = f[+2] - 2.0 * f[+1] + f[0];
  s2 = (13. / 12.) * c2 * c2 + 0.25 * c1 * c1;
  s0 = 1.0 / (s0 * s0 + eps);
  s1 = 1.0 / (s1 * s1 + eps);
  s2 = 1.0 / (s2 * s2 + eps);
  /* linear weights 0.075/0.650/0.275 */
  w0 = 0.075 * s0;
  w1 = 0.650 * s1;
  w2 = 0.275 * s2;
  dn = 1.0 / (w0 + w1 + w2);
  w0 *= dn;
  w1 *= dn;
  w2 = 1.0 - w0 - w1;
  *fl = 0.125 * (+w0 * (3.0 * f[-2] - 10.0 * f[-1] + 15.0 * f[0])
                 + w1 * (-f[-1] + 6.0 * f[0] + 3.0 * f[+1])
                 + w2 * (+3.0 * f[0] + 6.0 * f[+1] - f[+2]));
  w0 = 0.275 * s0;
  w1 = 0.650 * s1;
  w2 = 0.075 * s2;
  dn = 1.0 / (w0 + w1 + w2);
  w0 *= dn;
  w1 *= dn;
  w2 = 1.0 - w0 - w1;
  *fr = 0.125 * (+w2 * (3.0 * f[+2] - 10.0 * f[+1] + 15.0 * f[0])
                 + w1 * (-f[+1] + 6.0 * f[0] + 3.0 * f[-1])
                 + w0 * (+3.0 * f[0] + 6.0 * f[-1] - f[-2]));
}

/* scheme tables: common/mhd_class.hpp:107-113 */
static lr_fn lin_interp(int odr)
{
  static const lr_fn t[4] = {flr1, flr2, flr3, flr4};
  return t[odr - 1];
}
static lr_fn nl_interp(int odr)
{
  static const lr_fn t[4] = {flr1, muscl_mm, wcns3, wcns4};
  return t[odr - 1];
}
static pt_fn face_to_centre(int odr) { return odr >= 3 ? fcen4 : fcen2; }
static pt_fn first_diff(int odr) { return odr >= 3 ? dfc4 : dfc2; }

/* ------------------------------------------------------------------------ */
/* equation of state: common/mhd_func.c:6-28, common/mhd_class.hpp:59-85     */
/* ------------------------------------------------------------------------ */
static double ieos(double ro, double vx, double vy, double vz, double bx, double by, double bz,
                   double en, double gamma)
{
  double v2 = vx * vx + vy * vy + vz * vz;
  double b2 = bx * bx + by * by + bz * bz;
  return (gamma - 1) * (en - 0.5 * (ro * v2 + b2));
}
static double energy(double ro, double vx, double vy, double vz, double bx, double by, double bz,
                     double pr, double gamma)
{
  double v2 = vx * vx + vy * vy + vz * vz;
  double b2 = bx * bx + by * by + bz * bz;
  return pr / (gamma - 1) + 0.5 * (ro * v2 + b2);
}

/* ------------------------------------------------------------------------ */
/* approximate eigenvectors: common/mhd_eigen.c:175-434                     */
/* L[k][n]: k-th left eigenvector (row), R[k][n]: k-th right eigenvector     */
/* ------------------------------------------------------------------------ */
static void eig_fast_alfven(double ro, double bx, double by, double bz, double pr, double gamma,
                            double L[7][7], double R[7][7])
{
  double iro = 1.0 / ro;
  double cs2 = gamma * pr * iro;
  double ca2 = bx * bx * iro;
  double ct2 = (by * by + bz * bz) * iro;
  double cb2 = cs2 + ca2 + ct2;
  double cf2 = 0.5 * (cb2 + sqrt(fabs(cb2 * cb2 - 4.0 * cs2 * ca2)));
  double cf = sqrt(cf2);
  double rcf = ro * cf;
  double sro = sqrt(ro);
  double isroh = 0.5 / sro;
  double icf2 = 1.0 / cf2;
  double icf2h = 0.5 * icf2;
  double ircfh = 0.5 / rcf;
  double byh = 0.5 * by, bzh = 0.5 * bz;
  memset(L, 0, sizeof(double) * 49);
  memset(R, 0, sizeof(double) * 49);
  L[0][1] = -rcf; L[0][4] = +by; L[0][5] = +bz; L[0][6] = +1.0;
  L[1][0] = cf2;  L[1][4] = -by; L[1][5] = -bz; L[1][6] = -1.0;
  L[2][1] = +rcf; L[2][4] = +by; L[2][5] = +bz; L[2][6] = +1.0;
  L[3][2] = +sro; L[3][4] = +1.0;
  L[4][2] = +sro; L[4][4] = -1.0;
  L[5][3] = +sro; L[5][5] = +1.0;
  L[6][3] = +sro; L[6][5] = -1.0;
  R[0][0] = +icf2h; R[0][1] = -ircfh; R[0][6] = +0.5;
  R[1][0] = +icf2;
  R[2][0] = +icf2h; R[2][1] = +ircfh; R[2][6] = +0.5;
  R[3][2] = +isroh; R[3][4] = +0.5; R[3][6] = -byh;
  R[4][2] = +isroh; R[4][4] = -0.5; R[4][6] = +byh;
  R[5][3] = +isroh; R[5][5] = +0.5; R[5][6] = -bzh;
  R[6][3] = +isroh; R[6][5] = -0.5; R[6][6] = +bzh;
}

static void eig_alfven_entropy(double ro, double bx, double by, double bz, double pr, double gamma,
                               double L[7][7], double R[7][7])
{
  double iro = 1.0 / ro;
  double cs2 = gamma * pr * iro;
  double ca2 = bx * bx * iro;
  double ct2 = (by * by + bz * bz) * iro;
  double cb2 = cs2 + ca2 + ct2;
  double cf2 = 0.5 * (cb2 + sqrt(fabs(cb2 * cb2 - 4.0 * cs2 * ca2)));
  double sro = sqrt(ro);
  double isroh = 0.5 / sro;
  double icf2 = 1.0 / cf2;
  double byh = 0.5 * by, bzh = 0.5 * bz;
  memset(L, 0, sizeof(double) * 49);
  memset(R, 0, sizeof(double) * 49);
  L[0][1] = +1.0;
  L[1][0] = cf2;  L[1][4] = -by; L[1][5] = -bz; L[1][6] = -1.0;
  L[2][4] = +by;  L[2][5] = +bz; L[2][6] = +1.0;
  L[3][2] = +sro; L[3][4] = +1.0;
  L[4][2] = +sro; L[4][4] = -1.0;
  L[5][3] = +sro; L[5][5] = +1.0;
  L[6][3] = +sro; L[6][5] = -1.0;
  R[0][1] = +1.0;
  R[1][0] = +icf2;
  R[2][0] = +icf2; R[2][6] = +1.0;
  R[3][2] = +isroh; R[3][4] = +0.5; R[3][6] = -byh;
  R[4][2] = +isroh; R[4][4] = -0.5; R[4][6] = +byh;
  R[5][3] = +isroh; R[5][5] = +0.5; R[5][6] = -bzh;
  R[6][3] = +isroh; R[6][5] = -0.5; R[6][6] = +bzh;
}

/* Athena-type eigenvectors of the non-conservative form: mhd_eigen_st (common/mhd_eigen.c:5-173);
 * L[k] = row l(k+1), R[k] = column r(k+1) */
static void eig_athena(double ro, double bx, double by, double bz, double pr, double gamma,
                       double L[7][7], double R[7][7])
{
  double eps = 1e-12;
  double sqrt2 = sqrt(2.0);
  double iro = 1.0 / ro;
  double sro = sqrt(ro);
  double isro = 1.0 / sro;
  double bxsr = bx * isro, bysr = by * isro, bzsr = bz * isro;
  double bx2 = bxsr * bxsr;
  double bt2 = bysr * bysr + bzsr * bzsr;
  double b2 = bx2 + bt2;
  double a2 = fabs(gamma * pr / ro);
  double aa = sqrt(a2);
  double ca2 = bx2;
  double junk = sqrt(fabs((a2 + b2) * (a2 + b2) - 4.0 * a2 * ca2));
  double cf2 = fabs(0.5 * (a2 + b2 + junk));
  double cf = sqrt(cf2);
  double cs2 = fabs(0.5 * (a2 + b2 - junk));
  double cs = sqrt(cs2);
  bx2 = bx * bx;
  bt2 = by * by + bz * bz;
  b2 = bx2 + bt2;
  double denom = 1.0 / sqrt(bt2);
  int flag = (bt2 > eps * b2);
  double betay = (flag) ? (by * denom) : (0.5 * sqrt2);
  double betaz = (flag) ? (bz * denom) : (0.5 * sqrt2);
  denom = 1.0 / sqrt(fabs(cf2 - cs2));
  flag = ((bt2 > eps * b2) || (fabs(gamma * pr - bx2) > eps * gamma * pr));
  double alphaf = (flag) ? (sqrt(fabs(a2 - cs2)) * denom) : 1.0;
  double alphas = (flag) ? (sqrt(fabs(cf2 - a2)) * denom) : 0.0;
  double sgnbx = (bx > 0) ? (1.0) : (-1.0);
  double cfalf = cf * alphaf, csals = cs * alphas, aaalf = aa * alphaf, aaals = aa * alphas;
  int n;
  denom = 0.5 / a2;
  memset(L, 0, sizeof(double) * 49);
  memset(R, 0, sizeof(double) * 49);
  L[0][1] = -cfalf * denom; L[0][2] = +csals * denom * sgnbx * betay; L[0][3] = +csals * denom * sgnbx * betaz;
  L[0][4] = +aaals * denom * isro * betay; L[0][5] = +aaals * denom * isro * betaz; L[0][6] = alphaf * denom * iro;
  L[1][2] = -0.5 * betaz; L[1][3] = +0.5 * betay;
  L[1][4] = -0.5 * isro * betaz * sgnbx; L[1][5] = +0.5 * isro * betay * sgnbx;
  L[2][1] = -csals * denom; L[2][2] = -cfalf * denom * sgnbx * betay; L[2][3] = -cfalf * denom * sgnbx * betaz;
  L[2][4] = -aaalf * denom * isro * betay; L[2][5] = -aaalf * denom * isro * betaz; L[2][6] = alphas * denom * iro;
  L[3][0] = 1.0; L[3][6] = -1.0 / a2;
  R[0][0] = ro * alphaf; R[0][1] = -cfalf; R[0][2] = +csals * sgnbx * betay; R[0][3] = +csals * sgnbx * betaz;
  R[0][4] = +aaals * sro * betay; R[0][5] = +aaals * sro * betaz; R[0][6] = alphaf * gamma * pr;
  R[1][2] = -betaz; R[1][3] = +betay; R[1][4] = -sro * betaz * sgnbx; R[1][5] = +sro * betay * sgnbx;
  R[2][0] = ro * alphas; R[2][1] = -csals; R[2][2] = -cfalf * sgnbx * betay; R[2][3] = -cfalf * sgnbx * betaz;
  R[2][4] = -aaalf * sro * betay; R[2][5] = -aaalf * sro * betaz; R[2][6] = alphas * gamma * pr;
  R[3][0] = 1.0;
  /* l7, l6, l5 (r7, r6, r5) mirror l1, l2, l3: +, -, -, -, +, +, + */
  for (n = 0; n < 7; n++) {
    const double sg = (n >= 1 && n <= 3) ? -1.0 : 1.0;
    L[6][n] = sg > 0 ? +L[0][n] : -L[0][n];
    L[5][n] = sg > 0 ? +L[1][n] : -L[1][n];
    L[4][n] = sg > 0 ? +L[2][n] : -L[2][n];
    R[6][n] = sg > 0 ? +R[0][n] : -R[0][n];
    R[5][n] = sg > 0 ? +R[1][n] : -R[1][n];
    R[4][n] = sg > 0 ? +R[2][n] : -R[2][n];
  }
}

/* characteristic reconstruction: common/mhd_eigen.c:513-665 (mode 0: mhd_m_reconst's
 * eigenvectors when fast, mhd_a_reconst's else) and :436-511 (mode 2: mhd_c_reconst).
 * q[v][m]: primitive v (ro,vn,vt,vu,bt,bu,pr) at stencil point m=0..4 */
static void char_reconst(int fast, int mode, const double q[7][5], double bn, double gamma, lr_fn lr,
                         double *ul, double *ur)
{
  double L[7][7], R[7][7], w[7][5], wl[7], wr[7];
  int k, m, n;
  if (mode == 2)
    eig_athena(q[0][2], bn, q[4][2], q[5][2], q[6][2], gamma, L, R);
  else if (fast)
    eig_fast_alfven(q[0][2], bn, q[4][2], q[5][2], q[6][2], gamma, L, R);
  else
    eig_alfven_entropy(q[0][2], bn, q[4][2], q[5][2], q[6][2], gamma, L, R);
  for (m = 0; m < 5; m++) {
    for (k = 0; k < 7; k++) {
      w[k][m] = (+L[k][0] * q[0][m] + L[k][1] * q[1][m] + L[k][2] * q[2][m] + L[k][3] * q[3][m]
                 + L[k][4] * q[4][m] + L[k][5] * q[5][m] + L[k][6] * q[6][m]);
    }
  }
  for (k = 0; k < 7; k++) lr(&w[k][2], &wl[k], &wr[k]);
  for (n = 0; n < 7; n++)
    ul[n] = R[0][n] * wl[0] + R[1][n] * wl[1] + R[2][n] * wl[2] + R[3][n] * wl[3] + R[4][n] * wl[4]
            + R[5][n] * wl[5] + R[6][n] * wl[6];
  for (n = 0; n < 7; n++)
    ur[n] = R[0][n] * wr[0] + R[1][n] * wr[1] + R[2][n] * wr[2] + R[3][n] * wr[3] + R[4][n] * wr[4]
            + R[5][n] * wr[5] + R[6][n] * wr[6];
  /* keep exactly-zero velocity / transverse field exactly zero */
  for (n = 1; n <= 5; n++) {
    int allzero = 1;
    for (m = 0; m < 5; m++)
      if (q[n][m] != 0.0) allzero = 0;
    if (allzero) ul[n] = ur[n] = 0.0;
  }
}

/* mhd_lrstate (common/mhd_func.c:108-161); mode 1: the reconstruction call replaced by the
 * primitive-variable mhd_reconst (common/mhd_eigen.c:667-706), mode 2: by the Athena-type
 * mhd_c_reconst (:436-511) */
static void face_states(const double q[7][5], double bn, double gamma, lr_fn lr, double *vl, double *vr, int mode)
{
  const double eps = 1e-12;
  if (mode == 1) {
    for (int n = 0; n < 7; n++) lr(&q[n][2], &vl[n], &vr[n]);
  } else {
    int fast = (q[0][2] * (q[1][2] * q[1][2] + q[2][2] * q[2][2] + q[3][2] * q[3][2]) > gamma * q[6][2]);
    char_reconst(fast, mode, q, bn, gamma, lr, vl, vr);
  }
  if (vl[0] <= eps || vl[6] <= eps) {
    vl[0] = q[0][2];
    vl[1] = q[1][2];
    vl[6] = q[6][2];
  }
  if (vr[0] <= eps || vr[6] <= eps) {
    vr[0] = q[0][2];
    vr[1] = q[1][2];
    vr[6] = q[6][2];
  }
}

/* ------------------------------------------------------------------------ */
/* Riemann solvers: common/mhd_flux.c.  L/R = (ro,vn,vt,vu,bt,bu,pr),        */
/* F = (fro,fmn,fmt,fmu,fbt,fbu,fen)                                         */
/* ------------------------------------------------------------------------ */
#define FL_EPS (1e-8)

/* MLAU: common/mhd_flux.c:7-192 */
static void flux_mlau(const double *L, const double *R, double bnc, double gamma, const double *dv, double *F)
{
  double rol = L[0], vnl = L[1], vtl = L[2], vul = L[3], btl = L[4], bul = L[5], prl = L[6];
  double ror = R[0], vnr = R[1], vtr = R[2], vur = R[3], btr = R[4], bur = R[5], prr = R[6];
  double gammam1i = 1.0 / (gamma - 1.0);
  double bnc2 = bnc * bnc;
  double sgn = (bnc > 0) ? (1.0) : (-1.0);
  double bnca = sgn * bnc;
  double roli = 1.0 / rol;
  double vl2 = vnl * vnl + vtl * vtl + vul * vul;
  double pml = 0.5 * (btl * btl + bul * bul);
  double ptl = prl + pml;
  double enl = gammam1i * prl + pml + 0.5 * rol * vl2;
  double hnl = (enl + ptl) * roli;
  double rori = 1.0 / ror;
  double vr2 = vnr * vnr + vtr * vtr + vur * vur;
  double pmr = 0.5 * (btr * btr + bur * bur);
  double ptr = prr + pmr;
  double enr = gammam1i * prr + pmr + 0.5 * ror * vr2;
  double hnr = (enr + ptr) * rori;
  double cl2 = gamma * prl * roli;
  double cr2 = gamma * prr * rori;
  double cal2 = bnc2 * roli;
  double car2 = bnc2 * rori;
  double cbl2 = cl2 + cal2 + 2.0 * pml * roli;
  double cbr2 = cr2 + car2 + 2.0 * pmr * rori;
  double cfl2 = 0.5 * (cbl2 + sqrt(fabs(cbl2 * cbl2 - 4.0 * cl2 * cal2)));
  double cfr2 = 0.5 * (cbr2 + sqrt(fabs(cbr2 * cbr2 - 4.0 * cr2 * car2)));
  cbl2 = vl2 + cal2 + 2.0 * pml * roli;
  cbr2 = vr2 + car2 + 2.0 * pmr * rori;
  double ccl2 = 0.5 * (cbl2 + sqrt(fabs(cbl2 * cbl2 - 4.0 * vl2 * cal2)));
  double ccr2 = 0.5 * (cbr2 + sqrt(fabs(cbr2 * cbr2 - 4.0 * vr2 * car2)));
  double cmax = sqrt(qmax(cfl2, cfr2));
  double cfn = cmax;
  double cfni = 1.0 / cfn;
  double sl = qmin(0.0, qmin(vnl, vnr) - cmax);
  double sr = qmax(0.0, qmax(vnl, vnr) + cmax);
  double mal = vnl * cfni;
  double mar = vnr * cfni;
  double snl = (mal > 0) ? 1.0 : (-1.0);
  double snr = (mar > 0) ? 1.0 : (-1.0);
  double theta = qmin(1.0, (cfn - qmin(dv[0], 0.0)) / (cfn - qmin(dv[1], 0.0)));
  theta *= theta;
  theta *= theta;
  double alpha = 0.1875, beta = 0.125;
  double malp1 = mal + 1.0;
  double marm1 = mar - 1.0;
  double mal2m1 = mal * mal - 1.0;
  double mar2m1 = mar * mar - 1.0;
  double bfl, ffl, bfr, ffr;
  if (snl * mal > 1.0) {
    bfl = 0.5 * (1.0 + snl);
    ffl = bfl * mal;
  } else {
    bfl = +0.25 * malp1 * malp1 * (2.0 - mal) + alpha * mal * mal2m1 * mal2m1;
    ffl = +0.25 * malp1 * malp1 + beta * mal2m1 * mal2m1;
  }
  if (snr * mar > 1.0) {
    bfr = 0.5 * (1.0 - snr);
    ffr = bfr * mar;
  } else {
    bfr = +0.25 * marm1 * marm1 * (2.0 + mar) - alpha * mar * mar2m1 * mar2m1;
    ffr = -0.25 * marm1 * marm1 - beta * mar2m1 * mar2m1;
  }
  double mnc = ffl + ffr;
  double mflux = mnc * cfn;
  mflux -= qmax(1.0 - fabs(mnc), 0.0) * theta * cfni * (ptr - ptl) / (rol + ror);
  double dir = (mflux > 0) ? 1.0 : (-1.0);
  double dirl = 0.5 * (1.0 + dir);
  double dirr = 1.0 - dirl;
  mflux *= (dirl * rol + dirr * ror);
  double mfl = mflux * dirl;
  double mfr = mflux - mfl;
  double ptot = bfl * ptl + bfr * ptr;
  double cfmod = sqrt(qmax(ccl2, ccr2));
  ptot -= 0.25 * bfl * bfr * (rol + ror) * cfmod * (vnr - vnl);
  ptot -= 0.5 * (1.0 - cfmod * cfni) * (bfl + bfr - 1.0) * (ptl + ptr);
  double slvl = sl - vnl;
  double srvr = sr - vnr;
  double snc = dirl * sl + dirr * sr;
  double vndnm = mflux + dirl * rol * slvl + dirr * ror * srvr;
  double vnc = ((fabs(vndnm) > FL_EPS) && (snc != 0)) ? (mflux * snc / vndnm) : (dirl * vnl + dirr * vnr);
  double slvc = sl - vnc;
  double srvc = sr - vnc;
  double slvci = 1.0 / slvc;
  double srvci = 1.0 / srvc;
  double rhdl = rol * slvl * slvc - bnc2;
  double rhdr = ror * srvr * srvc - bnc2;
  double dvtl = 0.0, dvul = 0.0, dbtl = 0.0, dbul = 0.0;
  double dvtr = 0.0, dvur = 0.0, dbtr = 0.0, dbur = 0.0;
  if (fabs(rhdl) > FL_EPS) {
    double q = (vnc - vnl) / rhdl;
    dvtl = -bnc * btl * q;
    dvul = -bnc * bul * q;
    dbtl = bnc2 * btl * q * slvci;
    dbul = bnc2 * bul * q * slvci;
  }
  if (fabs(rhdr) > FL_EPS) {
    double q = (vnc - vnr) / rhdr;
    dvtr = -bnc * btr * q;
    dvur = -bnc * bur * q;
    dbtr = bnc2 * btr * q * srvci;
    dbur = bnc2 * bur * q * srvci;
  }
  double cmpl = slvl * slvci;
  double cmpr = srvr * srvci;
  double ro2l = rol * cmpl;
  double srol = sqrt(ro2l);
  double vt2l = dvtl + vtl;
  double vu2l = dvul + vul;
  double bt2l = dbtl + btl * cmpl;
  double bu2l = dbul + bul * cmpl;
  double ro2r = ror * cmpr;
  double sror = sqrt(ro2r);
  double vt2r = dvtr + vtr;
  double vu2r = dvur + vur;
  double bt2r = dbtr + btr * cmpr;
  double bu2r = dbur + bur * cmpr;
  double sroi = 1.0 / (srol + sror);
  double srollri = srol * sroi;
  double srorlri = sror * sroi;
  double bnflb = sgn * qmin(qmax(0.0, srollri * (bnca + sror * vnc)), bnca);
  double bnfrb = sgn * qmin(qmax(0.0, srorlri * (bnca - srol * vnc)), bnca);
  double bnflv = sgn * qmin(qmax(0.0, srorlri * (bnca + mflux / sror)), bnca);
  double bnfrv = sgn * qmin(qmax(0.0, srollri * (bnca - mflux / srol)), bnca);
  double bnsrv = qmax(bnca - dir * vnc * (dirl * srol + dirr * sror), 0.0);
  double ccb = sroi * bnsrv;
  double ccv = srol * sror * ccb;
  double bnvt = bnflb * vt2l + bnfrb * vt2r + ccb * (bt2r - bt2l);
  double bnvu = bnflb * vu2l + bnfrb * vu2r + ccb * (bu2r - bu2l);
  double bnbt = bnflv * bt2l + bnfrv * bt2r + ccv * (vt2r - vt2l);
  double bnbu = bnflv * bu2l + bnfrv * bu2r + ccv * (vu2r - vu2l);
  bnvt -= vnc * (dirl * dbtl + dirr * dbtr);
  bnvu -= vnc * (dirl * dbul + dirr * dbur);
  bnbt -= mflux * (dirl * dvtl + dirr * dvtr);
  bnbu -= mflux * (dirl * dvul + dirr * dvur);
  F[0] = mflux;
  F[1] = mfl * vnl + mfr * vnr + ptot - 0.5 * bnc2;
  F[2] = mfl * vtl + mfr * vtr - bnbt;
  F[3] = mfl * vul + mfr * vur - bnbu;
  F[4] = mfl * btl * roli + mfr * btr * rori - bnvt;
  F[5] = mfl * bul * roli + mfr * bur * rori - bnvu;
  double vb1 = dirl * (vtl * btl + vul * bul) + dirr * (vtr * btr + vur * bur);
  double vb2 = dirl * (vt2l * bt2l + vu2l * bu2l) + dirr * (vt2r * bt2r + vu2r * bu2r);
  double rv2b2 = (mflux * vnc - bnc2);
  rv2b2 *= rv2b2;
  double vb3 = 0.0;
  if (rv2b2 > FL_EPS * FL_EPS) {
    vb3 = (+(F[2] * vnc + F[4] * bnc) * (F[2] * bnc + F[4] * mflux)
           + (F[3] * vnc + F[5] * bnc) * (F[3] * bnc + F[5] * mflux)) / rv2b2;
  }
  double bnvb = sgn * (bnca * (snc * vb2 - vnc * vb1) * (dirl * slvci + dirr * srvci) + bnsrv * (vb3 - vb2));
  F[6] = mfl * hnl + mfr * hnr - bnvb;
}

/* Roe: common/mhd_flux.c:194-433 */
static void flux_roe(const double *L, const double *R, double bnc, double gamma, const double *dv, double *F)
{
  double rol = L[0], vnl = L[1], vtl = L[2], vul = L[3], btl = L[4], bul = L[5], prl = L[6];
  double ror = R[0], vnr = R[1], vtr = R[2], vur = R[3], btr = R[4], bur = R[5], prr = R[6];
  (void)dv;
  double gammam1 = gamma - 1.0;
  double gammam2 = gamma - 2.0;
  double gammam1i = 1.0 / gammam1;
  double roli = 1.0 / rol;
  double rori = 1.0 / ror;
  double rrol = sqrt(rol);
  double rror = sqrt(ror);
  double rroi = 1.0 / (rrol + rror);
  double robar = rrol * rror;
  double robari = 1.0 / robar;
  double rrobar = sqrt(robar);
  double rrobai = sqrt(robari);
  double vnbar = (rrol * vnl + rror * vnr) * rroi;
  double vtbar = (rrol * vtl + rror * vtr) * rroi;
  double vubar = (rrol * vul + rror * vur) * rroi;
  double bnbar = bnc;
  double btbar = (rrol * btr + rror * btl) * rroi;
  double bubar = (rrol * bur + rror * bul) * rroi;
  double hl = (+gamma * gammam1i * prl * roli + 0.5 * (vnl * vnl + vtl * vtl + vul * vul)
               + (bnbar * bnbar + btl * btl + bul * bul) * roli);
  double hr = (+gamma * gammam1i * prr * rori + 0.5 * (vnr * vnr + vtr * vtr + vur * vur)
               + (bnbar * bnbar + btr * btr + bur * bur) * rori);
  double hbar = (rrol * hl + rror * hr) * rroi;
  double btave = 0.5 * (btl + btr);
  double buave = 0.5 * (bul + bur);
  double sgn = (bnbar > 0) ? (1.0) : (-1.0);
  double db2 = 0.5 * gammam2 * gammam1i * ((btr - btl) * (btr - btl) + (bur - bul) * (bur - bul)) * rroi * rroi;
  double c2 = gammam1 * (+hbar - 0.5 * (vnbar * vnbar + vtbar * vtbar + vubar * vubar) - db2
                         - (bnbar * bnbar + btbar * btbar + bubar * bubar) * robari);
  double a2 = (gammam1 * (+hbar - 0.5 * (vnbar * vnbar + vtbar * vtbar + vubar * vubar) - db2)
               - gammam2 * (bnbar * bnbar + btbar * btbar + bubar * bubar) * robari);
  double ca2 = bnbar * bnbar * robari;
  double cb2 = (btbar * btbar + bubar * bubar) * robari;
  double cf2 = 0.5 * (a2 + sqrt(cb2 * (a2 + c2 + ca2) + (c2 - ca2) * (c2 - ca2)));
  double cs2 = c2 * ca2 / cf2;
  double cf = sqrt(cf2);
  double cs = sqrt(cs2);
  double ca = sqrt(ca2);
  double c = sqrt(c2);
  double cfi = 1.0 / cf;
  double sgr1 = btbar * btbar + bubar * bubar - FL_EPS;
  double sf11 = (sgr1 > 0) ? 1.0 : 0.0;
  double sf21 = 1.0 - sf11;
  double beti = 1.0 / sqrt(btbar * btbar + bubar * bubar + sf21);
  double bett = sf11 * btbar * beti + sf21 * sqrt(0.5);
  double betu = sf11 * bubar * beti + sf21 * sqrt(0.5);
  double sgr2 = (btbar * btbar + bubar * bubar) * robari + fabs(ca2 - c2) - FL_EPS;
  double sf12 = (sgr2 > 0) ? 1.0 : 0.0;
  double sf22 = 1.0 - sf12;
  double cfca = qmax(0.0, cf2 - ca2);
  double cfcs = qmax(0.0, cf2 - cs2);
  double cfa = qmax(0.0, cf2 - c2);
  double alpi = 1.0 / sqrt(cfcs + sf22);
  double alpf = sf12 * sqrt(cfca) * alpi + sf22;
  double alps = sf12 * sqrt(cfa) * alpi;
  double eeps = 0.0;
  double evpf = qmax(fabs(vnbar + cf), eeps);
  double evmf = qmax(fabs(vnbar - cf), eeps);
  double evps = qmax(fabs(vnbar + cs), eeps);
  double evms = qmax(fabs(vnbar - cs), eeps);
  double evpa = qmax(fabs(vnbar + ca), eeps);
  double evma = qmax(fabs(vnbar - ca), eeps);
  double ev00 = qmax(fabs(vnbar), eeps);
  double dltro = ror - rol;
  double dltmn = robar * (vnr - vnl);
  double dltmt = robar * (vtr - vtl);
  double dltmu = robar * (vur - vul);
  double dltbt = btr - btl;
  double dltbu = bur - bul;
  double t1 = bett * dltbt + betu * dltbu;
  double t2 = (prr - prl + (btave * dltbt + buave * dltbu) + gammam2 * (btbar * dltbt + bubar * dltbu)) * gammam1i;
  double t3 = betu * dltbt - bett * dltbu;
  double s1 = dltmn;
  double s2 = bett * dltmt + betu * dltmu;
  double s3 = betu * dltmt - bett * dltmu;
  double p11 = alps * cf * rrobai;
  double p12 = -alpf * c2 * cfi * rrobai;
  double p21 = alpf * (cf2 - c2 * gammam2 * gammam1i);
  double p22 = alps * (cs2 - c2 * gammam2 * gammam1i);
  double q11 = alpf * cf;
  double q12 = alps * cs;
  double q21 = -alps * ca * sgn;
  double q22 = alpf * c * sgn;
  double detpi = 1.0 / (p11 * p22 - p12 * p21);
  double detqi = 1.0 / (q11 * q22 - q12 * q21);
  double wvpf = 0.5 * ((p22 * t1 - p12 * t2) * detpi + (q22 * s1 - q12 * s2) * detqi);
  double wvmf = 0.5 * ((p22 * t1 - p12 * t2) * detpi - (q22 * s1 - q12 * s2) * detqi);
  double wvps = 0.5 * ((-p21 * t1 + p11 * t2) * detpi + (-q21 * s1 + q11 * s2) * detqi);
  double wvms = 0.5 * ((-p21 * t1 + p11 * t2) * detpi - (-q21 * s1 + q11 * s2) * detqi);
  double wvpa = 0.5 * (rrobar * t3 - sgn * s3);
  double wvma = 0.5 * (rrobar * t3 + sgn * s3);
  double wv00 = dltro - alpf * (wvpf + wvmf) - alps * (wvps + wvms);
  double frol = rol * vnl;
  double fmnl = rol * vnl * vnl + prl + 0.5 * (-bnbar * bnbar + btl * btl + bul * bul);
  double fmtl = rol * vnl * vtl - bnbar * btl;
  double fmul = rol * vnl * vul - bnbar * bul;
  double fbtl = vnl * btl - vtl * bnbar;
  double fbul = vnl * bul - vul * bnbar;
  double fenl = rol * vnl * hl - bnbar * (bnbar * vnl + btl * vtl + bul * vul);
  double fror = ror * vnr;
  double fmnr = ror * vnr * vnr + prr + 0.5 * (-bnbar * bnbar + btr * btr + bur * bur);
  double fmtr = ror * vnr * vtr - bnbar * btr;
  double fmur = ror * vnr * vur - bnbar * bur;
  double fbtr = vnr * btr - vtr * bnbar;
  double fbur = vnr * bur - vur * bnbar;
  double fenr = ror * vnr * hr - bnbar * (bnbar * vnr + btr * vtr + bur * vur);
  double v2h = 0.5 * (vnbar * vnbar + vtbar * vtbar + vubar * vubar);
  double rvpfro = alpf;
  double rvpfmn = alpf * (vnbar + cf);
  double rvpfmt = alpf * vtbar - alps * bett * ca * sgn;
  double rvpfmu = alpf * vubar - alps * betu * ca * sgn;
  double rvpfbt = alps * bett * cf * rrobai;
  double rvpfbu = alps * betu * cf * rrobai;
  double rvpfen = alpf * (v2h + db2 + cf * vnbar + cf2 * gammam1i + (cf2 - c2) * gammam2 * gammam1i)
                  - alps * ca * (bett * vtbar + betu * vubar) * sgn;
  double rvmfro = alpf;
  double rvmfmn = alpf * (vnbar - cf);
  double rvmfmt = alpf * vtbar + alps * bett * ca * sgn;
  double rvmfmu = alpf * vubar + alps * betu * ca * sgn;
  double rvmfbt = rvpfbt;
  double rvmfbu = rvpfbu;
  double rvmfen = alpf * (v2h + db2 - cf * vnbar + cf2 * gammam1i + (cf2 - c2) * gammam2 * gammam1i)
                  + alps * ca * (bett * vtbar + betu * vubar) * sgn;
  double rvpsro = alps;
  double rvpsmn = alps * (vnbar + cs);
  double rvpsmt = alps * vtbar + c * sgn * alpf * bett;
  double rvpsmu = alps * vubar + c * sgn * alpf * betu;
  double rvpsbt = -rrobai * c2 * alpf * bett * cfi;
  double rvpsbu = -rrobai * c2 * alpf * betu * cfi;
  double rvpsen = alps * (v2h + db2 + cs * vnbar + cs2 * gammam1i + (cs2 - c2) * gammam2 * gammam1i)
                  + alpf * c * (bett * vtbar + betu * vubar) * sgn;
  double rvmsro = alps;
  double rvmsmn = alps * (vnbar - cs);
  double rvmsmt = alps * vtbar - c * sgn * alpf * bett;
  double rvmsmu = alps * vubar - c * sgn * alpf * betu;
  double rvmsbt = rvpsbt;
  double rvmsbu = rvpsbu;
  double rvmsen = alps * (v2h + db2 - cs * vnbar + cs2 * gammam1i + (cs2 - c2) * gammam2 * gammam1i)
                  - alpf * c * (bett * vtbar + betu * vubar) * sgn;
  double rvparo = 0.0, rvpamn = 0.0;
  double rvpamt = -sgn * betu;
  double rvpamu = sgn * bett;
  double rvpabt = rrobai * betu;
  double rvpabu = -rrobai * bett;
  double rvpaen = -(betu * vtbar - bett * vubar) * sgn;
  double rvmaro = 0.0, rvmamn = 0.0;
  double rvmamt = -rvpamt;
  double rvmamu = -rvpamu;
  double rvmabt = rvpabt;
  double rvmabu = rvpabu;
  double rvmaen = -rvpaen;
  double rv00ro = 1.0;
  double rv00mn = vnbar;
  double rv00mt = vtbar;
  double rv00mu = vubar;
  double rv00bt = 0.0, rv00bu = 0.0;
  double rv00en = v2h + db2;
  F[0] = 0.5 * (+frol + fror - evpf * wvpf * rvpfro - evmf * wvmf * rvmfro - evps * wvps * rvpsro
                - evms * wvms * rvmsro - evpa * wvpa * rvparo - evma * wvma * rvmaro - ev00 * wv00 * rv00ro);
  F[1] = 0.5 * (+fmnl + fmnr - evpf * wvpf * rvpfmn - evmf * wvmf * rvmfmn - evps * wvps * rvpsmn
                - evms * wvms * rvmsmn - evpa * wvpa * rvpamn - evma * wvma * rvmamn - ev00 * wv00 * rv00mn);
  F[2] = 0.5 * (fmtl + fmtr - evpf * wvpf * rvpfmt - evmf * wvmf * rvmfmt - evps * wvps * rvpsmt
                - evms * wvms * rvmsmt - evpa * wvpa * rvpamt - evma * wvma * rvmamt - ev00 * wv00 * rv00mt);
  F[3] = 0.5 * (fmul + fmur - evpf * wvpf * rvpfmu - evmf * wvmf * rvmfmu - evps * wvps * rvpsmu
                - evms * wvms * rvmsmu - evpa * wvpa * rvpamu - evma * wvma * rvmamu - ev00 * wv00 * rv00mu);
  F[4] = 0.5 * (fbtl + fbtr - evpf * wvpf * rvpfbt - evmf * wvmf * rvmfbt - evps * wvps * rvpsbt
                - evms * wvms * rvmsbt - evpa * wvpa * rvpabt - evma * wvma * rvmabt - ev00 * wv00 * rv00bt);
  F[5] = 0.5 * (fbul + fbur - evpf * wvpf * rvpfbu - evmf * wvmf * rvmfbu - evps * wvps * rvpsbu
                - evms * wvms * rvmsbu - evpa * wvpa * rvpabu - evma * wvma * rvmabu - ev00 * wv00 * rv00bu);
  F[6] = 0.5 * (fenl + fenr - evpf * wvpf * rvpfen - evmf * wvmf * rvmfen - evps * wvps * rvpsen
                - evms * wvms * rvmsen - evpa * wvpa * rvpaen - evma * wvma * rvmaen - ev00 * wv00 * rv00en);
}

/* HLLD (lowdiss=0, common/mhd_flux.c:435-561) and LHLLD (lowdiss=1, :563-698) */
static void flux_hlld_common(int lowdiss, const double *L, const double *R, double bnc, double gamma,
                             const double *dv, double *F)
{
  double rol = L[0], vnl = L[1], vtl = L[2], vul = L[3], btl = L[4], bul = L[5], prl = L[6];
  double ror = R[0], vnr = R[1], vtr = R[2], vur = R[3], btr = R[4], bur = R[5], prr = R[6];
  double gammam1i = 1.0 / (gamma - 1.0);
  double bnc2 = bnc * bnc;
  double sgn = (bnc > 0) ? (1.0) : (-1.0);
  double roli = 1.0 / rol;
  double pml = 0.5 * (btl * btl + bul * bul);
  double ptl = prl + pml;
  double vl2 = 0.0, vr2 = 0.0, enl, enr;
  if (lowdiss) {
    vl2 = vnl * vnl + vtl * vtl + vul * vul;
    enl = gammam1i * prl + pml + 0.5 * rol * vl2;
  } else {
    enl = gammam1i * prl + pml + 0.5 * rol * (vnl * vnl + vtl * vtl + vul * vul);
  }
  double vbl = vtl * btl + vul * bul;
  double rori = 1.0 / ror;
  double pmr = 0.5 * (btr * btr + bur * bur);
  double ptr = prr + pmr;
  if (lowdiss) {
    vr2 = vnr * vnr + vtr * vtr + vur * vur;
    enr = gammam1i * prr + pmr + 0.5 * ror * vr2;
  } else {
    enr = gammam1i * prr + pmr + 0.5 * ror * (vnr * vnr + vtr * vtr + vur * vur);
  }
  double vbr = vtr * btr + vur * bur;
  double cl2 = gamma * prl * roli;
  double cr2 = gamma * prr * rori;
  double cal2 = bnc2 * roli;
  double car2 = bnc2 * rori;
  double cbl2 = cl2 + cal2 + 2.0 * pml * roli;
  double cbr2 = cr2 + car2 + 2.0 * pmr * rori;
  double cfl2 = 0.5 * (cbl2 + sqrt(fabs(cbl2 * cbl2 - 4.0 * cl2 * cal2)));
  double cfr2 = 0.5 * (cbr2 + sqrt(fabs(cbr2 * cbr2 - 4.0 * cr2 * car2)));
  double cmax, ccl2 = 0.0, ccr2 = 0.0;
  if (lowdiss) {
    cbl2 = vl2 + cal2 + 2.0 * pml * roli;
    cbr2 = vr2 + car2 + 2.0 * pmr * rori;
    ccl2 = 0.5 * (cbl2 + sqrt(fabs(cbl2 * cbl2 - 4.0 * vl2 * cal2)));
    ccr2 = 0.5 * (cbr2 + sqrt(fabs(cbr2 * cbr2 - 4.0 * vr2 * car2)));
    cmax = sqrt(qmax(cfl2, cfr2));
  } else {
    double cfl = sqrt(cfl2);
    double cfr = sqrt(cfr2);
    cmax = qmax(cfl, cfr);
  }
  double sl = qmin(0.0, qmin(vnl, vnr) - cmax);
  double sr = qmax(0.0, qmax(vnl, vnr) + cmax);
  double slvl = sl - vnl;
  double srvr = sr - vnr;
  double rslvl = rol * slvl;
  double rsrvr = ror * srvr;
  double drsvi = 1.0 / (rsrvr - rslvl);
  double vnc, ptc;
  if (lowdiss) {
    double theta = qmin(1.0, (cmax - qmin(dv[0], 0.0)) / (cmax - qmin(dv[1], 0.0)));
    theta *= theta;
    theta *= theta;
    vnc = (rsrvr * vnr - rslvl * vnl - theta * (ptr - ptl)) * drsvi;
    double mcc = qmin(1.0, sqrt(qmax(ccl2, ccr2)) / cmax);
    ptc = (rsrvr * ptl - rslvl * ptr + (mcc * (2.0 - mcc)) * rsrvr * rslvl * (vnr - vnl)) * drsvi;
  } else {
    vnc = (rsrvr * vnr - rslvl * vnl - ptr + ptl) * drsvi;
    ptc = (rsrvr * ptl - rslvl * ptr + rsrvr * rslvl * (vnr - vnl)) * drsvi;
  }
  double slvc = sl - vnc;
  double srvc = sr - vnc;
  double ro2l = rslvl / slvc;
  double ro2r = rsrvr / srvc;
  double rhdl = rslvl * slvc - bnc2;
  double rhdr = rsrvr * srvc - bnc2;
  double vt2l, vu2l, bt2l, bu2l, vt2r, vu2r, bt2r, bu2r;
  if (fabs(rhdl) > FL_EPS) {
    double rhdli = 1.0 / rhdl;
    double rhnvl = (vnl - vnc) * bnc;
    double rhnbl = rslvl * slvl - bnc2;
    vt2l = vtl + rhnvl * rhdli * btl;
    vu2l = vul + rhnvl * rhdli * bul;
    bt2l = rhnbl * rhdli * btl;
    bu2l = rhnbl * rhdli * bul;
  } else {
    vt2l = vtl; vu2l = vul; bt2l = btl; bu2l = bul;
  }
  if (fabs(rhdr) > FL_EPS) {
    double rhdri = 1.0 / rhdr;
    double rhnvr = (vnr - vnc) * bnc;
    double rhnbr = rsrvr * srvr - bnc2;
    vt2r = vtr + rhnvr * rhdri * btr;
    vu2r = vur + rhnvr * rhdri * bur;
    bt2r = rhnbr * rhdri * btr;
    bu2r = rhnbr * rhdri * bur;
  } else {
    vt2r = vtr; vu2r = vur; bt2r = btr; bu2r = bur;
  }
  double vb2l = vt2l * bt2l + vu2l * bu2l;
  double vb2r = vt2r * bt2r + vu2r * bu2r;
  double en2l = (slvl * enl - ptl * vnl + ptc * vnc + bnc * (vbl - vb2l)) / slvc;
  double en2r = (srvr * enr - ptr * vnr + ptc * vnc + bnc * (vbr - vb2r)) / srvc;
  double rro2l = sqrt(ro2l);
  double rro2r = sqrt(ro2r);
  double rro2i = 1.0 / (rro2r + rro2l);
  double vt3m = (rro2r * vt2r + rro2l * vt2l + (bt2r - bt2l) * sgn) * rro2i;
  double vu3m = (rro2r * vu2r + rro2l * vu2l + (bu2r - bu2l) * sgn) * rro2i;
  double bt3m = (rro2l * bt2r + rro2r * bt2l + rro2r * rro2l * (vt2r - vt2l) * sgn) * rro2i;
  double bu3m = (rro2l * bu2r + rro2r * bu2l + rro2r * rro2l * (vu2r - vu2l) * sgn) * rro2i;
  double vb3m = vt3m * bt3m + vu3m * bu3m;
  double en3l = en2l - rro2l * (vb2l - vb3m) * sgn;
  double en3r = en2r + rro2r * (vb2r - vb3m) * sgn;
  double hl = (vnc > 0) ? (1.0) : (0.0);
  double hr = 1.0 - hl;
  double h2l = (vnc - fabs(bnc) / rro2l > 0) ? (1.0) : (0.0);
  double h3l = (1.0 - h2l) * hl;
  double h2r = (vnc + fabs(bnc) / rro2r > 0) ? (0.0) : (1.0);
  double h3r = (1.0 - h2r) * hr;
  double rou = ro2l * hl + ro2r * hr;
  double vtu = vt2l * h2l + vt3m * (h3l + h3r) + vt2r * h2r;
  double vuu = vu2l * h2l + vu3m * (h3l + h3r) + vu2r * h2r;
  double btu = bt2l * h2l + bt3m * (h3l + h3r) + bt2r * h2r;
  double buu = bu2l * h2l + bu3m * (h3l + h3r) + bu2r * h2r;
  double enu = en2l * h2l + en3l * h3l + en3r * h3r + en2r * h2r;
  F[0] = rou * vnc;
  F[1] = rou * vnc * vnc + ptc - bnc2 * 0.5;
  F[2] = rou * vtu * vnc - bnc * btu;
  F[3] = rou * vuu * vnc - bnc * buu;
  F[4] = btu * vnc - bnc * vtu;
  F[5] = buu * vnc - bnc * vuu;
  F[6] = (enu + ptc) * vnc - bnc * (vtu * btu + vuu * buu);
}
static void flux_hlld(const double *L, const double *R, double bnc, double gamma, const double *dv, double *F)
{
  flux_hlld_common(0, L, R, bnc, gamma, dv, F);
}
static void flux_lhlld(const double *L, const double *R, double bnc, double gamma, const double *dv, double *F)
{
  flux_hlld_common(1, L, R, bnc, gamma, dv, F);
}
static flux_fn riemann(int rmn)
{
  static const flux_fn t[4] = {flux_roe, flux_hlld, flux_lhlld, flux_mlau};
  return t[rmn];
}

/* CUCT weight: common/mhd_func.c:56-76 (p[] holds the 4 cells (i-1,j-1),(i,j-1),(i-1,j),(i,j)) */
static double cuct_weight(const double *ro, const double *va, const double *vb, const double *ba,
                          const double *bb, long oa, long ob)
{
  const double eps = 1e-12;
  long s0 = -oa - ob, s1 = -ob, s2 = -oa, s3 = 0;
  double roc = 0.25 * (ro[s0] + ro[s1] + ro[s2] + ro[s3]);
  roc = 1.0 / sqrt(roc);
  double vac = 0.25 * (va[s0] + va[s1] + va[s2] + va[s3]);
  double vbc = 0.25 * (vb[s0] + vb[s1] + vb[s2] + vb[s3]);
  double bac = 0.5 * (ba[s1] + ba[s3]);
  double bbc = 0.5 * (bb[s2] + bb[s3]);
  vac = fabs(vac) + fabs(bac * roc);
  vbc = fabs(vbc) + fabs(bbc * roc);
  return (vac + 0.5 * eps) / (vac + vbc + eps);
}

/* ------------------------------------------------------------------------ */
/* grid bookkeeping                                                          */
/* ------------------------------------------------------------------------ */
typedef struct {
  const qo_grid *g;
  int nx, ny, nz;
  long nd, sx, sy, sz;
} geo;

static geo mkgeo(const qo_grid *g)
{
  geo e;
  e.g = g;
  e.nx = g->nxm + 2 * GH;
  e.ny = g->dim >= 2 ? g->nym + 2 * GH : 1;
  e.nz = g->dim >= 3 ? g->nzm + 2 * GH : 1;
  e.nd = (long)e.nx * e.ny * e.nz;
  e.sx = 1;
  e.sy = e.nx;
  e.sz = (long)e.nx * e.ny;
  return e;
}

#define IDX(e, i, j, k) ((long)(e).nx * ((long)(e).ny * (k) + (j)) + (i))

/* ------------------------------------------------------------------------ */
/* ghost fill passes                                                          */
/* 1D: common/common_func.c:34-58 (no staggering); 2D: :60-138 (x then y);    */
/* 3D on one rank: mpi/common_mpi.c:198-391 periodic copies for every field   */
/* (decided by the first field's flag) then :392-525 physical passes.         */
/* ------------------------------------------------------------------------ */
static void pass_periodic(const geo *e, double *f, int axis)
{
  int n = axis == 0 ? e->nx : axis == 1 ? e->ny : e->nz;
  long s = axis == 0 ? e->sx : axis == 1 ? e->sy : e->sz;
  int a, b;
  int na = axis == 0 ? e->ny : e->nx, nb = axis == 2 ? e->ny : e->nz;
  long sa = axis == 0 ? e->sy : e->sx, sb = axis == 2 ? e->sy : e->sz;
  for (b = 0; b < nb; b++)
    for (a = 0; a < na; a++) {
      double *p = f + sa * a + sb * b;
      for (int i = 0; i < GH; i++) {
        p[s * (n - 1 - i)] = p[s * (2 * GH - 1 - i)];
        p[s * i] = p[s * (n - 2 * GH + i)];
      }
    }
}

static void pass_physical(const geo *e, double *f, int axis, int st, int dn)
{
  int n = axis == 0 ? e->nx : axis == 1 ? e->ny : e->nz;
  long s = axis == 0 ? e->sx : axis == 1 ? e->sy : e->sz;
  int na = axis == 0 ? e->ny : e->nx, nb = axis == 2 ? e->ny : e->nz;
  long sa = axis == 0 ? e->sy : e->sx, sb = axis == 2 ? e->sy : e->sz;
  int a, b, i;
  if (abs(dn) == 1) {
    for (b = 0; b < nb; b++)
      for (a = 0; a < na; a++) {
        double *p = f + sa * a + sb * b;
        for (i = 0; i < GH; i++) p[s * i] = dn * p[s * (2 * GH - 1 + st - i)];
        for (i = 0; i < GH - st; i++) p[s * (n - 1 - i)] = dn * p[s * (n - 2 * GH + st + i)];
      }
  } else if (abs(dn) == 2) {
    for (b = 0; b < nb; b++)
      for (a = 0; a < na; a++) {
        double *p = f + sa * a + sb * b;
        for (i = 0; i < GH; i++) p[s * i] = 0.25 * (2 + dn) * p[s * GH];
        for (i = 0; i < GH - st; i++) p[s * (n - 1 - i)] = 0.25 * (2 + dn) * p[s * (n - 1 - GH + st)];
      }
  }
}

/* apply the fill to nf fields with per-field flags dn[axis][m] and staggering st[axis][m] */
static void fill_ghosts(const geo *e, double *const *f, int nf, const int *const dn[3], const int *const st[3])
{
  int m, ax;
  int dim = e->g->dim;
  if (dim == 1) {
    for (m = 0; m < nf; m++) {
      if (dn[0][m] == 0)
        pass_periodic(e, f[m], 0);
      else
        pass_physical(e, f[m], 0, 0, dn[0][m]);
    }
  } else if (dim == 2) {
    for (m = 0; m < nf; m++) {
      for (ax = 0; ax < 2; ax++) {
        if (dn[ax][m] == 0)
          pass_periodic(e, f[m], ax);
        else
          pass_physical(e, f[m], ax, st[ax][m], dn[ax][m]);
      }
    }
  } else {
    for (ax = 0; ax < 3; ax++)
      if (dn[ax][0] == 0)
        for (m = 0; m < nf; m++) pass_periodic(e, f[m], ax);
    for (m = 0; m < nf; m++)
      for (ax = 0; ax < 3; ax++) pass_physical(e, f[m], ax, st[ax][m], dn[ax][m]);
  }
}

/* staggering flags of the state: bx on x faces, by on y faces, bz on z faces
 * (mhd2d_class.cpp:146-163, mhd3d_class.cpp:178-204; 1D ignores them). */
static const int ST_X[8] = {0, 0, 0, 0, 1, 0, 0, 0};
static const int ST_Y[8] = {0, 0, 0, 0, 0, 1, 0, 0};
static const int ST_Z[8] = {0, 0, 0, 0, 0, 0, 1, 0};
static const int ST_0[8] = {0, 0, 0, 0, 0, 0, 0, 0};

void qo_bound(const qo_grid *g, double *u)
{
  geo e = mkgeo(g);
  double *f[8];
  for (int m = 0; m < 8; m++) f[m] = u + (long)m * e.nd;
  const int *dn[3] = {g->dnx, g->dny, g->dnz};
  const int *st[3] = {ST_X, ST_Y, ST_Z};
  fill_ghosts(&e, f, 8, dn, st);
  if (g->phi && g->dim >= 2) {
    /* gravity drivers: the energy in the ghost layers of the last axis from the first/last
     * interior layer and the potential difference (2D/SERIAL/RTI/mhd2d_class.cpp:10-32,
     * 3D/MPI/RTI/mhd3d_class.cpp:14-40) */
    const double *phi = g->phi;
    double *ro = f[0], *en = f[7];
    double fac = (2.0 - g->gam) / (g->gam - 1.0);
    int n = g->dim == 3 ? e.nz : e.ny;
    long sl = g->dim == 3 ? e.sz : e.sy;    /* stride of the last axis */
    long layer = sl;                         /* cells per layer */
    for (int q = 0; q < GH; q++)
      for (long c = 0; c < layer; c++) {
        long ss = (long)q * sl + c, sb = (long)GH * sl + c;
        en[ss] = en[sb] - fac * ro[sb] * (phi[ss] - phi[sb]);
      }
    for (int q = n - GH; q < n; q++)
      for (long c = 0; c < layer; c++) {
        long ss = (long)q * sl + c, sb = (long)(n - GH - 1) * sl + c;
        en[ss] = en[sb] - fac * ro[sb] * (phi[ss] - phi[sb]);
      }
  }
}

/* ------------------------------------------------------------------------ */
/* one ideal stage, shared by 1D/2D/3D                                        */
/* ------------------------------------------------------------------------ */
typedef struct {
  double *vx, *vy, *vz, *pr, *cx, *cy, *cz;
  double *ct[3];
  double *dv[3];
  double *flx[3];   /* per direction: 8*nd SoA face fluxes */
  double *fcd[3];   /* per direction: 2*nd central parts of the induction fluxes */
  double *ex, *ey, *ez;
  double *ut;
} work;

static void *xcalloc(long n) { return calloc((size_t)n, sizeof(double)); }

static int work_alloc(work *w, const geo *e)
{
  long nd = e->nd;
  memset(w, 0, sizeof(*w));
  w->vx = xcalloc(nd); w->vy = xcalloc(nd); w->vz = xcalloc(nd); w->pr = xcalloc(nd);
  w->cx = xcalloc(nd); w->cy = xcalloc(nd); w->cz = xcalloc(nd);
  for (int a = 0; a < 3; a++) {
    w->ct[a] = xcalloc(nd);
    w->dv[a] = xcalloc(nd);
    w->flx[a] = xcalloc(8 * nd);
    w->fcd[a] = xcalloc(2 * nd);
  }
  w->ex = xcalloc(nd); w->ey = xcalloc(nd); w->ez = xcalloc(nd);
  w->ut = xcalloc(8 * nd);
  if (!w->vx || !w->vy || !w->vz || !w->pr || !w->cx || !w->cy || !w->cz || !w->ex || !w->ey || !w->ez || !w->ut)
    return -1;
  for (int a = 0; a < 3; a++)
    if (!w->ct[a] || !w->dv[a] || !w->flx[a] || !w->fcd[a]) return -1;
  return 0;
}

static void work_free(work *w)
{
  free(w->vx); free(w->vy); free(w->vz); free(w->pr); free(w->cx); free(w->cy); free(w->cz);
  for (int a = 0; a < 3; a++) { free(w->ct[a]); free(w->dv[a]); free(w->flx[a]); free(w->fcd[a]); }
  free(w->ex); free(w->ey); free(w->ez); free(w->ut);
}

/* gather a 5-point stencil centred on ss along stride s */
static inline void gather5(double *q, const double *f, long ss, long s)
{
  q[0] = f[ss - 2 * s]; q[1] = f[ss - s]; q[2] = f[ss]; q[3] = f[ss + s]; q[4] = f[ss + 2 * s];
}

/* L/R induction-flux states for CUCT: common/mhd_func.c:163-188.
 * vn,vt: normal and transverse velocity; bnf: normal B on faces; btc: transverse B at centres */
static inline void induction_states(const double *vn, const double *vt, const double *bnf, const double *btc,
                                    long ss, long s, lr_fn lin, double *vl, double *vr)
{
  double vns[5], vts[5], bns[5], bts[5], prod[5], fl0, fr0, fl1, fr1;
  gather5(vns, vn, ss, s);
  gather5(vts, vt, ss, s);
  gather5(bns, bnf, ss, s);
  gather5(bts, btc, ss, s);
  for (int m = 0; m < 5; m++) prod[m] = bts[m] * vns[m];
  lin(&prod[2], &fl0, &fr0);
  lin(&vts[2], &fl1, &fr1);
  *vl = fl0 - bns[3] * fl1;
  *vr = fr0 - bns[2] * fr1;
}

/* one direction's face sweep: lrstate + Riemann flux + central/upwind split.
 * axis a: normal velocity va, transverse (vb,vc), cell-centre (bb,bc) with bn=ca (centre) and ba_face.
 * Mirrors mhd2d_solve.cpp:127-199 (x), :234-306 (y) and mhd3d_solve.cpp:166-258, :330-422, :494-586. */
static void sweep(const geo *e, const double *const *u, work *w, int axis)
{
  const qo_grid *g = e->g;
  int dim = g->dim;
  long s = axis == 0 ? e->sx : axis == 1 ? e->sy : e->sz;
  int n = axis == 0 ? e->nx : axis == 1 ? e->ny : e->nz;
  const double *ro = u[0], *pr = w->pr;
  const double *v[3] = {w->vx, w->vy, w->vz};
  const double *c[3] = {w->cx, w->cy, w->cz};
  const double *bf[3] = {u[4], u[5], u[6]};
  int a = axis, b = (axis + 1) % 3, cc = (axis + 2) % 3;
  lr_fn lr = nl_interp(g->odr), lin = lin_interp(g->odr);
  flux_fn fl = riemann(g->rmn);
  double *F = w->flx[axis];
  double *FC = w->fcd[axis];
  /* flux components written by this sweep: (ro, m_a, m_b, m_c, B_a=0, B_b, B_c, en) */
  int mcomp[3] = {1 + a, 1 + b, 1 + cc};
  int bcomp[3] = {4 + a, 4 + b, 4 + cc};
  long nd = e->nd;
  int i, j, k;
  int ilo = 0, ihi = e->nx, jlo = 0, jhi = e->ny, klo = 0, khi = e->nz;
#pragma omp parallel for collapse(2) schedule(static) private(i)
  for (k = klo; k < khi; k++) {
    for (j = jlo; j < jhi; j++) {
      for (i = ilo; i < ihi; i++) {
        int pos = axis == 0 ? i : axis == 1 ? j : k;
        if (pos < 3 || pos >= n - 2) continue;
        long ssf = IDX(*e, i, j, k);   /* face pos between cells pos-1 and pos */
        double ql[7][5], qr[7][5], vl[7], vr[7], tmp[7], L[7], R[7], Fl[7];
        /* left state at this face: lrstate of cell pos-1 (its vl), right: cell pos (its vr) */
        long sl = ssf - s, sr = ssf;
        gather5(ql[0], ro, sl, s); gather5(ql[1], v[a], sl, s); gather5(ql[2], v[b], sl, s);
        gather5(ql[3], v[cc], sl, s); gather5(ql[4], c[b], sl, s); gather5(ql[5], c[cc], sl, s);
        gather5(ql[6], pr, sl, s);
        gather5(qr[0], ro, sr, s); gather5(qr[1], v[a], sr, s); gather5(qr[2], v[b], sr, s);
        gather5(qr[3], v[cc], sr, s); gather5(qr[4], c[b], sr, s); gather5(qr[5], c[cc], sr, s);
        gather5(qr[6], pr, sr, s);
        face_states(ql, c[a][sl], g->gam, lr, vl, tmp, g->char_mode);
        face_states(qr, c[a][sr], g->gam, lr, tmp, vr, g->char_mode);
        for (int m = 0; m < 7; m++) { L[m] = vl[m]; R[m] = vr[m]; }
        double bn = 0.5 * (bf[a][ssf] + bf[a][ssf]);
        double dvsd[2];
        dvsd[0] = v[a][ssf] - v[a][ssf - s];
        if (dim == 1) {
          dvsd[1] = 0.0;
        } else if (dim == 2) {
          const double *dvt = w->dv[axis == 0 ? 1 : 0];
          dvsd[1] = qmin(dvt[ssf - s], dvt[ssf]);
        } else {
          const double *d1 = w->dv[b], *d2 = w->dv[cc];
          dvsd[1] = qmin(qmin(d1[ssf - s], d1[ssf]), qmin(d2[ssf - s], d2[ssf]));
        }
        fl(L, R, bn, g->gam, dvsd, Fl);
        F[0 * nd + ssf] = Fl[0];
        F[(long)mcomp[0] * nd + ssf] = Fl[1];
        F[(long)mcomp[1] * nd + ssf] = Fl[2];
        F[(long)mcomp[2] * nd + ssf] = Fl[3];
        F[(long)bcomp[0] * nd + ssf] = 0;
        F[(long)bcomp[1] * nd + ssf] = Fl[4];
        F[(long)bcomp[2] * nd + ssf] = Fl[5];
        F[7 * nd + ssf] = Fl[6];
        /* work done by gravity (2D/SERIAL/RTI/mhd2d_solve.cpp:197, :305; 3D/MPI/RTI :247, :412, :577) */
        if (g->phi) F[7 * nd + ssf] += Fl[0] * 0.5 * (g->phi[sl] + g->phi[sr]);
        if (dim >= 2) {
          /* induction fluxes split (2D: only B_b for x, B_a... see below) */
          double q0l, q0r, q1l, q1r, dummy;
          if (dim == 2) {
            /* 2D: x sweep splits By flux (bt=cy), y sweep splits Bx flux (bt=cx) */
            const double *vt = axis == 0 ? w->vy : w->vx;
            const double *btc = axis == 0 ? w->cy : w->cx;
            induction_states(v[a], vt, bf[a], btc, sl, s, lin, &q0l, &dummy);
            induction_states(v[a], vt, bf[a], btc, sr, s, lin, &dummy, &q0r);
            int comp = axis == 0 ? 5 : 4;
            double fcv = 0.5 * (q0l + q0r);
            FC[0 * nd + ssf] = fcv;
            F[(long)comp * nd + ssf] -= fcv;
          } else {
            /* 3D: component order per mhd3d_solve.cpp:215-221, :379-385, :543-549 */
            int t0 = axis == 0 ? 1 : axis == 1 ? 2 : 0;   /* By for x, Bz for y, Bx for z */
            int t1 = axis == 0 ? 2 : axis == 1 ? 0 : 1;   /* Bz for x, Bx for y, By for z */
            induction_states(v[a], v[t0], bf[a], c[t0], sl, s, lin, &q0l, &dummy);
            induction_states(v[a], v[t0], bf[a], c[t0], sr, s, lin, &dummy, &q0r);
            induction_states(v[a], v[t1], bf[a], c[t1], sl, s, lin, &q1l, &dummy);
            induction_states(v[a], v[t1], bf[a], c[t1], sr, s, lin, &dummy, &q1r);
            double fc0 = 0.5 * (q0l + q0r);
            double fc1 = 0.5 * (q1l + q1r);
            FC[0 * nd + ssf] = fc0;
            F[(long)(4 + t0) * nd + ssf] -= fc0;
            FC[1 * nd + ssf] = fc1;
            F[(long)(4 + t1) * nd + ssf] -= fc1;
          }
        }
      }
    }
  }
}

/* corner EMF contribution: interpolate the upwind induction flux `up` and its central part `cen`
 * from face centres to the edge along stride s; returns the sign-weighted term
 * sgn*0.5*((upL+upR) + w*(cenL+cenR)) with w = ct or 1-ct.
 * Mirrors mhd2d_solve.cpp:201-232, :308-339 and mhd3d_solve.cpp:259-328, :423-492, :587-656. */
static inline double emf_term(const double *up, const double *cen, long ss, long s, lr_fn lin,
                              double sgn, double wgt)
{
  double f[5], l0, r0, l1, r1, d;
  gather5(f, up, ss - s, s);
  lin(&f[2], &l0, &d);
  gather5(f, up, ss, s);
  lin(&f[2], &d, &r0);
  gather5(f, cen, ss - s, s);
  lin(&f[2], &l1, &d);
  gather5(f, cen, ss, s);
  lin(&f[2], &d, &r1);
  return sgn * ((l0 + r0) + wgt * (l1 + r1));
}

static void corner_emfs(const geo *e, work *w)
{
  const qo_grid *g = e->g;
  lr_fn lin = lin_interp(g->odr);
  long nd = e->nd;
  int i, j, k;
  if (g->dim == 2) {
    const double *fx = w->flx[0], *fy = w->flx[1];
    const double *ct = w->ct[0];
#pragma omp parallel for schedule(static) private(i)
    for (j = 0; j < e->ny; j++)
      for (i = 0; i < e->nx; i++) {
        long ss = IDX(*e, i, j, 0);
        double ez = 0.0;
        if (j >= 3 && j < e->ny - 2 && i >= 3 && i < e->nx - 2) {
          ez += emf_term(fx + 5 * nd, w->fcd[0], ss, e->sy, lin, -0.5, (1.0 - ct[ss]));
          ez += emf_term(fy + 4 * nd, w->fcd[1], ss, e->sx, lin, +0.5, ct[ss]);
        }
        w->ez[ss] = ez;
      }
    return;
  }
  /* 3D */
  const double *fx = w->flx[0], *fy = w->flx[1], *fz = w->flx[2];
#pragma omp parallel for collapse(2) schedule(static) private(i)
  for (k = 0; k < e->nz; k++)
    for (j = 0; j < e->ny; j++)
      for (i = 0; i < e->nx; i++) {
        long ss = IDX(*e, i, j, k);
        double ex = 0.0, ey = 0.0, ez = 0.0;
        int ii = (i >= 3 && i < e->nx - 2), jj = (j >= 3 && j < e->ny - 2), kk = (k >= 3 && k < e->nz - 2);
        if (ii && jj) {
          ez += emf_term(fx + 5 * nd, w->fcd[0] + 0 * nd, ss, e->sy, lin, -0.5, (1.0 - w->ct[0][ss]));
          ez += emf_term(fy + 4 * nd, w->fcd[1] + 1 * nd, ss, e->sx, lin, +0.5, w->ct[0][ss]);
        }
        if (ii && kk) {
          ey += emf_term(fx + 6 * nd, w->fcd[0] + 1 * nd, ss, e->sz, lin, +0.5, w->ct[2][ss]);
          ey += emf_term(fz + 4 * nd, w->fcd[2] + 0 * nd, ss, e->sx, lin, -0.5, (1.0 - w->ct[2][ss]));
        }
        if (jj && kk) {
          ex += emf_term(fy + 6 * nd, w->fcd[1] + 0 * nd, ss, e->sz, lin, -0.5, (1.0 - w->ct[1][ss]));
          ex += emf_term(fz + 5 * nd, w->fcd[2] + 1 * nd, ss, e->sy, lin, +0.5, w->ct[1][ss]);
        }
        w->ex[ss] = ex;
        w->ey[ss] = ey;
        w->ez[ss] = ez;
      }
}

static const double RKF[3][3][2] = {
    /* rk_fac table of mhd2d_solve.cpp:7 evaluated for R_K = 1, 2, 3 */
    {{0.0, 1.0}, {0.5 + (1 - 2) * 0.25, 0.5 - (1 - 2) * 0.25}, {1. / 3., 2. / 3.}},
    {{0.0, 1.0}, {0.5 + (2 - 2) * 0.25, 0.5 - (2 - 2) * 0.25}, {1. / 3., 2. / 3.}},
    {{0.0, 1.0}, {0.5 + (3 - 2) * 0.25, 0.5 - (3 - 2) * 0.25}, {1. / 3., 2. / 3.}}};

/* centre update du = -dt/dx D_x F - ... (common/mhd_func.c:207-284) */
static inline double div_flux(const geo *e, const work *w, int m, long ss, const double dtd[3], pt_fn df)
{
  const qo_grid *g = e->g;
  long nd = e->nd;
  double f[4];
  const double *F0 = w->flx[0] + (long)m * nd;
  f[0] = F0[ss - 1]; f[1] = F0[ss]; f[2] = F0[ss + 1]; f[3] = F0[ss + 2];
  double du0 = df(&f[1]);
  if (g->dim == 1) return -dtd[0] * du0;
  const double *F1 = w->flx[1] + (long)m * nd;
  f[0] = F1[ss - e->sy]; f[1] = F1[ss]; f[2] = F1[ss + e->sy]; f[3] = F1[ss + 2 * e->sy];
  double du1 = df(&f[1]);
  if (g->dim == 2) return (-dtd[0] * du0 - dtd[1] * du1);
  const double *F2 = w->flx[2] + (long)m * nd;
  f[0] = F2[ss - e->sz]; f[1] = F2[ss]; f[2] = F2[ss + e->sz]; f[3] = F2[ss + 2 * e->sz];
  double du2 = df(&f[1]);
  return (-dtd[0] * du0 - dtd[1] * du1 - dtd[2] * du2);
}

static inline double d4(const double *p, long ss, long s, pt_fn df)
{
  double f[4] = {p[ss - s], p[ss], p[ss + s], p[ss + 2 * s]};
  return df(&f[1]);
}

/* bc1d (common/common_func.c:34-58) of one array with any flag value (flags outside
 * {0, +-1, +-2} leave the ghosts alone) */
static void bc1d_any(double *f, int nx, int dn)
{
  int i;
  if (dn == 0) {
    for (i = 0; i < GH; i++) { f[i] = f[nx - 2 * GH + i]; f[nx - 1 - i] = f[2 * GH - 1 - i]; }
  } else if (abs(dn) == 1) {
    for (i = 0; i < GH; i++) { f[i] = dn * f[2 * GH - 1 - i]; f[nx - 1 - i] = dn * f[nx - 2 * GH + i]; }
  } else if (abs(dn) == 2) {
    for (i = 0; i < GH; i++) { f[i] = 0.25 * (2 + dn) * f[GH]; f[nx - 1 - i] = 0.25 * (2 + dn) * f[nx - 1 - GH]; }
  }
}

static double d2f2(const double *f) { return ((f[1] + f[-1]) - 2.0 * f[0]); }
static double d2f4(const double *f) { return ((-(f[2] + f[-2]) + 16.0 * (f[1] + f[-1]) - 30.0 * f[0]) / 12.0); }

/* HMHD1D::crcte (1D/SERIAL/h-shock/hmhd1d_solve.cpp:275-300) with eorg2enew_cg (:326-403):
 * fbt/fen = the by (or bz) and energy fluxes (stride 1 here), bt = by (or bz), dn = the flag
 * product; the density passed to the solve is 1 everywhere, as crcte does.  Faces 0..2 and
 * nx-2.. are never read by the update, so their (reference: uninitialised) inputs do not matter. */
static void crcte(double *fbt, double *fen, const double *bt, int nx, int dn, double de, double dx, int odr)
{
  int i;
  double *eorg = xcalloc(nx), *enew = xcalloc(nx), *rk = xcalloc(nx), *pk = xcalloc(nx), *ap = xcalloc(nx);
  const double one = 1.0;
  pt_fn d2f = odr >= 3 ? d2f4 : d2f2;
  for (i = 0; i < nx; i++) eorg[i] = enew[i] = fbt[i];
  const int cmax = nx;
  const double eps = 1e-8, fac = (de * de) / (dx * dx);
  int cnt = 0;
  double numer = 0.0, denom, coef, anorm, anormf = 0.0;
  bc1d_any(enew, nx, dn);
  for (i = GH; i < nx - GH; i++) {
    rk[i] = one * eorg[i] - (one * enew[i] - fac * d2f(&enew[i]));
    pk[i] = rk[i];
    numer += rk[i] * rk[i];
    anormf += fabs(rk[i]);
  }
  do {
    bc1d_any(pk, nx, dn);
    denom = 0.0;
    for (i = GH; i < nx - GH; i++) {
      ap[i] = (one * pk[i] - fac * d2f(&pk[i]));
      denom += pk[i] * ap[i];
    }
    coef = (denom == 0) ? 0 : numer / denom;
    anorm = 0.0;
    for (i = GH; i < nx - GH; i++) {
      enew[i] += coef * pk[i];
      rk[i] -= coef * ap[i];
      anorm += fabs(rk[i]);
    }
    denom = numer;
    numer = 0.0;
    for (i = GH; i < nx - GH; i++) numer += rk[i] * rk[i];
    coef = (denom == 0) ? 0 : numer / denom;
    for (i = GH; i < nx - GH; i++) pk[i] = rk[i] + coef * pk[i];
  } while ((anorm > eps * anormf) && (++cnt < cmax));
  bc1d_any(enew, nx, dn);
  for (i = 1; i < nx; i++) {
    double dd = enew[i] - eorg[i];
    double bb = 0.5 * (bt[i - 1] + bt[i]);
    fbt[i] = enew[i];
    fen[i] += dd * bb;
  }
  free(eorg); free(enew); free(rk); free(pk); free(ap);
}

static void ideal_stage(const geo *e, double *const *u, work *w, int rk, double dt)
{
  const qo_grid *g = e->g;
  int dim = g->dim;
  int nx = e->nx, ny = e->ny, nz = e->nz;
  long nd = e->nd, sy = e->sy, sz = e->sz;
  pt_fn fc = face_to_centre(g->odr), df = first_diff(g->odr);
  int i, j, k;
  long ss;
  double dtd[3] = {dt / g->dx, dim >= 2 ? dt / g->dy : 0.0, dim >= 3 ? dt / g->dz : 0.0};
  const double *rkf = RKF[g->rk - 1][rk];

  /* cell-centre B: 2D mhd2d_solve.cpp:51-79; 3D mhd3d_solve.cpp:49-88; 1D aliases */
  if (dim == 1) {
    memcpy(w->cx, u[4], sizeof(double) * nd);
    memcpy(w->cy, u[5], sizeof(double) * nd);
    memcpy(w->cz, u[6], sizeof(double) * nd);
  } else {
#pragma omp parallel for collapse(2) schedule(static) private(i, ss)
    for (k = 0; k < nz; k++)
      for (j = 0; j < ny; j++)
        for (i = 0; i < nx; i++) {
          ss = IDX(*e, i, j, k);
          if (i >= 1 && i < nx - 2) w->cx[ss] = fc(&((double[4]){u[4][ss - 1], u[4][ss], u[4][ss + 1], u[4][ss + 2]})[1]);
          if (j >= 1 && j < ny - 2) w->cy[ss] = fc(&((double[4]){u[5][ss - sy], u[5][ss], u[5][ss + sy], u[5][ss + 2 * sy]})[1]);
          if (dim == 3 && k >= 1 && k < nz - 2)
            w->cz[ss] = fc(&((double[4]){u[6][ss - sz], u[6][ss], u[6][ss + sz], u[6][ss + 2 * sz]})[1]);
        }
    if (dim == 2) memcpy(w->cz, u[6], sizeof(double) * nd);
    double *pc[3] = {w->cx, w->cy, w->cz};
    const int *dn[3] = {g->dnx + 4, g->dny + 4, g->dnz + 4};
    const int *st[3] = {ST_0, ST_0, ST_0};
    fill_ghosts(e, pc, dim, dn, st);
  }

  /* primitives everywhere: prmtv (common/mhd_class.hpp:80-85) */
#pragma omp parallel for schedule(static)
  for (ss = 0; ss < nd; ss++) {
    /* gravity drivers: en -= ro*phi; prmtv; en += ro*phi (2D/SERIAL/RTI/mhd2d_solve.cpp:85-88) */
    if (g->phi) u[7][ss] -= u[0][ss] * g->phi[ss];
    double iro = 1.0 / u[0][ss];
    w->vx[ss] = u[1][ss] * iro;
    w->vy[ss] = u[2][ss] * iro;
    w->vz[ss] = u[3][ss] * iro;
    w->pr[ss] = ieos(u[0][ss], w->vx[ss], w->vy[ss], w->vz[ss], w->cx[ss], w->cy[ss], w->cz[ss], u[7][ss], g->gam);
    if (g->phi) u[7][ss] += u[0][ss] * g->phi[ss];
  }

  if (dim >= 2) {
    /* CUCT weights: mhd2d_solve.cpp:81-103, mhd3d_solve.cpp:90-136 */
#pragma omp parallel for collapse(2) schedule(static) private(i, ss)
    for (k = 0; k < nz; k++)
      for (j = 0; j < ny; j++)
        for (i = 0; i < nx; i++) {
          ss = IDX(*e, i, j, k);
          double c0 = 0.5, c1 = 0.5, c2 = 0.5;
          if (g->ctw) {
            if (j >= 1 && i >= 1) c0 = cuct_weight(&u[0][ss], &w->vx[ss], &w->vy[ss], &u[4][ss], &u[5][ss], 1, sy);
            if (dim == 3) {
              if (k >= 1 && j >= 1) c1 = cuct_weight(&u[0][ss], &w->vy[ss], &w->vz[ss], &u[5][ss], &u[6][ss], sy, sz);
              if (k >= 1 && i >= 1) c2 = cuct_weight(&u[0][ss], &w->vz[ss], &w->vx[ss], &u[6][ss], &u[4][ss], sz, 1);
            }
          }
          w->ct[0][ss] = c0;
          w->ct[1][ss] = c1;
          w->ct[2][ss] = c2;
        }
    /* shock detector dv: mhd2d_solve.cpp:105-125, mhd3d_solve.cpp:138-164 */
#pragma omp parallel for collapse(2) schedule(static) private(i, ss)
    for (k = (dim == 3 ? 1 : 0); k < (dim == 3 ? nz - 1 : 1); k++)
      for (j = 1; j < ny - 1; j++)
        for (i = 1; i < nx - 1; i++) {
          ss = IDX(*e, i, j, k);
          w->dv[0][ss] = qmin((w->vx[ss + 1] - w->vx[ss]), (w->vx[ss] - w->vx[ss - 1]));
          w->dv[1][ss] = qmin((w->vy[ss + sy] - w->vy[ss]), (w->vy[ss] - w->vy[ss - sy]));
          if (dim == 3) w->dv[2][ss] = qmin((w->vz[ss + sz] - w->vz[ss]), (w->vz[ss] - w->vz[ss - sz]));
        }
    int fdx[3] = {-g->dnx[1], g->dnx[2], g->dnx[3]};
    int fdy[3] = {g->dny[1], -g->dny[2], g->dny[3]};
    int fdz[3] = {g->dnz[1], g->dnz[2], -g->dnz[3]};
    const int *dn[3] = {fdx, fdy, fdz};
    const int *st[3] = {ST_0, ST_0, ST_0};
    fill_ghosts(e, w->dv, dim, dn, st);
  }

  /* face sweeps */
  for (int a = 0; a < dim; a++) sweep(e, (const double *const *)u, w, a);
  if (dim >= 2) corner_emfs(e, w);
  if (dim == 1 && g->hall_de != 0) {
    /* HMHD1D::ideal's electron-inertia correction (1D/SERIAL/h-shock/hmhd1d_solve.cpp:98-108) */
    double *F = w->flx[0];
    crcte(F + 5 * nd, F + 7 * nd, u[5], nx, g->dnx[1] * g->dnx[5], g->hall_de, g->dx, g->odr);
    crcte(F + 6 * nd, F + 7 * nd, u[6], nx, g->dnx[1] * g->dnx[6], g->hall_de, g->dx, g->odr);
  }

  /* centre update: mhd2d_solve.cpp:341-358, mhd3d_solve.cpp:658-676, mhd1d_solve.cpp:97-113 */
  int cen1[7] = {0, 1, 2, 3, 5, 6, 7};
  int cen2[6] = {0, 1, 2, 3, 6, 7};
  int cen3[5] = {0, 1, 2, 3, 7};
  const int *cen = dim == 1 ? cen1 : dim == 2 ? cen2 : cen3;
  int ncen = dim == 1 ? 7 : dim == 2 ? 6 : 5;
  int k0 = dim == 3 ? GH : 0, k1 = dim == 3 ? nz - GH : 1;
  int j0 = dim >= 2 ? GH : 0, j1 = dim >= 2 ? ny - GH : 1;
#pragma omp parallel for collapse(2) schedule(static) private(i, ss)
  for (k = k0; k < k1; k++)
    for (j = j0; j < j1; j++)
      for (i = GH; i < nx - GH; i++) {
        ss = IDX(*e, i, j, k);
        for (int c = 0; c < ncen; c++) {
          int m = cen[c];
          double d = div_flux(e, w, m, ss, dtd, df);
          rk_combine(&u[m][ss], w->ut[(long)m * nd + ss], d, rkf[0], rkf[1]);
        }
        if (g->phi) {
          /* work done by gravity on the momentum, with the updated density
           * (2D/SERIAL/RTI/mhd2d_solve.cpp:361-362, 3D/MPI/RTI/mhd3d_solve.cpp:679-681) */
          const double *phi = g->phi;
          u[1][ss] += -rkf[1] * u[0][ss] * 0.5 * (phi[ss + 1] - phi[ss - 1]) * dtd[0];
          u[2][ss] += -rkf[1] * u[0][ss] * 0.5 * (phi[ss + sy] - phi[ss - sy]) * dtd[1];
          if (dim == 3) u[3][ss] += -rkf[1] * u[0][ss] * 0.5 * (phi[ss + sz] - phi[ss - sz]) * dtd[2];
        }
      }

  /* CT update */
  if (dim == 2) {
    /* mhd2d_solve.cpp:359-380 via mhd_updt2d_ctb (common/mhd_func.c:286-300) */
#pragma omp parallel for schedule(static) private(i, ss)
    for (j = GH; j < ny - GH + 1; j++)
      for (i = GH; i < nx - GH + 1; i++) {
        ss = IDX(*e, i, j, 0);
        if (j < ny - GH) {
          double du = d4(w->ez, ss, sy, df);
          rk_combine(&u[4][ss], w->ut[4 * nd + ss], -(+dtd[1]) * du, rkf[0], rkf[1]);
        }
        if (i < nx - GH) {
          double du = d4(w->ez, ss, 1, df);
          rk_combine(&u[5][ss], w->ut[5 * nd + ss], -(-dtd[0]) * du, rkf[0], rkf[1]);
        }
      }
  } else if (dim == 3) {
    /* mhd3d_solve.cpp:677-709 via mhd_updt3d_ctb (common/mhd_func.c:302-325) */
#pragma omp parallel for collapse(2) schedule(static) private(i, ss)
    for (k = GH; k < nz - GH + 1; k++)
      for (j = GH; j < ny - GH + 1; j++)
        for (i = GH; i < nx - GH + 1; i++) {
          ss = IDX(*e, i, j, k);
          int in_k = k < nz - GH, in_j = j < ny - GH, in_i = i < nx - GH;
          if (in_k && in_j) { /* bx: ey along z, ez along y */
            double du0 = +d4(w->ez, ss, sy, df);
            double du1 = -d4(w->ey, ss, sz, df);
            rk_combine(&u[4][ss], w->ut[4 * nd + ss], -dtd[1] * du0 - dtd[2] * du1, rkf[0], rkf[1]);
          }
          if (in_k && in_i) { /* by: ez along x, ex along z */
            double du0 = +d4(w->ex, ss, sz, df);
            double du1 = -d4(w->ez, ss, 1, df);
            rk_combine(&u[5][ss], w->ut[5 * nd + ss], -dtd[2] * du0 - dtd[0] * du1, rkf[0], rkf[1]);
          }
          if (in_j && in_i) { /* bz: ex along y, ey along x */
            double du0 = +d4(w->ey, ss, 1, df);
            double du1 = -d4(w->ex, ss, sy, df);
            rk_combine(&u[6][ss], w->ut[6 * nd + ss], -dtd[0] * du0 - dtd[1] * du1, rkf[0], rkf[1]);
          }
        }
  }
}

int qo_step(const qo_grid *g, double *u, double dt)
{
  geo e = mkgeo(g);
  work w;
  if (work_alloc(&w, &e) != 0) { work_free(&w); return -1; }
  double *f[8];
  for (int m = 0; m < 8; m++) f[m] = u + (long)m * e.nd;
  memcpy(w.ut, u, sizeof(double) * 8 * e.nd);
  for (int rk = 0; rk < g->rk; rk++) {
    ideal_stage(&e, f, &w, rk, dt);
    qo_bound(g, u);
  }
  work_free(&w);
  return 0;
}

/* setdt reduction (mhd1d_class.cpp:11-30, mhd2d_class.cpp:11-33, mhd3d_class.cpp:15-46; the
 * gravity drivers' energy rewrite: 2D/SERIAL/RTI/mhd2d_class.cpp:46-48, 3D/MPI/RTI
 * mhd3d_class.cpp:56-58) */
double qo_cfl_dt(const qo_grid *g, double *u, double unused)
{
  (void)unused;
  geo e = mkgeo(g);
  const double *ro = u, *mx = u + e.nd, *my = u + 2 * e.nd, *mz = u + 3 * e.nd;
  const double *bx = u + 4 * e.nd, *by = u + 5 * e.nd, *bz = u + 6 * e.nd;
  double *en = u + 7 * e.nd;
  double vmax = 1.0;
  int k0 = g->dim == 3 ? GH : 0, k1 = g->dim == 3 ? e.nz - GH : 1;
  int j0 = g->dim >= 2 ? GH : 0, j1 = g->dim >= 2 ? e.ny - GH : 1;
  for (int k = k0; k < k1; k++)
    for (int j = j0; j < j1; j++)
      for (int i = GH; i < e.nx - GH; i++) {
        long ss = IDX(e, i, j, k);
        double cx, cy, cz;
        if (g->dim == 1) {
          cx = bx[ss]; cy = by[ss]; cz = bz[ss];
        } else {
          cx = 0.5 * (bx[ss] + bx[ss + 1]);
          cy = 0.5 * (by[ss] + by[ss + e.sy]);
          cz = g->dim == 3 ? 0.5 * (bz[ss] + bz[ss + e.sz]) : bz[ss];
        }
        if (g->phi) en[ss] -= ro[ss] * g->phi[ss];  /* 2D/SERIAL/RTI/mhd2d_class.cpp:46-48 */
        double iro = 1.0 / ro[ss];
        double vx = mx[ss] * iro, vy = my[ss] * iro, vz = mz[ss] * iro;
        double pr = ieos(ro[ss], vx, vy, vz, cx, cy, cz, en[ss], g->gam);
        if (g->phi) en[ss] += ro[ss] * g->phi[ss];
        double vf = sqrt((g->gam * pr + (cx * cx + cy * cy + cz * cz)) / ro[ss]);
        double vt;
        if (g->dim == 1)
          vt = fabs(vx) + vf;
        else if (g->dim == 2)
          vt = sqrt(vx * vx + vy * vy) + vf;
        else
          vt = sqrt(vx * vx + vy * vy + vz * vz) + vf;
        if (vt > vmax) vmax = vt;
      }
  return vmax;
}

/* ------------------------------------------------------------------------ */
/* visco-resistive step: 2D/SERIAL/MRX/dmhd2d_solve.cpp:3-151 (2D),          */
/* 3D/MPI/MRX/dmhd3d_solve.cpp:3-179 (3D)                                      */
/* ------------------------------------------------------------------------ */

/* eta*J on the CT edges: common/mhd_func.c:78-106 with zoffset = 0 */
static void ct_eres2(const geo *e, const double *bx, const double *by, const double *bz, const double *eta,
                     double idx, double idy, pt_fn df, long ss, double *ex, double *ey, double *ez)
{
  long xo = 1, yo = e->sy, zo = 0;
  double idz = 0.0;
  long si[4] = {-2 * xo, -xo, 0, +xo}, sj[4] = {-2 * yo, -yo, 0, +yo}, sk[4] = {-2 * zo, -zo, 0, +zo};
  double bxj[4] = {bx[ss + sj[0]], bx[ss + sj[1]], bx[ss + sj[2]], bx[ss + sj[3]]};
  double bxk[4] = {bx[ss + sk[0]], bx[ss + sk[1]], bx[ss + sk[2]], bx[ss + sk[3]]};
  double byk[4] = {by[ss + sk[0]], by[ss + sk[1]], by[ss + sk[2]], by[ss + sk[3]]};
  double byi[4] = {by[ss + si[0]], by[ss + si[1]], by[ss + si[2]], by[ss + si[3]]};
  double bzi[4] = {bz[ss + si[0]], bz[ss + si[1]], bz[ss + si[2]], bz[ss + si[3]]};
  double bzj[4] = {bz[ss + sj[0]], bz[ss + sj[1]], bz[ss + sj[2]], bz[ss + sj[3]]};
  double jx = df(&bzj[1]) * idy - df(&byk[1]) * idz;
  double jy = df(&bxk[1]) * idz - df(&bzi[1]) * idx;
  double jz = df(&byi[1]) * idx - df(&bxj[1]) * idy;
  const double *et = eta + ss;
  *ex = 0.25 * (et[-yo - zo] + et[-zo] + et[-yo] + et[0]) * jx;
  *ey = 0.25 * (et[-zo - xo] + et[-xo] + et[-zo] + et[0]) * jy;
  *ez = 0.25 * (et[-xo - yo] + et[-yo] + et[-xo] + et[0]) * jz;
}

/* eta*J on the CT edges in 3D: common/mhd_func.c:78-106 with zoffset = nx*ny */
static void ct_eres3(const geo *e, const double *bx, const double *by, const double *bz, const double *eta,
                     double idx, double idy, double idz, pt_fn df, long ss, double *ex, double *ey, double *ez)
{
  long xo = 1, yo = e->sy, zo = e->sz;
  long si[4] = {-2 * xo, -xo, 0, +xo}, sj[4] = {-2 * yo, -yo, 0, +yo}, sk[4] = {-2 * zo, -zo, 0, +zo};
  double bxj[4] = {bx[ss + sj[0]], bx[ss + sj[1]], bx[ss + sj[2]], bx[ss + sj[3]]};
  double bxk[4] = {bx[ss + sk[0]], bx[ss + sk[1]], bx[ss + sk[2]], bx[ss + sk[3]]};
  double byk[4] = {by[ss + sk[0]], by[ss + sk[1]], by[ss + sk[2]], by[ss + sk[3]]};
  double byi[4] = {by[ss + si[0]], by[ss + si[1]], by[ss + si[2]], by[ss + si[3]]};
  double bzi[4] = {bz[ss + si[0]], bz[ss + si[1]], bz[ss + si[2]], bz[ss + si[3]]};
  double bzj[4] = {bz[ss + sj[0]], bz[ss + sj[1]], bz[ss + sj[2]], bz[ss + sj[3]]};
  double jx = df(&bzj[1]) * idy - df(&byk[1]) * idz;
  double jy = df(&bxk[1]) * idz - df(&bzi[1]) * idx;
  double jz = df(&byi[1]) * idx - df(&bxj[1]) * idy;
  const double *et = eta + ss;
  *ex = 0.25 * (et[-yo - zo] + et[-zo] + et[-yo] + et[0]) * jx;
  *ey = 0.25 * (et[-zo - xo] + et[-xo] + et[-zo] + et[0]) * jy;
  *ez = 0.25 * (et[-xo - yo] + et[-yo] + et[-xo] + et[0]) * jz;
}

/* viscous face flux at i-1/2 along offset xo (transverse yo, zo): common/mhd_flux.c:700-752 */
static void visc_flux(const double *vx, const double *vy, const double *vz, long ss, double rnu,
                      double idx, double idy, double idz, long xo, long yo, long zo, pt_fn fc, pt_fn df,
                      double *fmx, double *fmy, double *fmz, double *fen)
{
  long s4[4] = {-2 * xo, -xo, 0, +xo};
  double c2 = 2. / 3., c4 = 4. / 3.;
  double vxi[4], vyi[4], vzi[4], dv[4];
  int m;
  for (m = 0; m < 4; m++) { vxi[m] = vx[ss + s4[m]]; vyi[m] = vy[ss + s4[m]]; vzi[m] = vz[ss + s4[m]]; }
  double vx0 = fc(&vxi[1]), vy0 = fc(&vyi[1]), vz0 = fc(&vzi[1]);
  double dvxdx = df(&vxi[1]) * idx, dvydx = df(&vyi[1]) * idx, dvzdx = df(&vzi[1]) * idx;
  for (m = 0; m < 4; m++) dv[m] = 0.5 * (vx[ss + s4[m] + yo] - vx[ss + s4[m] - yo]);
  double dvxdy = fc(&dv[1]) * idy;
  for (m = 0; m < 4; m++) dv[m] = 0.5 * (vy[ss + s4[m] + yo] - vy[ss + s4[m] - yo]);
  double dvydy = fc(&dv[1]) * idy;
  for (m = 0; m < 4; m++) dv[m] = 0.5 * (vx[ss + s4[m] + zo] - vx[ss + s4[m] - zo]);
  double dvxdz = fc(&dv[1]) * idz;
  for (m = 0; m < 4; m++) dv[m] = 0.5 * (vz[ss + s4[m] + zo] - vz[ss + s4[m] - zo]);
  double dvzdz = fc(&dv[1]) * idz;
  *fmx = -rnu * (c4 * dvxdx - c2 * (dvydy + dvzdz));
  *fmy = -rnu * (dvydx + dvxdy);
  *fmz = -rnu * (dvzdx + dvxdz);
  *fen = (*fmx) * vx0 + (*fmy) * vy0 + (*fmz) * vz0;
}

/* resistive face flux at i-1/2: common/mhd_flux.c:754-782 */
static void resist_flux(const double *by, const double *bz, const double *ey, const double *ez, long ss,
                        long xo, long yo, long zo, pt_fn fc, double *fby, double *fbz, double *fen)
{
  long s4[4] = {-2 * xo, -xo, 0, +xo};
  double ey0 = 0.5 * (ey[ss] + ey[ss + zo]);
  double ez0 = 0.5 * (ez[ss] + ez[ss + yo]);
  double byi[4], bzi[4];
  for (int m = 0; m < 4; m++) {
    byi[m] = 0.5 * (by[ss + s4[m]] + by[ss + s4[m] + yo]);
    bzi[m] = 0.5 * (bz[ss + s4[m]] + bz[ss + s4[m] + zo]);
  }
  double by0 = fc(&byi[1]), bz0 = fc(&bzi[1]);
  *fby = -ez0;
  *fbz = +ey0;
  *fen = ey0 * bz0 - ez0 * by0;
}

static int qo_dsptv3(const qo_grid *g, double *u, double dt, double nu0, double eta0);

int qo_dsptv(const qo_grid *g, double *u, double dt, double nu0, double eta0)
{
  if (g->dim == 3) return qo_dsptv3(g, u, dt, nu0, eta0);
  if (g->dim != 2) return -1;
  geo e = mkgeo(g);
  long nd = e.nd, sy = e.sy;
  int nx = e.nx, ny = e.ny, i, j;
  long ss;
  double *ut = xcalloc(8 * nd), *fx = xcalloc(8 * nd), *fy = xcalloc(8 * nd);
  double *ex = xcalloc(nd), *ey = xcalloc(nd), *ez = xcalloc(nd);
  double *vx = xcalloc(nd), *vy = xcalloc(nd), *vz = xcalloc(nd), *nu = xcalloc(nd), *eta = xcalloc(nd);
  if (!ut || !fx || !fy || !ex || !ey || !ez || !vx || !vy || !vz || !nu || !eta) return -1;
  for (ss = 0; ss < nd; ss++) {  /* setdc: the given profiles, else uniform */
    nu[ss] = g->nu ? g->nu[ss] : nu0;
    eta[ss] = g->eta ? g->eta[ss] : eta0;
  }
  pt_fn fc = face_to_centre(g->odr), df = first_diff(g->odr);
  double idx = 1.0 / g->dx, idy = 1.0 / g->dy;
  double dtdx = dt * idx, dtdy = dt * idy;
  double *f[8];
  for (int m = 0; m < 8; m++) f[m] = u + (long)m * nd;
  memcpy(ut, u, sizeof(double) * 8 * nd);
  for (int rk = 0; rk < g->rk; rk++) {
    const double *rkf = RKF[g->rk - 1][rk];
    for (ss = 0; ss < nd; ss++) {
      double iro = 1.0 / f[0][ss];
      vx[ss] = f[1][ss] * iro; vy[ss] = f[2][ss] * iro; vz[ss] = f[3][ss] * iro;
    }
#pragma omp parallel for schedule(static) private(i, ss)
    for (j = 2; j < ny - 1; j++)
      for (i = 2; i < nx - 1; i++) {
        ss = (long)nx * j + i;
        ct_eres2(&e, f[4], f[5], f[6], eta, idx, idy, df, ss, &ex[ss], &ey[ss], &ez[ss]);
      }
#pragma omp parallel for schedule(static) private(i, ss)
    for (j = 2; j < ny - 1; j++)
      for (i = 2; i < nx - 1; i++) {
        ss = (long)nx * j + i;
        double rnu, fl[2][8];
        memset(fl, 0, sizeof(fl));
        rnu = 0.5 * (f[0][ss - 1] * nu[ss - 1] + f[0][ss] * nu[ss]);
        visc_flux(vx, vy, vz, ss, rnu, idx, idy, 0.0, 1, sy, 0, fc, df, &fl[0][1], &fl[0][2], &fl[0][3], &fl[0][7]);
        resist_flux(f[5], f[6], ey, ez, ss, 1, sy, 0, fc, &fl[1][5], &fl[1][6], &fl[1][7]);
        fx[0 * nd + ss] = fl[0][0] + fl[1][0];
        fx[1 * nd + ss] = fl[0][1] + fl[1][1];
        fx[2 * nd + ss] = fl[0][2] + fl[1][2];
        fx[3 * nd + ss] = fl[0][3] + fl[1][3];
        fx[4 * nd + ss] = 0;
        fx[5 * nd + ss] = fl[0][5] + fl[1][5];
        fx[6 * nd + ss] = fl[0][6] + fl[1][6];
        fx[7 * nd + ss] = fl[0][7] + fl[1][7];
        rnu = 0.5 * (f[0][ss - sy] * nu[ss - sy] + f[0][ss] * nu[ss]);
        visc_flux(vy, vz, vx, ss, rnu, idy, 0.0, idx, sy, 0, 1, fc, df, &fl[0][1], &fl[0][2], &fl[0][3], &fl[0][7]);
        resist_flux(f[6], f[4], ez, ex, ss, sy, 0, 1, fc, &fl[1][5], &fl[1][6], &fl[1][7]);
        fy[0 * nd + ss] = fl[0][0] + fl[1][0];
        fy[2 * nd + ss] = fl[0][1] + fl[1][1];
        fy[3 * nd + ss] = fl[0][2] + fl[1][2];
        fy[1 * nd + ss] = fl[0][3] + fl[1][3];
        fy[5 * nd + ss] = 0;
        fy[6 * nd + ss] = fl[0][5] + fl[1][5];
        fy[4 * nd + ss] = fl[0][6] + fl[1][6];
        fy[7 * nd + ss] = fl[0][7] + fl[1][7];
      }
    int cen2[6] = {0, 1, 2, 3, 6, 7};
#pragma omp parallel for schedule(static) private(i, ss)
    for (j = GH; j < ny - GH; j++)
      for (i = GH; i < nx - GH; i++) {
        ss = (long)nx * j + i;
        for (int c = 0; c < 6; c++) {
          int m = cen2[c];
          double du0 = d4(fx + (long)m * nd, ss, 1, df);
          double du1 = d4(fy + (long)m * nd, ss, sy, df);
          rk_combine(&f[m][ss], ut[(long)m * nd + ss], (-dtdx * du0 - dtdy * du1), rkf[0], rkf[1]);
        }
      }
#pragma omp parallel for schedule(static) private(i, ss)
    for (j = GH; j < ny - GH + 1; j++)
      for (i = GH; i < nx - GH + 1; i++) {
        ss = (long)nx * j + i;
        if (j < ny - GH) {
          double du = d4(ez, ss, sy, df);
          rk_combine(&f[4][ss], ut[4 * nd + ss], -(+dtdy) * du, rkf[0], rkf[1]);
        }
        if (i < nx - GH) {
          double du = d4(ez, ss, 1, df);
          rk_combine(&f[5][ss], ut[5 * nd + ss], -(-dtdx) * du, rkf[0], rkf[1]);
        }
      }
    qo_bound(g, u);
  }
  free(ut); free(fx); free(fy); free(ex); free(ey); free(ez); free(vx); free(vy); free(vz); free(nu); free(eta);
  return 0;
}

/* 3D: DMHD3D::dsptv (3D/MPI/MRX/dmhd3d_solve.cpp:3-179) */
static int qo_dsptv3(const qo_grid *g, double *u, double dt, double nu0, double eta0)
{
  geo e = mkgeo(g);
  long nd = e.nd, sy = e.sy, sz = e.sz;
  int nx = e.nx, ny = e.ny, nz = e.nz, i, j, k;
  long ss;
  double *ut = xcalloc(8 * nd), *fx = xcalloc(8 * nd), *fy = xcalloc(8 * nd), *fz = xcalloc(8 * nd);
  double *ex = xcalloc(nd), *ey = xcalloc(nd), *ez = xcalloc(nd);
  double *vx = xcalloc(nd), *vy = xcalloc(nd), *vz = xcalloc(nd), *nu = xcalloc(nd), *eta = xcalloc(nd);
  if (!ut || !fx || !fy || !fz || !ex || !ey || !ez || !vx || !vy || !vz || !nu || !eta) return -1;
  for (ss = 0; ss < nd; ss++) {  /* setdc: the given profiles, else uniform */
    nu[ss] = g->nu ? g->nu[ss] : nu0;
    eta[ss] = g->eta ? g->eta[ss] : eta0;
  }
  pt_fn fc = face_to_centre(g->odr), df = first_diff(g->odr);
  double idx = 1.0 / g->dx, idy = 1.0 / g->dy, idz = 1.0 / g->dz;
  double dtdx = dt * idx, dtdy = dt * idy, dtdz = dt * idz;
  double *f[8];
  for (int m = 0; m < 8; m++) f[m] = u + (long)m * nd;
  memcpy(ut, u, sizeof(double) * 8 * nd);
  for (int rk = 0; rk < g->rk; rk++) {
    const double *rkf = RKF[g->rk - 1][rk];
    for (ss = 0; ss < nd; ss++) {
      double iro = 1.0 / f[0][ss];
      vx[ss] = f[1][ss] * iro; vy[ss] = f[2][ss] * iro; vz[ss] = f[3][ss] * iro;
    }
#pragma omp parallel for collapse(2) schedule(static) private(i, ss)
    for (k = 2; k < nz - 1; k++)
      for (j = 2; j < ny - 1; j++)
        for (i = 2; i < nx - 1; i++) {
          ss = IDX(e, i, j, k);
          ct_eres3(&e, f[4], f[5], f[6], eta, idx, idy, idz, df, ss, &ex[ss], &ey[ss], &ez[ss]);
        }
#pragma omp parallel for collapse(2) schedule(static) private(i, ss)
    for (k = 2; k < nz - 1; k++)
      for (j = 2; j < ny - 1; j++)
        for (i = 2; i < nx - 1; i++) {
          ss = IDX(e, i, j, k);
          double rnu, fl[2][8];
          memset(fl, 0, sizeof(fl));
          rnu = 0.5 * (f[0][ss - 1] * nu[ss - 1] + f[0][ss] * nu[ss]);
          visc_flux(vx, vy, vz, ss, rnu, idx, idy, idz, 1, sy, sz, fc, df, &fl[0][1], &fl[0][2], &fl[0][3], &fl[0][7]);
          resist_flux(f[5], f[6], ey, ez, ss, 1, sy, sz, fc, &fl[1][5], &fl[1][6], &fl[1][7]);
          fx[0 * nd + ss] = fl[0][0] + fl[1][0];
          fx[1 * nd + ss] = fl[0][1] + fl[1][1];
          fx[2 * nd + ss] = fl[0][2] + fl[1][2];
          fx[3 * nd + ss] = fl[0][3] + fl[1][3];
          fx[4 * nd + ss] = 0;
          fx[5 * nd + ss] = fl[0][5] + fl[1][5];
          fx[6 * nd + ss] = fl[0][6] + fl[1][6];
          fx[7 * nd + ss] = fl[0][7] + fl[1][7];
          rnu = 0.5 * (f[0][ss - sy] * nu[ss - sy] + f[0][ss] * nu[ss]);
          visc_flux(vy, vz, vx, ss, rnu, idy, idz, idx, sy, sz, 1, fc, df, &fl[0][1], &fl[0][2], &fl[0][3], &fl[0][7]);
          resist_flux(f[6], f[4], ez, ex, ss, sy, sz, 1, fc, &fl[1][5], &fl[1][6], &fl[1][7]);
          fy[0 * nd + ss] = fl[0][0] + fl[1][0];
          fy[2 * nd + ss] = fl[0][1] + fl[1][1];
          fy[3 * nd + ss] = fl[0][2] + fl[1][2];
          fy[1 * nd + ss] = fl[0][3] + fl[1][3];
          fy[5 * nd + ss] = 0;
          fy[6 * nd + ss] = fl[0][5] + fl[1][5];
          fy[4 * nd + ss] = fl[0][6] + fl[1][6];
          fy[7 * nd + ss] = fl[0][7] + fl[1][7];
          rnu = 0.5 * (f[0][ss - sz] * nu[ss - sz] + f[0][ss] * nu[ss]);
          visc_flux(vz, vx, vy, ss, rnu, idz, idx, idy, sz, 1, sy, fc, df, &fl[0][1], &fl[0][2], &fl[0][3], &fl[0][7]);
          resist_flux(f[4], f[5], ex, ey, ss, sz, 1, sy, fc, &fl[1][5], &fl[1][6], &fl[1][7]);
          fz[0 * nd + ss] = fl[0][0] + fl[1][0];
          fz[3 * nd + ss] = fl[0][1] + fl[1][1];
          fz[1 * nd + ss] = fl[0][2] + fl[1][2];
          fz[2 * nd + ss] = fl[0][3] + fl[1][3];
          fz[6 * nd + ss] = 0;
          fz[4 * nd + ss] = fl[0][5] + fl[1][5];
          fz[5 * nd + ss] = fl[0][6] + fl[1][6];
          fz[7 * nd + ss] = fl[0][7] + fl[1][7];
        }
    int cen3[5] = {0, 1, 2, 3, 7};
#pragma omp parallel for collapse(2) schedule(static) private(i, ss)
    for (k = GH; k < nz - GH; k++)
      for (j = GH; j < ny - GH; j++)
        for (i = GH; i < nx - GH; i++) {
          ss = IDX(e, i, j, k);
          for (int c = 0; c < 5; c++) {
            int m = cen3[c];
            double du0 = d4(fx + (long)m * nd, ss, 1, df);
            double du1 = d4(fy + (long)m * nd, ss, sy, df);
            double du2 = d4(fz + (long)m * nd, ss, sz, df);
            rk_combine(&f[m][ss], ut[(long)m * nd + ss], (-dtdx * du0 - dtdy * du1 - dtdz * du2), rkf[0], rkf[1]);
          }
        }
#pragma omp parallel for collapse(2) schedule(static) private(i, ss)
    for (k = GH; k < nz - GH + 1; k++)
      for (j = GH; j < ny - GH + 1; j++)
        for (i = GH; i < nx - GH + 1; i++) {
          ss = IDX(e, i, j, k);
          int in_k = k < nz - GH, in_j = j < ny - GH, in_i = i < nx - GH;
          if (in_k && in_j) { /* mhd_updt3d_ctb(&bx[ss], .., &ey, &ez, dtdy, dtdz, .., nx, nxy) */
            double du0 = +d4(ez, ss, sy, df);
            double du1 = -d4(ey, ss, sz, df);
            rk_combine(&f[4][ss], ut[4 * nd + ss], -dtdy * du0 - dtdz * du1, rkf[0], rkf[1]);
          }
          if (in_k && in_i) { /* (&by[ss], .., &ez, &ex, dtdz, dtdx, .., nxy, 1) */
            double du0 = +d4(ex, ss, sz, df);
            double du1 = -d4(ez, ss, 1, df);
            rk_combine(&f[5][ss], ut[5 * nd + ss], -dtdz * du0 - dtdx * du1, rkf[0], rkf[1]);
          }
          if (in_j && in_i) { /* (&bz[ss], .., &ex, &ey, dtdx, dtdy, .., 1, nx) */
            double du0 = +d4(ey, ss, 1, df);
            double du1 = -d4(ex, ss, sy, df);
            rk_combine(&f[6][ss], ut[6 * nd + ss], -dtdx * du0 - dtdy * du1, rkf[0], rkf[1]);
          }
        }
    qo_bound(g, u);
  }
  free(ut); free(fx); free(fy); free(fz); free(ex); free(ey); free(ez);
  free(vx); free(vy); free(vz); free(nu); free(eta);
  return 0;
}

int qo_dissipate(const qo_grid *g, double *u, double dt, double nu0, double eta0)
{
  if (g->dim < 2) return -1;
  double dx = g->dx, dy = g->dy;
  double dr = g->dim == 3 ? qmin(qmin(dx, dy), g->dz) : qmin(dx, dy);
  /* setdc's reduction (2D/SERIAL/MRX/dmhd2d_init_.cpp:85-106): max over every cell of
   * max(2 nu, eta), from 0 */
  double dcmax = 0.0;
  geo e = mkgeo(g);
  for (long ss = 0; ss < e.nd; ss++) {
    double dtmp = qmax(2 * (g->nu ? g->nu[ss] : nu0), g->eta ? g->eta[ss] : eta0);
    if (dtmp > dcmax) dcmax = dtmp;
  }
  if (dcmax > 1e-15) {
    int ncmax = 1 + (int)(2 * (dcmax * dt) / (dr * dr));
    for (int nc = 0; nc < ncmax; nc++) {
      qo_bound(g, u);
      if (qo_dsptv(g, u, dt / ncmax, nu0, eta0) != 0) return -1;
    }
  }
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Hall term of the 1D Hall driver: 1D/SERIAL/h-shock/hmhd1d_solve.cpp:138-264 */
/* ------------------------------------------------------------------------ */

/* HMHD1D::hallv (hmhd1d_class.hpp:28-35) with rotc (common/common_interp.h:39-43) on the
 * cell-centre field, which is the state's own B in 1D */
static void hall_velocity(const double *ro, const double *bx, const double *by, const double *bz, double di,
                          double idx, long i, double *hx, double *hy, double *hz)
{
  double fac = di / ro[i];
  hx[i] = 0.0;
  hy[i] = -fac * (0.5 * ((bx[i + 0] - bx[i - 0]) * 0.0 - (bz[i + 1] - bz[i - 1]) * idx));
  hz[i] = -fac * (0.5 * ((by[i + 1] - by[i - 1]) * idx - (bx[i + 0] - bx[i - 0]) * 0.0));
}

double qo_haldt(const qo_grid *g, const double *u, double cfl, double di, double vphix)
{
  geo e = mkgeo(g);
  long nx = e.nx;
  const double *ro = u, *bx = u + 4 * nx, *by = u + 5 * nx, *bz = u + 6 * nx;
  double *h = xcalloc(3 * nx);
  if (!h) return -1.0;
  double idx = 1.0 / g->dx, vmax = 1.0;
  for (long i = GH; i < nx - GH; i++) {
    hall_velocity(ro, bx, by, bz, di, idx, i, h, h + nx, h + 2 * nx);
    double vt = fabs(h[i]) + vphix * fabs(bx[i] / ro[i]);
    if (vt > vmax) vmax = vt;
  }
  free(h);
  return cfl * g->dx / vmax;
}

/* Lax-Friedrichs Hall flux: calc_flux_hall_lf (common/mhd_flux.c:784-813) */
static void flux_hall_lf(const double *L, const double *R, double bnc, double smax, double *fbt, double *fbu,
                         double *fen)
{
  double pml = 0.5 * (bnc * bnc + L[4] * L[4] + L[5] * L[5]);
  double vbl = L[1] * bnc + L[2] * L[4] + L[3] * L[5];
  double pmr = 0.5 * (bnc * bnc + R[4] * R[4] + R[5] * R[5]);
  double vbr = R[1] * bnc + R[2] * R[4] + R[3] * R[5];
  double fbtl = L[4] * L[1] - bnc * L[2];
  double fbul = L[5] * L[1] - bnc * L[3];
  double fenl = 2.0 * pml * L[1] - bnc * vbl;
  double fbtr = R[4] * R[1] - bnc * R[2];
  double fbur = R[5] * R[1] - bnc * R[3];
  double fenr = 2.0 * pmr * R[1] - bnc * vbr;
  *fbt = 0.5 * (fbtl + fbtr - smax * (R[4] - L[4]));
  *fbu = 0.5 * (fbul + fbur - smax * (R[5] - L[5]));
  *fen = 0.5 * (fenl + fenr - smax * (pmr - pml));
}

int qo_hall(const qo_grid *g, double *u, double dt, double di, double vphix)
{
  if (g->dim != 1) return -1;
  geo e = mkgeo(g);
  long nx = e.nx, i;
  double *f[8];
  for (int m = 0; m < 8; m++) f[m] = u + (long)m * nx;
  double *ut = xcalloc(8 * nx), *h = xcalloc(3 * nx), *vl = xcalloc(7 * nx), *vr = xcalloc(7 * nx);
  double *fx = xcalloc(3 * nx);
  if (!ut || !h || !vl || !vr || !fx) return -1;
  double *hv[3] = {h, h + nx, h + 2 * nx};
  memcpy(ut, u, sizeof(double) * 8 * nx);
  lr_fn lr = nl_interp(g->odr);
  pt_fn df = first_diff(g->odr);
  double idx = 1.0 / g->dx, dtdx = dt / g->dx;
  for (int rk = 0; rk < g->rk; rk++) {
    const double *rkf = RKF[g->rk - 1][rk];
    for (i = 1; i < nx - 1; i++) hall_velocity(f[0], f[4], f[5], f[6], di, idx, i, hv[0], hv[1], hv[2]);
    {  /* bound(pv,3,&dnxs[1]) */
      const int *dn[3] = {g->dnx + 1, g->dny + 1, g->dnz + 1};
      const int *st[3] = {ST_0, ST_0, ST_0};
      fill_ghosts(&e, hv, 3, dn, st);
    }
    /* mhd_lr_single of ro, hx, hy, hz, by, bz, en: left state at face i+1, right at face i */
    const double *q[7] = {f[0], hv[0], hv[1], hv[2], f[5], f[6], f[7]};
    for (i = 2; i < nx - 2; i++)
      for (int m = 0; m < 7; m++) {
        double s5[5] = {q[m][i - 2], q[m][i - 1], q[m][i], q[m][i + 1], q[m][i + 2]};
        lr(&s5[2], &vl[(long)m * nx + i + 1], &vr[(long)m * nx + i]);
      }
    for (i = 3; i < nx - 2; i++) {
      double L[7], R[7];
      for (int m = 0; m < 7; m++) { L[m] = vl[(long)m * nx + i]; R[m] = vr[(long)m * nx + i]; }
      double bn = 0.5 * (f[4][i] + f[4][i]);
      double rn = qmin(L[0], R[0]);
      double smax = 0.0;
      smax += qmax(fabs(L[1]), fabs(R[1]));
      smax += vphix * fabs(bn / rn);
      flux_hall_lf(L, R, bn, smax, &fx[i], &fx[nx + i], &fx[2 * nx + i]);
    }
    if (g->hall_de != 0) {  /* hmhd1d_solve.cpp:232-240 */
      crcte(fx, fx + 2 * nx, f[5], nx, g->dnx[1] * g->dnx[5], g->hall_de, g->dx, g->odr);
      crcte(fx + nx, fx + 2 * nx, f[6], nx, g->dnx[1] * g->dnx[6], g->hall_de, g->dx, g->odr);
    }
    /* update of by, bz, en (mhd_updt1d) */
    for (i = GH; i < nx - GH; i++) {
      const int mm[3] = {5, 6, 7};
      for (int c = 0; c < 3; c++) {
        double d = -dtdx * d4(fx + (long)c * nx, i, 1, df);
        rk_combine(&f[mm[c]][i], ut[(long)mm[c] * nx + i], d, rkf[0], rkf[1]);
      }
    }
    qo_bound(g, u);
  }
  free(ut); free(h); free(vl); free(vr); free(fx);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* known-answer entry (layouts of oracle/ref_harness/ref_kat.cpp)            */
/* ------------------------------------------------------------------------ */
int qo_kat(int func, int ncase, int nin, int nout, const double *in, double *out)
{
  static const lr_fn lrs[10] = {flr1, flr2, flr3, flr4, muscl_mm, wcns3, wcns4, muscl_mc, muscl_vl, muscl_kr};
  for (int c = 0; c < ncase; c++) {
    const double *a = in + (long)c * nin;
    double *o = out + (long)c * nout;
    if (func >= 0 && func <= 3) {
      riemann(func)(&a[0], &a[7], a[14], a[15], &a[16], o);
    } else if (func >= 10 && func <= 19) {
      lrs[func - 10](&a[2], &o[0], &o[1]);
    } else if ((func >= 20 && func <= 27) || (func >= 40 && func <= 43)) {
      /* 24..27: primitive reconstruction, 40..43: Athena-type */
      double q[7][5];
      const int mode = func >= 40 ? 2 : (func >= 24 ? 1 : 0);
      const int odr = func >= 40 ? func - 39 : (func >= 24 ? func - 23 : func - 19);
      for (int v = 0; v < 7; v++)
        for (int m = 0; m < 5; m++) q[v][m] = a[5 * v + m];
      face_states(q, a[35], a[36], nl_interp(odr), &o[0], &o[7], mode);
    } else if (func == 30) {
      o[0] = cuct_weight(&a[3], &a[7], &a[11], &a[15], &a[19], 1, 2);
    } else if (func == 31) {
      o[0] = ieos(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8]);
    } else if (func == 32) {
      o[0] = energy(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8]);
    } else {
      return -1;
    }
  }
  return 0;
}
