// Host build of the forward point functions and their reverse-mode (VJP)
// counterparts, for finite-difference checks on the CPU.
#include "qas_adjoint.cuh"

using namespace qas;

extern "C" {

void t_wcns4(const double *f, double *out) { wcns4_lr(f, out[0], out[1]); }
void t_wcns4_vjp(const double *f, double gl, double gr, double *gf) { wcns4_vjp(f, gl, gr, gf); }

void t_face_states(const double *q, double bn, double gam, double *vl, double *vr)
{
  double qq[7][5];
  for (int v = 0; v < 7; v++)
    for (int m = 0; m < 5; m++) qq[v][m] = q[5 * v + m];
  face_states<4>(qq, bn, gam, vl, vr);
}
void t_face_states_vjp(const double *q, double bn, double gam, const double *gvl, const double *gvr, double *gq,
                       double *gbn)
{
  double qq[7][5], g[7][5] = {};
  for (int v = 0; v < 7; v++)
    for (int m = 0; m < 5; m++) qq[v][m] = q[5 * v + m];
  double b = 0.0;
  face_states_vjp(qq, bn, gam, gvl, gvr, g, b);
  for (int v = 0; v < 7; v++)
    for (int m = 0; m < 5; m++) gq[5 * v + m] = g[v][m];
  *gbn = b;
}

void t_roe(const double *L, const double *R, double bn, double gam, double *F) { flux_roe(L, R, bn, gam, F); }
void t_roe_vjp(const double *L, const double *R, double bn, double gam, const double *gF, double *gL, double *gR,
               double *gbn)
{
  double b = 0.0;
  for (int k = 0; k < 7; k++) gL[k] = gR[k] = 0.0;
  flux_roe_vjp(L, R, bn, gam, gF, gL, gR, b);
  *gbn = b;
}

double t_cuct(const double *a)
{
  return cuct_weight(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8], a[9], a[10], a[11], a[12], a[13], a[14],
                     a[15]);
}
void t_cuct_vjp(const double *a, double g, double *gi)
{
  for (int k = 0; k < 16; k++) gi[k] = 0.0;
  cuct_weight_vjp(a, g, gi);
}
}
