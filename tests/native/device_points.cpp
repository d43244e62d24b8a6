// Host build of the device point functions of the step (qas_device.cuh is host+device): the
// Riemann solvers, the face interpolations, the characteristic face states (both the
// per-field and the grouped-stencil forms the kernels use), the primitive-variable and the
// Athena-type characteristic face states and the CUCT weight, with the
// argument layout of the known-answer vectors of the reference's own point functions.
#include "qas_device.cuh"

using namespace qas;

namespace {

struct ArrayStencil {  // P(v, m) over a 7 x 5 stencil in row-major order
  const double *a;
  double operator()(int v, int m) const { return a[5 * v + m]; }
};

template <int ODR>
void face_states_of(const double *a, int grouped, double *o)
{
  if (grouped) {
    face_states_grouped<ODR>(ArrayStencil{a}, a[35], a[36], &o[0], &o[7]);
  } else {
    double q[7][5];
    for (int v = 0; v < 7; v++)
      for (int m = 0; m < 5; m++) q[v][m] = a[5 * v + m];
    face_states<ODR>(q, a[35], a[36], &o[0], &o[7]);
  }
}

}  // namespace

extern "C" {

// a: L[7], R[7], bn, gamma, dv0, dv1 -> F[7]
void t_flux(int rmn, const double *a, double *o)
{
  switch (rmn) {
    case 0: riemann<0>(&a[0], &a[7], a[14], a[15], a[16], a[17], o); break;
    case 1: riemann<1>(&a[0], &a[7], a[14], a[15], a[16], a[17], o); break;
    case 2: riemann<2>(&a[0], &a[7], a[14], a[15], a[16], a[17], o); break;
    default: riemann<3>(&a[0], &a[7], a[14], a[15], a[16], a[17], o); break;
  }
}

// a: 5-point stencil -> (left state at the right face, right state at the left face)
void t_lin(int odr, const double *a, double *o)
{
  switch (odr) {
    case 1: lin_lr<1>(a, o[0], o[1]); break;
    case 2: lin_lr<2>(a, o[0], o[1]); break;
    case 3: lin_lr<3>(a, o[0], o[1]); break;
    default: lin_lr<4>(a, o[0], o[1]); break;
  }
}
void t_nl(int odr, const double *a, double *o)
{
  switch (odr) {
    case 1: nl_lr<1>(a, o[0], o[1]); break;
    case 2: nl_lr<2>(a, o[0], o[1]); break;
    case 3: nl_lr<3>(a, o[0], o[1]); break;
    default: nl_lr<4>(a, o[0], o[1]); break;
  }
}

// a: q[7][5] (ro, vn, vt, vu, bt, bu, pr), bn, gamma -> vl[7], vr[7]
void t_face_states(int odr, int grouped, const double *a, double *o)
{
  switch (odr) {
    case 1: face_states_of<1>(a, grouped, o); break;
    case 2: face_states_of<2>(a, grouped, o); break;
    case 3: face_states_of<3>(a, grouped, o); break;
    default: face_states_of<4>(a, grouped, o); break;
  }
}

// the same with the Athena-type characteristic reconstruction (mhd_c_reconst, mhd_eigen_st)
void t_face_states_char(int odr, const double *a, double *o)
{
  const ArrayStencil st{a};
  switch (odr) {
    case 1: face_states_athena<1>(st, a[35], a[36], &o[0], &o[7]); break;
    case 2: face_states_athena<2>(st, a[35], a[36], &o[0], &o[7]); break;
    case 3: face_states_athena<3>(st, a[35], a[36], &o[0], &o[7]); break;
    default: face_states_athena<4>(st, a[35], a[36], &o[0], &o[7]); break;
  }
}

// the same with the primitive reconstruction (mhd_reconst): each field interpolated on its own
void t_face_states_prim(int odr, const double *a, double *o)
{
  const ArrayStencil st{a};
  switch (odr) {
    case 1: face_states_prim<1>(st, &o[0], &o[7]); break;
    case 2: face_states_prim<2>(st, &o[0], &o[7]); break;
    case 3: face_states_prim<3>(st, &o[0], &o[7]); break;
    default: face_states_prim<4>(st, &o[0], &o[7]); break;
  }
}

// a: ro, va, vb, ba, bb at the four cells (c-oa-ob, c-ob, c-oa, c) of a corner
double t_cuct(const double *a)
{
  return cuct_weight(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8], a[9], a[10], a[11], a[13], a[15], a[18],
                     a[19]);
}

}  // extern "C"
