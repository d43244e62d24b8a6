/*
 * qas_oracle.h -- plain-C restatement of qasMHD's per-step update.
 *
 * TEST INFRASTRUCTURE.  This library is the CPU checker used by tests/,
 * __graft_entry__.smoke() and the CPU-baseline leg of bench.py.  The product
 * (libqas, include/qas.h) never links or calls it.
 *
 * State layout: one contiguous block of 8*nd doubles, field m at u + m*nd,
 * fields (ro,mx,my,mz,bx,by,bz,en), cell ss = nx*(ny*k+j)+i with 4 ghost
 * cells per side (2D/SERIAL/OTvortex/mhd2d_class.cpp:116-164).
 */
#ifndef QAS_ORACLE_H
#define QAS_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int dim;             /* 1, 2 or 3 */
  int nxm, nym, nzm;   /* interior cells per axis (1 for unused axes) */
  int rmn;             /* 0 Roe, 1 HLLD, 2 LHLLD, 3 MLAU (common/mhd_class.hpp:102-105) */
  int odr;             /* spatial order 1..4 */
  int rk;              /* SSP-RK order 1..3 */
  int ctw;             /* CUCT upwind weighting on/off */
  double gam, dx, dy, dz;
  int dnx[8], dny[8], dnz[8];   /* boundary flags per field */
  const double *phi;   /* gravitational potential phi_g (nd doubles), NULL without gravity:
                          the gravity form of the 2D/3D drivers (2D/SERIAL/RTI, 3D/MPI/RTI) */
  double hall_de;      /* 1D Hall driver's electron inertia length de (absolute); when non-zero
                          the by/bz fluxes of ideal() and hall_() get the crcte correction */
  const double *nu, *eta;  /* per-cell viscosity / resistivity of the dissipative drivers (the
                              API's nu/eta, nd doubles each); NULL: uniform nu0/eta0 arguments */
  int char_mode;       /* 0 characteristic reconstruction (mhd_m/a_reconst), 1 primitive (mhd_reconst),
                          2 Athena-type characteristic (mhd_c_reconst) */
} qo_grid;

/* Ghost fill of the 8 state fields (bound(): mhd1d_class.cpp:3-9, mhd2d_class.cpp:3-9,
 * mhd3d_class.cpp:3-13). */
void qo_bound(const qo_grid *g, double *u);

/* One SSP-RK step of the ideal equations, i.e. MHD{1,2,3}D::ideal(dt), including the
 * per-stage ghost fill.  Returns 0 on success, -1 on allocation failure. */
int qo_step(const qo_grid *g, double *u, double dt);

/* max(1, max over interior of |v| + c_f), the reduction inside setdt()
 * (mhd1d_class.cpp:11-30, mhd2d_class.cpp:11-33, mhd3d_class.cpp:15-46).  `unused`
 * is ignored (kept for ABI stability of the test binding).  With gravity the energy of each
 * interior cell is rewritten as (en - ro*phi) + ro*phi, as the gravity drivers' setdt does
 * (2D/SERIAL/RTI/mhd2d_class.cpp:46-48). */
double qo_cfl_dt(const qo_grid *g, double *u, double unused);

/* One visco-resistive stage loop, DMHD2D::dsptv(dt) (2D/SERIAL/MRX/dmhd2d_solve.cpp:3-151)
 * with uniform nu0, eta0.  2D only. */
int qo_dsptv(const qo_grid *g, double *u, double dt, double nu0, double eta0);

/* setdc() + sub-cycled dsptv (2D/SERIAL/MRX/dmhd2d_class.cpp:19-26) with uniform nu0, eta0. */
int qo_dissipate(const qo_grid *g, double *u, double dt, double nu0, double eta0);

/* Hall term of the 1D Hall driver (1D/SERIAL/h-shock): one hall_(dt) call
 * (hmhd1d_solve.cpp:138-264) with ion inertia length di and whistler speed factor vphix and
 * no electron inertia (de = 0), and haldt() (hmhd1d_class.cpp:3-13), which returns the
 * Hall sub-cycle time step cfl*dx/max(1, max_i |hx| + vphix |bx/ro|).  With g->hall_de != 0
 * both hall_ and the 1D ideal step apply the electron-inertia correction (crcte with a CG
 * solve, hmhd1d_solve.cpp:266-426). */
int qo_hall(const qo_grid *g, double *u, double dt, double di, double vphix);
double qo_haldt(const qo_grid *g, const double *u, double cfl, double di, double vphix);

/* Point-function known answers; same function ids and layouts as oracle/ref_harness/ref_kat.cpp,
 * plus 24..27: mhd_lrstate at ODR 1..4 with the primitive reconstruction mhd_reconst (the ids
 * 20..23 of the harness built against it, oracle/_ref/ref_kat_prim), and 40..43: the same with
 * the Athena-type reconstruction mhd_c_reconst (oracle/_ref/ref_kat_char). */
int qo_kat(int func, int ncase, int nin, int nout, const double *in, double *out);

#ifdef __cplusplus
}
#endif
#endif
