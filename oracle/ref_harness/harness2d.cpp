/*
 * Oracle harness for the reference's 2D stepping code.
 *
 * Built (oracle/Makefile) against the reference sources where they lie:
 *   2D/SERIAL/MRX/{mhd2d_class,mhd2d_solve,dmhd2d_class,dmhd2d_solve}.cpp
 *   (mhd2d_solve.cpp and mhd2d_class.cpp are byte-identical to the OTvortex
 *   and KHI copies) plus common/*.c.
 * The harness loads a state, runs the reference's own bound()/ideal()/setdt()
 * (and dsptv() for the resistive form) with the loop semantics of
 * MHD2D::exec_ (2D/SERIAL/OTvortex/mhd2d_class.cpp:35-61) and
 * DMHD2D::exec_ (2D/SERIAL/MRX/dmhd2d_class.cpp:3-39), and writes the result.
 * Test infrastructure only.
 */
#include <omp.h>
#ifdef QAS_GRAVITY
/* gravity form: built against 2D/SERIAL/RTI (MHD2D with phi_g; no dissipative driver) */
#include "mhd2d_class.hpp"
typedef MHD2D RefBase;
#else
#include "dmhd2d_class.hpp"
typedef DMHD2D RefBase;
#endif
#include "qas_ref_io.h"

int qh_xmesh = 1, qh_ymesh = 1, qh_zmesh = 1, qh_nout = 1, qh_rmn = 1, qh_odr = 4, qh_rk = 3;
double qh_dtrec = 1.0, qh_cfl = 0.4;

static double g_nu0 = 0.0, g_eta0 = 0.0;
static const double *g_nu_arr = nullptr, *g_eta_arr = nullptr;  /* per-cell profiles, if given */

#ifndef QAS_GRAVITY

/* Uniform visco-resistive coefficients; same reduction as the reference's
 * localized-profile version (2D/SERIAL/MRX/dmhd2d_init_.cpp:85-106). */
double DMHD2D::setdc()
{
  double dcmax = 0.0, dtmp;
  for (int j = 0; j < ny; j++) {
    for (int i = 0; i < nx; i++) {
      int ss = nx * j + i;
      nu[ss] = g_nu_arr ? g_nu_arr[ss] : g_nu0;
      eta[ss] = g_eta_arr ? g_eta_arr[ss] : g_eta0;
      dtmp = max(2 * nu[ss], eta[ss]);
      if (dtmp > dcmax) dcmax = dtmp;
    }
  }
  return dcmax;
}

#endif

class RefHarness2D : public RefBase {
 public:
  void setup(const RefCaseHeader &h, const double *data)
  {
    setgam(h.gam);
    xmin = h.xmin; xmax = h.xmax; ymin = h.ymin; ymax = h.ymax;
    dx = (xmax - xmin) / XMESH;
    dy = (ymax - ymin) / YMESH;
    dr = min(dx, dy);
    dt = cfl * dr;
    for (int i = 0; i < nx; i++) x[i] = (i - xoff + 0.5) * dx + xmin;
    for (int j = 0; j < ny; j++) y[j] = (j - yoff + 0.5) * dy + ymin;
    for (int m = 0; m < nm; m++) { dnxs[m] = h.dnx[m]; dnys[m] = h.dny[m]; }
    for (int m = 0; m < nm; m++) memcpy(val[m], data + (size_t)m * nd, sizeof(double) * nd);
#ifdef QAS_GRAVITY
    if (!(h.has_phi & 1)) ref_die("the gravity build needs phi_g in the case");
    memcpy(phi_g, data + (size_t)8 * nd, sizeof(double) * nd);
#else
    if (h.has_phi & 1) ref_die("phi_g given to a build without gravity");
#endif
    if (h.has_phi & 2) {  /* per-cell nu, eta after the state (and phi_g) */
      const size_t o = (size_t)(8 + (h.has_phi & 1)) * nd;
      g_nu_arr = data + o;
      g_eta_arr = data + o + nd;
    }
  }
  void dissipate()
  {
#ifdef QAS_GRAVITY
    ref_die("no dissipative form in the gravity build");
#else
    double dcmax = setdc();
    if (dcmax > 1e-15) {
      int nc, ncmax = 1 + (int)(2 * (dcmax * dt) / (dr * dr));
      for (nc = 0; nc < ncmax; nc++) {
        bound(val, nm, stxs, dnxs, stys, dnys);
        dsptv(dt / ncmax);
      }
    }
#endif
  }
  void one_step(int flg, bool resist, std::vector<double> *dts)
  {
    tim += dt;
    dts->push_back(dt);
    bound(val, nm, stxs, dnxs, stys, dnys);
    ideal(dt);
    if (resist) dissipate();
    setdt(flg * (n % 2 == 0));
  }
  int run(const RefCaseHeader &h, std::vector<double> *dts, double *elapsed)
  {
    int steps = 0;
    double t0 = omp_get_wtime();
    if (h.mode == REF_MODE_STEP) {
      dt = h.dt;
      dts->push_back(dt);
      bound(val, nm, stxs, dnxs, stys, dnys);
      ideal(dt);
      steps = 1;
    } else if (h.mode == REF_MODE_DSTEP) {
#ifdef QAS_GRAVITY
      ref_die("no dissipative form in the gravity build");
#else
      dt = h.dt;
      dts->push_back(dt);
      setdc();
      bound(val, nm, stxs, dnxs, stys, dnys);
      dsptv(dt);
#endif
      steps = 1;
    } else if (h.mode == REF_MODE_RUN || h.mode == REF_MODE_DRUN) {
      setdt(1);
      for (int s = 0; s < h.nsteps; s++) {
        double ts = omp_get_wtime();
        n++;
        one_step(h.flg, h.mode == REF_MODE_DRUN, dts);
        step_times.push_back(omp_get_wtime() - ts);
        steps++;
      }
    } else if (h.mode == REF_MODE_EXEC) {
      setdt(1);
      while (n++ < nmax && tim < tmax) {
        one_step(h.flg, false, dts);
        steps++;
      }
    } else {
      ref_die("unknown mode");
    }
    *elapsed = omp_get_wtime() - t0;
    return steps;
  }
  /* the reference's own writers / reader on this state (I/O pins) */
  void io(const RefCaseHeader &h, const char *dir)
  {
    snprintf(fildir, sizeof(fildir), "%s", dir);
    if (h.mode == REF_MODE_IO) {
      n = h.nsteps;
      cnt = h.flg;
      tim = h.dt;
      dt = h.cfl;
      trec = h.dtrec;
      dout_(0);
      bkup_save(val, nm, nd, n, cnt, tim, dt, trec, 0, fildir);
    } else {
      bkup_load(val, nm, nd, &n, &cnt, &tim, &dt, &trec, 0, fildir);
      ref_write_loaded(dir, n, cnt, tim, dt, trec);
    }
  }
  double time_now() const { return tim; }
  double dt_now() const { return dt; }
  double *const *state() const { return val; }
  std::vector<double> step_times;
};

int main(int argc, char **argv)
{
  if (argc != 3 && argc != 4) ref_die("usage: ref2d <case.bin> <result.bin> [io dir]");
  RefCaseHeader h;
  std::vector<double> data;
  ref_read_case(argv[1], &h, &data);
  if (h.dim != 2) ref_die("ref2d needs dim=2");
  if (h.ctw != CTW) ref_die("binary built for the other CTW setting");
  qh_xmesh = h.nxm; qh_ymesh = h.nym; qh_zmesh = 1;
  qh_rmn = h.rmn; qh_odr = h.odr; qh_rk = h.rk;
  qh_cfl = h.cfl; qh_dtrec = h.dtrec; qh_nout = h.nout;
  g_nu0 = h.nu0; g_eta0 = h.eta0;
  if (h.nthreads > 0) omp_set_num_threads(h.nthreads);

  RefHarness2D *sim = new RefHarness2D();
  sim->setup(h, data.data());
  std::vector<double> dts;
  double elapsed = 0.0;
  int steps = 0;
  if (h.mode == REF_MODE_IO || h.mode == REF_MODE_IOLOAD) {
    if (argc != 4) ref_die("I/O modes need the directory argument");
    sim->io(h, argv[3]);
  } else {
    steps = sim->run(h, &dts, &elapsed);
  }

  RefResultHeader r;
  memset(&r, 0, sizeof(r));
  r.magic = QAS_REF_MAGIC_OUT;
  r.nsteps_done = steps;
  r.n_dt = (int)dts.size();
  r.nd = (h.nxm + 8) * (h.nym + 8);
  r.tim = sim->time_now();
  r.dt = sim->dt_now();
  r.elapsed_s = elapsed;
  ref_write_result(argv[2], r, dts, sim->state(), r.nd);
  ref_append_times(argv[2], sim->step_times);
  delete sim;
  return 0;
}
