/*
 * Oracle harness for the reference's 1D stepping code
 * (1D/SERIAL/shock/mhd1d_solve.cpp:3-124, mhd1d_class.cpp:3-53).
 * Loop semantics follow MHD1D::exec_ (1D/SERIAL/shock/mhd1d_class.cpp:32-53):
 * the 1D driver calls exec_(0) (1D/SERIAL/shock/main.cpp), i.e. a constant dt
 * from the first setdt(1) and nmax = nrec*nout steps.  Test infrastructure only.
 */
#include <omp.h>
#ifdef QAS_HALL
/* Hall form: built against 1D/SERIAL/h-shock (HMHD1D: hmhd1d_class.cpp, hmhd1d_solve.cpp),
 * with the Hall parameters taken from the case (di = nu0, de = eta0 fields) and vphix set as
 * HMHD1D::paras does (1D/SERIAL/h-shock/hmhd1d_paras.cpp:29-34). */
#include "hmhd1d_class.hpp"
typedef HMHD1D RefBase;
#else
#include "mhd1d_class.hpp"
typedef MHD1D RefBase;
#endif
#include "qas_ref_io.h"

int qh_xmesh = 1, qh_ymesh = 1, qh_zmesh = 1, qh_nout = 1, qh_rmn = 1, qh_odr = 4, qh_rk = 3;
double qh_dtrec = 1.0, qh_cfl = 0.4;

class RefHarness1D : public RefBase {
 public:
  void setup(const RefCaseHeader &h, const double *data)
  {
    setgam(h.gam);
    xmin = h.xmin; xmax = h.xmax;
    dx = (xmax - xmin) / XMESH;
    dt = cfl * dx;
    for (int i = 0; i < nx; i++) x[i] = (i - xoff + 0.5) * dx + xmin;
    for (int m = 0; m < nm; m++) dnxs[m] = h.dnx[m];
    for (int m = 0; m < nm; m++) memcpy(val[m], data + (size_t)m * nx, sizeof(double) * nx);
#ifdef QAS_HALL
    di = h.nu0;
    de = h.eta0;
    idx = 1.0 / dx;
    double kpeak = M_PI * idx;
    if (de != 0) kpeak = min(kpeak, 1.0 / de);
    vphix = di * kpeak;
#endif
  }
  void one_step(int flg, std::vector<double> *dts)
  {
    tim += dt;
    dts->push_back(dt);
    bound(val, nm, dnxs);
#ifdef QAS_HALL
    /* Hall sub-cycles of HMHD1D::exec_ (1D/SERIAL/h-shock/hmhd1d_class.cpp:26-33) */
    if (di != 0) {
      int hmax = 1 + (int)(dt / haldt());
      for (int hs = 0; hs < hmax; hs++) {
        hall_(dt / hmax);
        bound(val, nm, dnxs);
      }
    }
#endif
    ideal(dt);
    setdt(flg * (n % 2 == 0));
  }
  int run(const RefCaseHeader &h, std::vector<double> *dts, double *elapsed)
  {
    int steps = 0;
    double t0 = omp_get_wtime();
    if (h.mode == REF_MODE_STEP) {
      dt = h.dt;
      dts->push_back(dt);
      bound(val, nm, dnxs);
      ideal(dt);
      steps = 1;
#ifdef QAS_HALL
    } else if (h.mode == REF_MODE_DSTEP) {  /* Hall build: bound; one hall_(dt) */
      dt = h.dt;
      dts->push_back(dt);
      bound(val, nm, dnxs);
      hall_(dt);
      steps = 1;
#endif
    } else if (h.mode == REF_MODE_RUN) {
      setdt(1);
      for (int s = 0; s < h.nsteps; s++) {
        double ts = omp_get_wtime();
        n++;
        one_step(h.flg, dts);
        step_times.push_back(omp_get_wtime() - ts);
        steps++;
      }
    } else if (h.mode == REF_MODE_EXEC) {
      setdt(1);
      int flg = h.flg;
      while ((flg) ? (n++ < nmax && tim < tmax) : (n++ < nmax)) {
        one_step(flg, dts);
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
      dout_();
      bkup_save(val, nm, nx, n, cnt, tim, dt, trec, 0, fildir);
    } else {
      bkup_load(val, nm, nx, &n, &cnt, &tim, &dt, &trec, 0, fildir);
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
  if (argc != 3 && argc != 4) ref_die("usage: ref1d <case.bin> <result.bin> [io dir]");
  RefCaseHeader h;
  std::vector<double> data;
  ref_read_case(argv[1], &h, &data);
  if (h.dim != 1) ref_die("ref1d needs dim=1");
  qh_xmesh = h.nxm; qh_ymesh = 1; qh_zmesh = 1;
  qh_rmn = h.rmn; qh_odr = h.odr; qh_rk = h.rk;
  qh_cfl = h.cfl; qh_dtrec = h.dtrec; qh_nout = h.nout;
  if (h.nthreads > 0) omp_set_num_threads(h.nthreads);

  RefHarness1D *sim = new RefHarness1D();
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
  r.nd = h.nxm + 8;
  r.tim = sim->time_now();
  r.dt = sim->dt_now();
  r.elapsed_s = elapsed;
  ref_write_result(argv[2], r, dts, sim->state(), r.nd);
  ref_append_times(argv[2], sim->step_times);
  delete sim;
  return 0;
}
