/*
 * Tangent-linear run of the reference's 2D stepping code: the sources of
 * 2D/SERIAL/MRX (mhd2d_class, mhd2d_solve, dmhd2d_class, dmhd2d_solve) and
 * common/*.c compiled with a forward-mode dual number in place of double
 * (qas_dual.h).  It steps the exec_ body -- bound(), ideal(dt), and with eta0 > 0
 * setdc() + the sub-cycled dsptv (DMHD2D::exec_, 2D/SERIAL/MRX/dmhd2d_class.cpp:
 * 19-26) -- with a given dt per step held constant, from a state seeded with a
 * tangent direction (and an eta tangent), and writes the final state and its
 * directional derivative.  Test infrastructure: the reference dual-number
 * gradient the adjoint is checked against.
 *
 * Input : DualCaseHeader, dts[nsteps], state[8*nd], tangent[8*nd]
 * Output: state[8*nd], tangent[8*nd]
 */
#include "qas_dual.h"
#define double qd
#include "dmhd2d_class.hpp"

static qd g_eta_dual(0.0);
static double g_nu_plain;  // `double` is qd here: plain values below go through .v

qd DMHD2D::setdc()
{
  qd dcmax = 0.0, dtmp;
  for (int j = 0; j < ny; j++) {
    for (int i = 0; i < nx; i++) {
      int ss = nx * j + i;
      nu[ss] = g_nu_plain;
      eta[ss] = g_eta_dual;
      dtmp = max(2 * nu[ss], eta[ss]);
      if (dtmp > dcmax) dcmax = dtmp;
    }
  }
  return dcmax;
}
#undef double

int qh_xmesh = 1, qh_ymesh = 1, qh_zmesh = 1, qh_nout = 1, qh_rmn = 0, qh_odr = 4, qh_rk = 3;
double qh_dtrec = 1.0, qh_cfl = 0.4;

#pragma pack(push, 1)
struct DualCaseHeader {
  int32_t magic;  // "QASD"
  int32_t nxm, nym, rmn, odr, rk, ctw, nsteps, nthreads, pad;
  double gam, xmin, xmax, ymin, ymax, eta0, deta;
  int32_t dnx[8], dny[8];
};
#pragma pack(pop)

static void die(const char *m)
{
  fprintf(stderr, "ref2d_dual: %s\n", m);
  exit(2);
}

class DualHarness2D : public DMHD2D {
 public:
  void setup(const DualCaseHeader &h, const double *st, const double *tg)
  {
    setgam(h.gam);
    xmin = h.xmin; xmax = h.xmax; ymin = h.ymin; ymax = h.ymax;
    dx = (xmax - xmin) / XMESH;
    dy = (ymax - ymin) / YMESH;
    dr = min(dx, dy);
    for (int i = 0; i < nx; i++) x[i] = (i - xoff + 0.5) * dx + xmin;
    for (int j = 0; j < ny; j++) y[j] = (j - yoff + 0.5) * dy + ymin;
    for (int m = 0; m < nm; m++) { dnxs[m] = h.dnx[m]; dnys[m] = h.dny[m]; }
    for (int m = 0; m < nm; m++)
      for (int s = 0; s < nd; s++) val[m][s] = qd(st[(size_t)m * nd + s], tg[(size_t)m * nd + s]);
  }
  void run(const std::vector<double> &dts, bool resist)
  {
    for (size_t n = 0; n < dts.size(); n++) {
      dt = qd(dts[n], 0.0);
      tim += dt;
      bound(val, nm, stxs, dnxs, stys, dnys);
      ideal(dt);
      if (resist) {
        qd dcmax = setdc();
        if (dcmax > 1e-15) {
          int nc, ncmax = 1 + (int)(2 * (dcmax * dt) / (dr * dr));
          for (nc = 0; nc < ncmax; nc++) {
            bound(val, nm, stxs, dnxs, stys, dnys);
            dsptv(dt / ncmax);
          }
        }
      }
    }
  }
  void write(FILE *f) const
  {
    std::vector<double> buf((size_t)nd);
    for (int part = 0; part < 2; part++)
      for (int m = 0; m < nm; m++) {
        for (int s = 0; s < nd; s++) buf[s] = part ? val[m][s].d : val[m][s].v;
        fwrite(buf.data(), sizeof(double), (size_t)nd, f);
      }
  }
};

int main(int argc, char **argv)
{
  if (argc != 3) die("usage: ref2d_dual <case.bin> <result.bin>");
  FILE *f = fopen(argv[1], "rb");
  if (!f) die("cannot open input");
  DualCaseHeader h;
  if (fread(&h, sizeof(h), 1, f) != 1 || h.magic != 0x44534151) die("bad header");
  if (h.ctw != CTW) die("binary built for the other CTW setting");
  const size_t nd = (size_t)(h.nxm + 8) * (h.nym + 8);
  std::vector<double> dts((size_t)h.nsteps), st(8 * nd), tg(8 * nd);
  if (fread(dts.data(), sizeof(double), dts.size(), f) != dts.size() ||
      fread(st.data(), sizeof(double), st.size(), f) != st.size() ||
      fread(tg.data(), sizeof(double), tg.size(), f) != tg.size())
    die("short input");
  fclose(f);
  qh_xmesh = h.nxm; qh_ymesh = h.nym; qh_zmesh = 1;
  qh_rmn = h.rmn; qh_odr = h.odr; qh_rk = h.rk;
  g_nu_plain = 0.0;
  g_eta_dual = qd(h.eta0, h.deta);
  if (h.nthreads > 0) omp_set_num_threads(h.nthreads);
  DualHarness2D *sim = new DualHarness2D();
  sim->setup(h, st.data(), tg.data());
  sim->run(dts, h.eta0 > 0.0);
  FILE *o = fopen(argv[2], "wb");
  if (!o) die("cannot open output");
  sim->write(o);
  fclose(o);
  delete sim;
  return 0;
}
