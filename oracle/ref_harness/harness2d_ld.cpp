/*
 * Central finite differences of the 2D Kelvin-Helmholtz inversion loss on the reference's
 * 2D stepping code (2D/SERIAL/MRX: mhd2d_class, mhd2d_solve, dmhd2d_class, dmhd2d_solve, and
 * common/*.c) compiled in long double (qas_ld_define.h).  Each evaluation steps the exec_ body
 * -- bound(), ideal(dt), setdc() + the sub-cycled dsptv with uniform eta (DMHD2D::exec_,
 * 2D/SERIAL/MRX/dmhd2d_class.cpp:19-26) -- with the given dt per step, from the state
 *   my = ro vy, en = en_base + ro vy^2 / 2, vy = amp * (dvy + s * eps * d)   (interior cells),
 * and returns L = sum over the interior of (mx/ro - tvx)^2 + (my/ro - tvy)^2 + (bx - tbx)^2 +
 * (by - tby)^2, all in long double.  For each direction d_k it writes
 * (L(+eps d_k) - L(-eps d_k)) / (2 eps), and for eta (L(eta + he) - L(eta - he)) / (2 he).
 * Test infrastructure: the finite-difference reference of the adjoint's gradient.
 *
 * Input : LdCaseHeader, dts[nsteps], base[8*nd], amp[n*n], dvy[n*n], d[ndir][n*n], target[4][n*n]
 * Output: fd[ndir + 1] (double; the last is eta's), loss at the centre point (double)
 */
#include "qas_ld_define.h"
#include "dmhd2d_class.hpp"

// `double` is long double in this part of the file
static double g_eta_ld = 0.0L;

double DMHD2D::setdc()
{
  double dcmax = 0.0, dtmp;
  for (int j = 0; j < ny; j++) {
    for (int i = 0; i < nx; i++) {
      int ss = nx * j + i;
      nu[ss] = 0.0L;
      eta[ss] = g_eta_ld;
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
struct LdCaseHeader {
  int32_t magic;  // "QASL"
  int32_t nxm, nym, rmn, odr, rk, ctw, nsteps, nthreads, ndir;
  double gam, xmin, xmax, ymin, ymax, eta0, eps, eps_eta;
  int32_t dnx[8], dny[8];
};
#pragma pack(pop)

static void die(const char *m)
{
  fprintf(stderr, "ref2d_ld: %s\n", m);
  exit(2);
}

class LdHarness2D : public DMHD2D {
 public:
  void geometry(const LdCaseHeader &h)
  {
    setgam(h.gam);
    xmin = h.xmin; xmax = h.xmax; ymin = h.ymin; ymax = h.ymax;
    dx = (xmax - xmin) / XMESH;
    dy = (ymax - ymin) / YMESH;
    dr = min(dx, dy);
    for (int i = 0; i < nx; i++) x[i] = (i - xoff + 0.5) * dx + xmin;
    for (int j = 0; j < ny; j++) y[j] = (j - yoff + 0.5) * dy + ymin;
    for (int m = 0; m < nm; m++) { dnxs[m] = h.dnx[m]; dnys[m] = h.dny[m]; }
  }
  // initial state of the inversion at dvy + s * d
  void load(const double *base, const double *amp, const double *dvy, const double *d, long double s)
  {
    const int n = XMESH;
    for (int m = 0; m < nm; m++)
      for (int q = 0; q < nd; q++) val[m][q] = base[(size_t)m * nd + q];
    for (int j = 0; j < YMESH; j++)
      for (int i = 0; i < n; i++) {
        const int k = n * j + i, q = nx * (j + yoff) + (i + xoff);
        long double f = (long double)dvy[k];
        if (d) f += s * (long double)d[k];
        const long double vy = (long double)amp[k] * f;
        val[2][q] = val[0][q] * vy;
        val[7][q] = val[7][q] + 0.5L * val[0][q] * vy * vy;
      }
    tim = 0.0L;
  }
  void run(const std::vector<double> &dts)
  {
    for (size_t n = 0; n < dts.size(); n++) {
      dt = dts[n];
      tim += dt;
      bound(val, nm, stxs, dnxs, stys, dnys);
      ideal(dt);
      long double dcmax = setdc();
      if (dcmax > 1e-15) {
        int nc, ncmax = 1 + (int)(2 * (dcmax * dt) / (dr * dr));
        for (nc = 0; nc < ncmax; nc++) {
          bound(val, nm, stxs, dnxs, stys, dnys);
          dsptv(dt / ncmax);
        }
      }
    }
  }
  long double loss(const double *target) const
  {
    const int n = XMESH, nn = XMESH * YMESH;
    long double sum = 0.0L;
    for (int j = 0; j < YMESH; j++)
      for (int i = 0; i < n; i++) {
        const int k = n * j + i, q = nx * (j + yoff) + (i + xoff);
        const long double obs[4] = {val[1][q] / val[0][q], val[2][q] / val[0][q], val[4][q], val[5][q]};
        for (int c = 0; c < 4; c++) {
          const long double e = obs[c] - (long double)target[(size_t)c * nn + k];
          sum += e * e;
        }
      }
    return sum;
  }
};

int main(int argc, char **argv)
{
  if (argc != 3) die("usage: ref2d_ld <case.bin> <result.bin>");
  FILE *f = fopen(argv[1], "rb");
  if (!f) die("cannot open input");
  LdCaseHeader h;
  if (fread(&h, sizeof(h), 1, f) != 1 || h.magic != 0x4c534151) die("bad header");
  if (h.ctw != CTW) die("binary built for the other CTW setting");
  const size_t nd = (size_t)(h.nxm + 8) * (h.nym + 8), nn = (size_t)h.nxm * h.nym;
  std::vector<double> dts((size_t)h.nsteps), base(8 * nd), amp(nn), dvy(nn), dirs((size_t)h.ndir * nn), tgt(4 * nn);
  if (fread(dts.data(), sizeof(double), dts.size(), f) != dts.size() ||
      fread(base.data(), sizeof(double), base.size(), f) != base.size() ||
      fread(amp.data(), sizeof(double), nn, f) != nn || fread(dvy.data(), sizeof(double), nn, f) != nn ||
      fread(dirs.data(), sizeof(double), dirs.size(), f) != dirs.size() ||
      fread(tgt.data(), sizeof(double), tgt.size(), f) != tgt.size())
    die("short input");
  fclose(f);
  qh_xmesh = h.nxm; qh_ymesh = h.nym; qh_zmesh = 1;
  qh_rmn = h.rmn; qh_odr = h.odr; qh_rk = h.rk;
  if (h.nthreads > 0) omp_set_num_threads(h.nthreads);
  LdHarness2D *sim = new LdHarness2D();
  sim->geometry(h);
  const long double eps = h.eps, he = h.eps_eta, eta0 = h.eta0;
  std::vector<double> out((size_t)h.ndir + 2);
  auto eval = [&](const double *d, long double s, long double eta) {
    g_eta_ld = eta;
    sim->load(base.data(), amp.data(), dvy.data(), d, s);
    sim->run(dts);
    return sim->loss(tgt.data());
  };
  for (int k = 0; k < h.ndir; k++) {
    const double *d = dirs.data() + (size_t)k * nn;
    const long double lp = eval(d, eps, eta0), lm = eval(d, -eps, eta0);
    out[k] = (double)((lp - lm) / (2.0L * eps));
    fprintf(stderr, "direction %d: fd %.17g\n", k, out[k]);
  }
  const long double lp = eval(nullptr, 0.0L, eta0 + he), lm = eval(nullptr, 0.0L, eta0 - he);
  out[h.ndir] = (double)((lp - lm) / (2.0L * he));
  out[h.ndir + 1] = (double)eval(nullptr, 0.0L, eta0);
  FILE *o = fopen(argv[2], "wb");
  if (!o) die("cannot open output");
  fwrite(out.data(), sizeof(double), out.size(), o);
  fclose(o);
  delete sim;
  return 0;
}
