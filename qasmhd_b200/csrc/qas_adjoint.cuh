// qas_adjoint.cuh -- hand-written reverse-mode (vector-Jacobian products) of
// the point functions of the step: WCNS4 and the 4th-order linear face
// interpolation, the characteristic reconstruction (mhd_lrstate with the
// mhd_eigen_mi/ae eigenvectors), the Roe flux, the CUCT weight and the
// primitive recovery.  Each VJP recomputes its forward intermediates and then
// sweeps them backwards; results are ADDED into the output adjoints.
// Conventions at non-smooth points: d|x|/dx = sign(x) with sign(0) = 0,
// dmax(0,x)/dx = [x > 0], d sqrt(x)/dx = 0 at x = 0, discrete branches
// (eigen-system choice, zero-preservation flags, positivity fallback, Roe
// renormalisation switches) keep the branch the forward pass took.
// Host+device so tests can check them against finite differences on the CPU.
#pragma once

#include "qas_device.cuh"

namespace qas {

QAS_HD double sgn0(double x) { return x > 0.0 ? 1.0 : (x < 0.0 ? -1.0 : 0.0); }
QAS_HD double dsqrt_safe(double s) { return s > 0.0 ? 0.5 / s : 0.0; }  // d sqrt(x)/dx given s = sqrt(x)

// ---------------------------------------------------------------------------
// 4th-order linear interpolation (cal_flr_4th) VJP
// ---------------------------------------------------------------------------
QAS_HD void lin4_vjp(double gl, double gr, double gf[5])
{
  gf[0] += 0.003125 * (9.0 * gl - 11.0 * gr);
  gf[1] += 0.003125 * (-56.0 * gl + 144.0 * gr);
  gf[2] += 0.003125 * (234.0 * gl + 234.0 * gr);
  gf[3] += 0.003125 * (144.0 * gl - 56.0 * gr);
  gf[4] += 0.003125 * (-11.0 * gl + 9.0 * gr);
}

// ---------------------------------------------------------------------------
// WCNS4 (wcns4_cal_flr, common/common_interp.c:102-150) VJP
// ---------------------------------------------------------------------------
QAS_HD void wcns4_vjp(const double f[5], double gl, double gr, double gf[5])
{
  const double eps = 1e-40;
  const double c1a = f[0] - 4.0 * f[1] + 3.0 * f[2], c2a = f[0] - 2.0 * f[1] + f[2];
  const double c1b = f[1] - f[3], c2b = f[1] - 2.0 * f[2] + f[3];
  const double c1c = f[4] - 4.0 * f[3] + 3.0 * f[2], c2c = f[4] - 2.0 * f[3] + f[2];
  const double s0 = (13. / 12.) * c2a * c2a + 0.25 * c1a * c1a;
  const double s1 = (13. / 12.) * c2b * c2b + 0.25 * c1b * c1b;
  const double s2 = (13. / 12.) * c2c * c2c + 0.25 * c1c * c1c;
  const double S0 = 1.0 / (s0 * s0 + eps), S1 = 1.0 / (s1 * s1 + eps), S2 = 1.0 / (s2 * s2 + eps);
  const double pl0 = 3.0 * f[0] - 10.0 * f[1] + 15.0 * f[2];
  const double pl1 = -f[1] + 6.0 * f[2] + 3.0 * f[3];
  const double pl2 = 3.0 * f[2] + 6.0 * f[3] - f[4];
  const double pr2 = 3.0 * f[4] - 10.0 * f[3] + 15.0 * f[2];
  const double pr1 = -f[3] + 6.0 * f[2] + 3.0 * f[1];
  const double pr0 = 3.0 * f[2] + 6.0 * f[1] - f[0];
  const double a0 = 0.075 * S0, a1 = 0.650 * S1, a2 = 0.275 * S2;
  const double D = 1.0 / (a0 + a1 + a2);
  const double w0 = a0 * D, w1 = a1 * D, w2 = 1.0 - w0 - w1;
  const double b0 = 0.275 * S0, b1 = 0.650 * S1, b2 = 0.075 * S2;
  const double E = 1.0 / (b0 + b1 + b2);
  const double v0 = b0 * E, v1 = b1 * E, v2 = 1.0 - v0 - v1;
  // fl = 0.125 (w0 pl0 + w1 pl1 + w2 pl2), fr = 0.125 (v2 pr2 + v1 pr1 + v0 pr0)
  const double gpl0 = 0.125 * gl * w0, gpl1 = 0.125 * gl * w1, gpl2 = 0.125 * gl * w2;
  const double gw0 = 0.125 * gl * (pl0 - pl2), gw1 = 0.125 * gl * (pl1 - pl2);
  const double gpr0 = 0.125 * gr * v0, gpr1 = 0.125 * gr * v1, gpr2 = 0.125 * gr * v2;
  const double gv0 = 0.125 * gr * (pr0 - pr2), gv1 = 0.125 * gr * (pr1 - pr2);
  const double gD = gw0 * a0 + gw1 * a1;
  const double gsa = -gD * D * D;
  const double ga0 = gw0 * D + gsa, ga1 = gw1 * D + gsa, ga2 = gsa;
  const double gE = gv0 * b0 + gv1 * b1;
  const double gsb = -gE * E * E;
  const double gb0 = gv0 * E + gsb, gb1 = gv1 * E + gsb, gb2 = gsb;
  const double gS0 = 0.075 * ga0 + 0.275 * gb0;
  const double gS1 = 0.650 * ga1 + 0.650 * gb1;
  const double gS2 = 0.275 * ga2 + 0.075 * gb2;
  const double gs0 = -2.0 * s0 * S0 * S0 * gS0, gs1 = -2.0 * s1 * S1 * S1 * gS1, gs2 = -2.0 * s2 * S2 * S2 * gS2;
  const double gc2a = gs0 * (13. / 6.) * c2a, gc1a = gs0 * 0.5 * c1a;
  const double gc2b = gs1 * (13. / 6.) * c2b, gc1b = gs1 * 0.5 * c1b;
  const double gc2c = gs2 * (13. / 6.) * c2c, gc1c = gs2 * 0.5 * c1c;
  gf[0] += gc1a + gc2a + 3.0 * gpl0 - gpr0;
  gf[1] += -4.0 * gc1a - 2.0 * gc2a + gc1b + gc2b - 10.0 * gpl0 - gpl1 + 3.0 * gpr1 + 6.0 * gpr0;
  gf[2] += 3.0 * gc1a + gc2a - 2.0 * gc2b + 3.0 * gc1c + gc2c + 15.0 * gpl0 + 6.0 * gpl1 + 3.0 * gpl2 +
           15.0 * gpr2 + 6.0 * gpr1 + 3.0 * gpr0;
  gf[3] += -gc1b + gc2b - 4.0 * gc1c - 2.0 * gc2c + 3.0 * gpl1 + 6.0 * gpl2 - 10.0 * gpr2 - gpr1;
  gf[4] += gc1c + gc2c - gpl2 + 3.0 * gpr2;
}

// ---------------------------------------------------------------------------
// characteristic reconstruction of one cell (face_states, ODR = 4) VJP.
// q[v][m] primitives (ro,vn,vt,vu,bt,bu,pr) at stencil points, bn centre
// normal field; gvl/gvr adjoints of the two face states -> gq, gbn (added).
// ---------------------------------------------------------------------------
QAS_HD void face_states_vjp(const double q[7][5], double bn, double gam, const double gvl_in[7],
                            const double gvr_in[7], double gq[7][5], double &gbn)
{
  const double ro = q[0][2], vn = q[1][2], vt = q[2][2], vu = q[3][2];
  const double by = q[4][2], bz = q[5][2], pr = q[6][2];
  const bool fast = (ro * (vn * vn + vt * vt + vu * vu) > gam * pr);
  const double iro = 1.0 / ro;
  const double cs2 = gam * pr * iro;
  const double ca2 = bn * bn * iro;
  const double ct2 = (by * by + bz * bz) * iro;
  const double cb2 = cs2 + ca2 + ct2;
  const double disc = cb2 * cb2 - 4.0 * cs2 * ca2;
  const double sq = sqrt(fabs(disc));
  const double cf2 = 0.5 * (cb2 + sq);
  const double sro = sqrt(ro);
  const double isroh = 0.5 / sro;
  const double icf2 = 1.0 / cf2;
  const double byh = 0.5 * by, bzh = 0.5 * bz;
  double cf = 0.0, rcf = 0.0, icf2h = 0.0, ircfh = 0.0;
  if (fast) {
    cf = sqrt(cf2);
    rcf = ro * cf;
    icf2h = 0.5 * icf2;
    ircfh = 0.5 / rcf;
  }
  // characteristic fields and their face values
  double w[7][5], wl[7], wr[7];
  for (int m = 0; m < 5; m++) {
    const double r_ = q[0][m], n_ = q[1][m], t_ = q[2][m], u_ = q[3][m], b_ = q[4][m], c_ = q[5][m], p_ = q[6][m];
    w[0][m] = fast ? (((-rcf) * n_ + by * b_) + bz * c_) + p_ : n_;
    w[1][m] = ((cf2 * r_ - by * b_) - bz * c_) - p_;
    w[2][m] = fast ? (((rcf * n_ + by * b_) + bz * c_) + p_) : ((by * b_ + bz * c_) + p_);
    w[3][m] = sro * t_ + b_;
    w[4][m] = sro * t_ - b_;
    w[5][m] = sro * u_ + c_;
    w[6][m] = sro * u_ - c_;
  }
  for (int k = 0; k < 7; k++) wcns4_lr(w[k], wl[k], wr[k]);
  double vl0, vl6, vr0, vr6;
  if (fast) {
    vl0 = icf2h * wl[0] + icf2 * wl[1] + icf2h * wl[2];
    vr0 = icf2h * wr[0] + icf2 * wr[1] + icf2h * wr[2];
    vl6 = ((((0.5 * wl[0] + 0.5 * wl[2]) - byh * wl[3]) + byh * wl[4]) - bzh * wl[5]) + bzh * wl[6];
    vr6 = ((((0.5 * wr[0] + 0.5 * wr[2]) - byh * wr[3]) + byh * wr[4]) - bzh * wr[5]) + bzh * wr[6];
  } else {
    vl0 = icf2 * wl[1] + icf2 * wl[2];
    vr0 = icf2 * wr[1] + icf2 * wr[2];
    vl6 = (((wl[2] - byh * wl[3]) + byh * wl[4]) - bzh * wl[5]) + bzh * wl[6];
    vr6 = (((wr[2] - byh * wr[3]) + byh * wr[4]) - bzh * wr[5]) + bzh * wr[6];
  }
  const double eps = 1e-12;
  const bool fb_l = (vl0 <= eps || vl6 <= eps), fb_r = (vr0 <= eps || vr6 <= eps);
  bool zero[7] = {false, false, false, false, false, false, false};
  for (int v = 1; v <= 5; v++)
    zero[v] = (q[v][0] == 0.0) && (q[v][1] == 0.0) && (q[v][2] == 0.0) && (q[v][3] == 0.0) && (q[v][4] == 0.0);

  double gvl[7], gvr[7];
  for (int v = 0; v < 7; v++) {
    gvl[v] = gvl_in[v];
    gvr[v] = gvr_in[v];
  }
  double g_ro = 0.0, g_vn = 0.0, g_by = 0.0, g_bz = 0.0, g_pr = 0.0;
  if (fb_l) {
    g_ro += gvl[0];
    g_vn += gvl[1];
    g_pr += gvl[6];
    gvl[0] = gvl[1] = gvl[6] = 0.0;
  }
  if (fb_r) {
    g_ro += gvr[0];
    g_vn += gvr[1];
    g_pr += gvr[6];
    gvr[0] = gvr[1] = gvr[6] = 0.0;
  }
  for (int v = 1; v <= 5; v++)
    if (zero[v]) gvl[v] = gvr[v] = 0.0;

  double gwl[7] = {0, 0, 0, 0, 0, 0, 0}, gwr[7] = {0, 0, 0, 0, 0, 0, 0};
  double g_icf2 = 0.0, g_icf2h = 0.0, g_ircfh = 0.0, g_isroh = 0.0, g_byh = 0.0, g_bzh = 0.0;
  // back-projection of both faces
  for (int side = 0; side < 2; side++) {
    const double *W = side ? wr : wl;
    const double *G = side ? gvr : gvl;
    double *GW = side ? gwr : gwl;
    if (fast) {
      GW[0] += icf2h * G[0];
      GW[1] += icf2 * G[0];
      GW[2] += icf2h * G[0];
      g_icf2h += (W[0] + W[2]) * G[0];
      g_icf2 += W[1] * G[0];
      GW[0] += -ircfh * G[1];
      GW[2] += ircfh * G[1];
      g_ircfh += (W[2] - W[0]) * G[1];
      GW[0] += 0.5 * G[6];
      GW[2] += 0.5 * G[6];
    } else {
      GW[1] += icf2 * G[0];
      GW[2] += icf2 * G[0];
      g_icf2 += (W[1] + W[2]) * G[0];
      GW[0] += G[1];
      GW[2] += G[6];
    }
    GW[3] += -byh * G[6];
    GW[4] += byh * G[6];
    GW[5] += -bzh * G[6];
    GW[6] += bzh * G[6];
    g_byh += (W[4] - W[3]) * G[6];
    g_bzh += (W[6] - W[5]) * G[6];
    GW[3] += isroh * G[2];
    GW[4] += isroh * G[2];
    g_isroh += (W[3] + W[4]) * G[2];
    GW[5] += isroh * G[3];
    GW[6] += isroh * G[3];
    g_isroh += (W[5] + W[6]) * G[3];
    GW[3] += 0.5 * G[4];
    GW[4] += -0.5 * G[4];
    GW[5] += 0.5 * G[5];
    GW[6] += -0.5 * G[5];
  }
  // interpolation and projection of the stencil
  double g_rcf = 0.0, g_cf2 = 0.0, g_sro = 0.0;
  for (int k = 0; k < 7; k++) {
    double gw[5] = {0, 0, 0, 0, 0};
    wcns4_vjp(w[k], gwl[k], gwr[k], gw);
    for (int m = 0; m < 5; m++) {
      const double r_ = q[0][m], n_ = q[1][m], t_ = q[2][m], u_ = q[3][m], b_ = q[4][m], c_ = q[5][m];
      const double g = gw[m];
      switch (k) {
        case 0:
          if (fast) {
            g_rcf += -n_ * g;
            gq[1][m] += -rcf * g;
            g_by += b_ * g;
            gq[4][m] += by * g;
            g_bz += c_ * g;
            gq[5][m] += bz * g;
            gq[6][m] += g;
          } else {
            gq[1][m] += g;
          }
          break;
        case 1:
          g_cf2 += r_ * g;
          gq[0][m] += cf2 * g;
          g_by += -b_ * g;
          gq[4][m] += -by * g;
          g_bz += -c_ * g;
          gq[5][m] += -bz * g;
          gq[6][m] += -g;
          break;
        case 2:
          if (fast) {
            g_rcf += n_ * g;
            gq[1][m] += rcf * g;
          }
          g_by += b_ * g;
          gq[4][m] += by * g;
          g_bz += c_ * g;
          gq[5][m] += bz * g;
          gq[6][m] += g;
          break;
        case 3:
          g_sro += t_ * g;
          gq[2][m] += sro * g;
          gq[4][m] += g;
          break;
        case 4:
          g_sro += t_ * g;
          gq[2][m] += sro * g;
          gq[4][m] += -g;
          break;
        case 5:
          g_sro += u_ * g;
          gq[3][m] += sro * g;
          gq[5][m] += g;
          break;
        default:
          g_sro += u_ * g;
          gq[3][m] += sro * g;
          gq[5][m] += -g;
          break;
      }
    }
  }
  // eigen-system prefix
  double g_cf = 0.0;
  if (fast) {
    g_rcf += -ircfh / rcf * g_ircfh;
    g_icf2 += 0.5 * g_icf2h;
    g_ro += cf * g_rcf;
    g_cf += ro * g_rcf;
    g_cf2 += g_cf * dsqrt_safe(cf);
  }
  g_by += 0.5 * g_byh;
  g_bz += 0.5 * g_bzh;
  g_cf2 += -icf2 * icf2 * g_icf2;
  g_sro += -isroh / sro * g_isroh;
  g_ro += g_sro * dsqrt_safe(sro);
  double g_cb2 = 0.5 * g_cf2;
  const double g_sq = 0.5 * g_cf2;
  const double g_disc = g_sq * dsqrt_safe(sq) * sgn0(disc);
  g_cb2 += 2.0 * cb2 * g_disc;
  double g_cs2 = -4.0 * ca2 * g_disc + g_cb2;
  double g_ca2 = -4.0 * cs2 * g_disc + g_cb2;
  const double g_ct2 = g_cb2;
  g_by += 2.0 * by * iro * g_ct2;
  g_bz += 2.0 * bz * iro * g_ct2;
  double g_iro = (by * by + bz * bz) * g_ct2;
  gbn += 2.0 * bn * iro * g_ca2;
  g_iro += bn * bn * g_ca2;
  g_pr += gam * iro * g_cs2;
  g_iro += gam * pr * g_cs2;
  g_ro += -iro * iro * g_iro;
  gq[0][2] += g_ro;
  gq[1][2] += g_vn;
  gq[4][2] += g_by;
  gq[5][2] += g_bz;
  gq[6][2] += g_pr;
}

// ---------------------------------------------------------------------------
// Roe flux (calc_flux_roe, common/mhd_flux.c:194-433) VJP:
// gF (7) -> gL (7), gR (7), gbn (added)
// ---------------------------------------------------------------------------
QAS_HD void flux_roe_vjp(const double L[7], const double R[7], double bnc, double gamma, const double gF[7],
                         double gL[7], double gR[7], double &gbn)
{
  const double rol = L[0], vnl = L[1], vtl = L[2], vul = L[3], btl = L[4], bul = L[5], prl = L[6];
  const double ror = R[0], vnr = R[1], vtr = R[2], vur = R[3], btr = R[4], bur = R[5], prr = R[6];
  const double FE = QAS_FL_EPS;
  // ---- forward ----
  const double gm1 = gamma - 1.0, gm2 = gamma - 2.0, gm1i = 1.0 / gm1;
  const double roli = 1.0 / rol, rori = 1.0 / ror, rrol = sqrt(rol), rror = sqrt(ror);
  const double rroi = 1.0 / (rrol + rror);
  const double robar = rrol * rror, robari = 1.0 / robar, rrobar = sqrt(robar), rrobai = sqrt(robari);
  const double vnbar = (rrol * vnl + rror * vnr) * rroi;
  const double vtbar = (rrol * vtl + rror * vtr) * rroi;
  const double vubar = (rrol * vul + rror * vur) * rroi;
  const double bn = bnc;
  const double btbar = (rrol * btr + rror * btl) * rroi;
  const double bubar = (rrol * bur + rror * bul) * rroi;
  const double hl = gamma * gm1i * prl * roli + 0.5 * (vnl * vnl + vtl * vtl + vul * vul) +
                    (bn * bn + btl * btl + bul * bul) * roli;
  const double hr = gamma * gm1i * prr * rori + 0.5 * (vnr * vnr + vtr * vtr + vur * vur) +
                    (bn * bn + btr * btr + bur * bur) * rori;
  const double hbar = (rrol * hl + rror * hr) * rroi;
  const double btave = 0.5 * (btl + btr), buave = 0.5 * (bul + bur);
  const double sgn = (bn > 0) ? 1.0 : -1.0;
  const double dbt = btr - btl, dbu = bur - bul;
  const double db2 = 0.5 * gm2 * gm1i * (dbt * dbt + dbu * dbu) * rroi * rroi;
  const double v2h = 0.5 * (vnbar * vnbar + vtbar * vtbar + vubar * vubar);
  const double B2 = bn * bn + btbar * btbar + bubar * bubar;
  const double b2r = B2 * robari;
  const double c2 = gm1 * (hbar - v2h - db2 - b2r);
  const double a2 = gm1 * (hbar - v2h - db2) - gm2 * B2 * robari;
  const double ca2 = bn * bn * robari;
  const double T2 = btbar * btbar + bubar * bubar;
  const double cb2 = T2 * robari;
  const double X = cb2 * (a2 + c2 + ca2) + (c2 - ca2) * (c2 - ca2);
  const double sX = sqrt(X);
  const double cf2 = 0.5 * (a2 + sX);
  const double cs2 = c2 * ca2 / cf2;
  const double cf = sqrt(cf2), cs = sqrt(cs2), ca = sqrt(ca2), c = sqrt(c2), cfi = 1.0 / cf;
  const double sf11 = (T2 - FE > 0) ? 1.0 : 0.0, sf21 = 1.0 - sf11;
  const double sZ = sqrt(T2 + sf21), beti = 1.0 / sZ;
  const double sqh = sqrt(0.5);
  const double bett = sf11 * btbar * beti + sf21 * sqh, betu = sf11 * bubar * beti + sf21 * sqh;
  const double sf12 = (T2 * robari + fabs(ca2 - c2) - FE > 0) ? 1.0 : 0.0, sf22 = 1.0 - sf12;
  const double xca = cf2 - ca2, xcs = cf2 - cs2, xa = cf2 - c2;
  const double cfca = qmax(0.0, xca), cfcs = qmax(0.0, xcs), cfa = qmax(0.0, xa);
  const double sW = sqrt(cfcs + sf22), alpi = 1.0 / sW;
  const double scfca = sqrt(cfca), scfa = sqrt(cfa);
  const double alpf = sf12 * scfca * alpi + sf22, alps = sf12 * scfa * alpi;
  const double xpf = vnbar + cf, xmf = vnbar - cf, xps = vnbar + cs, xms = vnbar - cs, xpa = vnbar + ca,
               xma = vnbar - ca;
  const double evpf = fabs(xpf), evmf = fabs(xmf), evps = fabs(xps), evms = fabs(xms), evpa = fabs(xpa),
               evma = fabs(xma), ev00 = fabs(vnbar);
  const double dltro = ror - rol, dvn = vnr - vnl, dvt = vtr - vtl, dvu = vur - vul;
  const double dltmn = robar * dvn, dltmt = robar * dvt, dltmu = robar * dvu;
  const double t1 = bett * dbt + betu * dbu;
  const double t2 = (prr - prl + (btave * dbt + buave * dbu) + gm2 * (btbar * dbt + bubar * dbu)) * gm1i;
  const double t3 = betu * dbt - bett * dbu;
  const double s1 = dltmn, s2 = bett * dltmt + betu * dltmu, s3 = betu * dltmt - bett * dltmu;
  const double k2 = gm2 * gm1i;
  const double p11 = alps * cf * rrobai, p12 = -alpf * c2 * cfi * rrobai, p21 = alpf * (cf2 - c2 * k2),
               p22 = alps * (cs2 - c2 * k2);
  const double q11 = alpf * cf, q12 = alps * cs, q21 = -alps * ca * sgn, q22 = alpf * c * sgn;
  const double dp = p11 * p22 - p12 * p21, detpi = 1.0 / dp;
  const double dq = q11 * q22 - q12 * q21, detqi = 1.0 / dq;
  const double A = (p22 * t1 - p12 * t2) * detpi, B = (q22 * s1 - q12 * s2) * detqi;
  const double C = (-p21 * t1 + p11 * t2) * detpi, D = (-q21 * s1 + q11 * s2) * detqi;
  const double wvpf = 0.5 * (A + B), wvmf = 0.5 * (A - B), wvps = 0.5 * (C + D), wvms = 0.5 * (C - D);
  const double wvpa = 0.5 * (rrobar * t3 - sgn * s3), wvma = 0.5 * (rrobar * t3 + sgn * s3);
  const double wv00 = dltro - alpf * (wvpf + wvmf) - alps * (wvps + wvms);
  const double apf = evpf * wvpf, amf = evmf * wvmf, aps = evps * wvps, ams = evms * wvms, apa = evpa * wvpa,
               ama = evma * wvma, a00 = ev00 * wv00;
  const double K = bett * vtbar + betu * vubar;
  const double cab = alps * ca * K * sgn, cfb = alpf * c * K * sgn;
  const double P1 = v2h + db2 + cf * vnbar + cf2 * gm1i + (cf2 - c2) * k2;
  const double M1 = v2h + db2 - cf * vnbar + cf2 * gm1i + (cf2 - c2) * k2;
  const double P2 = v2h + db2 + cs * vnbar + cs2 * gm1i + (cs2 - c2) * k2;
  const double M2 = v2h + db2 - cs * vnbar + cs2 * gm1i + (cs2 - c2) * k2;
  const double rvpfmn = alpf * (vnbar + cf), rvmfmn = alpf * (vnbar - cf);
  const double rvpfmt = alpf * vtbar - alps * bett * ca * sgn, rvmfmt = alpf * vtbar + alps * bett * ca * sgn;
  const double rvpfmu = alpf * vubar - alps * betu * ca * sgn, rvmfmu = alpf * vubar + alps * betu * ca * sgn;
  const double rvpfbt = alps * bett * cf * rrobai, rvpfbu = alps * betu * cf * rrobai;
  const double rvpfen = alpf * P1 - cab, rvmfen = alpf * M1 + cab;
  const double rvpsmn = alps * (vnbar + cs), rvmsmn = alps * (vnbar - cs);
  const double rvpsmt = alps * vtbar + c * sgn * alpf * bett, rvmsmt = alps * vtbar - c * sgn * alpf * bett;
  const double rvpsmu = alps * vubar + c * sgn * alpf * betu, rvmsmu = alps * vubar - c * sgn * alpf * betu;
  const double rvpsbt = -rrobai * c2 * alpf * bett * cfi, rvpsbu = -rrobai * c2 * alpf * betu * cfi;
  const double rvpsen = alps * P2 + cfb, rvmsen = alps * M2 - cfb;
  const double rvpamt = -sgn * betu, rvpamu = sgn * bett, rvpabt = rrobai * betu, rvpabu = -rrobai * bett;
  const double rvpaen = -(betu * vtbar - bett * vubar) * sgn;
  const double rv00en = v2h + db2;
  // ---- reverse ----
  double h[7];
  for (int k = 0; k < 7; k++) h[k] = 0.5 * gF[k];
  // physical fluxes: each side gets h
  double grol = 0, gvnl = 0, gvtl = 0, gvul = 0, gbtl = 0, gbul = 0, gprl = 0, ghl = 0;
  double gror = 0, gvnr = 0, gvtr = 0, gvur = 0, gbtr = 0, gbur = 0, gprr = 0, ghr = 0;
  double g_bn = 0;
  {
    // left
    grol += vnl * h[0];
    gvnl += rol * h[0];
    grol += vnl * vnl * h[1];
    gvnl += 2.0 * rol * vnl * h[1];
    gprl += h[1];
    g_bn += -bn * h[1];
    gbtl += btl * h[1];
    gbul += bul * h[1];
    grol += vnl * vtl * h[2];
    gvnl += rol * vtl * h[2];
    gvtl += rol * vnl * h[2];
    g_bn += -btl * h[2];
    gbtl += -bn * h[2];
    grol += vnl * vul * h[3];
    gvnl += rol * vul * h[3];
    gvul += rol * vnl * h[3];
    g_bn += -bul * h[3];
    gbul += -bn * h[3];
    gvnl += btl * h[4];
    gbtl += vnl * h[4];
    gvtl += -bn * h[4];
    g_bn += -vtl * h[4];
    gvnl += bul * h[5];
    gbul += vnl * h[5];
    gvul += -bn * h[5];
    g_bn += -vul * h[5];
    grol += vnl * hl * h[6];
    gvnl += rol * hl * h[6] - bn * bn * h[6];
    ghl += rol * vnl * h[6];
    g_bn += -(bn * vnl + btl * vtl + bul * vul) * h[6] - bn * vnl * h[6];
    gbtl += -bn * vtl * h[6];
    gvtl += -bn * btl * h[6];
    gbul += -bn * vul * h[6];
    gvul += -bn * bul * h[6];
    // right
    gror += vnr * h[0];
    gvnr += ror * h[0];
    gror += vnr * vnr * h[1];
    gvnr += 2.0 * ror * vnr * h[1];
    gprr += h[1];
    g_bn += -bn * h[1];
    gbtr += btr * h[1];
    gbur += bur * h[1];
    gror += vnr * vtr * h[2];
    gvnr += ror * vtr * h[2];
    gvtr += ror * vnr * h[2];
    g_bn += -btr * h[2];
    gbtr += -bn * h[2];
    gror += vnr * vur * h[3];
    gvnr += ror * vur * h[3];
    gvur += ror * vnr * h[3];
    g_bn += -bur * h[3];
    gbur += -bn * h[3];
    gvnr += btr * h[4];
    gbtr += vnr * h[4];
    gvtr += -bn * h[4];
    g_bn += -vtr * h[4];
    gvnr += bur * h[5];
    gbur += vnr * h[5];
    gvur += -bn * h[5];
    g_bn += -vur * h[5];
    gror += vnr * hr * h[6];
    gvnr += ror * hr * h[6] - bn * bn * h[6];
    ghr += ror * vnr * h[6];
    g_bn += -(bn * vnr + btr * vtr + bur * vur) * h[6] - bn * vnr * h[6];
    gbtr += -bn * vtr * h[6];
    gvtr += -bn * btr * h[6];
    gbur += -bn * vur * h[6];
    gvur += -bn * bur * h[6];
  }
  // wave amplitudes a_j
  const double g_apf = -(h[0] * alpf + h[1] * rvpfmn + h[2] * rvpfmt + h[3] * rvpfmu + h[4] * rvpfbt + h[5] * rvpfbu +
                         h[6] * rvpfen);
  const double g_amf = -(h[0] * alpf + h[1] * rvmfmn + h[2] * rvmfmt + h[3] * rvmfmu + h[4] * rvpfbt + h[5] * rvpfbu +
                         h[6] * rvmfen);
  const double g_aps = -(h[0] * alps + h[1] * rvpsmn + h[2] * rvpsmt + h[3] * rvpsmu + h[4] * rvpsbt + h[5] * rvpsbu +
                         h[6] * rvpsen);
  const double g_ams = -(h[0] * alps + h[1] * rvmsmn + h[2] * rvmsmt + h[3] * rvmsmu + h[4] * rvpsbt + h[5] * rvpsbu +
                         h[6] * rvmsen);
  const double g_apa = -(h[2] * rvpamt + h[3] * rvpamu + h[4] * rvpabt + h[5] * rvpabu + h[6] * rvpaen);
  const double g_ama = -(-h[2] * rvpamt - h[3] * rvpamu + h[4] * rvpabt + h[5] * rvpabu - h[6] * rvpaen);
  const double g_a00 = -(h[0] + h[1] * vnbar + h[2] * vtbar + h[3] * vubar + h[6] * rv00en);
  // eigenvector entries
  double g_alpf = -h[0] * (apf + amf), g_alps = -h[0] * (aps + ams);
  double g_vnbar = -h[1] * a00, g_vtbar = -h[2] * a00, g_vubar = -h[3] * a00;
  const double g_rvpfmn = -h[1] * apf, g_rvmfmn = -h[1] * amf, g_rvpsmn = -h[1] * aps, g_rvmsmn = -h[1] * ams;
  const double g_rvpfmt = -h[2] * apf, g_rvmfmt = -h[2] * amf, g_rvpsmt = -h[2] * aps, g_rvmsmt = -h[2] * ams;
  const double g_rvpamt = -h[2] * (apa - ama);
  const double g_rvpfmu = -h[3] * apf, g_rvmfmu = -h[3] * amf, g_rvpsmu = -h[3] * aps, g_rvmsmu = -h[3] * ams;
  const double g_rvpamu = -h[3] * (apa - ama);
  const double g_rvpfbt = -h[4] * (apf + amf), g_rvpsbt = -h[4] * (aps + ams), g_rvpabt = -h[4] * (apa + ama);
  const double g_rvpfbu = -h[5] * (apf + amf), g_rvpsbu = -h[5] * (aps + ams), g_rvpabu = -h[5] * (apa + ama);
  const double g_rvpfen = -h[6] * apf, g_rvmfen = -h[6] * amf, g_rvpsen = -h[6] * aps, g_rvmsen = -h[6] * ams;
  const double g_rvpaen = -h[6] * (apa - ama), g_rv00en = -h[6] * a00;
  double g_cf = 0, g_cs = 0, g_ca = 0, g_c = 0, g_c2 = 0, g_cf2 = 0, g_cs2 = 0, g_cfi = 0, g_rrobai = 0;
  double g_bett = 0, g_betu = 0, g_v2h = 0, g_db2 = 0, g_K = 0;
  // rv*mn
  g_alpf += (vnbar + cf) * g_rvpfmn + (vnbar - cf) * g_rvmfmn;
  g_vnbar += alpf * (g_rvpfmn + g_rvmfmn);
  g_cf += alpf * (g_rvpfmn - g_rvmfmn);
  g_alps += (vnbar + cs) * g_rvpsmn + (vnbar - cs) * g_rvmsmn;
  g_vnbar += alps * (g_rvpsmn + g_rvmsmn);
  g_cs += alps * (g_rvpsmn - g_rvmsmn);
  // rv*mt, rv*mu (fast, slow)
  g_alpf += vtbar * (g_rvpfmt + g_rvmfmt) + vubar * (g_rvpfmu + g_rvmfmu);
  g_vtbar += alpf * (g_rvpfmt + g_rvmfmt);
  g_vubar += alpf * (g_rvpfmu + g_rvmfmu);
  {
    const double dt_ = g_rvmfmt - g_rvpfmt, du_ = g_rvmfmu - g_rvpfmu;  // coefficient of alps*bet*ca*sgn
    g_alps += (bett * dt_ + betu * du_) * ca * sgn;
    g_bett += alps * ca * sgn * dt_;
    g_betu += alps * ca * sgn * du_;
    g_ca += alps * sgn * (bett * dt_ + betu * du_);
  }
  g_alps += vtbar * (g_rvpsmt + g_rvmsmt) + vubar * (g_rvpsmu + g_rvmsmu);
  g_vtbar += alps * (g_rvpsmt + g_rvmsmt);
  g_vubar += alps * (g_rvpsmu + g_rvmsmu);
  {
    const double dt_ = g_rvpsmt - g_rvmsmt, du_ = g_rvpsmu - g_rvmsmu;  // coefficient of c*sgn*alpf*bet
    g_c += sgn * alpf * (bett * dt_ + betu * du_);
    g_alpf += c * sgn * (bett * dt_ + betu * du_);
    g_bett += c * sgn * alpf * dt_;
    g_betu += c * sgn * alpf * du_;
  }
  // rv*bt, rv*bu
  g_alps += (bett * g_rvpfbt + betu * g_rvpfbu) * cf * rrobai;
  g_bett += alps * cf * rrobai * g_rvpfbt;
  g_betu += alps * cf * rrobai * g_rvpfbu;
  g_cf += alps * rrobai * (bett * g_rvpfbt + betu * g_rvpfbu);
  g_rrobai += alps * cf * (bett * g_rvpfbt + betu * g_rvpfbu);
  {
    const double e_ = bett * g_rvpsbt + betu * g_rvpsbu;
    g_rrobai += -c2 * alpf * cfi * e_;
    g_c2 += -rrobai * alpf * cfi * e_;
    g_alpf += -rrobai * c2 * cfi * e_;
    g_cfi += -rrobai * c2 * alpf * e_;
    g_bett += -rrobai * c2 * alpf * cfi * g_rvpsbt;
    g_betu += -rrobai * c2 * alpf * cfi * g_rvpsbu;
  }
  // rv*en
  g_alpf += P1 * g_rvpfen + M1 * g_rvmfen;
  {
    const double gP = alpf * g_rvpfen, gM = alpf * g_rvmfen;
    g_v2h += gP + gM;
    g_db2 += gP + gM;
    g_cf += vnbar * (gP - gM);
    g_vnbar += cf * (gP - gM);
    g_cf2 += (gm1i + k2) * (gP + gM);
    g_c2 += -k2 * (gP + gM);
  }
  {
    const double g_cab = -g_rvpfen + g_rvmfen;
    g_alps += ca * K * sgn * g_cab;
    g_ca += alps * K * sgn * g_cab;
    g_K += alps * ca * sgn * g_cab;
  }
  g_alps += P2 * g_rvpsen + M2 * g_rvmsen;
  {
    const double gP = alps * g_rvpsen, gM = alps * g_rvmsen;
    g_v2h += gP + gM;
    g_db2 += gP + gM;
    g_cs += vnbar * (gP - gM);
    g_vnbar += cs * (gP - gM);
    g_cs2 += (gm1i + k2) * (gP + gM);
    g_c2 += -k2 * (gP + gM);
  }
  {
    const double g_cfb = g_rvpsen - g_rvmsen;
    g_alpf += c * K * sgn * g_cfb;
    g_c += alpf * K * sgn * g_cfb;
    g_K += alpf * c * sgn * g_cfb;
  }
  // Alfven and entropy eigenvectors
  g_betu += -sgn * g_rvpamt;
  g_bett += sgn * g_rvpamu;
  g_rrobai += betu * g_rvpabt - bett * g_rvpabu;
  g_betu += rrobai * g_rvpabt;
  g_bett += -rrobai * g_rvpabu;
  g_betu += -vtbar * sgn * g_rvpaen;
  g_vtbar += -betu * sgn * g_rvpaen;
  g_bett += vubar * sgn * g_rvpaen;
  g_vubar += bett * sgn * g_rvpaen;
  g_v2h += g_rv00en;
  g_db2 += g_rv00en;
  g_bett += vtbar * g_K;
  g_vtbar += bett * g_K;
  g_betu += vubar * g_K;
  g_vubar += betu * g_K;
  // amplitudes a = ev * wv
  double g_wvpf = evpf * g_apf, g_wvmf = evmf * g_amf, g_wvps = evps * g_aps, g_wvms = evms * g_ams;
  const double g_wvpa = evpa * g_apa, g_wvma = evma * g_ama, g_wv00 = ev00 * g_a00;
  {
    const double gx_pf = sgn0(xpf) * wvpf * g_apf, gx_mf = sgn0(xmf) * wvmf * g_amf;
    const double gx_ps = sgn0(xps) * wvps * g_aps, gx_ms = sgn0(xms) * wvms * g_ams;
    const double gx_pa = sgn0(xpa) * wvpa * g_apa, gx_ma = sgn0(xma) * wvma * g_ama;
    g_vnbar += gx_pf + gx_mf + gx_ps + gx_ms + gx_pa + gx_ma + sgn0(vnbar) * wv00 * g_a00;
    g_cf += gx_pf - gx_mf;
    g_cs += gx_ps - gx_ms;
    g_ca += gx_pa - gx_ma;
  }
  // wv00 = dltro - alpf (wvpf + wvmf) - alps (wvps + wvms)
  double g_dltro = g_wv00;
  g_alpf += -(wvpf + wvmf) * g_wv00;
  g_wvpf += -alpf * g_wv00;
  g_wvmf += -alpf * g_wv00;
  g_alps += -(wvps + wvms) * g_wv00;
  g_wvps += -alps * g_wv00;
  g_wvms += -alps * g_wv00;
  double g_rrobar = 0.5 * t3 * (g_wvpa + g_wvma);
  double g_t3 = 0.5 * rrobar * (g_wvpa + g_wvma);
  double g_s3 = 0.5 * sgn * (g_wvma - g_wvpa);
  const double g_A = 0.5 * (g_wvpf + g_wvmf), g_B = 0.5 * (g_wvpf - g_wvmf);
  const double g_C = 0.5 * (g_wvps + g_wvms), g_D = 0.5 * (g_wvps - g_wvms);
  double g_p11 = 0, g_p12 = 0, g_p21 = 0, g_p22 = 0, g_q11 = 0, g_q12 = 0, g_q21 = 0, g_q22 = 0;
  double g_t1 = 0, g_t2 = 0, g_s1 = 0, g_s2 = 0;
  g_p22 += t1 * detpi * g_A;
  g_t1 += p22 * detpi * g_A;
  g_p12 += -t2 * detpi * g_A;
  g_t2 += -p12 * detpi * g_A;
  g_p21 += -t1 * detpi * g_C;
  g_t1 += -p21 * detpi * g_C;
  g_p11 += t2 * detpi * g_C;
  g_t2 += p11 * detpi * g_C;
  const double g_detpi = (p22 * t1 - p12 * t2) * g_A + (-p21 * t1 + p11 * t2) * g_C;
  g_q22 += s1 * detqi * g_B;
  g_s1 += q22 * detqi * g_B;
  g_q12 += -s2 * detqi * g_B;
  g_s2 += -q12 * detqi * g_B;
  g_q21 += -s1 * detqi * g_D;
  g_s1 += -q21 * detqi * g_D;
  g_q11 += s2 * detqi * g_D;
  g_s2 += q11 * detqi * g_D;
  const double g_detqi = (q22 * s1 - q12 * s2) * g_B + (-q21 * s1 + q11 * s2) * g_D;
  const double g_dp = -detpi * detpi * g_detpi, g_dq = -detqi * detqi * g_detqi;
  g_p11 += p22 * g_dp;
  g_p22 += p11 * g_dp;
  g_p12 += -p21 * g_dp;
  g_p21 += -p12 * g_dp;
  g_q11 += q22 * g_dq;
  g_q22 += q11 * g_dq;
  g_q12 += -q21 * g_dq;
  g_q21 += -q12 * g_dq;
  g_alpf += cf * g_q11 + c * sgn * g_q22;
  g_cf += alpf * g_q11;
  g_c += alpf * sgn * g_q22;
  g_alps += cs * g_q12 - ca * sgn * g_q21;
  g_cs += alps * g_q12;
  g_ca += -alps * sgn * g_q21;
  g_alps += cf * rrobai * g_p11 + (cs2 - c2 * k2) * g_p22;
  g_cf += alps * rrobai * g_p11;
  g_rrobai += alps * cf * g_p11 - alpf * c2 * cfi * g_p12;
  g_alpf += -c2 * cfi * rrobai * g_p12 + (cf2 - c2 * k2) * g_p21;
  g_c2 += -alpf * cfi * rrobai * g_p12 - alpf * k2 * g_p21 - alps * k2 * g_p22;
  g_cfi += -alpf * c2 * rrobai * g_p12;
  g_cf2 += alpf * g_p21;
  g_cs2 += alps * g_p22;
  // t's and s's
  double g_dbt = 0, g_dbu = 0, g_btave = 0, g_buave = 0, g_btbar = 0, g_bubar = 0;
  double g_dltmn = g_s1, g_dltmt = 0, g_dltmu = 0;
  g_bett += dltmt * g_s2 - dltmu * g_s3 + dbt * g_t1 - dbu * g_t3;
  g_betu += dltmu * g_s2 + dltmt * g_s3 + dbu * g_t1 + dbt * g_t3;
  g_dltmt += bett * g_s2 + betu * g_s3;
  g_dltmu += betu * g_s2 - bett * g_s3;
  g_dbt += bett * g_t1 + betu * g_t3;
  g_dbu += betu * g_t1 - bett * g_t3;
  {
    const double gg = gm1i * g_t2;
    gprr += gg;
    gprl += -gg;
    g_btave += dbt * gg;
    g_dbt += btave * gg + gm2 * btbar * gg;
    g_buave += dbu * gg;
    g_dbu += buave * gg + gm2 * bubar * gg;
    g_btbar += gm2 * dbt * gg;
    g_bubar += gm2 * dbu * gg;
  }
  double g_robar = dvn * g_dltmn + dvt * g_dltmt + dvu * g_dltmu;
  gvnr += robar * g_dltmn;
  gvnl += -robar * g_dltmn;
  gvtr += robar * g_dltmt;
  gvtl += -robar * g_dltmt;
  gvur += robar * g_dltmu;
  gvul += -robar * g_dltmu;
  gror += g_dltro;
  grol += -g_dltro;
  // alpf, alps
  const double g_scfca = sf12 * alpi * g_alpf, g_scfa = sf12 * alpi * g_alps;
  const double g_alpi = sf12 * scfca * g_alpf + sf12 * scfa * g_alps;
  const double g_cfca = g_scfca * dsqrt_safe(scfca), g_cfa = g_scfa * dsqrt_safe(scfa);
  const double g_cfcs = -alpi * alpi * g_alpi * dsqrt_safe(sW);
  double g_ca2 = 0;
  if (xca > 0) {
    g_cf2 += g_cfca;
    g_ca2 += -g_cfca;
  }
  if (xcs > 0) {
    g_cf2 += g_cfcs;
    g_cs2 += -g_cfcs;
  }
  if (xa > 0) {
    g_cf2 += g_cfa;
    g_c2 += -g_cfa;
  }
  // bett, betu
  g_btbar += sf11 * beti * g_bett;
  g_bubar += sf11 * beti * g_betu;
  const double g_beti = sf11 * (btbar * g_bett + bubar * g_betu);
  double g_T2 = -beti * beti * g_beti * dsqrt_safe(sZ);
  // cfi, c, ca, cs, cf
  g_cf += -cfi * cfi * g_cfi;
  g_c2 += g_c * dsqrt_safe(c);
  g_ca2 += g_ca * dsqrt_safe(ca);
  g_cs2 += g_cs * dsqrt_safe(cs);
  g_cf2 += g_cf * dsqrt_safe(cf);
  // cs2 = c2 ca2 / cf2
  g_c2 += ca2 / cf2 * g_cs2;
  g_ca2 += c2 / cf2 * g_cs2;
  g_cf2 += -cs2 / cf2 * g_cs2;
  // cf2 = 0.5 (a2 + sX)
  double g_a2 = 0.5 * g_cf2;
  const double g_X = 0.5 * g_cf2 * dsqrt_safe(sX);
  double g_cb2 = (a2 + c2 + ca2) * g_X;
  g_a2 += cb2 * g_X;
  g_c2 += cb2 * g_X + 2.0 * (c2 - ca2) * g_X;
  g_ca2 += cb2 * g_X - 2.0 * (c2 - ca2) * g_X;
  g_T2 += robari * g_cb2;
  double g_robari = T2 * g_cb2;
  g_btbar += 2.0 * btbar * g_T2;
  g_bubar += 2.0 * bubar * g_T2;
  g_bn += 2.0 * bn * robari * g_ca2;
  g_robari += bn * bn * g_ca2;
  // a2 and c2
  double g_hbar = gm1 * g_a2 + gm1 * g_c2;
  g_v2h += -gm1 * g_a2 - gm1 * g_c2;
  g_db2 += -gm1 * g_a2 - gm1 * g_c2;
  double g_B2 = -gm2 * robari * g_a2;
  g_robari += -gm2 * B2 * g_a2;
  const double g_b2r = -gm1 * g_c2;
  g_B2 += robari * g_b2r;
  g_robari += B2 * g_b2r;
  g_bn += 2.0 * bn * g_B2;
  g_btbar += 2.0 * btbar * g_B2;
  g_bubar += 2.0 * bubar * g_B2;
  g_vnbar += vnbar * g_v2h;
  g_vtbar += vtbar * g_v2h;
  g_vubar += vubar * g_v2h;
  // db2
  double g_rroi = gm2 * gm1i * (dbt * dbt + dbu * dbu) * rroi * g_db2;
  g_dbt += gm2 * gm1i * dbt * rroi * rroi * g_db2;
  g_dbu += gm2 * gm1i * dbu * rroi * rroi * g_db2;
  gbtr += g_dbt + 0.5 * g_btave;
  gbtl += -g_dbt + 0.5 * g_btave;
  gbur += g_dbu + 0.5 * g_buave;
  gbul += -g_dbu + 0.5 * g_buave;
  // hbar = (rrol hl + rror hr) rroi
  double g_rrol = hl * rroi * g_hbar, g_rror = hr * rroi * g_hbar;
  ghl += rrol * rroi * g_hbar;
  ghr += rror * rroi * g_hbar;
  g_rroi += (rrol * hl + rror * hr) * g_hbar;
  double g_roli = (gamma * gm1i * prl + bn * bn + btl * btl + bul * bul) * ghl;
  gprl += gamma * gm1i * roli * ghl;
  gvnl += vnl * ghl;
  gvtl += vtl * ghl;
  gvul += vul * ghl;
  g_bn += 2.0 * bn * roli * ghl + 2.0 * bn * rori * ghr;
  gbtl += 2.0 * btl * roli * ghl;
  gbul += 2.0 * bul * roli * ghl;
  double g_rori = (gamma * gm1i * prr + bn * bn + btr * btr + bur * bur) * ghr;
  gprr += gamma * gm1i * rori * ghr;
  gvnr += vnr * ghr;
  gvtr += vtr * ghr;
  gvur += vur * ghr;
  gbtr += 2.0 * btr * rori * ghr;
  gbur += 2.0 * bur * rori * ghr;
  // Roe averages
  g_rrol += btr * rroi * g_btbar + bur * rroi * g_bubar + vnl * rroi * g_vnbar + vtl * rroi * g_vtbar +
            vul * rroi * g_vubar;
  g_rror += btl * rroi * g_btbar + bul * rroi * g_bubar + vnr * rroi * g_vnbar + vtr * rroi * g_vtbar +
            vur * rroi * g_vubar;
  gbtr += rrol * rroi * g_btbar;
  gbtl += rror * rroi * g_btbar;
  gbur += rrol * rroi * g_bubar;
  gbul += rror * rroi * g_bubar;
  gvnl += rrol * rroi * g_vnbar;
  gvnr += rror * rroi * g_vnbar;
  gvtl += rrol * rroi * g_vtbar;
  gvtr += rror * rroi * g_vtbar;
  gvul += rrol * rroi * g_vubar;
  gvur += rror * rroi * g_vubar;
  g_rroi += (rrol * btr + rror * btl) * g_btbar + (rrol * bur + rror * bul) * g_bubar +
            (rrol * vnl + rror * vnr) * g_vnbar + (rrol * vtl + rror * vtr) * g_vtbar +
            (rrol * vul + rror * vur) * g_vubar;
  g_robari += g_rrobai * dsqrt_safe(rrobai);
  g_robar += g_rrobar * dsqrt_safe(rrobar);
  g_robar += -robari * robari * g_robari;
  g_rrol += rror * g_robar;
  g_rror += rrol * g_robar;
  const double g_sum = -rroi * rroi * g_rroi;
  g_rrol += g_sum;
  g_rror += g_sum;
  grol += g_rrol * dsqrt_safe(rrol) - roli * roli * g_roli;
  gror += g_rror * dsqrt_safe(rror) - rori * rori * g_rori;
  gL[0] += grol; gL[1] += gvnl; gL[2] += gvtl; gL[3] += gvul; gL[4] += gbtl; gL[5] += gbul; gL[6] += gprl;
  gR[0] += gror; gR[1] += gvnr; gR[2] += gvtr; gR[3] += gvur; gR[4] += gbtr; gR[5] += gbur; gR[6] += gprr;
  gbn += g_bn;
}

// ---------------------------------------------------------------------------
// CUCT weight VJP (mhd_cuct_weight): g -> the 16 inputs in cuct_weight order
// (r0..r3, va0..va3, vb0..vb3, ba1, ba3, bb2, bb3), added into gi[16]
// ---------------------------------------------------------------------------
QAS_HD void cuct_weight_vjp(const double in[16], double g, double gi[16])
{
  const double eps = 1e-12;
  const double rsum = 0.25 * (in[0] + in[1] + in[2] + in[3]);
  const double sr = sqrt(rsum), roc = 1.0 / sr;
  const double vac0 = 0.25 * (in[4] + in[5] + in[6] + in[7]);
  const double vbc0 = 0.25 * (in[8] + in[9] + in[10] + in[11]);
  const double bac = 0.5 * (in[12] + in[13]), bbc = 0.5 * (in[14] + in[15]);
  const double ba_r = bac * roc, bb_r = bbc * roc;
  const double vac = fabs(vac0) + fabs(ba_r), vbc = fabs(vbc0) + fabs(bb_r);
  const double den = vac + vbc + eps;
  const double w = (vac + 0.5 * eps) / den;
  // w = (vac + e/2) / den
  const double g_vac = g / den - g * w / den;
  const double g_vbc = -g * w / den;
  const double g_vac0 = sgn0(vac0) * g_vac, g_bar = sgn0(ba_r) * g_vac;
  const double g_vbc0 = sgn0(vbc0) * g_vbc, g_bbr = sgn0(bb_r) * g_vbc;
  const double g_bac = roc * g_bar, g_bbc = roc * g_bbr;
  const double g_roc = bac * g_bar + bbc * g_bbr;
  const double g_rsum = -roc * roc * g_roc * dsqrt_safe(sr);
  for (int q = 0; q < 4; q++) {
    gi[q] += 0.25 * g_rsum;
    gi[4 + q] += 0.25 * g_vac0;
    gi[8 + q] += 0.25 * g_vbc0;
  }
  gi[12] += 0.5 * g_bac;
  gi[13] += 0.5 * g_bac;
  gi[14] += 0.5 * g_bbc;
  gi[15] += 0.5 * g_bbc;
}

}  // namespace qas
