/*
 * Known-answer harness for the reference's point functions (common/*.c).
 * Reads  : int32 func, int32 ncase, int32 nin, int32 nout, then ncase*nin doubles.
 * Writes : ncase*nout doubles.
 * func ids:
 *   0..3   riemann[RMN] (common/mhd_class.hpp:102-105: Roe, HLLD, LHLLD, MLAU),
 *          in  = rol,vnl,vtl,vul,btl,bul,prl, ror,vnr,vtr,vur,btr,bur,prr, bnc, gamma, dv0, dv1
 *          out = fro,fmn,fmt,fmu,fbt,fbu,fen
 *   10..13 cal_flr_1st..4th, 14 muscl_mm, 15 wcns3, 16 wcns4, 17 muscl_mc,
 *          18 muscl_vl, 19 muscl_kr (common/common_interp.c): in = f[-2..2], out = fl, fr
 *   20..23 mhd_lrstate with interpol[ODR-1], ODR=1..4 (common/mhd_func.c:108-161):
 *          in = 7 primitives x 5 stencil points (ro,vx,vy,vz,by,bz,pr), bx, gamma
 *          out = vl[0..6], vr[0..6]
 *   30     mhd_cuct_weight on a 2x2 patch (common/mhd_func.c:56-76):
 *          in = ro[4],vx[4],vy[4],bx[4],by[4] (index = 2*j+i), out = weight at corner (1,1)
 *   31     mhd_ieos,  in = ro,vx,vy,vz,bx,by,bz,en,gamma
 *   32     mhd_energy, in = ro,vx,vy,vz,bx,by,bz,pr,gamma
 * Test infrastructure only.
 */
#include <stdio.h>
#include <stdlib.h>
#include <stdint.h>
#include <vector>
#include "mhd_common.h"

typedef void (*flux_fn)(double, double, double, double, double, double, double,
                        double, double, double, double, double, double, double,
                        double, double, const double *,
                        double *, double *, double *, double *, double *, double *, double *);
typedef void (*lr_fn)(const double *, double *, double *);

int main(int argc, char **argv)
{
  if (argc != 3) { fprintf(stderr, "usage: ref_kat <in> <out>\n"); return 2; }
  FILE *f = fopen(argv[1], "rb");
  if (!f) return 2;
  int32_t hdr[4];
  if (fread(hdr, sizeof(int32_t), 4, f) != 4) return 2;
  int func = hdr[0], ncase = hdr[1], nin = hdr[2], nout = hdr[3];
  std::vector<double> in((size_t)ncase * nin), out((size_t)ncase * nout, 0.0);
  if (fread(in.data(), sizeof(double), in.size(), f) != in.size()) return 2;
  fclose(f);

  flux_fn fluxes[4] = {calc_flux_roe, calc_flux_hlld, calc_flux_lhlld, calc_flux_mlau};
  lr_fn lrs[10] = {cal_flr_1st, cal_flr_2nd, cal_flr_3rd, cal_flr_4th, muscl_mm_cal_flr,
                   wcns3_cal_flr, wcns4_cal_flr, muscl_mc_cal_flr, muscl_vl_cal_flr, muscl_kr_cal_flr};
  lr_fn interpol[4] = {cal_flr_1st, muscl_mm_cal_flr, wcns3_cal_flr, wcns4_cal_flr};

  for (int c = 0; c < ncase; c++) {
    const double *a = &in[(size_t)c * nin];
    double *o = &out[(size_t)c * nout];
    if (func >= 0 && func <= 3) {
      fluxes[func](a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8], a[9], a[10], a[11], a[12], a[13],
                   a[14], a[15], &a[16], &o[0], &o[1], &o[2], &o[3], &o[4], &o[5], &o[6]);
    } else if (func >= 10 && func <= 19) {
      lrs[func - 10](&a[2], &o[0], &o[1]);
    } else if (func >= 20 && func <= 23) {
      mhd_lrstate(&a[2], &a[7], &a[12], &a[17], &a[22], &a[27], &a[32], a[35], a[36], 1,
                  interpol[func - 20], &o[0], &o[7]);
    } else if (func == 30) {
      o[0] = mhd_cuct_weight(&a[3], &a[7], &a[11], &a[15], &a[19], 1, 2);
    } else if (func == 31) {
      o[0] = mhd_ieos(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8]);
    } else if (func == 32) {
      o[0] = mhd_energy(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8]);
    } else {
      fprintf(stderr, "unknown func %d\n", func);
      return 2;
    }
  }
  f = fopen(argv[2], "wb");
  if (!f) return 2;
  fwrite(out.data(), sizeof(double), out.size(), f);
  fclose(f);
  return 0;
}
