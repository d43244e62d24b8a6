// qas_mhd2d_dropin.hpp -- drop-in GPU stepping for the reference's 2D driver class.
//
// Include it in place of "mhd2d_class.hpp" in a problem directory (2D/SERIAL/<problem>/) and
// link libqas (g++ ... -I<repo>/include -L<repo>/qasmhd_b200 -lqas).  GpuMHD2D keeps paras(),
// init_(), setdt() and dout_() of MHD2D and adds exec_gpu(flg), which replaces exec_(flg)
// (2D/SERIAL/OTvortex/mhd2d_class.cpp:35-61; exec_ is not virtual, so main() calls exec_gpu):
// the same loop -- dt refreshed by setdt every 2nd step when flg is set, the stop rule
// n < nmax && tim < tmax, dout_(1) whenever tim passes trec -- with the state on the GPU.  The
// host arrays val[] are refreshed only at output times.  A failing library call throws
// std::runtime_error with the library's status text.
#ifndef QAS_MHD2D_DROPIN_HPP
#define QAS_MHD2D_DROPIN_HPP

#include <stdexcept>
#include <string>

#include "mhd2d_class.hpp"
#include "qas.h"

class GpuMHD2D : public MHD2D {
 public:
  void exec_gpu(int flg)
  {
    qas_grid g = {2, XMESH, YMESH, 1, dx, dy, 0.0, gam};
    qas_scheme s = {RMN, ODR, R_K, CTW, 0};  // char_mode 0: mhd_lrstate's characteristic form
    qas_bc bc;
    for (int m = 0; m < 8; m++) {
      bc.dnx[m] = dnxs[m];
      bc.dny[m] = dnys[m];
      bc.dnz[m] = 0;
    }
    qas_ctx *ctx = nullptr;
    check(qas_create(&ctx, &g, &s, &bc, -1));
    check(qas_upload(ctx, val));  // val[8]: ro,mx,my,mz,bx,by,bz,en (host, nd each)
    if (n == 0) dout_(0);
    // one exec_ step per call: setdt as main()+exec_ do it, stop rule n < nmax && tim < tmax
    qas_run_opts o = {1, flg, 1, cfl, dtrec, nout, 1, 0.0, 0.0};
    qas_run_info info = {0, 0, 0, 0.0, 0.0};
    while (true) {
      do {
        check(qas_run(ctx, &o, &info));
      } while (info.steps && info.tim < trec);
      n = info.n;
      tim = info.tim;
      dt = info.dt;
      nmax = info.nmax;
      if (tim < trec) break;  // the run stopped before the next output time
      check(qas_download(ctx, val));
      cnt++;
      trec += dtrec;
      dout_(1);
    }
    check(qas_destroy(ctx));
  }

 private:
  static void check(qas_status st)
  {
    if (st != QAS_OK) throw std::runtime_error(std::string("libqas: ") + qas_status_str(st));
  }
};

#endif
