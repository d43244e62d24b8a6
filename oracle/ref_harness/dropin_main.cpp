/*
 * The reference's 2D main (2D/SERIAL/OTvortex/main.cpp) with the drop-in subclass: the same
 * paras / init_ / setdt(1) sequence, then exec_gpu(1) where the reference calls exec_(1).
 * Writes the reference's own output files (dout_) under ./dat/.  Test infrastructure only.
 */
#include "qas_mhd2d_dropin.hpp"

int main()
{
  GpuMHD2D mhd2d;
  mhd2d.paras();
  mhd2d.init_();
  mhd2d.setdt(1);
  mhd2d.exec_gpu(1);
  return 0;
}
