/*
 * Binary case format shared by the reference harnesses (oracle/_ref/*) and the
 * Python test helpers (qasmhd oracle tooling in tests/).  Test infrastructure.
 *
 * Input  : RefCaseHeader, then 8 arrays (ro,mx,my,mz,bx,by,bz,en) of nd doubles,
 *          each in the reference layout ss = nx*(ny*k+j)+i with 4 ghost cells
 *          per side (2D/SERIAL/OTvortex/mhd2d_class.hpp:10-12), then phi_g when has_phi.
 * Output : RefResultHeader, n_dt doubles (dt used by each step), the 8 arrays
 *          after the run, then int32 count + per-step wall times (RUN modes).
 */
#ifndef QAS_REF_IO_H
#define QAS_REF_IO_H

#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <vector>

#define QAS_REF_MAGIC_IN  0x31534151   /* "QAS1" */
#define QAS_REF_MAGIC_OUT 0x32534151   /* "QAS2" */

enum RefMode {
  REF_MODE_STEP = 0,   /* bound(val); ideal(dt) once, with the given dt            */
  REF_MODE_RUN  = 1,   /* setdt(1); nsteps x { tim+=dt; bound; ideal; setdt(flg) } */
  REF_MODE_EXEC = 2,   /* exec_(flg) loop termination: n<nmax && tim<tmax          */
  REF_MODE_DRUN = 3,   /* RUN with the dissipative sub-cycle after ideal (2D, 3D)  */
  REF_MODE_DSTEP = 4,  /* bound; dsptv(dt) once (2D, 3D)                           */
  REF_MODE_IO = 5,     /* dout_ + bkup_save of the state into argv[3] (n = nsteps,
                          cnt = flg, tim = dt, dt = cfl, trec = dtrec)             */
  REF_MODE_IOLOAD = 6  /* bkup_load from argv[3]; the loaded counters go to
                          argv[3]/loaded.txt, the loaded state to the result       */
};


#pragma pack(push, 1)
struct RefCaseHeader {
  int32_t magic;
  int32_t dim, nxm, nym, nzm;
  int32_t rmn, odr, rk, ctw;
  int32_t mode, nsteps, flg, nthreads;
  int32_t nout, has_phi;  /* bit 0: nd doubles of phi_g follow the 8 state arrays;
                             bit 1: then the nu and eta arrays (nd doubles each) */
  double gam, cfl, dtrec, dt;
  double xmin, xmax, ymin, ymax, zmin, zmax;
  double nu0, eta0;
  int32_t dnx[8], dny[8], dnz[8];
};
struct RefResultHeader {
  int32_t magic, nsteps_done, n_dt, nd;
  double tim, dt, elapsed_s, pad;
};
#pragma pack(pop)

static inline void ref_die(const char *msg)
{
  fprintf(stderr, "qas ref harness: %s\n", msg);
  exit(2);
}

/* Counters of a bkup_load, for the I/O pins. */
static inline void ref_write_loaded(const char *dir, int n, int cnt, double tim, double dt, double trec)
{
  char path[512];
  snprintf(path, sizeof(path), "%s/loaded.txt", dir);
  FILE *f = fopen(path, "w");
  if (!f) ref_die("cannot write loaded.txt");
  fprintf(f, "%d %d %.17g %.17g %.17g\n", n, cnt, tim, dt, trec);
  fclose(f);
}

static inline void ref_read_case(const char *path, RefCaseHeader *h, std::vector<double> *data)
{
  FILE *f = fopen(path, "rb");
  if (!f) ref_die("cannot open input");
  if (fread(h, sizeof(*h), 1, f) != 1) ref_die("short header");
  if (h->magic != QAS_REF_MAGIC_IN) ref_die("bad magic");
  long nx = h->nxm + 8;
  long ny = h->dim >= 2 ? h->nym + 8 : 1;
  long nz = h->dim >= 3 ? h->nzm + 8 : 1;
  size_t n = (size_t)((8 + ((h->has_phi & 1) ? 1 : 0) + ((h->has_phi & 2) ? 2 : 0)) * nx * ny * nz);
  data->resize(n);
  if (fread(data->data(), sizeof(double), n, f) != n) ref_die("short data");
  fclose(f);
}

static inline void ref_write_result(const char *path, const RefResultHeader &r,
                                    const std::vector<double> &dts, double *const val[8], long nd)
{
  FILE *f = fopen(path, "wb");
  if (!f) ref_die("cannot open output");
  fwrite(&r, sizeof(r), 1, f);
  if (!dts.empty()) fwrite(dts.data(), sizeof(double), dts.size(), f);
  for (int m = 0; m < 8; m++) fwrite(val[m], sizeof(double), (size_t)nd, f);
  fclose(f);
}

/* Per-step wall times of the RUN modes, appended after the state (count, then values). */
static inline void ref_append_times(const char *path, const std::vector<double> &t)
{
  FILE *f = fopen(path, "ab");
  if (!f) ref_die("cannot append output");
  int32_t n = (int32_t)t.size();
  fwrite(&n, sizeof(n), 1, f);
  if (n) fwrite(t.data(), sizeof(double), t.size(), f);
  fclose(f);
}

#endif
