/*
 * Forced-include settings for the drop-in check: the reference's 2D Orszag-Tang problem
 * directory (2D/SERIAL/OTvortex) built at 64^2 with its own solver choice (mymacros.hpp:4-14:
 * LHLLD, ODR 2, RK3, CTW) and outputs every 0.2*3.1416 up to 6 outputs.  Defining the
 * include guard _MYMACROS_ first makes the directory's mymacros.hpp a no-op.
 * Test infrastructure only.
 */
#ifndef QAS_DROPIN_MACROS_H
#define QAS_DROPIN_MACROS_H
#define _MYMACROS_
#define XMESH (64)
#define YMESH (64)
#define N_OUT (6)
#define DTREC (0.2 * 3.1416)
#define CFL (0.4)
#define RMN (2)
#define ODR (2)
#define R_K (3)
#define CTW (1)
#endif
