// qas_pipe.cuh -- kernels of the pipelined host round trip (qas_step_host): the cell kernels
// of one exec_ step restricted to a window of planes along the last axis (rows in 2D, z planes
// in 3D).  Every kernel calls the same per-cell body as its full-grid counterpart, so a value
// computed here is bit-identical to the one the full-grid kernel computes at that cell from
// the same inputs.
#pragma once

#include "qas_kernels.cuh"

namespace qas {

// Launched with programmatic dependent launch: a kernel may start while the previous one in
// its stream drains, and waits for its completion (and its memory) before touching anything.
#define QAS_PDL_WAIT() cudaGridDependencySynchronize()

// planes [lo, hi) of the last axis, padded index
struct Rows {
  int lo, hi;
};

// the eight state arrays of one stage buffer
struct StatePtrs {
  double *p[8];
};

// up to two disjoint plane ranges handled by one launch (b empty for one range); the
// launch's last grid axis counts the planes of a, then those of b
struct Rows2 {
  Rows a, b;
};

__device__ __forceinline__ int rows_len(Rows r) { return r.hi > r.lo ? r.hi - r.lo : 0; }
__device__ __forceinline__ bool rows_has(Rows r, int h) { return h >= r.lo && h < r.hi; }
__device__ __forceinline__ bool rows2_has(const Rows2 &r, int h) { return rows_has(r.a, h) || rows_has(r.b, h); }

// the t-th plane of r, or -1 past its end
__device__ __forceinline__ int rows2_plane(const Rows2 &r, int t)
{
  const int na = rows_len(r.a);
  if (t < na) return r.a.lo + t;
  t -= na;
  return t < rows_len(r.b) ? r.b.lo + t : -1;
}

__device__ __forceinline__ bool win_cell(const Geo &g, const Rows2 &r, int &i, int &j, int &k)
{
  i = blockIdx.x * blockDim.x + threadIdx.x;
  j = blockIdx.y * blockDim.y + threadIdx.y;
  k = blockIdx.z * blockDim.z + threadIdx.z;
  int &h = g.dim == 3 ? k : j;
  h = rows2_plane(r, h);
  return h >= 0 && i < g.nx && j < g.ny && k < g.nz;
}

// the primitives on planes pr, one launch over rows r (pr and cp together); on a finished run
// (stop flag set) instead the copy of the eight state arrays v.u -> dst on planes cp, so that the
// state passes through unchanged (otherwise the update writes every interior cell of dst from
// v.u and the ghost fill the rest)
template <int ODR>
__global__ void QAS_PRIM_BOUNDS kw_prim_copy(View v, Rows2 r, Rows2 pr, Rows2 cp, StatePtrs dst)
{
  QAS_PDL_WAIT();
  int i, j, k;
  if (!win_cell(v.g, r, i, j, k)) return;
  const int h = v.g.dim == 3 ? k : j;
  if (v.ctl->done && rows2_has(cp, h)) {
    const long long c = cidx(v.g, i, j, k);
#pragma unroll
    for (int m = 0; m < 8; m++) dst.p[m][c] = v.u[m][c];
  }
  if (!v.ctl->done && rows2_has(pr, h)) prim_body<ODR>(v, i, j, k);
}

__global__ void kw_dv(View v, Rows2 r)
{
  QAS_PDL_WAIT();
  if (v.ctl->done) return;
  int i, j, k;
  if (!win_cell(v.g, r, i, j, k)) return;
  dv_body(v, i, j, k);
}

template <int ODR, int A, int PR>
__global__ void __launch_bounds__(128, QAS_LR_MINB) kw_lr(View v, Rows2 r)
{
  QAS_PDL_WAIT();
  if (v.ctl->done) return;
  int i, j, k;
  if (!win_cell(v.g, r, i, j, k)) return;
  lr_body<ODR, A, PR>(v, i, j, k);
}

template <int RMN, int A>
__global__ void __launch_bounds__(128, QAS_FLUX_MINB_OF(RMN)) kw_flux(View v, Rows2 r)
{
  QAS_PDL_WAIT();
  if (v.ctl->done) return;
  int i, j, k;
  if (!win_cell(v.g, r, i, j, k)) return;
  flux_body<RMN, A>(v, i, j, k);
}

template <int A>
__global__ void __launch_bounds__(128, QAS_FLUX_MLAU_MINB) kw_flux_mlau(View v, Rows2 r)
{
  QAS_PDL_WAIT();
  if (v.ctl->done) return;
  int i, j, k;
  if (!win_cell(v.g, r, i, j, k)) return;
  flux_body<3, A>(v, i, j, k);
}

// fused face sweeps on a window (the default form in 3D, see k_sweep_x / k_sweep_m)
// x sweep over the flattened cells of the rows of planes r
template <int ODR, int RMN, int PR>
__global__ void __launch_bounds__(128, QAS_SWEEP_MINB_OF(RMN)) kw_sweep_x(View v, Rows2 r, long long nwarps)
{
  QAS_PDL_WAIT();
  if (v.ctl->done) return;
  const Geo &g = v.g;
  const int lane = threadIdx.x & 31;
  const long long w = (long long)blockIdx.x * 4 + (threadIdx.x >> 5);
  if (w >= nwarps) return;  // the whole warp leaves together
  const long long ncell = g.nx - 4;
  const long long per_plane = g.dim == 3 ? g.ny : 1;
  const long long total = ncell * per_plane * (rows_len(r.a) + rows_len(r.b));
  long long t = w * 31 + lane;
  const bool have_cell = t < total;
  if (!have_cell) t = total - 1;
  const long long row = t / ncell;
  const int i = 2 + (int)(t - row * ncell);
  const int j = g.dim == 3 ? (int)(row % g.ny) : rows2_plane(r, (int)row);
  const int k = g.dim == 3 ? rows2_plane(r, (int)(row / g.ny)) : 0;
  sweep_x_cell<ODR, RMN, PR>(v, i, j, k, lane, have_cell);
}

// y sweep of a 3D window (an in-plane axis): columns (i, k) with k on planes r, every y face
// [3, ny-2) in segments of `seg`
template <int ODR, int RMN, int PR>
__global__ void __launch_bounds__(128, QAS_SWEEP_MINB_OF(RMN)) kw_sweep_y3(View v, Rows2 r, int seg)
{
  QAS_PDL_WAIT();
  if (v.ctl->done) return;
  const Geo &g = v.g;
  __shared__ double carry[9][128];
  const int tid = threadIdx.x;
  const long long col = (long long)blockIdx.x * 128 + tid;
  if (col >= (long long)g.nx * (rows_len(r.a) + rows_len(r.b))) return;
  const int p0 = 3 + blockIdx.y * seg;
  sweep_column<ODR, RMN, 1, PR>(v, (int)(col % g.nx), rows2_plane(r, (int)(col / g.nx)), p0, min(p0 + seg, g.ny - 2),
                            carry, tid);
}

// sweep along the last axis A (y in 2D, z in 3D): every column (i, j in 3D), the faces of
// f = r clipped to [3, n-2), chunk q of `seg` faces per blockIdx.y: first those of r.a, then r.b
template <int ODR, int RMN, int A, int PR>
__global__ void __launch_bounds__(128, QAS_SWEEP_MINB_OF(RMN)) kw_sweep_last(View v, Rows2 f, int seg)
{
  QAS_PDL_WAIT();
  if (v.ctl->done) return;
  const Geo &g = v.g;
  __shared__ double carry[9][128];
  const int tid = threadIdx.x;
  const long long col = (long long)blockIdx.x * 128 + tid;
  if (col >= (long long)g.nx * (A == 2 ? g.ny : 1)) return;
  const int n = g.n[A];
  const Rows a{max(f.a.lo, 3), min(f.a.hi, n - 2)}, b{max(f.b.lo, 3), min(f.b.hi, n - 2)};
  const int ca = (rows_len(a) + seg - 1) / seg;
  const int q = blockIdx.y;
  const Rows &x = q < ca ? a : b;
  const int p0 = x.lo + (q < ca ? q : q - ca) * seg;
  if (p0 >= x.hi) return;
  sweep_column<ODR, RMN, A, PR>(v, (int)(col % g.nx), (int)(col / g.nx), p0, min(p0 + seg, x.hi), carry, tid);
}

template <int ODR>
__global__ void QAS_EMF_BOUNDS kw_emf(View v, Rows2 r)
{
  QAS_PDL_WAIT();
  if (v.ctl->done) return;
  int i, j, k;
  if (!win_cell(v.g, r, i, j, k)) return;
  emf_body<ODR>(v, i, j, k);
}

// the update cells of k_update (i in [GH, nx-GH], likewise j in 3D) on planes [lo, hi), which
// lie in [GH, n-GH] (the last face plane of the staggered field included)
template <int ODR>
__global__ void QAS_UPDATE_BOUNDS kw_update(View v, Rows2 r, double c0, double c1, StatePtrs src)
{
  QAS_PDL_WAIT();
  if (v.ctl->done) return;
  const Geo &g = v.g;
  const int i = GH + blockIdx.x * blockDim.x + threadIdx.x;
  const int tj = blockIdx.y * blockDim.y + threadIdx.y;
  const int tk = blockIdx.z * blockDim.z + threadIdx.z;
  int j, k;
  if (g.dim == 3) {
    j = GH + tj;
    k = rows2_plane(r, tk);
    if (j > g.ny - GH || k < 0) return;
  } else {
    j = rows2_plane(r, tj);
    k = 0;
    if (tk > 0 || j < 0) return;
  }
  if (i > g.nx - GH) return;
  update_body<ODR>(v, i, j, k, c0, c1, src.p);  // U_r of the cell from U_{r-1} (src) and ut
}

// ghost fill of the cells of planes [lo, hi) that are ghosts along an in-plane axis (x in 2D;
// x or y in 3D).  Their sources lie in the same plane.
__global__ void kw_bound_cols(View v, Rows2 r)
{
  QAS_PDL_WAIT();
  if (v.ctl->done) return;
  const Geo &g = v.g;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int planes = rows_len(r.a) + rows_len(r.b);
  int i, j, k;
  if (g.dim == 2) {
    const long long per = 2 * GH;
    if (t >= per * planes) return;
    const int col = (int)(t % per);
    i = col < GH ? col : g.nx - 2 * GH + col;
    j = rows2_plane(r, (int)(t / per));
    k = 0;
  } else {
    const long long per = (long long)g.nx * g.ny - (long long)(g.nx - 2 * GH) * (g.ny - 2 * GH);
    if (t >= per * planes) return;
    Geo g2 = g;
    g2.dim = 2;
    int kk;
    shell_cell(g2, t % per, i, j, kk);
    k = rows2_plane(r, (int)(t / per));
  }
  bound_body(v, i, j, k);
}

// ghost fill of the ghost planes of the last axis ([0, GH) and [n-GH, n), every in-plane cell)
__global__ void kw_bound_ends(View v)
{
  QAS_PDL_WAIT();
  if (v.ctl->done) return;
  const Geo &g = v.g;
  const long long plane = g.dim == 3 ? (long long)g.nx * g.ny : (long long)g.nx;
  const int n = g.dim == 3 ? g.nz : g.ny;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 2 * GH * plane) return;
  const int h = (int)(t / plane);
  const int hh = h < GH ? h : n - 2 * GH + h;
  const long long q = t % plane;
  int i, j, k;
  if (g.dim == 3) {
    i = (int)(q % g.nx);
    j = (int)(q / g.nx);
    k = hh;
  } else {
    i = (int)q;
    j = hh;
    k = 0;
  }
  bound_body(v, i, j, k);
}

}  // namespace qas
