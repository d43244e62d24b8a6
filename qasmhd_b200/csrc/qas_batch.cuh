// qas_batch.cuh -- batched-ensemble kernels: one launch per stage covers every
// instance of the ensemble.  Blocks are persistent (grid-stride over the block
// list); a block map gives each block its instance and its block index inside
// that instance's launch grid, so every block works on one instance with that
// instance's View (its own sizes, boundary maps, scheme and dt).  The per-cell
// arithmetic is the single-instance kernels' device bodies.
#pragma once

#include "qas_kernels.cuh"

namespace qas {

struct BMap {
  int nblocks;
  const int2 *blk;   // (instance, local block index) per block
  const int4 *grid;  // per instance: launch grid in blocks (x, y, z, 0), or the thread extent
                     // (x, y, z, -1) of a linear map
};

// the thread's index in its instance's launch extent.  Tiled: block lb is tile (bx, by, bz) of
// the instance's grid.  Linear: block lb covers threads [lb*T, (lb+1)*T) of the extent in x-fastest
// order, so no thread idles at the end of a row whatever the instance's size; threads past the
// extent get an index that fails every range test.
__device__ __forceinline__ void batch_thread(int4 gd, int lb, int &ti, int &tj, int &tk)
{
  if (gd.w < 0) {
    const int nt = blockDim.x * blockDim.y * blockDim.z;
    const int lin = lb * nt + (threadIdx.z * blockDim.y + threadIdx.y) * blockDim.x + threadIdx.x;
    const int r = lin / gd.x;
    ti = lin - r * gd.x;
    tj = r % gd.y;
    tk = r / gd.y;
    if (tk >= gd.z) ti = tj = tk = 1 << 29;
  } else {
    const int bx = lb % gd.x, by = (lb / gd.x) % gd.y, bz = lb / (gd.x * gd.y);
    ti = bx * blockDim.x + threadIdx.x;
    tj = by * blockDim.y + threadIdx.y;
    tk = bz * blockDim.z + threadIdx.z;
  }
}

// Block loop of a persistent batched kernel.  0 (default): grid-stride over the block list.
// QAS_BATCH_CONTIGUOUS = 1: each CTA takes one contiguous run of the (instance-major) list, so
// that its consecutive blocks share an instance (View, control word and launch grid in L1), with
// the next map entry loaded while the current block works -- measured slower on B200 (512-member
// C4 ensemble: 551 against 587 Mcell-updates/s): the long runs of one instance per CTA balance
// the SMs worse than the interleaved stride.
#ifndef QAS_BATCH_CONTIGUOUS
#define QAS_BATCH_CONTIGUOUS 0
#endif
#if QAS_BATCH_CONTIGUOUS
#define QAS_BATCH_BLOCKS(map)                                                         \
  const int bper_ = ((map).nblocks + gridDim.x - 1) / gridDim.x;                      \
  const int bend_ = min((map).nblocks, (int)(blockIdx.x + 1) * bper_);                \
  int2 bnext_ = make_int2(0, 0);                                                      \
  if ((int)blockIdx.x * bper_ < bend_) bnext_ = (map).blk[blockIdx.x * bper_];       \
  for (int b_ = blockIdx.x * bper_; b_ < bend_; b_++) {                               \
    const int2 bi_ = bnext_;                                                          \
    if (b_ + 1 < bend_) bnext_ = (map).blk[b_ + 1];                                   \
    const View &v = views[bi_.x];                                                     \
    if (v.ctl->done) continue;                                                        \
    const int4 gd_ = (map).grid[bi_.x];                                               \
    int ti, tj, tk;                                                                   \
    batch_thread(gd_, bi_.y, ti, tj, tk);
#else
#define QAS_BATCH_BLOCKS(map)                                                         \
  for (int b_ = blockIdx.x; b_ < (map).nblocks; b_ += gridDim.x) {                    \
    const int2 bi_ = (map).blk[b_];                                                   \
    const View &v = views[bi_.x];                                                     \
    if (v.ctl->done) continue;                                                        \
    const int4 gd_ = (map).grid[bi_.x];                                               \
    int ti, tj, tk;                                                                   \
    batch_thread(gd_, bi_.y, ti, tj, tk);
#endif

#define QAS_BATCH_END }

#define QAS_BATCH_CELL_OK (ti < v.g.nx && tj < v.g.ny && tk < v.g.nz)

// resident-block caps of the light batched kernels (0: the single-grid kernels' 16).  The block
// loop keeps the instance View and map entry live, so at the single-grid cap (32 registers) both
// spill (96-180 B); at 8 blocks (64 registers) neither does.  Measured on the 512-member C4
// ensemble, same box back to back: both at 16 / 12 / 8 blocks 580-582 / 573-576 / 592-593
// Mcell-updates/s; with the primitives at 8, the update at 16 / 12 / 8 594-598 / 583-586 /
// 594-597 -- the gain is the primitives', so the update keeps the single-grid cap.
#ifndef QAS_BATCH_PRIM_MINB
#define QAS_BATCH_PRIM_MINB 8
#endif
#ifndef QAS_BATCH_UPDATE_MINB
#define QAS_BATCH_UPDATE_MINB 0
#endif
#if QAS_BATCH_PRIM_MINB > 0
#define QAS_BATCH_PRIM_BOUNDS __launch_bounds__(128, QAS_BATCH_PRIM_MINB)
#else
#define QAS_BATCH_PRIM_BOUNDS QAS_PRIM_BOUNDS
#endif
#if QAS_BATCH_UPDATE_MINB > 0
#define QAS_BATCH_UPDATE_BOUNDS __launch_bounds__(128, QAS_BATCH_UPDATE_MINB)
#else
#define QAS_BATCH_UPDATE_BOUNDS QAS_UPDATE_BOUNDS
#endif

template <int ODR>
__global__ void QAS_BATCH_PRIM_BOUNDS kb_prim(const View *__restrict__ views, BMap map)
{
  QAS_BATCH_BLOCKS(map)
  if (QAS_BATCH_CELL_OK) prim_body<ODR>(v, ti, tj, tk);
  QAS_BATCH_END
}

__global__ void kb_dv(const View *__restrict__ views, BMap map)
{
  QAS_BATCH_BLOCKS(map)
  if (QAS_BATCH_CELL_OK) dv_body(v, ti, tj, tk);
  QAS_BATCH_END
}

// PR: the face-value form of every instance (0 characteristic, 1 primitive) or -1 (mixed: each
// instance's View decides)
#ifndef QAS_BATCH_LR_MINB
#define QAS_BATCH_LR_MINB QAS_LR_MINB
#endif
template <int ODR, int A, int PR>
__global__ void __launch_bounds__(128, QAS_BATCH_LR_MINB) kb_lr(const View *__restrict__ views, BMap map)
{
  QAS_BATCH_BLOCKS(map)
  if (QAS_BATCH_CELL_OK) {
    const int pos = A == 0 ? ti : (A == 1 ? tj : tk);
    if (pos >= 2 && pos < v.g.n[A] - 2) lr_body<ODR, A, PR>(v, ti, tj, tk);
  }
  QAS_BATCH_END
}

template <int RMN, int A>
__global__ void __launch_bounds__(128, QAS_FLUX_MINB_OF(RMN)) kb_flux(const View *__restrict__ views, BMap map)
{
  QAS_BATCH_BLOCKS(map)
  if (QAS_BATCH_CELL_OK) {
    const int pos = A == 0 ? ti : (A == 1 ? tj : tk);
    if (pos >= 3 && pos < v.g.n[A] - 2) flux_body<RMN, A>(v, ti, tj, tk);
  }
  QAS_BATCH_END
}

// MLAU with the register cap of the single-grid k_flux_mlau
template <int A>
__global__ void __launch_bounds__(128, QAS_FLUX_MLAU_MINB) kb_flux_mlau(const View *__restrict__ views, BMap map)
{
  QAS_BATCH_BLOCKS(map)
  if (QAS_BATCH_CELL_OK) {
    const int pos = A == 0 ? ti : (A == 1 ? tj : tk);
    if (pos >= 3 && pos < v.g.n[A] - 2) flux_body<3, A>(v, ti, tj, tk);
  }
  QAS_BATCH_END
}

template <int ODR>
__global__ void kb_emf(const View *__restrict__ views, BMap map)
{
  QAS_BATCH_BLOCKS(map)
  if (QAS_BATCH_CELL_OK) emf_body<ODR>(v, ti, tj, tk);
  QAS_BATCH_END
}

template <int ODR>
__global__ void QAS_BATCH_UPDATE_BOUNDS kb_update(const View *__restrict__ views, BMap map, double c0, double c1)
{
  QAS_BATCH_BLOCKS(map)
  int i, j, k;
  if (update_cell(v.g, ti, tj, tk, i, j, k)) update_body<ODR>(v, i, j, k, c0, c1);
  QAS_BATCH_END
}

// ghost shell (1D block index over the shell cells of each instance)
__global__ void kb_bound(const View *__restrict__ views, BMap map)
{
  QAS_BATCH_BLOCKS(map)
  (void)tj;
  (void)tk;
  if (ti < shell_cells(v.g)) {
    int i, j, k;
    shell_cell(v.g, ti, i, j, k);
    bound_body(v, i, j, k);
  }
  QAS_BATCH_END
}

// u0 = u for all cells of every instance (the copy of ut at the start of ideal)
__global__ void kb_copy_u0(const View *__restrict__ views, BMap map)
{
  QAS_BATCH_BLOCKS(map)
  if (QAS_BATCH_CELL_OK) {
    const long long c = cidx(v.g, ti, tj, tk);
#pragma unroll
    for (int m = 0; m < 8; m++) v.u0[m][c] = v.u[m][c];
  }
  QAS_BATCH_END
}

// per-instance control: one thread per instance
__global__ void kb_begin(const View *__restrict__ views, int n, int check_tim)
{
  const int inst = blockIdx.x * blockDim.x + threadIdx.x;
  if (inst < n) begin_body(views[inst], check_tim);
}
__global__ void kb_vmax_reset(const View *__restrict__ views, int n)
{
  const int inst = blockIdx.x * blockDim.x + threadIdx.x;
  if (inst < n && !views[inst].ctl->done)
    views[inst].ctl->vmax_bits = (unsigned long long)__double_as_longlong(1.0);
}
__global__ void kb_setdt(const View *__restrict__ views, int n, double cfl, int rule, double dtrec, int nout)
{
  const int inst = blockIdx.x * blockDim.x + threadIdx.x;
  if (inst < n) setdt_body(views[inst], cfl, views[inst].dr, rule, dtrec, nout);
}

// per-instance max of |v|+c_f over the interior (1D blocks of 128 threads)
__global__ void kb_vmax(const View *__restrict__ views, BMap map)
{
  __shared__ double red[4];
  for (int b_ = blockIdx.x; b_ < map.nblocks; b_ += gridDim.x) {
    const int2 bi = map.blk[b_];
    const View &v = views[bi.x];
    if (v.ctl->done) continue;  // uniform over the block
    const int4 gd = map.grid[bi.x];
    const int bx = bi.y % gd.x, by = (bi.y / gd.x) % gd.y, bz = bi.y / (gd.x * gd.y);
    const Geo &g = v.g;
    const int i = GH + bx * blockDim.x + threadIdx.x;
    const int j = (g.dim >= 2 ? GH : 0) + by;
    const int k = (g.dim >= 3 ? GH : 0) + bz;
    double best = 1.0;
    if (i < g.nx - GH) {
      const double vt = vmax_cell(v, i, j, k);
      if (vt > best) best = vt;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double other = __shfl_xor_sync(0xffffffffu, best, o);
      best = (other > best) ? other : best;
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) red[wid] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
      double m = red[0];
      for (int q = 1; q < (int)(blockDim.x >> 5); q++) m = (red[q] > m) ? red[q] : m;
      atomicMax(&v.ctl->vmax_bits, (unsigned long long)__double_as_longlong(m));
    }
    __syncthreads();
  }
}

}  // namespace qas
