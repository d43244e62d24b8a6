// qas_tma.cuh -- the characteristic reconstruction (k_lr) with its stencil staged in shared
// memory by the Tensor Memory Accelerator (sm_100a).
//
// The seven primitives a face state reads (ro, vn, vb, vc, cb, cc, pr along axis A) are moved
// from HBM into a ring of shared-memory planes by cp.async.bulk.tensor, one mbarrier per slot.
// Each CTA (TX x TR threads, one cell each) owns a TX x TR column of the transverse plane and
// a segment along the march axis MA:
//   * A == MA (y or z faces): the CTA marches along A with a 5-plane window (points m-2..m+2 of
//     the stencil are ring slots), so every primitive is read from HBM/L2 once per column;
//   * A == 0 (x faces): each plane is an x-tile with a +-2 halo, streamed along MA.
// One elected thread issues the loads of the next plane while all threads compute the
// current cell; the arithmetic is lr_cell, the same function as the global-memory k_lr, so
// the results are bit-identical.  Every mbarrier wait is bounded (two seconds of device time
// by %globaltimer, LrTmaPlan::wait_ns): on expiry the kernel latches an error bit, waits
// (bounded) for its own loads in flight and returns.
#pragma once

#include <cuda.h>

#include "qas_kernels.cuh"

namespace qas {

// one tensor map per stencil field of an axis: ro, vn, vb, vc, cb, cc, pr
struct LrTmaMaps {
  CUtensorMap m[7];
};

// work decomposition of one axis
struct LrTmaPlan {
  int xt, rt, ms;  // tiles along x, along the row axis, segments along the march axis
  int items;       // xt * rt * ms
  int seg;         // march cells per segment
  int mlo, mhi;    // computed range along the march axis
  int xlo, xhi;    // computed range along x
  int nr;          // extent of the row axis
  // bound of every mbarrier wait in ns of device time (2 s), and a failure hook for tests: when
  // stall_plane >= 0, no CTA issues its plane number stall_plane (counted from the CTA's first),
  // so the wait for that plane runs out and the kernel takes its timeout path
  unsigned long long wait_ns;
  int stall_plane;
};

constexpr int LR_TMA_TIMEOUT_BIT = 8;

__device__ __forceinline__ unsigned smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long *bar, unsigned bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity)
{
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns()
{
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// wait for phase `parity` of the barrier, giving up after `limit_ns` of device time
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long *bar, unsigned parity,
                                                  unsigned long long limit_ns)
{
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (!mbar_try_wait(bar, parity)) {
    if (global_ns() - t0 > limit_ns) return false;
  }
  return true;
}

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z,
                                            unsigned long long *bar)
{
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
      : "memory");
}

// stencil accessor over the shared-memory ring: field f at stencil point m (0..4).  Holds
// 32-bit indices only: idx = the thread's element in a field plane, sl = the ring slot of
// stencil point 0 (A != 0: point m is slot sl+m mod R) or of the plane (A == 0: point m is
// element idx+m of the halo tile).
template <bool XS, int PD, int R>
struct SmemStencil {
  const double *ring;
  int idx, sl;
  __device__ __forceinline__ double operator()(int f, int m) const
  {
    if (XS) return ring[(sl * 7 + f) * PD + idx + m];
    int q = sl + m;
    if (q >= R) q -= R;
    return ring[(q * 7 + f) * PD + idx];
  }
  __device__ __forceinline__ double late(int f, int m) const { return (*this)(f, m); }
};

// dynamic shared memory of one configuration: ring slots x 7 fields x PD doubles + barriers
template <int A, int TX, int TR>
struct LrTmaShape {
  static constexpr bool XS = (A == 0);
  static constexpr int BX = TX + (XS ? 4 : 0);          // plane width along x
  static constexpr int PD = ((BX * TR + 15) / 16) * 16;  // doubles per field per slot (128-byte multiple)
  static constexpr int W = XS ? 1 : 5;                   // planes in the stencil window
  static constexpr int H = (W - 1) / 2;
  static constexpr int R = XS ? 3 : 6;                   // ring slots
  static constexpr unsigned PLANE_BYTES = 7u * BX * TR * 8u;
  static constexpr size_t SMEM = (size_t)R * 7 * PD * sizeof(double) + R * sizeof(unsigned long long);
};

template <int ODR, int A, int TX, int TR, int MA>
__global__ void __launch_bounds__(TX *TR, 5) k_lr_tma(View v, const __grid_constant__ LrTmaMaps maps, LrTmaPlan pl)
{
  using S = LrTmaShape<A, TX, TR>;
  constexpr int NF = 7;
  extern __shared__ __align__(128) double lr_ring[];
  unsigned long long *bar = reinterpret_cast<unsigned long long *>(lr_ring + S::R * NF * S::PD);
  if (v.ctl->done) return;
  const Geo &g = v.g;
  const int tid = threadIdx.x;
  const int lx = tid % TX, lrow = tid / TX;
  if (tid == 0) {
#pragma unroll
    for (int q = 0; q < S::R; q++) mbar_init(&bar[q], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
  const long long sA = g.s[A];
  const double *cn = A == 0 ? v.cx : (A == 1 ? v.cy : v.cz);
  unsigned gbase = 0;  // planes issued by this CTA before the current item
  for (int item = blockIdx.x; item < pl.items; item += gridDim.x) {
    int t = item;
    const int tx = t % pl.xt;
    t /= pl.xt;
    const int tr = t % pl.rt;
    const int sg = t / pl.rt;
    const int xb = pl.xlo + tx * TX;  // first computed x of the tile
    const int r0 = tr * TR;
    const int m0 = pl.mlo + sg * pl.seg;
    const int m1 = min(m0 + pl.seg, pl.mhi);
    const int ns = m1 - m0;
    const int Q = ns + 2 * S::H;      // planes of this item
    const int bx0 = xb - (S::XS ? 2 : 0);
    int issued = 0, waited = 0;
    auto issue = [&](int q) {  // thread 0 only
      const unsigned gq = gbase + q;
      const int slot = (int)(gq % S::R);
      const int m = m0 - S::H + q;
      const int cy = MA == 1 ? m : r0, cz = MA == 1 ? r0 : m;
      if ((int)gq == pl.stall_plane) return;  // test hook: this plane is never loaded
      mbar_arrive_expect_tx(&bar[slot], S::PLANE_BYTES);
#pragma unroll
      for (int f = 0; f < NF; f++) tma_load_3d(lr_ring + (slot * NF + f) * S::PD, &maps.m[f], bx0, cy, cz, &bar[slot]);
    };
    if (tid == 0) {
      const int n0 = Q < S::R ? Q : S::R;
      for (int q = 0; q < n0; q++) issue(q);
    }
    issued = Q < S::R ? Q : S::R;
    const int i = xb + lx;
    const int rr = r0 + lrow;
    const bool live = i < pl.xhi && rr < pl.nr;
    int timeout = 0;
    for (int s = 0; s < ns; s++) {
      for (int q = waited; q <= s + S::W - 1; q++) {
        const unsigned gq = gbase + q;
        if (!mbar_wait_bounded(&bar[gq % S::R], (gq / S::R) & 1, pl.wait_ns)) timeout = 1;
      }
      waited = s + S::W;
      if (!timeout && live) {
        const int m = m0 + s;
        const int j = MA == 1 ? m : rr, k = MA == 1 ? rr : m;
        const long long c = cidx(g, i, j, k);
        const SmemStencil<S::XS, S::PD, S::R> st{lr_ring, lrow * S::BX + lx, (int)((gbase + s) % S::R)};
        lr_cell<ODR, A>(v, c, sA, st, __ldg(cn + c));
      }
      if (__syncthreads_or(timeout)) {
        if (tid == 0) {
          atomicOr(&v.ctl->err, LR_TMA_TIMEOUT_BIT);
          for (int q = waited; q < issued; q++) {  // own loads still in flight
            const unsigned gq = gbase + q;
            mbar_wait_bounded(&bar[gq % S::R], (gq / S::R) & 1, pl.wait_ns);
          }
        }
        __syncthreads();
        return;
      }
      if (s + S::R < Q) {
        if (tid == 0) issue(s + S::R);
        issued = s + S::R + 1;
      }
    }
    gbase += Q;
  }
}

}  // namespace qas
