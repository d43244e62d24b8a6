// qas_api.cu -- C-ABI of libqas (include/qas.h): contexts, ghost-fill maps,
// stage sequencing, the device-resident exec_() loop and its CUDA graphs.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/qas.h"
#include "qas_adjoint_kernels.cuh"
#include "qas_batch.cuh"
#include "qas_dissip.cuh"
#include "qas_kernels.cuh"
#include "qas_tma.cuh"
#include "qas_hall.cuh"
#include "qas_pipe.cuh"

using namespace qas;

namespace {

thread_local std::string g_last_cuda_error;

constexpr int BLK = 128;     // threads per block of the cell kernels
constexpr int NSUB_CAP = 8;  // device-guarded cap on dissipative sub-cycles per step

qas_status cuda_fail(cudaError_t e, const char *what)
{
  g_last_cuda_error = std::string(what) + ": " + cudaGetErrorString(e);
  return e == cudaErrorMemoryAllocation ? QAS_ERR_NOMEM : QAS_ERR_CUDA;
}

#define QAS_CUDA(call)                                 \
  do {                                                 \
    cudaError_t e_ = (call);                           \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
  } while (0)

double hmin(double a, double b) { return (a >= b) ? b : a; }  // common/common_func.h:11-15

// No C++ exception crosses the C-ABI: every entry point's body runs inside QAS_API_TRY /
// QAS_API_CATCH, which turn a failed host allocation into QAS_ERR_NOMEM and any other exception
// of the host code (a thread the file writer could not start, ...) into QAS_ERR_HOST, with the
// message kept for qas_last_cuda_error.
qas_status host_fail(qas_status s, const char *what) noexcept
{
  try {
    g_last_cuda_error = std::string("host exception: ") + what;
  } catch (...) {
  }
  return s;
}

#define QAS_API_TRY try {
#define QAS_API_CATCH                                                               \
  }                                                                                 \
  catch (const std::bad_alloc &) {                                                  \
    return host_fail(QAS_ERR_NOMEM, "host memory allocation failed");               \
  }                                                                                 \
  catch (const std::exception &e_) {                                                \
    return host_fail(QAS_ERR_HOST, e_.what());                                      \
  }                                                                                 \
  catch (...) {                                                                     \
    return host_fail(QAS_ERR_HOST, "unknown exception");                            \
  }

}  // namespace

struct AdjState;  // discrete-adjoint run state (qas_adjoint_api.inc)
static void adj_free(qas_ctx *c);
struct IoState;  // asynchronous output writer (qas_io.inc)
static void io_free(qas_ctx *c);
struct PipeState;  // host round trip with overlapped copies (qas_pipe.inc)
static void pipe_free(qas_ctx *c);
static qas_status pipe_set_items(qas_ctx *c, int value);
static qas_status pipe_set_lanes(qas_ctx *c, int value);

struct qas_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  qas_grid grid{};
  qas_scheme scheme{};
  qas_bc bc{};
  Geo geo{};
  double dr = 0.0;
  // device memory
  void *pool = nullptr;
  size_t pool_bytes = 0;
  int *d_src = nullptr;
  double *d_fac = nullptr;
  Ctl *d_ctl = nullptr;
  DCtl *d_dctl = nullptr;
  unsigned long long *d_scratch = nullptr;
  Ctl *h_ctl = nullptr;  // pinned mirror
  View view{};
  // run state
  bool run_initialised = false;
  // graph of two exec_ steps (odd then even n), keyed by its settings
  cudaGraphExec_t graph = nullptr;
  int graph_flg = -1, graph_rule = -1;
  double graph_cfl = 0.0, graph_nu0 = -1.0, graph_eta0 = -1.0, graph_dtrec = 0.0;
  int graph_nout = 0;
  long long graph_kernels = 0;
  long long launches = 0;
  bool capturing = false;
  qas_status latched = QAS_OK;
  // thread-block tile (x,y,z extents, 128 threads) of every cell kernel, by kernel id
  dim3 tile[32];
  // face sweep form: two kernels with the face states in HBM, or one fused kernel (the
  // default in 3D, set at creation)
  bool fused = false;
  int sweep_seg[3] = {0, 0, 0};  // segment length of the fused y / z sweeps (0: not chosen yet)
  // live per-kernel timing (qas_profile_run): an event pair around every launch
  bool prof = false;
  std::vector<cudaEvent_t> prof_events;
  std::vector<int> prof_kids;  // kernel id of each recorded pair
  double prof_ms[32] = {0};
  long long prof_n[32] = {0};
  AdjState *adj = nullptr;
  IoState *io = nullptr;
  // reconstruction with TMA-staged stencils (qas_tma.cuh): per-axis tensor maps, work plan
  // and persistent grid size; lr_tma_ok = supported by this grid, lr_tma = in use
  bool lr_tma_ok = false, lr_tma = false;
  double *d_phi = nullptr;  // gravitational potential of the gravity drivers (qas_set_gravity)
  // per-cell viscosity / resistivity (qas_set_dissipation) and their setdc maximum
  double *d_nu = nullptr, *d_eta = nullptr;
  double diss_dcmax = 0.0;
  // Hall driver (qas_set_hall): ion inertia length, whistler speed factor, haldt reduction
  bool hall = false;
  double hall_di = 0.0, hall_vphix = 0.0, hall_de = 0.0;
  unsigned long long *d_hvmax = nullptr, *h_hvmax = nullptr;
  LrTmaMaps lr_maps[3];
  LrTmaPlan lr_plan[3];
  int lr_grid[3] = {0, 0, 0};
  PipeState *pipe = nullptr;  // qas_step_host: stage buffers, copy streams, item plan
};

// ---------------------------------------------------------------------------
// ghost-fill maps: replay the reference's fill passes on (source, factor) pairs
// ---------------------------------------------------------------------------
namespace {

struct AxisMap {
  std::vector<int> src;
  std::vector<double> fac;
  explicit AxisMap(int n) : src(n), fac(n, 1.0)
  {
    for (int i = 0; i < n; i++) src[i] = i;
  }
  void write(int dst, int s, double f)
  {
    src[dst] = src[s];
    fac[dst] = f * fac[s];
  }
};

// periodic copies (common/common_func.c:67-74; mpi/common_mpi.c:256-268)
void pass_periodic(AxisMap &m, int n)
{
  for (int i = 0; i < GH; i++) {
    m.write(n - 1 - i, 2 * GH - 1 - i, 1.0);
    m.write(i, n - 2 * GH + i, 1.0);
  }
}

// Neumann/Dirichlet (|dn|=1) and open/zero-fixed (|dn|=2) passes (common_func.c:75-99)
void pass_physical(AxisMap &m, int n, int st, int dn)
{
  if (dn == 1 || dn == -1) {
    for (int i = 0; i < GH; i++) m.write(i, 2 * GH - 1 + st - i, (double)dn);
    for (int i = 0; i < GH - st; i++) m.write(n - 1 - i, n - 2 * GH + st + i, (double)dn);
  } else if (dn == 2 || dn == -2) {
    const double c = 0.25 * (2 + dn);
    for (int i = 0; i < GH; i++) m.write(i, GH, c);
    for (int i = 0; i < GH - st; i++) m.write(n - 1 - i, n - 1 - GH + st, c);
  }
}

bool flag_ok(int dn) { return dn == 0 || dn == 1 || dn == -1 || dn == 2 || dn == -2; }

// Build one axis map.  dim 1/2: the field's own flag decides periodic vs physical
// (bc1d/bc2d).  dim 3: the group's first flag decides the periodic copy for all its
// fields, then the field's physical pass (mpi_sdrv3d + mpi_x/y/zbc3d).
bool build_axis(AxisMap &m, int dim, int n, int st, int dn, int group_dn)
{
  if (!flag_ok(dn) || !flag_ok(group_dn)) return false;
  if (dim <= 2) {
    if (dn == 0)
      pass_periodic(m, n);
    else
      pass_physical(m, n, dim == 1 ? 0 : st, dn);
  } else {
    if (group_dn == 0) pass_periodic(m, n);
    if (dn != 0) pass_physical(m, n, st, dn);
    if (dn == 0 && group_dn != 0) return false;  // ghosts left unset by the reference
  }
  // every source must be a cell this axis' passes never write
  for (int i = 0; i < n; i++)
    if (m.src[m.src[i]] != m.src[i]) return false;
  return true;
}

}  // namespace

// One (group, field, axis) map.  Groups: 0 the state (bound(val)), 1 cell-centre B
// (bound(cx,cy,cz) with bx/by/bz's flags, unstaggered: mhd2d_solve.cpp:75-79), 2 the shock
// detector dv (normal component's flag sign-flipped: mhd2d_solve.cpp:119-125), 3 the Hall
// velocity (the momentum flags, 1D/SERIAL/h-shock/hmhd1d_solve.cpp:185-188).
static bool map_for(int dim, const qas_bc &bc, int G, int f, int a, int n, AxisMap &m)
{
  if (a >= dim) return true;
  const int *dn[3] = {bc.dnx, bc.dny, bc.dnz};
  const int st_state[3][8] = {{0, 0, 0, 0, 1, 0, 0, 0}, {0, 0, 0, 0, 0, 1, 0, 0}, {0, 0, 0, 0, 0, 0, 1, 0}};
  int fdn, gdn, st;
  if (G == 0) {
    fdn = dn[a][f];
    gdn = dn[a][0];
    st = st_state[a][f];
  } else if (G == 1) {
    fdn = dn[a][4 + f];
    gdn = dn[a][4];
    st = 0;
  } else if (G == 2) {
    auto dvflag = [&](int comp) { return comp == a ? -dn[a][1 + comp] : dn[a][1 + comp]; };
    fdn = dvflag(f);
    gdn = dvflag(0);
    st = 0;
  } else {  // G == 3: Hall velocity with the momentum flags, bound(pv,3,&dnxs[1]) (hmhd1d_solve.cpp:185-188)
    fdn = dn[a][1 + f];
    gdn = dn[a][1];
    st = 0;
  }
  return build_axis(m, dim, n, st, fdn, gdn);
}

static qas_status build_maps(qas_ctx *c)
{
  const int dim = c->grid.dim;
  const int nmax = std::max(c->geo.nx, std::max(c->geo.ny, c->geo.nz));
  std::vector<int> src((size_t)4 * 8 * 3 * nmax, 0);
  std::vector<double> fac((size_t)4 * 8 * 3 * nmax, 1.0);
  for (int G = 0; G < 4; G++) {
    if (G == 3 && dim != 1) {  // the Hall driver is 1D; identity maps elsewhere
      for (int f = 0; f < 3; f++)
        for (int a = 0; a < 3; a++)
          for (int i = 0; i < nmax; i++) src[(size_t)((G * 8 + f) * 3 + a) * nmax + i] = i;
      continue;
    }
    const int nf = G == 0 ? 8 : 3;
    for (int f = 0; f < nf; f++) {
      for (int a = 0; a < 3; a++) {
        const int n = c->geo.n[a];
        AxisMap m(n);
        if (!map_for(dim, c->bc, G, f, a, n, m)) return QAS_ERR_INVALID;
        const size_t base = (size_t)((G * 8 + f) * 3 + a) * nmax;
        for (int i = 0; i < n; i++) {
          src[base + i] = m.src[i];
          fac[base + i] = m.fac[i];
        }
      }
    }
  }
  QAS_CUDA(cudaMalloc(&c->d_src, src.size() * sizeof(int)));
  QAS_CUDA(cudaMalloc(&c->d_fac, fac.size() * sizeof(double)));
  QAS_CUDA(cudaMemcpy(c->d_src, src.data(), src.size() * sizeof(int), cudaMemcpyHostToDevice));
  QAS_CUDA(cudaMemcpy(c->d_fac, fac.data(), fac.size() * sizeof(double), cudaMemcpyHostToDevice));
  c->view.maps.src = c->d_src;
  c->view.maps.fac = c->d_fac;
  c->view.maps.nmax = nmax;
  return QAS_OK;
}

// ---------------------------------------------------------------------------
// launch helpers
// ---------------------------------------------------------------------------
namespace {

enum Kid {
  KID_PRIM, KID_DV, KID_LR, KID_FLUX, KID_EMF, KID_UPDATE, KID_BOUND, KID_BEGIN, KID_VMAX, KID_SETDT,
  KID_DVEL, KID_ERES, KID_DFLUX, KID_DUPDATE, KID_DBOUND, KID_DCOPY, KID_DSUB, KID_SWEEP, KID_COUNT
};
const char *const KID_NAMES[KID_COUNT] = {"k_prim", "k_dv", "k_lr", "k_flux", "k_emf", "k_update", "k_bound",
                                          "k_begin_step", "k_vmax", "k_setdt", "k_dvel", "k_eres", "k_dflux",
                                          "k_dupdate", "k_dbound", "k_dcopy", "k_dsub", "k_sweep"};

void prof_mark(qas_ctx *c, int kid)
{
  const size_t n = c->prof_kids.size();
  if (c->prof_events.size() < 2 * (n + 1)) {
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    c->prof_events.push_back(a);
    c->prof_events.push_back(b);
  }
  c->prof_kids.push_back(kid);
  cudaEventRecord(c->prof_events[2 * n], c->stream);
}
void prof_done(qas_ctx *c) { cudaEventRecord(c->prof_events[2 * (c->prof_kids.size() - 1) + 1], c->stream); }

// launch `expr` (one kernel) with optional event timing
#define QL(c, kid, ...)                    \
  do {                                     \
    if ((c)->prof) prof_mark((c), (kid));  \
    __VA_ARGS__;                           \
    if ((c)->prof) prof_done((c));         \
  } while (0)

dim3 cells_grid(const Geo &g, dim3 t = dim3(BLK, 1, 1))
{
  return dim3((g.nx + t.x - 1) / t.x, (g.ny + t.y - 1) / t.y, (g.nz + t.z - 1) / t.z);
}
dim3 update_grid(const Geo &g, dim3 t = dim3(BLK, 1, 1))
{
  const int ny = g.dim >= 2 ? g.ny - 2 * GH + 1 : 1, nz = g.dim >= 3 ? g.nz - 2 * GH + 1 : 1;
  return dim3((g.nx - 2 * GH + 1 + t.x - 1) / t.x, (ny + t.y - 1) / t.y, (nz + t.z - 1) / t.z);
}
dim3 shell_grid(const Geo &g) { return dim3((unsigned)((shell_cells(g) + BLK - 1) / BLK)); }
dim3 interior_grid(const Geo &g)
{
  return dim3((g.nx - 2 * GH + BLK - 1) / BLK, g.dim >= 2 ? g.ny - 2 * GH : 1, g.dim >= 3 ? g.nz - 2 * GH : 1);
}

// ---- reconstruction with TMA-staged stencils: configurations, tensor maps, plans ----
// (tile width TX along x, TR rows, march axis MA) per dim and face axis: 2D x faces stream
// 32x4 tiles; 2D y faces march along y in 128-wide columns; 3D faces use 32x4 columns
// marching along z (x and z faces) or y (y faces).
struct LrCfg {
  int tx, tr, ma;
};
LrCfg lr_cfg(int dim, int a)
{
  if (dim == 2) return a == 0 ? LrCfg{32, 4, 2} : LrCfg{128, 1, 1};
  return a == 1 ? LrCfg{32, 4, 1} : LrCfg{32, 4, 2};
}
void *lr_tma_fn(int dim, int a)
{
  if (dim == 2) return a == 0 ? (void *)k_lr_tma<4, 0, 32, 4, 2> : (void *)k_lr_tma<4, 1, 128, 1, 1>;
  if (a == 0) return (void *)k_lr_tma<4, 0, 32, 4, 2>;
  if (a == 1) return (void *)k_lr_tma<4, 1, 32, 4, 1>;
  return (void *)k_lr_tma<4, 2, 32, 4, 2>;
}
size_t lr_tma_smem(int dim, int a)
{
  if (dim == 2) return a == 0 ? LrTmaShape<0, 32, 4>::SMEM : LrTmaShape<1, 128, 1>::SMEM;
  if (a == 0) return LrTmaShape<0, 32, 4>::SMEM;
  return a == 1 ? LrTmaShape<1, 32, 4>::SMEM : LrTmaShape<2, 32, 4>::SMEM;
}

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    cudaGetLastError();
  });
  return fn;
}

// tensor maps of the seven stencil fields of every axis and the per-axis work plans; false
// when the grid cannot use them (1D, or an odd padded x extent: TMA rows must be 16-byte
// multiples), in which case k_lr reads its stencils from global memory
bool setup_lr_tma(qas_ctx *c)
{
  const Geo &g = c->geo;
  if (g.dim < 2 || (g.nx % 2) != 0) return false;
  PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc) return false;
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device) != cudaSuccess || sms < 1) {
    cudaGetLastError();
    return false;
  }
  const View &v = c->view;
  double *vel[3] = {v.vx, v.vy, v.vz}, *ccb[3] = {v.cx, v.cy, v.cz};
  for (int a = 0; a < g.dim; a++) {
    const LrCfg k = lr_cfg(g.dim, a);
    const bool xs = a == 0;
    const int b = (a + 1) % 3, cc = (a + 2) % 3;
    double *fld[7] = {v.u[0], vel[a], vel[b], vel[cc], ccb[b], ccb[cc], v.pr};
    const cuuint64_t dims[3] = {(cuuint64_t)g.nx, (cuuint64_t)g.ny, (cuuint64_t)g.nz};
    const cuuint64_t strides[2] = {(cuuint64_t)g.nx * 8, (cuuint64_t)g.nx * g.ny * 8};
    const cuuint32_t box[3] = {(cuuint32_t)(k.tx + (xs ? 4 : 0)), (cuuint32_t)(k.ma == 1 ? 1 : k.tr),
                               (cuuint32_t)(k.ma == 1 ? k.tr : 1)};
    const cuuint32_t estr[3] = {1, 1, 1};
    for (int f = 0; f < 7; f++) {
      if (enc(&c->lr_maps[a].m[f], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, fld[f], dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
    }
    void *fn = lr_tma_fn(g.dim, a);
    const size_t smem = lr_tma_smem(g.dim, a);
    int occ = 0;
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, k.tx * k.tr, smem) != cudaSuccess || occ < 1) {
      cudaGetLastError();
      return false;
    }
    LrTmaPlan &p = c->lr_plan[a];
    p.xlo = xs ? 2 : 0;
    p.xhi = xs ? g.nx - 2 : g.nx;
    p.xt = (p.xhi - p.xlo + k.tx - 1) / k.tx;
    p.nr = k.ma == 1 ? g.nz : g.ny;
    p.rt = (p.nr + k.tr - 1) / k.tr;
    const int nm = k.ma == 1 ? g.ny : g.nz;
    const bool march = a == k.ma;
    p.mlo = march ? 2 : 0;
    p.mhi = march ? nm - 2 : nm;
    const int len = p.mhi - p.mlo;
    const long long slots = (long long)sms * occ;
    // segment length: fewest plane-steps per CTA over the persistent waves (the 4 halo
    // planes of a marching segment cost their loads, about a quarter of a computed plane)
    double best = 1e300;
    int bseg = len;
    for (int ms = 1; ms <= len && ms <= 512; ms++) {
      const int seg = (len + ms - 1) / ms;
      const long long items = (long long)p.xt * p.rt * ((len + seg - 1) / seg);
      const long long waves = (items + slots - 1) / slots;
      const double cost = (double)waves * (seg + (march ? 1.0 : 0.0));
      if (cost < best - 1e-9) {
        best = cost;
        bseg = seg;
      }
    }
    p.seg = bseg;
    p.wait_ns = 2000000000ull;  // 2 s of device time per mbarrier wait
    p.stall_plane = -1;
    p.ms = (len + bseg - 1) / bseg;
    p.items = p.xt * p.rt * p.ms;
    c->lr_grid[a] = (int)std::min<long long>(p.items, slots);
  }
  return true;
}

void launch_lr_tma(qas_ctx *c, int a)
{
  const int dim = c->geo.dim;
  const size_t sm = lr_tma_smem(dim, a);
  const dim3 grid((unsigned)c->lr_grid[a]);
  if (dim == 2) {
    if (a == 0)
      QL(c, KID_LR, k_lr_tma<4, 0, 32, 4, 2><<<grid, 128, sm, c->stream>>>(c->view, c->lr_maps[0], c->lr_plan[0]));
    else
      QL(c, KID_LR, k_lr_tma<4, 1, 128, 1, 1><<<grid, 128, sm, c->stream>>>(c->view, c->lr_maps[1], c->lr_plan[1]));
  } else if (a == 0) {
    QL(c, KID_LR, k_lr_tma<4, 0, 32, 4, 2><<<grid, 128, sm, c->stream>>>(c->view, c->lr_maps[0], c->lr_plan[0]));
  } else if (a == 1) {
    QL(c, KID_LR, k_lr_tma<4, 1, 32, 4, 1><<<grid, 128, sm, c->stream>>>(c->view, c->lr_maps[1], c->lr_plan[1]));
  } else {
    QL(c, KID_LR, k_lr_tma<4, 2, 32, 4, 2><<<grid, 128, sm, c->stream>>>(c->view, c->lr_maps[2], c->lr_plan[2]));
  }
}

template <int ODR>
void launch_lr(qas_ctx *c, int a)
{
  if (ODR == 4 && c->lr_tma) {
    launch_lr_tma(c, a);
    return;
  }
  const dim3 grid = cells_grid(c->geo, c->tile[KID_LR]), blk = c->tile[KID_LR];
  if (c->view.recon == 1) {
    if (a == 0) QL(c, KID_LR, k_lr<ODR, 0, 1><<<grid, blk, 0, c->stream>>>(c->view));
    if (a == 1) QL(c, KID_LR, k_lr<ODR, 1, 1><<<grid, blk, 0, c->stream>>>(c->view));
    if (a == 2) QL(c, KID_LR, k_lr<ODR, 2, 1><<<grid, blk, 0, c->stream>>>(c->view));
    return;
  }
  if (c->view.recon == 2) {
    if (a == 0) QL(c, KID_LR, k_lr<ODR, 0, 2><<<grid, blk, 0, c->stream>>>(c->view));
    if (a == 1) QL(c, KID_LR, k_lr<ODR, 1, 2><<<grid, blk, 0, c->stream>>>(c->view));
    if (a == 2) QL(c, KID_LR, k_lr<ODR, 2, 2><<<grid, blk, 0, c->stream>>>(c->view));
    return;
  }
  if (a == 0) QL(c, KID_LR, k_lr<ODR, 0><<<grid, blk, 0, c->stream>>>(c->view));
  if (a == 1) QL(c, KID_LR, k_lr<ODR, 1><<<grid, blk, 0, c->stream>>>(c->view));
  if (a == 2) QL(c, KID_LR, k_lr<ODR, 2><<<grid, blk, 0, c->stream>>>(c->view));
}
template <int RMN>
void launch_flux(qas_ctx *c, int a)
{
  if constexpr (RMN == 3) {
    if (a == 0) QL(c, KID_FLUX, k_flux_mlau<0><<<cells_grid(c->geo, c->tile[KID_FLUX]), c->tile[KID_FLUX], 0, c->stream>>>(c->view));
    if (a == 1) QL(c, KID_FLUX, k_flux_mlau<1><<<cells_grid(c->geo, c->tile[KID_FLUX]), c->tile[KID_FLUX], 0, c->stream>>>(c->view));
    if (a == 2) QL(c, KID_FLUX, k_flux_mlau<2><<<cells_grid(c->geo, c->tile[KID_FLUX]), c->tile[KID_FLUX], 0, c->stream>>>(c->view));
    return;
  } else {
    if (a == 0) QL(c, KID_FLUX, k_flux<RMN, 0><<<cells_grid(c->geo, c->tile[KID_FLUX]), c->tile[KID_FLUX], 0, c->stream>>>(c->view));
    if (a == 1) QL(c, KID_FLUX, k_flux<RMN, 1><<<cells_grid(c->geo, c->tile[KID_FLUX]), c->tile[KID_FLUX], 0, c->stream>>>(c->view));
    if (a == 2) QL(c, KID_FLUX, k_flux<RMN, 2><<<cells_grid(c->geo, c->tile[KID_FLUX]), c->tile[KID_FLUX], 0, c->stream>>>(c->view));
  }
}

// segment length of the y / z sweeps: fewest cell computations per resident block slot over
// the waves of blocks (each segment recomputes the cell before its first face)
int sweep_seg(qas_ctx *c, int a, const void *fn)
{
  if (c->sweep_seg[a] > 0) return c->sweep_seg[a];
  const Geo &g = c->geo;
  int dev = 0, sms = 148, occ = 1;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, 128, 0) != cudaSuccess || occ < 1) {
    cudaGetLastError();
    occ = 1;
  }
  const long long colb = ((long long)g.nx * (a == 1 ? g.nz : g.ny) + 127) / 128;
  const long long slots = (long long)sms * occ;
  const int len = g.n[a] - 5;  // faces 3 .. n-3
  double best = 1e300;
  int bseg = len;
  for (int ns = 1; ns <= len; ns++) {
    const int seg = (len + ns - 1) / ns;
    const long long blocks = colb * ((len + seg - 1) / seg);
    const double cost = (double)((blocks + slots - 1) / slots) * (seg + 1);
    if (cost < best - 1e-9) {
      best = cost;
      bseg = seg;
    }
  }
  c->sweep_seg[a] = bseg;
  return bseg;
}

// shared-memory carveout hint of the fused sweeps (percent of the SM's maximum; -1: the driver's
// choice): the y / z sweeps read each stencil plane five times along their march, from L1
// when the rest of the SM's 256 KB is left to it
#ifndef QAS_SWEEP_CARVEOUT
#define QAS_SWEEP_CARVEOUT -1
#endif
// choose the y / z segment lengths outside any stream capture (occupancy query); the fused
// sweeps are built for 4th-order interpolation only (other orders take the two-kernel form)
template <int RMN>
void sweep_prepare_t(qas_ctx *c)
{
  if (QAS_SWEEP_CARVEOUT >= 0) {
    const void *fns[6] = {(const void *)k_sweep_x<4, RMN, 0>, (const void *)k_sweep_m<4, RMN, 1, 0>,
                          (const void *)k_sweep_m<4, RMN, 2, 0>, (const void *)k_sweep_x<4, RMN, -1>,
                          (const void *)k_sweep_m<4, RMN, 1, -1>, (const void *)k_sweep_m<4, RMN, 2, -1>};
    for (const void *f : fns)
      cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, QAS_SWEEP_CARVEOUT);
    cudaGetLastError();
  }
  if (c->geo.dim >= 2) sweep_seg(c, 1, (const void *)k_sweep_m<4, RMN, 1, 0>);
  if (c->geo.dim >= 3) sweep_seg(c, 2, (const void *)k_sweep_m<4, RMN, 2, 0>);
}
void sweep_prepare(qas_ctx *c)
{
  if (c->scheme.odr != 4) return;
  switch (c->scheme.rmn) {
    case 0: sweep_prepare_t<0>(c); break;
    case 1: sweep_prepare_t<1>(c); break;
    case 2: sweep_prepare_t<2>(c); break;
    default: sweep_prepare_t<3>(c); break;
  }
}

template <int RMN, int PR>
void launch_sweep_pr(qas_ctx *c, int a)
{
  const Geo &g = c->geo;
  if (a == 0) {
    // warp w takes flattened cells [31w, 31w+32); the last cell needing a flux is total-1
    const long long total = (long long)(g.nx - 4) * g.ny * g.nz;
    const long long nwarps = (total - 2) / 31 + 1;
    const unsigned nb = (unsigned)((nwarps + 3) / 4);
    QL(c, KID_SWEEP, k_sweep_x<4, RMN, PR><<<nb, 128, 0, c->stream>>>(c->view, nwarps));
    return;
  }
  const unsigned colb = (unsigned)(((long long)g.nx * (a == 1 ? g.nz : g.ny) + 127) / 128);
  const int len = g.n[a] - 5;
  if (a == 1) {
    const int seg = sweep_seg(c, 1, (const void *)k_sweep_m<4, RMN, 1, 0>);
    QL(c, KID_SWEEP, k_sweep_m<4, RMN, 1, PR><<<dim3(colb, (len + seg - 1) / seg), 128, 0, c->stream>>>(c->view, seg));
  } else {
    const int seg = sweep_seg(c, 2, (const void *)k_sweep_m<4, RMN, 2, 0>);
    QL(c, KID_SWEEP, k_sweep_m<4, RMN, 2, PR><<<dim3(colb, (len + seg - 1) / seg), 128, 0, c->stream>>>(c->view, seg));
  }
}
template <int RMN>
void launch_sweep(qas_ctx *c, int a)
{
  if (c->view.recon != 2)
    launch_sweep_pr<RMN, 0>(c, a);
  else
    launch_sweep_pr<RMN, -1>(c, a);
}

// HMHD1D::crcte on the by and bz fluxes (1D Hall driver with electron inertia), after the
// flux and before the update of ideal() and hall_(); scratch = the face-state arrays, which
// the stage no longer needs at that point
long long launch_crcte(qas_ctx *c)
{
  if (!(c->hall && c->hall_de != 0 && c->geo.dim == 1)) return 0;
  View &v = c->view;
  const double fac = (c->hall_de * c->hall_de) / (c->grid.dx * c->grid.dx);
  const int *dn = c->bc.dnx;
  double *w[5] = {v.vl[0], v.vl[1], v.vl[2], v.vl[3], v.vl[4]};
  for (int q = 0; q < 2; q++) {
    double *fbt = v.f[0][5 + q];
    const double *bt = v.u[5 + q];
    const int flag = dn[1] * dn[5 + q];
    switch (c->scheme.odr) {
#define QAS_CRCTE(O)                                                                                  \
  case O:                                                                                             \
    k_crcte<O><<<1, 1024, 0, c->stream>>>(v, fbt, v.f[0][7], bt, flag, fac, w[0], w[1], w[2], w[3], w[4]); \
    break;
      QAS_CRCTE(1)
      QAS_CRCTE(2)
      QAS_CRCTE(3)
      default:
      QAS_CRCTE(4)
#undef QAS_CRCTE
    }
  }
  return 2;
}

// one SSP-RK stage in three phases (a domain split into slabs exchanges ghost planes
// between them): primitives + cell-centre B; the shock detector; sweeps, EMF, update, fill
template <int ODR>
long long stage_prim(qas_ctx *c)
{
  QL(c, KID_PRIM, k_prim<ODR><<<cells_grid(c->geo, c->tile[KID_PRIM]), c->tile[KID_PRIM], 0, c->stream>>>(c->view));
  return 1;
}
bool stage_has_dv(const qas_ctx *c) { return c->scheme.rmn >= 2 && c->geo.dim >= 2; }
long long stage_dv(qas_ctx *c)
{
  if (!stage_has_dv(c)) return 0;
  QL(c, KID_DV, k_dv<<<cells_grid(c->geo, c->tile[KID_DV]), c->tile[KID_DV], 0, c->stream>>>(c->view));
  return 1;
}
template <int ODR>
long long stage_rest(qas_ctx *c, double c0, double c1)
{
  const Geo &g = c->geo;
  long long nk = 0;
  for (int a = 0; a < g.dim; a++) {
    if constexpr (ODR == 4) {
      if (c->fused) {
        switch (c->scheme.rmn) {
          case 0: launch_sweep<0>(c, a); break;
          case 1: launch_sweep<1>(c, a); break;
          case 2: launch_sweep<2>(c, a); break;
          default: launch_sweep<3>(c, a); break;
        }
        nk += 1;
        continue;
      }
    }
    launch_lr<ODR>(c, a);
    switch (c->scheme.rmn) {
      case 0: launch_flux<0>(c, a); break;
      case 1: launch_flux<1>(c, a); break;
      case 2: launch_flux<2>(c, a); break;
      default: launch_flux<3>(c, a); break;
    }
    nk += 2;
  }
  nk += launch_crcte(c);  // 1D Hall driver with electron inertia (hmhd1d_solve.cpp:98-108)
  if (g.dim >= 2) {
    QL(c, KID_EMF, k_emf<ODR><<<cells_grid(g, c->tile[KID_EMF]), c->tile[KID_EMF], 0, c->stream>>>(c->view));
    nk++;
  }
  QL(c, KID_UPDATE, k_update<ODR><<<update_grid(g, c->tile[KID_UPDATE]), c->tile[KID_UPDATE], 0, c->stream>>>(c->view, c0, c1));
  QL(c, KID_BOUND, k_bound<<<shell_grid(g), BLK, 0, c->stream>>>(c->view));
  nk += 2;
  return nk;
}

template <int ODR>
long long stage_odr(qas_ctx *c, double c0, double c1)
{
  long long nk = stage_prim<ODR>(c);
  nk += stage_dv(c);
  return nk + stage_rest<ODR>(c, c0, c1);
}

// phase helpers by run-time order
long long stage_prim_any(qas_ctx *c)
{
  switch (c->scheme.odr) {
    case 1: return stage_prim<1>(c);
    case 2: return stage_prim<2>(c);
    case 3: return stage_prim<3>(c);
    default: return stage_prim<4>(c);
  }
}
long long stage_rest_any(qas_ctx *c, double c0, double c1)
{
  switch (c->scheme.odr) {
    case 1: return stage_rest<1>(c, c0, c1);
    case 2: return stage_rest<2>(c, c0, c1);
    case 3: return stage_rest<3>(c, c0, c1);
    default: return stage_rest<4>(c, c0, c1);
  }
}

// rk_fac table of mhd2d_solve.cpp:7 for the context's R_K
void rk_factors(int R_K, int rk, double &c0, double &c1)
{
  const double t[3][2] = {{0.0, 1.0}, {0.5 + (R_K - 2) * 0.25, 0.5 - (R_K - 2) * 0.25}, {1. / 3., 2. / 3.}};
  c0 = t[rk][0];
  c1 = t[rk][1];
}

// ideal(dt) on the device, dt and dt/dx already in the control block
long long launch_ideal(qas_ctx *c)
{
  long long nk = 0;
  const size_t bytes = (size_t)c->geo.nd * sizeof(double);
  for (int m = 0; m < 8; m++) cudaMemcpyAsync(c->view.u0[m], c->view.u[m], bytes, cudaMemcpyDeviceToDevice, c->stream);
  for (int rk = 0; rk < c->scheme.rk; rk++) {
    double c0, c1;
    rk_factors(c->scheme.rk, rk, c0, c1);
    switch (c->scheme.odr) {
      case 1: nk += stage_odr<1>(c, c0, c1); break;
      case 2: nk += stage_odr<2>(c, c0, c1); break;
      case 3: nk += stage_odr<3>(c, c0, c1); break;
      default: nk += stage_odr<4>(c, c0, c1); break;
    }
  }
  return nk;
}

template <int ODR>
long long dsptv_odr(qas_ctx *c, int nc, double nu0, double eta0)
{
  const Geo &g = c->geo;
  const double idx = 1.0 / c->grid.dx, idy = 1.0 / c->grid.dy;
  const double idz = g.dim == 3 ? 1.0 / c->grid.dz : 0.0;
  long long nk = 0;
  QL(c, KID_DBOUND, k_dbound<<<shell_grid(g), BLK, 0, c->stream>>>(c->view, c->d_dctl, nc));
  QL(c, KID_DCOPY, k_dcopy<<<(unsigned)((g.nd + 255) / 256), 256, 0, c->stream>>>(c->view, c->d_dctl, nc));
  nk += 2;
  for (int rk = 0; rk < c->scheme.rk; rk++) {
    double c0, c1;
    rk_factors(c->scheme.rk, rk, c0, c1);
    QL(c, KID_DVEL, k_dvel<<<cells_grid(g), BLK, 0, c->stream>>>(c->view, c->d_dctl, nc));
    QL(c, KID_ERES, k_eres<ODR><<<cells_grid(g), BLK, 0, c->stream>>>(c->view, c->d_dctl, nc, eta0, idx, idy, idz));
    QL(c, KID_DFLUX,
       k_dflux<ODR><<<cells_grid(g), BLK, 0, c->stream>>>(c->view, c->d_dctl, nc, nu0, idx, idy, idz));
    QL(c, KID_DUPDATE, k_dupdate<ODR><<<update_grid(g), BLK, 0, c->stream>>>(c->view, c->d_dctl, nc, c0, c1));
    QL(c, KID_DBOUND, k_dbound<<<shell_grid(g), BLK, 0, c->stream>>>(c->view, c->d_dctl, nc));
    nk += 5;
  }
  return nk;
}

long long launch_dsptv(qas_ctx *c, int nc, double nu0, double eta0)
{
  switch (c->scheme.odr) {
    case 1: return dsptv_odr<1>(c, nc, nu0, eta0);
    case 2: return dsptv_odr<2>(c, nc, nu0, eta0);
    case 3: return dsptv_odr<3>(c, nc, nu0, eta0);
    default: return dsptv_odr<4>(c, nc, nu0, eta0);
  }
}

// setdc + sub-cycled dsptv after ideal (dmhd2d_class.cpp:19-26, dmhd3d_class.cpp:20-28),
// device-guarded
bool diss_arrays(const qas_ctx *c) { return c->view.nu != nullptr; }

long long launch_dissipate(qas_ctx *c, double nu0, double eta0)
{
  // setdc's maximum of max(2 nu, eta) over every cell: the installed profiles, else uniform
  const double dcmax0 = (2 * nu0 >= eta0) ? 2 * nu0 : eta0;
  const double dcmax = diss_arrays(c) ? c->diss_dcmax : (dcmax0 > 0.0 ? dcmax0 : 0.0);
  if (!(dcmax > 1e-15)) return 0;
  const double idz = c->grid.dim == 3 ? 1.0 / c->grid.dz : 0.0;
  QL(c, KID_DSUB, k_dsub_setup<<<1, 1, 0, c->stream>>>(c->view, c->d_dctl, dcmax, c->dr, 1.0 / c->grid.dx,
                                                       1.0 / c->grid.dy, NSUB_CAP, idz));
  long long nk = 1;
  for (int nc = 0; nc < NSUB_CAP; nc++) nk += launch_dsptv(c, nc, nu0, eta0);
  return nk;
}

long long launch_setdt(qas_ctx *c, double cfl, int rule, double dtrec, int nout)
{
  QL(c, KID_VMAX, k_vmax_reset<<<1, 1, 0, c->stream>>>(c->view));
  QL(c, KID_VMAX, k_vmax<<<interior_grid(c->geo), BLK, 0, c->stream>>>(c->view));
  QL(c, KID_SETDT, k_setdt<<<1, 1, 0, c->stream>>>(c->view, cfl, c->dr, rule, dtrec, nout));
  return 3;
}

// one exec_ iteration
// one hall_(dt) call (1D/SERIAL/h-shock/hmhd1d_solve.cpp:138-264): ut = u, R_K stages
long long launch_hall(qas_ctx *c, double dt)
{
  const Geo &g = c->geo;
  const size_t bytes = (size_t)g.nd * sizeof(double);
  for (int m = 0; m < 8; m++) cudaMemcpyAsync(c->view.u0[m], c->view.u[m], bytes, cudaMemcpyDeviceToDevice, c->stream);
  const double dtdx = dt / c->grid.dx, idx = 1.0 / c->grid.dx;
  const unsigned nb = (unsigned)((g.nx + BLK - 1) / BLK);
  long long nk = 0;
  for (int rk = 0; rk < c->scheme.rk; rk++) {
    double c0, c1;
    rk_factors(c->scheme.rk, rk, c0, c1);
    k_hvel<<<nb, BLK, 0, c->stream>>>(c->view, c->hall_di, idx);
    switch (c->scheme.odr) {
      case 1: k_hlr<1><<<nb, BLK, 0, c->stream>>>(c->view); break;
      case 2: k_hlr<2><<<nb, BLK, 0, c->stream>>>(c->view); break;
      case 3: k_hlr<3><<<nb, BLK, 0, c->stream>>>(c->view); break;
      default: k_hlr<4><<<nb, BLK, 0, c->stream>>>(c->view); break;
    }
    k_hflux<<<nb, BLK, 0, c->stream>>>(c->view, c->hall_vphix);
    nk += launch_crcte(c);  // hmhd1d_solve.cpp:232-240
    switch (c->scheme.odr) {
      case 1: k_hupdate<1><<<nb, BLK, 0, c->stream>>>(c->view, dtdx, c0, c1); break;
      case 2: k_hupdate<2><<<nb, BLK, 0, c->stream>>>(c->view, dtdx, c0, c1); break;
      case 3: k_hupdate<3><<<nb, BLK, 0, c->stream>>>(c->view, dtdx, c0, c1); break;
      default: k_hupdate<4><<<nb, BLK, 0, c->stream>>>(c->view, dtdx, c0, c1); break;
    }
    k_bound<<<shell_grid(g), BLK, 0, c->stream>>>(c->view);
    nk += 5;
  }
  return nk;
}

// the Hall sub-cycles of HMHD1D::exec_ (1D/SERIAL/h-shock/hmhd1d_class.cpp:26-33): hmax =
// 1 + (int)(dt/haldt()) with haldt = cfl*dx/max(1, max |hx| + vphix |bx/ro|), read back to the
// host (1D grids are small; this is one short synchronisation per step)
long long launch_hall_subcycles(qas_ctx *c, double cfl)
{
  static const double one = 1.0;
  cudaMemcpyAsync(c->d_hvmax, &one, sizeof(one), cudaMemcpyHostToDevice, c->stream);
  const unsigned nb = (unsigned)((c->geo.nx - 2 * GH + BLK - 1) / BLK);
  k_hall_vmax<<<nb, BLK, 0, c->stream>>>(c->view, c->hall_vphix, c->d_hvmax);
  cudaMemcpyAsync(c->h_ctl, c->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, c->stream);
  cudaMemcpyAsync(c->h_hvmax, c->d_hvmax, sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess || c->h_ctl->done) return 1;
  const double dt = c->h_ctl->dt;
  const double vmax = __builtin_bit_cast(double, *c->h_hvmax);
  const double haldt = cfl * c->grid.dx / vmax;
  const int hmax = 1 + (int)(dt / haldt);
  long long nk = 1;
  for (int h = 0; h < hmax; h++) {
    nk += launch_hall(c, dt / hmax);
    k_bound<<<shell_grid(c->geo), BLK, 0, c->stream>>>(c->view);
    nk++;
  }
  return nk;
}

bool hall_active(const qas_ctx *c) { return c->hall && c->hall_di != 0; }

long long launch_exec_step(qas_ctx *c, const qas_run_opts &o, int n_after)
{
  long long nk = 0;
  QL(c, KID_BEGIN, k_begin_step<<<1, 1, 0, c->stream>>>(c->view, o.stop_rule == 2 ? 0 : 1));
  QL(c, KID_BOUND, k_bound<<<shell_grid(c->geo), BLK, 0, c->stream>>>(c->view));
  if (hall_active(c)) nk += launch_hall_subcycles(c, o.cfl);
  nk += 2 + launch_ideal(c);
  if (c->grid.dim >= 2 && (o.nu0 > 0.0 || o.eta0 > 0.0 || diss_arrays(c))) nk += launch_dissipate(c, o.nu0, o.eta0);
  if (o.flg && (n_after % 2 == 0)) nk += launch_setdt(c, o.cfl, o.stop_rule, o.dtrec, o.nout);
  return nk;
}

qas_status check_launch(qas_ctx *c)
{
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "kernel launch");
  return QAS_OK;
}

qas_status read_ctl(qas_ctx *c)
{
  QAS_CUDA(cudaMemcpyAsync(c->h_ctl, c->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, c->stream));
  QAS_CUDA(cudaStreamSynchronize(c->stream));
  if (c->h_ctl->err & LR_TMA_TIMEOUT_BIT) return QAS_ERR_TIMEOUT;
  if (c->h_ctl->err & 4) return QAS_ERR_UNSUPPORTED;
  if (c->h_ctl->err & 1) return QAS_ERR_NONFINITE;
  return QAS_OK;
}

qas_status write_ctl(qas_ctx *c)
{
  QAS_CUDA(cudaMemcpyAsync(c->d_ctl, c->h_ctl, sizeof(Ctl), cudaMemcpyHostToDevice, c->stream));
  QAS_CUDA(cudaStreamSynchronize(c->stream));
  return QAS_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// C-ABI
// ---------------------------------------------------------------------------
extern "C" {

const char *qas_status_str(qas_status s)
{
  switch (s) {
    case QAS_OK: return "ok";
    case QAS_ERR_INVALID: return "invalid argument";
    case QAS_ERR_CUDA: return "CUDA error";
    case QAS_ERR_NOMEM: return "out of memory";
    case QAS_ERR_NONFINITE: return "non-finite or non-positive state detected on the device";
    case QAS_ERR_TIMEOUT: return "bounded device wait timed out";
    case QAS_ERR_UNSUPPORTED: return "unsupported configuration";
    case QAS_ERR_NO_DEVICE: return "no CUDA device";
    case QAS_ERR_IO: return "file I/O failed";
    case QAS_ERR_HOST: return "exception in the library's host code";
  }
  return "unknown status";
}

int qas_abi_version(void) { return QAS_ABI_VERSION; }

const char *qas_last_cuda_error(void) { return g_last_cuda_error.c_str(); }

qas_status qas_create(qas_ctx **out, const qas_grid *grid, const qas_scheme *scheme, const qas_bc *bc, int device)
{
  QAS_API_TRY
  if (!out || !grid || !scheme || !bc) return QAS_ERR_INVALID;
  *out = nullptr;
  const qas_grid &gr = *grid;
  if (gr.dim < 1 || gr.dim > 3 || gr.nxm < 4) return QAS_ERR_INVALID;
  if (gr.dim >= 2 && gr.nym < 4) return QAS_ERR_INVALID;
  if (gr.dim >= 3 && gr.nzm < 4) return QAS_ERR_INVALID;
  if (!(gr.dx > 0) || (gr.dim >= 2 && !(gr.dy > 0)) || (gr.dim >= 3 && !(gr.dz > 0))) return QAS_ERR_INVALID;
  if (scheme->rmn < 0 || scheme->rmn > 3 || scheme->odr < 1 || scheme->odr > 4 || scheme->rk < 1 ||
      scheme->rk > 3 || scheme->char_mode < 0 || scheme->char_mode > 2)
    return QAS_ERR_INVALID;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return QAS_ERR_NO_DEVICE;
  qas_ctx *c = new (std::nothrow) qas_ctx();
  if (!c) return QAS_ERR_NOMEM;
  c->grid = gr;
  c->scheme = *scheme;
  c->bc = *bc;
  if (device >= 0) {
    if (cudaSetDevice(device) != cudaSuccess) {
      delete c;
      return QAS_ERR_NO_DEVICE;
    }
    c->device = device;
  } else {
    cudaGetDevice(&c->device);
  }
  Geo &g = c->geo;
  g.dim = gr.dim;
  g.nx = gr.nxm + 2 * GH;
  g.ny = gr.dim >= 2 ? gr.nym + 2 * GH : 1;
  g.nz = gr.dim >= 3 ? gr.nzm + 2 * GH : 1;
  g.nd = (long long)g.nx * g.ny * g.nz;
  g.s[0] = 1;
  g.s[1] = g.nx;
  g.s[2] = (long long)g.nx * g.ny;
  g.n[0] = g.nx;
  g.n[1] = g.ny;
  g.n[2] = g.nz;
  c->dr = gr.dim == 1 ? gr.dx : (gr.dim == 2 ? hmin(gr.dx, gr.dy) : hmin(hmin(gr.dx, gr.dy), gr.dz));

  qas_status st = QAS_OK;
  auto fail = [&](qas_status s) {
    qas_destroy(c);
    return s;
  };
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(QAS_ERR_CUDA);
  {
    const dim3 t = gr.dim == 1 ? dim3(128, 1, 1) : (gr.dim == 2 ? dim3(32, 4, 1) : dim3(32, 2, 2));
    for (int q = 0; q < 32; q++) c->tile[q] = t;
  }
  if ((st = build_maps(c)) != QAS_OK) return fail(st);

  // one pool for every field array, 256-byte aligned
  const size_t arr = ((size_t)g.nd * sizeof(double) + 255) & ~(size_t)255;
  const int n_arrays = 8 + 8 + 7 + 3 + 14 + 4 + 24 + 6 + 3;
  c->pool_bytes = arr * n_arrays;
  if (cudaMalloc(&c->pool, c->pool_bytes) != cudaSuccess) {
    cudaGetLastError();
    return fail(QAS_ERR_NOMEM);
  }
  if (cudaMemsetAsync(c->pool, 0, c->pool_bytes, c->stream) != cudaSuccess) return fail(QAS_ERR_CUDA);
  char *p = (char *)c->pool;
  auto take = [&]() {
    double *r = (double *)p;
    p += arr;
    return r;
  };
  View &v = c->view;
  v.g = g;
  v.rmn = scheme->rmn;
  v.odr = scheme->odr;
  v.rk = scheme->rk;
  v.ctw = scheme->ctw ? 1 : 0;
  v.recon = scheme->char_mode;
  v.gam = gr.gam;
  v.dx = gr.dx;
  v.dy = gr.dim >= 2 ? gr.dy : 1.0;
  v.dz = gr.dim >= 3 ? gr.dz : 1.0;
  v.dr = c->dr;
  for (int m = 0; m < 8; m++) v.u[m] = take();
  for (int m = 0; m < 8; m++) v.u0[m] = take();
  v.vx = take(); v.vy = take(); v.vz = take(); v.pr = take();
  v.cx = take(); v.cy = take(); v.cz = take();
  for (int a = 0; a < 3; a++) v.dv[a] = take();
  for (int m = 0; m < 7; m++) v.vl[m] = take();
  for (int m = 0; m < 7; m++) v.vr[m] = take();
  for (int t = 0; t < 2; t++) v.ql[t] = take();
  for (int t = 0; t < 2; t++) v.qr[t] = take();
  for (int a = 0; a < 3; a++)
    for (int m = 0; m < 8; m++) v.f[a][m] = take();
  for (int a = 0; a < 3; a++)
    for (int t = 0; t < 2; t++) v.fc[a][t] = take();
  v.ex = take(); v.ey = take(); v.ez = take();

  if (cudaMalloc(&c->d_ctl, sizeof(Ctl)) != cudaSuccess) return fail(QAS_ERR_NOMEM);
  if (cudaMalloc(&c->d_dctl, sizeof(DCtl)) != cudaSuccess) return fail(QAS_ERR_NOMEM);
  if (cudaMalloc(&c->d_scratch, 64) != cudaSuccess) return fail(QAS_ERR_NOMEM);
  if (cudaMallocHost(&c->h_ctl, sizeof(Ctl)) != cudaSuccess) return fail(QAS_ERR_NOMEM);
  memset(c->h_ctl, 0, sizeof(Ctl));
  c->h_ctl->nmax = INT_MAX;
  c->h_ctl->tmax = INFINITY;
  c->h_ctl->first = 1;
  v.ctl = c->d_ctl;
  // staged form available, global-load form the default: on B200 the reconstruction is bound
  // by FP64 dependency latency, and the staged form measured 9-35 % slower per launch
  c->lr_tma_ok = scheme->odr == 4 && setup_lr_tma(c);
  c->lr_tma = false;
  // face sweep form: fused (face states never in HBM) in 3D, where it measured faster on B200
  // (KH 256^3, MLAU: 2.78 ms per sweep against 1.90 + 1.21 ms for the two kernels, and a cooler
  // step under the power cap); two kernels in 1D/2D, where the y sweep has too few columns to
  // march long segments (OT 1024^2: 0.164 against 0.102 + 0.050 ms)
  c->fused = g.dim == 3;
  if (c->fused) sweep_prepare(c);
  if (cudaMemsetAsync(c->d_dctl, 0, sizeof(DCtl), c->stream) != cudaSuccess) return fail(QAS_ERR_CUDA);
  if ((st = write_ctl(c)) != QAS_OK) return fail(st);
  *out = c;
  return QAS_OK;
  QAS_API_CATCH
}

qas_status qas_destroy(qas_ctx *c)
{
  QAS_API_TRY
  if (!c) return QAS_ERR_INVALID;
  if (c->stream) cudaStreamSynchronize(c->stream);
  adj_free(c);
  io_free(c);
  pipe_free(c);
  if (c->graph) cudaGraphExecDestroy(c->graph);
  for (cudaEvent_t e : c->prof_events) cudaEventDestroy(e);
  if (c->pool) cudaFree(c->pool);
  if (c->d_src) cudaFree(c->d_src);
  if (c->d_fac) cudaFree(c->d_fac);
  if (c->d_ctl) cudaFree(c->d_ctl);
  if (c->d_dctl) cudaFree(c->d_dctl);
  if (c->d_scratch) cudaFree(c->d_scratch);
  if (c->d_phi) cudaFree(c->d_phi);
  if (c->d_nu) cudaFree(c->d_nu);
  if (c->d_eta) cudaFree(c->d_eta);
  if (c->d_hvmax) cudaFree(c->d_hvmax);
  if (c->h_hvmax) cudaFreeHost(c->h_hvmax);
  if (c->h_ctl) cudaFreeHost(c->h_ctl);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return QAS_OK;
  QAS_API_CATCH
}

qas_status qas_cells(const qas_ctx *c, long long *nd)
{
  QAS_API_TRY
  if (!c || !nd) return QAS_ERR_INVALID;
  *nd = c->geo.nd;
  return QAS_OK;
  QAS_API_CATCH
}

qas_status qas_upload(qas_ctx *c, double *const val[8])
{
  QAS_API_TRY
  if (!c || !val) return QAS_ERR_INVALID;
  const size_t bytes = (size_t)c->geo.nd * sizeof(double);
  for (int m = 0; m < 8; m++) {
    if (!val[m]) return QAS_ERR_INVALID;
    QAS_CUDA(cudaMemcpyAsync(c->view.u[m], val[m], bytes, cudaMemcpyHostToDevice, c->stream));
  }
  QAS_CUDA(cudaStreamSynchronize(c->stream));
  return QAS_OK;
  QAS_API_CATCH
}

qas_status qas_download(qas_ctx *c, double *val[8])
{
  QAS_API_TRY
  if (!c || !val) return QAS_ERR_INVALID;
  const size_t bytes = (size_t)c->geo.nd * sizeof(double);
  for (int m = 0; m < 8; m++) {
    if (!val[m]) return QAS_ERR_INVALID;
    QAS_CUDA(cudaMemcpyAsync(val[m], c->view.u[m], bytes, cudaMemcpyDeviceToHost, c->stream));
  }
  QAS_CUDA(cudaStreamSynchronize(c->stream));
  return QAS_OK;
  QAS_API_CATCH
}

qas_status qas_primitives(qas_ctx *c, double *prim[4], double *cc[3])
{
  QAS_API_TRY
  if (!c) return QAS_ERR_INVALID;
  const Geo &g = c->geo;
  const dim3 t = c->tile[KID_PRIM];
  switch (c->scheme.odr) {
    case 1: k_prim_eval<1><<<cells_grid(g, t), t, 0, c->stream>>>(c->view); break;
    case 2: k_prim_eval<2><<<cells_grid(g, t), t, 0, c->stream>>>(c->view); break;
    case 3: k_prim_eval<3><<<cells_grid(g, t), t, 0, c->stream>>>(c->view); break;
    default: k_prim_eval<4><<<cells_grid(g, t), t, 0, c->stream>>>(c->view); break;
  }
  c->launches++;
  qas_status s = check_launch(c);
  if (s != QAS_OK) return s;
  const size_t bytes = (size_t)g.nd * sizeof(double);
  double *src[7] = {c->view.vx, c->view.vy, c->view.vz, c->view.pr, c->view.cx, c->view.cy, c->view.cz};
  for (int m = 0; m < 7; m++) {
    double *dst = m < 4 ? (prim ? prim[m] : nullptr) : (cc ? cc[m - 4] : nullptr);
    if (dst) QAS_CUDA(cudaMemcpyAsync(dst, src[m], bytes, cudaMemcpyDeviceToHost, c->stream));
  }
  QAS_CUDA(cudaStreamSynchronize(c->stream));
  return QAS_OK;
  QAS_API_CATCH
}

qas_status qas_upload_block(qas_ctx *c, const double *block)
{
  QAS_API_TRY
  if (!c || !block) return QAS_ERR_INVALID;
  double *val[8];
  for (int m = 0; m < 8; m++) val[m] = (double *)block + (size_t)m * c->geo.nd;
  return qas_upload(c, val);
  QAS_API_CATCH
}

qas_status qas_download_block(qas_ctx *c, double *block)
{
  QAS_API_TRY
  if (!c || !block) return QAS_ERR_INVALID;
  double *val[8];
  for (int m = 0; m < 8; m++) val[m] = block + (size_t)m * c->geo.nd;
  return qas_download(c, val);
  QAS_API_CATCH
}

qas_status qas_upload_block_async(qas_ctx *c, const double *block)
{
  QAS_API_TRY
  if (!c || !block) return QAS_ERR_INVALID;
  const size_t n = (size_t)c->geo.nd;
  for (int m = 0; m < 8; m++)
    QAS_CUDA(cudaMemcpyAsync(c->view.u[m], block + m * n, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  return QAS_OK;
  QAS_API_CATCH
}

qas_status qas_download_block_async(qas_ctx *c, double *block)
{
  QAS_API_TRY
  if (!c || !block) return QAS_ERR_INVALID;
  const size_t n = (size_t)c->geo.nd;
  for (int m = 0; m < 8; m++)
    QAS_CUDA(cudaMemcpyAsync(block + m * n, c->view.u[m], n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  return QAS_OK;
  QAS_API_CATCH
}

qas_status qas_device_state(qas_ctx *c, double **d_block)
{
  QAS_API_TRY
  if (!c || !d_block) return QAS_ERR_INVALID;
  // the state arrays are consecutive in the pool with a 256-byte aligned stride; callers
  // that need a dense block use qas_upload_block / qas_download_block
  *d_block = c->view.u[0];
  return QAS_OK;
  QAS_API_CATCH
}

qas_status qas_stream(qas_ctx *c, void **stream)
{
  QAS_API_TRY
  if (!c || !stream) return QAS_ERR_INVALID;
  *stream = (void *)c->stream;
  return QAS_OK;
  QAS_API_CATCH
}

qas_status qas_bound(qas_ctx *c)
{
  QAS_API_TRY
  if (!c) return QAS_ERR_INVALID;
  QAS_CUDA(cudaMemsetAsync(&c->d_ctl->done, 0, sizeof(int), c->stream));
  k_bound<<<shell_grid(c->geo), BLK, 0, c->stream>>>(c->view);
  c->launches++;
  return check_launch(c);
  QAS_API_CATCH
}

qas_status qas_step(qas_ctx *c, double dt)
{
  QAS_API_TRY
  if (!c) return QAS_ERR_INVALID;
  // a single ideal(dt): make sure the loop's done flag does not mask the kernels
  QAS_CUDA(cudaMemsetAsync(&c->d_ctl->done, 0, sizeof(int), c->stream));
  k_set_dt<<<1, 1, 0, c->stream>>>(c->view, dt);
  c->launches += 1 + launch_ideal(c);
  return check_launch(c);
  QAS_API_CATCH
}

qas_status qas_cfl_vmax(qas_ctx *c, double *vmax)
{
  QAS_API_TRY
  if (!c || !vmax) return QAS_ERR_INVALID;
  QAS_CUDA(cudaMemsetAsync(&c->d_ctl->done, 0, sizeof(int), c->stream));
  k_vmax_reset<<<1, 1, 0, c->stream>>>(c->view);
  k_vmax<<<interior_grid(c->geo), BLK, 0, c->stream>>>(c->view);
  c->launches += 2;
  qas_status s = check_launch(c);
  if (s != QAS_OK) return s;
  QAS_CUDA(cudaMemcpyAsync(c->h_ctl, c->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, c->stream));
  QAS_CUDA(cudaStreamSynchronize(c->stream));
  unsigned long long b = c->h_ctl->vmax_bits;
  memcpy(vmax, &b, sizeof(double));
  return QAS_OK;
  QAS_API_CATCH
}

qas_status qas_cfl_dt(qas_ctx *c, double cfl, double *dt)
{
  QAS_API_TRY
  if (!dt) return QAS_ERR_INVALID;
  double vmax = 0.0;
  qas_status s = qas_cfl_vmax(c, &vmax);
  if (s != QAS_OK) return s;
  *dt = cfl * c->dr / vmax;
  return QAS_OK;
  QAS_API_CATCH
}

qas_status qas_run_reset(qas_ctx *c)
{
  QAS_API_TRY
  if (!c) return QAS_ERR_INVALID;
  c->run_initialised = false;
  return QAS_OK;
  QAS_API_CATCH
}

qas_status qas_run(qas_ctx *c, const qas_run_opts *opts, qas_run_info *info)
{
  QAS_API_TRY
  if (!c || !opts) return QAS_ERR_INVALID;
  qas_run_opts o = *opts;
  if (o.stop_rule < 0 || o.stop_rule > 2) return QAS_ERR_INVALID;
  if (o.stop_rule == 0 && o.max_steps <= 0) return QAS_ERR_INVALID;
  if ((o.nu0 > 0.0 || o.eta0 > 0.0) && (c->grid.dim < 2 || c->view.phi)) return QAS_ERR_UNSUPPORTED;
  if (diss_arrays(c) && (o.nu0 != 0.0 || o.eta0 != 0.0)) return QAS_ERR_INVALID;  // one source of coefficients
  qas_status s;
  if (!c->run_initialised) {
    // setdt(1) of main(): dt and nmax from the initial state
    memset(c->h_ctl, 0, sizeof(Ctl));
    c->h_ctl->first = 1;
    c->h_ctl->nmax = INT_MAX;
    c->h_ctl->tmax = o.stop_rule == 0 ? INFINITY : o.dtrec * o.nout;
    if ((s = write_ctl(c)) != QAS_OK) return s;
    c->launches += launch_setdt(c, o.cfl, o.stop_rule, o.dtrec, o.nout);
    if ((s = check_launch(c)) != QAS_OK) return s;
    c->run_initialised = true;
  } else {
    if ((s = read_ctl(c)) != QAS_OK) return s;
    c->h_ctl->done = 0;
    if (o.stop_rule == 0) c->h_ctl->nmax = INT_MAX;
    if ((s = write_ctl(c)) != QAS_OK) return s;
  }
  if ((s = read_ctl(c)) != QAS_OK) return s;
  const int n0 = c->h_ctl->n;
  int n_host = n0;
  const int limit = o.max_steps > 0 ? o.max_steps : INT_MAX;
  int launched = 0;
  // odd n: one eager step so graphs always start at an even n
  if (n_host % 2 == 1 && launched < limit) {
    c->launches += launch_exec_step(c, o, n_host + 1);
    n_host++;
    launched++;
  }
  const bool want_graph = o.use_graph != 0 && !hall_active(c);  // the Hall sub-cycle count is read back
  if (want_graph && launched + 2 <= limit) {
    const bool stale = !c->graph || c->graph_flg != o.flg || c->graph_rule != o.stop_rule || c->graph_cfl != o.cfl ||
                       c->graph_nu0 != o.nu0 || c->graph_eta0 != o.eta0 || c->graph_dtrec != o.dtrec ||
                       c->graph_nout != o.nout;
    if (stale) {
      if (c->graph) {
        cudaGraphExecDestroy(c->graph);
        c->graph = nullptr;
      }
      cudaGraph_t gph;
      QAS_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
      long long nk = launch_exec_step(c, o, 1) + launch_exec_step(c, o, 2);
      cudaError_t e = cudaStreamEndCapture(c->stream, &gph);
      if (e != cudaSuccess) return cuda_fail(e, "graph capture");
      e = cudaGraphInstantiate(&c->graph, gph, 0);
      cudaGraphDestroy(gph);
      if (e != cudaSuccess) return cuda_fail(e, "graph instantiate");
      c->graph_kernels = nk;
      c->graph_flg = o.flg;
      c->graph_rule = o.stop_rule;
      c->graph_cfl = o.cfl;
      c->graph_nu0 = o.nu0;
      c->graph_eta0 = o.eta0;
      c->graph_dtrec = o.dtrec;
      c->graph_nout = o.nout;
    }
  }
  const int chunk = 32;  // steps between host checks of the stop flag
  while (launched < limit) {
    int this_chunk = 0;
    while (this_chunk < chunk && launched < limit) {
      if (want_graph && c->graph && launched + 2 <= limit) {
        QAS_CUDA(cudaGraphLaunch(c->graph, c->stream));
        c->launches += c->graph_kernels;
        launched += 2;
        n_host += 2;
        this_chunk += 2;
      } else {
        c->launches += launch_exec_step(c, o, n_host + 1);
        launched++;
        n_host++;
        this_chunk++;
      }
    }
    if ((s = check_launch(c)) != QAS_OK) return s;
    if (o.stop_rule != 0) {
      if ((s = read_ctl(c)) != QAS_OK) return s;
      if (c->h_ctl->done) break;
    }
  }
  if ((s = read_ctl(c)) != QAS_OK) return s;
  if (info) {
    info->steps = c->h_ctl->n - n0;
    info->n = c->h_ctl->n;
    info->nmax = c->h_ctl->nmax;
    info->tim = c->h_ctl->tim;
    info->dt = c->h_ctl->dt;
  }
  return QAS_OK;
  QAS_API_CATCH
}

qas_status qas_dsptv(qas_ctx *c, double dt, double nu0, double eta0)
{
  QAS_API_TRY
  if (!c) return QAS_ERR_INVALID;
  if (c->grid.dim < 2 || c->view.phi) return QAS_ERR_UNSUPPORTED;
  if (diss_arrays(c) && (nu0 != 0.0 || eta0 != 0.0)) return QAS_ERR_INVALID;
  QAS_CUDA(cudaMemsetAsync(&c->d_ctl->done, 0, sizeof(int), c->stream));
  const Geo &g = c->geo;
  const double idx = 1.0 / c->grid.dx, idy = 1.0 / c->grid.dy;
  const double idz = g.dim == 3 ? 1.0 / c->grid.dz : 0.0;
  k_dsub_fixed<<<1, 1, 0, c->stream>>>(c->view, c->d_dctl, dt, idx, idy, idz);
  // dsptv itself does not fill the ghosts first; launch_dsptv starts with a fill, so
  // run the body without it: copy, stages
  k_dcopy<<<(unsigned)((g.nd + 255) / 256), 256, 0, c->stream>>>(c->view, c->d_dctl, 0);
  long long nk = 2;
  for (int rk = 0; rk < c->scheme.rk; rk++) {
    double c0, c1;
    rk_factors(c->scheme.rk, rk, c0, c1);
    switch (c->scheme.odr) {
#define QAS_DST(O)                                                                                        \
  case O:                                                                                                 \
    k_dvel<<<cells_grid(g), BLK, 0, c->stream>>>(c->view, c->d_dctl, 0);                                  \
    k_eres<O><<<cells_grid(g), BLK, 0, c->stream>>>(c->view, c->d_dctl, 0, eta0, idx, idy, idz);          \
    k_dflux<O><<<cells_grid(g), BLK, 0, c->stream>>>(c->view, c->d_dctl, 0, nu0, idx, idy, idz);          \
    k_dupdate<O><<<update_grid(g), BLK, 0, c->stream>>>(c->view, c->d_dctl, 0, c0, c1);                   \
    k_dbound<<<shell_grid(g), BLK, 0, c->stream>>>(c->view, c->d_dctl, 0);                                \
    break;
      QAS_DST(1)
      QAS_DST(2)
      QAS_DST(3)
      default:
      QAS_DST(4)
#undef QAS_DST
    }
    nk += 5;
  }
  c->launches += nk;
  return check_launch(c);
  QAS_API_CATCH
}

qas_status qas_dissipate(qas_ctx *c, double dt, double nu0, double eta0)
{
  QAS_API_TRY
  if (!c) return QAS_ERR_INVALID;
  if (c->grid.dim < 2 || c->view.phi) return QAS_ERR_UNSUPPORTED;
  if (diss_arrays(c) && (nu0 != 0.0 || eta0 != 0.0)) return QAS_ERR_INVALID;
  QAS_CUDA(cudaMemsetAsync(&c->d_ctl->done, 0, sizeof(int), c->stream));
  k_set_dt<<<1, 1, 0, c->stream>>>(c->view, dt);
  c->launches += 1 + launch_dissipate(c, nu0, eta0);
  return check_launch(c);
  QAS_API_CATCH
}

qas_status qas_max_divb(qas_ctx *c, double *maxdivb)
{
  QAS_API_TRY
  if (!c || !maxdivb) return QAS_ERR_INVALID;
  if (c->grid.dim < 2) {
    *maxdivb = 0.0;
    return QAS_OK;
  }
  QAS_CUDA(cudaMemsetAsync(c->d_scratch, 0, sizeof(unsigned long long), c->stream));
  switch (c->scheme.odr) {
    case 1: k_divb<1><<<interior_grid(c->geo), BLK, 0, c->stream>>>(c->view, c->d_scratch); break;
    case 2: k_divb<2><<<interior_grid(c->geo), BLK, 0, c->stream>>>(c->view, c->d_scratch); break;
    case 3: k_divb<3><<<interior_grid(c->geo), BLK, 0, c->stream>>>(c->view, c->d_scratch); break;
    default: k_divb<4><<<interior_grid(c->geo), BLK, 0, c->stream>>>(c->view, c->d_scratch); break;
  }
  c->launches++;
  qas_status s = check_launch(c);
  if (s != QAS_OK) return s;
  unsigned long long bits = 0;
  QAS_CUDA(cudaMemcpyAsync(&bits, c->d_scratch, sizeof(bits), cudaMemcpyDeviceToHost, c->stream));
  QAS_CUDA(cudaStreamSynchronize(c->stream));
  memcpy(maxdivb, &bits, sizeof(double));
  return QAS_OK;
  QAS_API_CATCH
}

qas_status qas_sync(qas_ctx *c)
{
  QAS_API_TRY
  if (!c) return QAS_ERR_INVALID;
  QAS_CUDA(cudaStreamSynchronize(c->stream));
  return read_ctl(c);
  QAS_API_CATCH
}

qas_status qas_bc_map(const qas_grid *grid, const qas_bc *bc, int group, int field, int axis, int *src,
                      double *fac, int n)
{
  QAS_API_TRY
  if (!grid || !bc || !src || !fac) return QAS_ERR_INVALID;
  if (group < 0 || group > 3 || field < 0 || field >= (group == 0 ? 8 : 3) || axis < 0 || axis > 2)
    return QAS_ERR_INVALID;
  const int ext[3] = {grid->nxm + 2 * GH, grid->dim >= 2 ? grid->nym + 2 * GH : 1,
                      grid->dim >= 3 ? grid->nzm + 2 * GH : 1};
  if (n != ext[axis]) return QAS_ERR_INVALID;
  AxisMap m(n);
  if (!map_for(grid->dim, *bc, group, field, axis, n, m)) return QAS_ERR_INVALID;
  for (int i = 0; i < n; i++) {
    src[i] = m.src[i];
    fac[i] = m.fac[i];
  }
  return QAS_OK;
  QAS_API_CATCH
}

qas_status qas_profile_run(qas_ctx *c, const qas_run_opts *opts, int nsteps, qas_kernel_time *out,
                           int max_entries, int *count)
{
  QAS_API_TRY
  if (!c || !opts || !out || !count || nsteps <= 0) return QAS_ERR_INVALID;
  qas_run_opts o = *opts;
  o.use_graph = 0;
  o.stop_rule = 0;
  o.max_steps = 1;
  qas_status s;
  // make sure the loop is initialised (setdt(1)) and the stop flag is clear
  if (!c->run_initialised) {
    qas_run_opts o0 = o;
    o0.max_steps = 1;
    if ((s = qas_run(c, &o0, nullptr)) != QAS_OK) return s;
  }
  if ((s = read_ctl(c)) != QAS_OK) return s;
  c->h_ctl->done = 0;
  c->h_ctl->nmax = INT_MAX;
  if ((s = write_ctl(c)) != QAS_OK) return s;
  for (int k = 0; k < KID_COUNT; k++) {
    c->prof_ms[k] = 0.0;
    c->prof_n[k] = 0;
  }
  int n_host = c->h_ctl->n;
  c->prof = true;
  for (int st = 0; st < nsteps; st++) {
    c->prof_kids.clear();
    c->launches += launch_exec_step(c, o, n_host + 1);
    n_host++;
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
      c->prof = false;
      return cuda_fail(e, "profile step");
    }
    for (size_t q = 0; q < c->prof_kids.size(); q++) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, c->prof_events[2 * q], c->prof_events[2 * q + 1]);
      c->prof_ms[c->prof_kids[q]] += ms;
      c->prof_n[c->prof_kids[q]] += 1;
    }
  }
  c->prof = false;
  c->prof_kids.clear();
  if ((s = check_launch(c)) != QAS_OK) return s;
  int w = 0;
  for (int k = 0; k < KID_COUNT && w < max_entries; k++) {
    if (!c->prof_n[k]) continue;
    snprintf(out[w].name, sizeof(out[w].name), "%s", KID_NAMES[k]);
    out[w].launches = c->prof_n[k];
    out[w].total_ms = c->prof_ms[k];
    w++;
  }
  *count = w;
  return read_ctl(c);
  QAS_API_CATCH
}

qas_status qas_set_dissipation(qas_ctx *c, const double *nu, const double *eta)
{
  QAS_API_TRY
  if (!c) return QAS_ERR_INVALID;
  if (c->grid.dim < 2 || c->view.phi) return QAS_ERR_UNSUPPORTED;
  QAS_CUDA(cudaStreamSynchronize(c->stream));
  if (c->graph) {  // captured launches carry the view by value
    cudaGraphExecDestroy(c->graph);
    c->graph = nullptr;
  }
  if (!nu && !eta) {
    c->view.nu = c->view.eta = nullptr;
    return QAS_OK;
  }
  const size_t nd = (size_t)c->geo.nd, bytes = nd * sizeof(double);
  if (!c->d_nu && cudaMalloc(&c->d_nu, bytes) != cudaSuccess) {
    cudaGetLastError();
    return QAS_ERR_NOMEM;
  }
  if (!c->d_eta && cudaMalloc(&c->d_eta, bytes) != cudaSuccess) {
    cudaGetLastError();
    return QAS_ERR_NOMEM;
  }
  std::vector<double> zero;
  if (!nu || !eta) zero.assign(nd, 0.0);
  const double *hn = nu ? nu : zero.data(), *he = eta ? eta : zero.data();
  // setdc's reduction (2D/SERIAL/MRX/dmhd2d_init_.cpp:85-106): dtmp = max(2 nu, eta) per cell
  double dcmax = 0.0;
  for (size_t q = 0; q < nd; q++) {
    const double dtmp = (2 * hn[q] >= he[q]) ? 2 * hn[q] : he[q];
    if (dtmp > dcmax) dcmax = dtmp;
  }
  QAS_CUDA(cudaMemcpy(c->d_nu, hn, bytes, cudaMemcpyHostToDevice));
  QAS_CUDA(cudaMemcpy(c->d_eta, he, bytes, cudaMemcpyHostToDevice));
  c->view.nu = c->d_nu;
  c->view.eta = c->d_eta;
  c->diss_dcmax = dcmax;
  return QAS_OK;
  QAS_API_CATCH
}

qas_status qas_set_hall(qas_ctx *c, double di, double de)
{
  QAS_API_TRY
  if (!c || !(di >= 0.0) || !(de >= 0.0)) return QAS_ERR_INVALID;
  if (c->grid.dim != 1) return QAS_ERR_UNSUPPORTED;
  QAS_CUDA(cudaStreamSynchronize(c->stream));
  if (c->graph) {
    cudaGraphExecDestroy(c->graph);
    c->graph = nullptr;
  }
  if (!c->d_hvmax && cudaMalloc(&c->d_hvmax, sizeof(unsigned long long)) != cudaSuccess) {
    cudaGetLastError();
    return QAS_ERR_NOMEM;
  }
  if (!c->h_hvmax && cudaMallocHost(&c->h_hvmax, sizeof(unsigned long long)) != cudaSuccess) {
    cudaGetLastError();
    return QAS_ERR_NOMEM;
  }
  // HMHD1D::paras (1D/SERIAL/h-shock/hmhd1d_paras.cpp:29-34)
  const double idx = 1.0 / c->grid.dx;
  double kpeak = M_PI * idx;
  if (de != 0) kpeak = hmin(kpeak, 1.0 / de);
  c->hall = true;
  c->hall_di = di;
  c->hall_de = de;
  c->hall_vphix = di * kpeak;
  return QAS_OK;
  QAS_API_CATCH
}

qas_status qas_hall(qas_ctx *c, double dt)
{
  QAS_API_TRY
  if (!c) return QAS_ERR_INVALID;
  if (!c->hall) return QAS_ERR_UNSUPPORTED;
  QAS_CUDA(cudaMemsetAsync(&c->d_ctl->done, 0, sizeof(int), c->stream));
  c->launches += launch_hall(c, dt);
  return check_launch(c);
  QAS_API_CATCH
}

qas_status qas_set_gravity(qas_ctx *c, const double *phi_g)
{
  QAS_API_TRY
  if (!c) return QAS_ERR_INVALID;
  if (c->grid.dim < 2) return QAS_ERR_UNSUPPORTED;
  QAS_CUDA(cudaStreamSynchronize(c->stream));
  if (c->graph) {  // captured launches carry the view by value
    cudaGraphExecDestroy(c->graph);
    c->graph = nullptr;
  }
  if (!phi_g) {
    c->view.phi = nullptr;
    return QAS_OK;
  }
  const size_t bytes = (size_t)c->geo.nd * sizeof(double);
  if (!c->d_phi && cudaMalloc(&c->d_phi, bytes) != cudaSuccess) {
    cudaGetLastError();
    return QAS_ERR_NOMEM;
  }
  QAS_CUDA(cudaMemcpy(c->d_phi, phi_g, bytes, cudaMemcpyHostToDevice));
  c->view.phi = c->d_phi;
  c->view.gfac = (2.0 - c->grid.gam) / (c->grid.gam - 1.0);  // fac of the drivers' bound()
  return QAS_OK;
  QAS_API_CATCH
}

qas_status qas_set_option(qas_ctx *c, int option, int value)
{
  QAS_API_TRY
  if (!c) return QAS_ERR_INVALID;
  if (option == QAS_OPT_FUSED_SWEEP) {
    const bool f = value != 0;
    if (f != c->fused && c->graph) {  // the captured graph holds the other form
      cudaStreamSynchronize(c->stream);
      cudaGraphExecDestroy(c->graph);
      c->graph = nullptr;
    }
    c->fused = f;
    if (f) sweep_prepare(c);
    return QAS_OK;
  }
  if (option == QAS_OPT_LR_STAGING) {
    const bool t = value != 0;
    if (t && !c->lr_tma_ok) return QAS_ERR_UNSUPPORTED;
    if (t != c->lr_tma && c->graph) {
      cudaStreamSynchronize(c->stream);
      cudaGraphExecDestroy(c->graph);
      c->graph = nullptr;
    }
    c->lr_tma = t;
    return QAS_OK;
  }
  if (option == QAS_OPT_TEST_TMA_STALL) {
    if (!c->lr_tma_ok) return QAS_ERR_UNSUPPORTED;
    if (c->graph) {  // the captured graph holds the plans by value
      cudaStreamSynchronize(c->stream);
      cudaGraphExecDestroy(c->graph);
      c->graph = nullptr;
    }
    for (int a = 0; a < 3; a++) {
      c->lr_plan[a].stall_plane = value >= 0 ? value : -1;
      c->lr_plan[a].wait_ns = value >= 0 ? 100000ull : 2000000000ull;
    }
    return QAS_OK;
  }
  if (option == QAS_OPT_PIPE_ITEMS) return pipe_set_items(c, value);
  if (option == QAS_OPT_PIPE_LANES) return pipe_set_lanes(c, value);
  return QAS_ERR_INVALID;
  QAS_API_CATCH
}

static int tile_kid(const char *k)
{
  if (!k) return -2;
  const int kids[6] = {KID_PRIM, KID_DV, KID_LR, KID_FLUX, KID_EMF, KID_UPDATE};
  if (!strcmp(k, "all")) return -1;
  for (int q = 0; q < 6; q++)
    if (!strcmp(k, KID_NAMES[kids[q]])) return kids[q];
  return -2;
}

static void drop_graph(qas_ctx *c)
{
  if (c->graph) {
    cudaStreamSynchronize(c->stream);
    cudaGraphExecDestroy(c->graph);
    c->graph = nullptr;
  }
}

qas_status qas_set_tile(qas_ctx *c, const char *kernel, int tx, int ty, int tz)
{
  QAS_API_TRY
  if (!c) return QAS_ERR_INVALID;
  const int kid = tile_kid(kernel);
  if (kid == -2 || tx < 32 || tx % 32 || ty < 1 || tz < 1 || tx * ty * tz > 128) return QAS_ERR_INVALID;
  if (c->grid.dim < 2 && ty != 1) return QAS_ERR_INVALID;
  if (c->grid.dim < 3 && tz != 1) return QAS_ERR_INVALID;
  drop_graph(c);
  const dim3 t(tx, ty, tz);
  if (kid == -1) {
    for (int q = 0; q < 32; q++) c->tile[q] = t;
  } else {
    c->tile[kid] = t;
  }
  return QAS_OK;
  QAS_API_CATCH
}

qas_status qas_get_tile(const qas_ctx *c, const char *kernel, int *tx, int *ty, int *tz)
{
  QAS_API_TRY
  if (!c || !tx || !ty || !tz) return QAS_ERR_INVALID;
  const int kid = tile_kid(kernel);
  if (kid < 0) return QAS_ERR_INVALID;
  *tx = c->tile[kid].x;
  *ty = c->tile[kid].y;
  *tz = c->tile[kid].z;
  return QAS_OK;
  QAS_API_CATCH
}

namespace {
struct TuneKey {
  int dim, odr, rmn, bucket;
  bool operator==(const TuneKey &o) const
  {
    return dim == o.dim && odr == o.odr && rmn == o.rmn && bucket == o.bucket;
  }
};
struct TuneEntry {
  TuneKey key;
  dim3 tiles[6];
};
std::vector<TuneEntry> g_tune_cache;
std::mutex g_tune_mu;
}  // namespace

qas_status qas_autotune(qas_ctx *c, int trial_steps)
{
  QAS_API_TRY
  if (!c || trial_steps <= 0) return QAS_ERR_INVALID;
  const int kids[6] = {KID_PRIM, KID_DV, KID_LR, KID_FLUX, KID_EMF, KID_UPDATE};
  int bucket = 0;
  for (long long n = c->geo.nd; n > 4096; n >>= 2) bucket++;
  const TuneKey key{c->grid.dim, c->scheme.odr, c->scheme.rmn, bucket};
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    for (const TuneEntry &e : g_tune_cache)
      if (e.key == key) {
        drop_graph(c);
        for (int q = 0; q < 6; q++) c->tile[kids[q]] = e.tiles[q];
        return QAS_OK;
      }
  }
  std::vector<dim3> cands;
  if (c->grid.dim == 1) {
    cands = {dim3(128, 1, 1), dim3(64, 1, 1), dim3(32, 1, 1)};
  } else if (c->grid.dim == 2) {
    cands = {dim3(128, 1, 1), dim3(64, 2, 1), dim3(32, 4, 1), dim3(32, 2, 1)};
  } else {
    cands = {dim3(128, 1, 1), dim3(64, 2, 1), dim3(32, 4, 1), dim3(32, 2, 2), dim3(32, 1, 4), dim3(64, 1, 2)};
  }
  // save the state and the loop counters
  qas_status s;
  if ((s = read_ctl(c)) != QAS_OK) return s;
  const Ctl saved_ctl = *c->h_ctl;
  const bool saved_init = c->run_initialised;
  const size_t bytes = (size_t)c->geo.nd * sizeof(double);
  double *backup = nullptr;
  QAS_CUDA(cudaMalloc(&backup, 8 * bytes));
  for (int m = 0; m < 8; m++)
    cudaMemcpyAsync(backup + (size_t)m * c->geo.nd, c->view.u[m], bytes, cudaMemcpyDeviceToDevice, c->stream);
  drop_graph(c);
  qas_run_opts o{};
  o.flg = 1;
  o.cfl = 0.4;
  o.dtrec = 1.0;
  o.nout = 1;
  double best_ms[6];
  dim3 best[6];
  for (int q = 0; q < 6; q++) {
    best_ms[q] = 1e300;
    best[q] = c->tile[kids[q]];
  }
  qas_kernel_time kt[32];
  int cnt = 0;
  for (const dim3 &t : cands) {
    for (int q = 0; q < 6; q++) c->tile[kids[q]] = t;
    // restore the state before each trial so every candidate sees the same work
    for (int m = 0; m < 8; m++)
      cudaMemcpyAsync(c->view.u[m], backup + (size_t)m * c->geo.nd, bytes, cudaMemcpyDeviceToDevice, c->stream);
    *c->h_ctl = saved_ctl;
    c->h_ctl->done = 0;
    if ((s = write_ctl(c)) != QAS_OK) break;
    c->run_initialised = true;
    if ((s = qas_profile_run(c, &o, trial_steps, kt, 32, &cnt)) != QAS_OK) break;
    for (int e = 0; e < cnt; e++)
      for (int q = 0; q < 6; q++)
        if (!strcmp(kt[e].name, KID_NAMES[kids[q]]) && kt[e].total_ms < best_ms[q]) {
          best_ms[q] = kt[e].total_ms;
          best[q] = t;
        }
  }
  for (int q = 0; q < 6; q++) c->tile[kids[q]] = best[q];
  for (int m = 0; m < 8; m++)
    cudaMemcpyAsync(c->view.u[m], backup + (size_t)m * c->geo.nd, bytes, cudaMemcpyDeviceToDevice, c->stream);
  *c->h_ctl = saved_ctl;
  qas_status s2 = write_ctl(c);
  c->run_initialised = saved_init;
  cudaFree(backup);
  if (s != QAS_OK) return s;
  if (s2 != QAS_OK) return s2;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  TuneEntry e;
  e.key = key;
  for (int q = 0; q < 6; q++) e.tiles[q] = best[q];
  g_tune_cache.push_back(e);
  return QAS_OK;
  QAS_API_CATCH
}

qas_status qas_fp64_peak(double *tflops)
{
  QAS_API_TRY
  if (!tflops) return QAS_ERR_INVALID;
  int dev = 0, sms = 0;
  QAS_CUDA(cudaGetDevice(&dev));
  QAS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  double *d = nullptr;
  QAS_CUDA(cudaMalloc(&d, sizeof(double)));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int threads = 256, blocks = sms * 8, iters = 20000;
  k_fp64_peak<<<blocks, threads>>>(d, 1000, 0.999999, 1e-7);  // warm-up
  cudaEventRecord(e0);
  k_fp64_peak<<<blocks, threads>>>(d, iters, 0.999999, 1e-7);
  cudaEventRecord(e1);
  cudaError_t e = cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d);
  if (e != cudaSuccess) return cuda_fail(e, "fp64 peak");
  *tflops = 2.0 * 8.0 * (double)iters * threads * blocks / (ms * 1e-3) / 1e12;
  return QAS_OK;
  QAS_API_CATCH
}

qas_status qas_kernel_launches(const qas_ctx *c, long long *count)
{
  QAS_API_TRY
  if (!c || !count) return QAS_ERR_INVALID;
  *count = c->launches;
  return QAS_OK;
  QAS_API_CATCH
}

}  // extern "C"

#include "qas_batch_api.inc"
#include "qas_adjoint_api.inc"
#include "qas_noalloc.inc"
#include "qas_io.inc"
#include "qas_dd.inc"
#include "qas_pipe.inc"
