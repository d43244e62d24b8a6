// Host-only entry points of libqas (the wave plan of qas_step_host, the ghost-fill maps, the slab
// plan of the domain decomposition, the status strings) swept over sizes and random boundary
// flags, for a build with AddressSanitizer and UndefinedBehaviorSanitizer
// (tests/test_host_sanitize.py).  No call touches a GPU.
#include <cstdio>
#include <cstdlib>
#include <vector>
#include "qas.h"

int main()
{
  long long checks = 0;
  // pipe plans
  for (int planes = 21; planes <= 700; planes += (planes < 80 ? 1 : 7))
    for (int w = 0; w <= 64; w += (w < 8 ? 1 : 4))
      for (int own = 0; own < 2; own++) {
        int n = 0, lag = 0;
        if (qas_pipe_plan(planes, w, own, nullptr, 0, &n, &lag) != QAS_OK) continue;
        std::vector<int> out((size_t)n * QAS_PIPE_ITEM_INTS);
        if (qas_pipe_plan(planes, w, own, out.data(), n, &n, &lag) != QAS_OK) { printf("pipe fail\n"); return 1; }
        checks++;
      }
  // ghost maps and slab plans over random flags
  srand(7);
  const int flags[6] = {0, 1, -1, 2, -2, 0};
  for (int t = 0; t < 3000; t++) {
    qas_grid g = {};
    g.dim = 1 + t % 3;
    g.nxm = 8 + rand() % 40;
    g.nym = g.dim >= 2 ? 8 + rand() % 40 : 1;
    g.nzm = g.dim >= 3 ? 8 + rand() % 40 : 1;
    g.dx = g.dy = g.dz = 0.1;
    g.gam = 5.0 / 3.0;
    qas_bc bc = {};
    for (int f = 0; f < 8; f++) {
      bc.dnx[f] = flags[rand() % 6];
      bc.dny[f] = flags[rand() % 6];
      bc.dnz[f] = flags[rand() % 6];
    }
    const int ext[3] = {g.nxm + 8, g.nym + 8, g.nzm + 8};
    for (int G = 0; G < 3; G++)
      for (int f = 0; f < (G == 0 ? 8 : 3); f++)
        for (int a = 0; a < g.dim; a++) {
          std::vector<int> src(ext[a]);
          std::vector<double> fac(ext[a]);
          qas_bc_map(&g, &bc, G, f, a, src.data(), fac.data(), ext[a]);
          checks++;
        }
    if (g.dim >= 2)
      for (int np = 1; np <= 4; np++) {
        std::vector<int> lo(np + 1);
        int nc = 0;
        if (qas_dd_plan(&g, &bc, np, lo.data(), nullptr, 0, &nc) != QAS_OK) continue;
        std::vector<qas_dd_copy> cp(nc > 0 ? nc : 1);
        qas_dd_plan(&g, &bc, np, lo.data(), cp.data(), nc, &nc);
        checks++;
      }
  }
  for (int s = 0; s < 12; s++) (void)qas_status_str((qas_status)s);
  printf("host plans ok: %lld calls\n", checks);
  return 0;
}
