// Property test of the segmented-reduction tile planner (HostPlan::add):
// random segment layouts with long runs of empty segments and segments far
// longer than a tile; checks position coverage, tile budgets, single
// ownership, owner position ranges and the split bookkeeping.
#include "host.hpp"
#include <cstdio>
#include <random>
using namespace wgpu;
int main() {
  std::mt19937_64 rng(1);
  for (int trial = 0; trial < 3000; ++trial) {
    int T = (trial % 3 == 0) ? 8 : (trial % 3 == 1) ? 32 : 2048;
    uint32_t nseg = rng() % 5000;
    std::vector<uint32_t> ptr(nseg + 1);
    uint32_t base = rng() % 100;
    ptr[0] = base;
    for (uint32_t s = 0; s < nseg; ++s) {
      uint32_t r = rng() % 10, len = r < 5 ? 0 : r < 8 ? rng() % 5 : rng() % (3 * T);
      ptr[s + 1] = ptr[s] + len;
    }
    HostPlan hp; hp.add(0, ptr.data(), nseg, T);
    std::vector<int> own(nseg, 0);
    uint32_t prevp = base;
    for (size_t t = 0; t < hp.tiles.size(); ++t) {
      auto& x = hp.tiles[t];
      if (x.p0 != prevp) { printf("gap trial %d\n", trial); return 1; }
      prevp = x.p1;
      if (x.p1 - x.p0 > (uint32_t)T || x.own_hi - x.own_lo > (uint32_t)T) { printf("budget trial %d\n", trial); return 1; }
      for (uint32_t s = x.own_lo; s < x.own_hi; ++s) {
        own[s]++;
        if (ptr[s+1] > ptr[s] && !(ptr[s] >= x.p0 && ptr[s] < x.p1)) { printf("owner mismatch trial %d\n", trial); return 1; }
        if (ptr[s+1] > x.p1 && ptr[s+1] > ptr[s] && x.tail_split < 0) { printf("missing tail trial %d\n", trial); return 1; }
      }
    }
    if (prevp != ptr[nseg]) { printf("end trial %d\n", trial); return 1; }
    for (uint32_t s = 0; s < nseg; ++s) if (own[s] != 1) { printf("own count trial %d seg %u\n", trial, s); return 1; }
    for (size_t id = 0; id < hp.splits.size(); ++id) {
      auto& sp = hp.splits[id];
      if (hp.tiles[sp.t0].tail_split != (int)id) { printf("tail id\n"); return 1; }
      for (uint32_t t = sp.t0 + 1; t <= sp.t1; ++t) if (hp.tiles[t].cont_split != (int)id || hp.tiles[t].p1 == hp.tiles[t].p0) { printf("cont id trial %d\n", trial); return 1; }
      if (!(ptr[sp.seg+1] - 1 >= hp.tiles[sp.t1].p0 && ptr[sp.seg+1] - 1 < hp.tiles[sp.t1].p1)) { printf("t1 wrong\n"); return 1; }
    }
  }
  printf("plan ok\n");
}
