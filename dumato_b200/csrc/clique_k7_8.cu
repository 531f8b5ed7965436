// k-clique kernel instantiations for k = 7 and 8 (compiled apart from clique.cu so the
// unrolled DFS of every k compiles in parallel).
#include "clique_kernel.cuh"

namespace dmb {

int clique_launch_k7_8(const CliqueArgs& a, int k, int m, LaunchCtx& ctx, int* grid) {
  return k == 7 ? launch_nw<7>(a, m, ctx, grid) : launch_nw<8>(a, m, ctx, grid);
}

int clique_cached_k7_8(CachedArgs* a, int k, int m, bool tma, bool multi, LaunchCtx& ctx, int* grid, bool query) {
  return k == 7 ? cached_nw<7>(a, m, tma, multi, ctx, grid, query) : cached_nw<8>(a, m, tma, multi, ctx, grid, query);
}

}  // namespace dmb
