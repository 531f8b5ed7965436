// k-clique kernel instantiations for k = 12 (compiled apart from clique.cu so the unrolled
// DFS of every k compiles in parallel).
#include "clique_kernel.cuh"

namespace dmb {

int clique_launch_k12(const CliqueArgs& a, int m, LaunchCtx& ctx, int* grid) { return launch_nw<12>(a, m, ctx, grid); }

}  // namespace dmb
