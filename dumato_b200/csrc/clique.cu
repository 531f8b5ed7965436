// k-clique counting kernel for sm_100a: the single-graph persistent launch. The per-task
// device code (semantics, bitmap and list paths) is in clique.cuh, the kernel template in
// clique_kernel.cuh; this unit instantiates k = 2..6 and dispatches the larger k to the units
// that instantiate them.
#include "clique_kernel.cuh"

namespace dmb {

int clique_max_warps(int num_sms) { return num_sms * 64; }

int clique_launch(const CliqueLaunch& L, LaunchCtx& ctx, int* grid) {
  CliqueArgs a;
  a.g = L.g;
  a.roots = L.roots;
  a.n_roots = L.n_roots;
  a.lb = LBArgs{L.ctr, reinterpret_cast<QHeader*>(L.queue),
                reinterpret_cast<QSlot*>(reinterpret_cast<char*>(L.queue) + sizeof(QHeader) * L.nq), L.qcap, 0,
                L.max_donations, (long long)ctx.donate_after_us * 1000ll, (long long)ctx.timeout_ms * 1000000ll,
                ctx.test_stall, 32, L.nq};
  a.arena = L.arena;
  a.arena_dcap = L.arena_dcap;
  a.list_threshold = L.list_threshold;
  a.per_root = L.per_root;
  a.parts = L.parts;
  switch (L.k) {
    case 2: return launch_nw<2>(a, L.nwmax, ctx, grid);
    case 3: return launch_nw<3>(a, L.nwmax, ctx, grid);
    case 4: return launch_nw<4>(a, L.nwmax, ctx, grid);
    case 5: return launch_nw<5>(a, L.nwmax, ctx, grid);
    case 6: return launch_nw<6>(a, L.nwmax, ctx, grid);
    case 7:
    case 8: return clique_launch_k7_8(a, L.k, L.nwmax, ctx, grid);
    case 9: return clique_launch_k9(a, L.nwmax, ctx, grid);
    case 10: return clique_launch_k10(a, L.nwmax, ctx, grid);
    case 11: return clique_launch_k11(a, L.nwmax, ctx, grid);
    case 12: return clique_launch_k12(a, L.nwmax, ctx, grid);
    default: return fail(DM_EINVAL, "k must be in [2, 12]");
  }
}

}  // namespace dmb
