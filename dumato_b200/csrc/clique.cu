// k-clique counting kernel for sm_100a: the single-graph persistent launch. The per-task
// device code (semantics, bitmap and list paths) is in clique.cuh, the kernel template in
// clique_kernel.cuh; this unit instantiates k = 2..6 and dispatches the larger k to the units
// that instantiate them.
#include "clique_kernel.cuh"

namespace dmb {

int clique_max_warps(int num_sms) { return num_sms * 64; }

static CliqueArgs clique_args(const CliqueLaunch& L, LaunchCtx& ctx) {
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
  a.list_vwarp = (L.list_vwarp == 8 || L.list_vwarp == 16) ? L.list_vwarp : 32;
  a.list_threshold = L.list_threshold;
  a.per_root = L.per_root;
  a.parts = L.parts;
  return a;
}

static int cached_dispatch(CachedArgs* a, int k, int m, bool tma, bool multi, LaunchCtx& ctx, int* grid,
                           bool query) {
  switch (k) {
    case 2: return cached_nw<2>(a, m, tma, multi, ctx, grid, query);
    case 3: return cached_nw<3>(a, m, tma, multi, ctx, grid, query);
    case 4: return cached_nw<4>(a, m, tma, multi, ctx, grid, query);
    case 5: return cached_nw<5>(a, m, tma, multi, ctx, grid, query);
    case 6: return cached_nw<6>(a, m, tma, multi, ctx, grid, query);
    case 7:
    case 8: return clique_cached_k7_8(a, k, m, tma, multi, ctx, grid, query);
    default: return fail(DM_EINVAL, "the clique index kernel covers k in [2, 8]");
  }
}

static CachedArgs cached_args(const CliqueLaunch& L, LaunchCtx& ctx) {
  CachedArgs a;
  a.c = clique_args(L, ctx);
  a.desc = L.desc;
  a.blocks = reinterpret_cast<const uint4*>(L.blocks);
  a.boff = L.boff;
  a.static_chunk = L.static_chunk;
  a.n_static = L.n_static;
  return a;
}

int clique_cached_grid(const CliqueLaunch& L, LaunchCtx& ctx, int* grid) {
  CachedArgs a = cached_args(L, ctx);
  *grid = 0;
  return cached_dispatch(&a, L.k, L.nwmax, L.tma, L.multi, ctx, grid, true);
}

int clique_cached_launch(const CliqueLaunch& L, LaunchCtx& ctx, int grid) {
  CachedArgs a = cached_args(L, ctx);
  int g = grid;
  return cached_dispatch(&a, L.k, L.nwmax, L.tma, L.multi, ctx, &g, false);
}

template <int M>
static int index_build_m(const GraphView& g, const int32_t* roots, int n, void* blocks, const uint32_t* boff,
                         LaunchCtx& ctx) {
  const size_t smem = (size_t)warp_layout(M).total * (CLIQUE_BLOCK / 32);
  auto kern = index_build_kernel<M>;
  static LaunchCache cache;
  int occ = 0;
  DM_CUDA(cached_occupancy(cache, kern, ctx.device, CLIQUE_BLOCK, smem, &occ));
  if (occ < 1) return fail(DM_EINVAL, "clique index build kernel does not fit on an SM");
  const int per_grid = (n + CLIQUE_BLOCK / 32 - 1) / (CLIQUE_BLOCK / 32);
  const int grid = std::max(1, std::min(ctx.num_sms * occ, per_grid));
  kern<<<grid, CLIQUE_BLOCK, smem, ctx.stream>>>(g, roots, n, reinterpret_cast<uint4*>(blocks), boff);
  ctx.launches++;
  DM_CUDA(cudaGetLastError());
  return DM_OK;
}

int clique_index_build(const GraphView& g, const int32_t* roots, int n, void* blocks, const uint32_t* boff, int m,
                       LaunchCtx& ctx) {
  if (n <= 0) return DM_OK;
  switch (m) {
    case 1: return index_build_m<1>(g, roots, n, blocks, boff, ctx);
    case 2: return index_build_m<2>(g, roots, n, blocks, boff, ctx);
    case 3: return index_build_m<3>(g, roots, n, blocks, boff, ctx);
    default: return index_build_m<4>(g, roots, n, blocks, boff, ctx);
  }
}

int clique_launch(const CliqueLaunch& L, LaunchCtx& ctx, int* grid) {
  CliqueArgs a = clique_args(L, ctx);
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
