// The single-graph k-clique kernel template and its launch helpers, shared by the
// translation units that instantiate it (clique.cu: k = 2..6; clique_k7_8.cu and
// clique_k9.cu .. clique_k12.cu: the larger k, split so the unrolled DFS of each k compiles
// in parallel).
#pragma once

#include <algorithm>
#include <climits>
#include <string>

#include "clique.cuh"
#include "clique_cached.cuh"

namespace dmb {

template <int K, int M>
__global__ void __launch_bounds__(256) clique_kernel(const __grid_constant__ CliqueArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  constexpr WarpLayout LY = warp_layout(M);
  const int lane = lane_id();
  unsigned char* wsm = smem + (size_t)LY.total * warp_in_block();
  const size_t gw = (size_t)blockIdx.x * (blockDim.x >> 5) + warp_in_block();
  const int total_warps = gridDim.x * (blockDim.x >> 5);
  int32_t* my_arena = a.arena ? a.arena + gw * (size_t)(32 / a.list_vwarp) * K * a.arena_dcap : nullptr;
  unsigned long long cnt = 0, ntasks = 0;
  while (true) {
    int first = 0, count = 0, b = 0, e = -1, ok = 0;
    bool donated = false;
    int level = 0, path[QPATH];
    if (lane == 0) ok = lb_next(a.lb, a.n_roots, total_warps, first, count, b, e, donated, level, path) ? 1 : 0;
    ok = __shfl_sync(FULL_MASK, ok, 0);
    if (!ok) break;
    first = __shfl_sync(FULL_MASK, first, 0);
    count = __shfl_sync(FULL_MASK, count, 0);
    b = __shfl_sync(FULL_MASK, b, 0);
    e = __shfl_sync(FULL_MASK, e, 0);
    donated = __shfl_sync(FULL_MASK, donated ? 1 : 0, 0) != 0;
    for (int ti = 0; ti < count; ++ti) {
      const int root = donated ? first : __ldg(a.roots + first + ti);
      int bb = b, ee = e;
      if (!donated && a.parts) part_bounds(__ldg(a.parts + first + ti), bb, ee);
      ++ntasks;
      const unsigned long long task_cnt = clique_task<K, M>(a, wsm, root, bb, ee, my_arena);
      cnt += task_cnt;
      if (a.per_root) {
        const unsigned long long tsum = warp_sum_u64(task_cnt);
        if (lane == 0 && tsum) atomicAdd(a.per_root + root, tsum);
      }
      __syncwarp();
    }
    if (lane == 0) lb_done(a.lb, count);
  }
  dm_gpm::aggregate_counter<32>(&a.lb.ctr->count, cnt);
  if (lane == 0) atomicAdd(&a.lb.ctr->tasks, ntasks);
}

// ---------------- host launcher ----------------

constexpr int CLIQUE_BLOCK = 256;

template <int K, int M>
static int launch_k(const CliqueArgs& a, LaunchCtx& ctx, int* grid_out) {
  const size_t smem = (size_t)warp_layout(M).total * (CLIQUE_BLOCK / 32);
  auto kern = clique_kernel<K, M>;
  static LaunchCache cache;
  int occ = 0;
  DM_CUDA(cached_occupancy(cache, kern, ctx.device, CLIQUE_BLOCK, smem, &occ));
  if (occ < 1) return fail(DM_EINVAL, "clique kernel does not fit on an SM");
  int grid = ctx.num_sms * occ;
  if (ctx.threads > 0) grid = std::max(1, std::min(grid, (ctx.threads + CLIQUE_BLOCK - 1) / CLIQUE_BLOCK));
  if (a.arena && grid * (CLIQUE_BLOCK / 32) > ctx.arena_warps) grid = std::max(1, ctx.arena_warps / (CLIQUE_BLOCK / 32));
  CliqueArgs args = a;
  const int warps = grid * (CLIQUE_BLOCK / 32);
  args.lb.hungry_trigger =
      ctx.threshold >= 100 ? 0 : std::max(1, (ctx.threshold * warps + 99) / 100);
  kern<<<grid, CLIQUE_BLOCK, smem, ctx.stream>>>(args);
  ctx.launches++;
  *grid_out = grid;
  DM_CUDA(cudaGetLastError());
  return DM_OK;
}

template <int K>
static int launch_nw(const CliqueArgs& a, int m, LaunchCtx& ctx, int* grid) {
  switch (m) {
    case 1: return launch_k<K, 1>(a, ctx, grid);
    case 2: return launch_k<K, 2>(a, ctx, grid);
    case 3: return launch_k<K, 3>(a, ctx, grid);
    default: return launch_k<K, 4>(a, ctx, grid);
  }
}

// Index-counting kernel: with query set, only the grid is computed.
template <int K, int M, bool TMA, bool MULTI>
static int cached_k(CachedArgs* a, LaunchCtx& ctx, int* grid_out, bool query) {
  const size_t smem = (size_t)cached_layout(M).total * (CLIQUE_BLOCK / 32);
  auto kern = clique_cached_kernel<K, M, TMA, MULTI>;
  static LaunchCache cache;
  int occ = 0;
  DM_CUDA(cached_occupancy(cache, kern, ctx.device, CLIQUE_BLOCK, smem, &occ));
  if (occ < 1) return fail(DM_EINVAL, "clique index kernel does not fit on an SM");
  int grid = ctx.num_sms * occ;
  if (ctx.threads > 0) grid = std::max(1, std::min(grid, (ctx.threads + CLIQUE_BLOCK - 1) / CLIQUE_BLOCK));
  if (a->c.arena && grid * (CLIQUE_BLOCK / 32) > ctx.arena_warps)
    grid = std::max(1, ctx.arena_warps / (CLIQUE_BLOCK / 32));
  if (!query && grid != *grid_out) return fail(DM_EINVAL, "clique index kernel: grid differs from its plan");
  *grid_out = grid;
  if (query) return DM_OK;
  const int warps = grid * (CLIQUE_BLOCK / 32);
  a->c.lb.hungry_trigger = ctx.threshold >= 100 ? 0 : std::max(1, (ctx.threshold * warps + 99) / 100);
  kern<<<grid, CLIQUE_BLOCK, smem, ctx.stream>>>(*a);
  ctx.launches++;
  DM_CUDA(cudaGetLastError());
  return DM_OK;
}

// Fused counts (every size up to K) are staged by bulk copies only.
template <int K, int M>
static int cached_m(CachedArgs* a, bool tma, bool multi, LaunchCtx& ctx, int* grid, bool query) {
  if (multi) {
    if constexpr (K >= 4) return cached_k<K, M, true, true>(a, ctx, grid, query);
    else return fail(DM_EINVAL, "fused clique counts need k >= 4");
  }
  return tma ? cached_k<K, M, true, false>(a, ctx, grid, query) : cached_k<K, M, false, false>(a, ctx, grid, query);
}

template <int K>
static int cached_nw(CachedArgs* a, int m, bool tma, bool multi, LaunchCtx& ctx, int* grid, bool query) {
  switch (m) {
    case 1: return cached_m<K, 1>(a, tma, multi, ctx, grid, query);
    case 2: return cached_m<K, 2>(a, tma, multi, ctx, grid, query);
    case 3: return cached_m<K, 3>(a, tma, multi, ctx, grid, query);
    default: return cached_m<K, 4>(a, tma, multi, ctx, grid, query);
  }
}

// Launchers of the k ranges compiled in the other translation units.
int clique_cached_k7_8(CachedArgs* a, int k, int m, bool tma, bool multi, LaunchCtx& ctx, int* grid, bool query);

int clique_launch_k7_8(const CliqueArgs& a, int k, int m, LaunchCtx& ctx, int* grid);
int clique_launch_k9(const CliqueArgs& a, int m, LaunchCtx& ctx, int* grid);
int clique_launch_k10(const CliqueArgs& a, int m, LaunchCtx& ctx, int* grid);
int clique_launch_k11(const CliqueArgs& a, int m, LaunchCtx& ctx, int* grid);
int clique_launch_k12(const CliqueArgs& a, int m, LaunchCtx& ctx, int* grid);

}  // namespace dmb
