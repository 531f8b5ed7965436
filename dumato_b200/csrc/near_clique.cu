// The reference's pattern-aware queries q4..q13 (src/main/q4_PA.cu .. q13_PA.cu; extension
// steps DuMatoGPU.cu:1222-1445): query q_n grows an (n-2)-clique v_0 < .. < v_{n-3}
// (extend_single from v_0 above v_0, then `intersect` of the previous set with N(v_l) above
// v_l), then takes v_{n-2} from the common neighbourhood of the clique (extend_single +
// intersect_unique over every clique vertex) and v_{n-1} from the same set above v_{n-2}
// (copy_extensions), counting at the last level. Every embedding it counts is therefore an
// (n-2)-clique C plus an unordered pair of vertices adjacent to all of C - a non-induced copy
// of K_n minus one edge - and the count is
//     q_n = sum over (n-2)-cliques C of  t_C (t_C - 1) / 2,   t_C = |common neighbourhood of C|.
//
// Here each (n-2)-clique is found once, from its lowest-ranked vertex, by a warp-cooperative
// list DFS on the degree-ordered DAG (dm_gpm::extend_intersect), and t_C is the size of the
// intersection of the members' rows in the undirected CSR (original ids), computed from the
// shortest row by dm_gpm::extend_intersect / intersect_count. Root tasks are claimed from the
// shared cursor in runs (lb.cuh); there is no donation in this kernel.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <string>

#include "engine.hpp"
#include "gpm.cuh"
#include "lb.cuh"

namespace dmb {

struct NearArgs {
  GraphView dag;          // rank-space out-lists
  GraphView und;          // undirected CSR, original ids
  const int32_t* orig;    // rank -> original id
  const int32_t* roots;   // roots (rank space)
  int n_roots;
  LBArgs lb;
  int32_t* arena;         // per warp: C levels of dag_cap ints, then 2 lists of und_cap ints
  int dag_cap, und_cap;
};

constexpr int NEAR_WARPS = 8;

// t (t - 1) / 2 for the common neighbourhood of the clique held in members[0..C) (rank space).
template <int C>
__device__ unsigned long long near_pairs(const NearArgs& a, const int32_t* members, int32_t* s0, int32_t* s1) {
  // the member with the shortest undirected row first
  int best = 0, best_deg = INT_MAX;
  int32_t ids[C];
#pragma unroll
  for (int i = 0; i < C; ++i) {
    ids[i] = __ldg(a.orig + members[i]);
    const int dg = __ldg(a.und.deg + ids[i]);
    if (dg < best_deg) {
      best_deg = dg;
      best = i;
    }
  }
  const int32_t* cur = a.und.adj + __ldg(a.und.row + ids[best]);
  int n = best_deg;
  int t = 0;
  int done = 1;
#pragma unroll
  for (int i = 0; i < C; ++i) {
    if (i == best) continue;
    const int32_t* B = a.und.adj + __ldg(a.und.row + ids[i]);
    const int nb = __ldg(a.und.deg + ids[i]);
    if (++done == C) {
      t = dm_gpm::intersect_count<32>(cur, n, B, nb);
    } else {
      int32_t* out = (done & 1) ? s0 : s1;
      n = dm_gpm::extend_intersect<32>(cur, n, B, nb, out);
      __syncwarp();
      cur = out;
    }
    if (n == 0) {
      t = 0;
      break;
    }
  }
  return (unsigned long long)t * (unsigned long long)(t > 0 ? t - 1 : 0) / 2ull;
}

template <int C>
__global__ void __launch_bounds__(32 * NEAR_WARPS) near_clique_kernel(const __grid_constant__ NearArgs a) {
  __shared__ int sN[NEAR_WARPS][C > 1 ? C : 2], sPos[NEAR_WARPS][C > 1 ? C : 2];
  __shared__ int32_t sMem[NEAR_WARPS][C];
  const int lane = lane_id();
  const int wib = warp_in_block();
  const int gw = blockIdx.x * NEAR_WARPS + wib;
  const int total_warps = gridDim.x * NEAR_WARPS;
  int32_t* base = a.arena + (size_t)gw * ((size_t)C * a.dag_cap + 2 * (size_t)a.und_cap);
  int32_t* s0 = base + (size_t)C * a.dag_cap;
  int32_t* s1 = s0 + a.und_cap;
  int* N = sN[wib];
  int* Pos = sPos[wib];
  int32_t* mem = sMem[wib];
  unsigned long long cnt = 0, ntasks = 0;
  while (true) {
    int first = 0, count = 0, b = 0, e = -1, ok = 0, level = 0;
    int path[QPATH];
    bool donated = false;
    if (lane == 0) ok = lb_next(a.lb, a.n_roots, total_warps, first, count, b, e, donated, level, path) ? 1 : 0;
    ok = __shfl_sync(FULL_MASK, ok, 0);
    if (!ok) break;
    first = __shfl_sync(FULL_MASK, first, 0);
    count = __shfl_sync(FULL_MASK, count, 0);
    ntasks += count;
    for (int ti = 0; ti < count; ++ti) {
      const int root = __ldg(a.roots + first + ti);
      if (lane == 0) mem[0] = root;
      const int32_t* L = a.dag.adj + __ldg(a.dag.row + root);
      const int d = __ldg(a.dag.deg + root);
      if constexpr (C == 2) {
        for (int i = 0; i < d; ++i) {
          if (lane == 0) mem[1] = __ldg(L + i);
          __syncwarp();
          cnt += near_pairs<C>(a, mem, s0, s1);
          __syncwarp();
        }
      } else {
        // level l (1..C-1) holds the candidates of the (l+1)-th member: level 1 = N+(root)
        if (lane == 0) {
          N[1] = d;
          Pos[1] = 0;
        }
        __syncwarp();
        int lvl = 1;
        while (lvl >= 1) {
          const int pos = Pos[lvl];
          const int rem = N[lvl] - pos;
          if (rem < C - lvl) {  // not enough candidates left to complete the clique
            --lvl;
            continue;
          }
          const int32_t* P = lvl == 1 ? L : base + (size_t)lvl * a.dag_cap;
          const int v = P[pos];
          __syncwarp();
          if (lane == 0) {
            Pos[lvl] = pos + 1;
            mem[lvl] = v;
            if ((pos & 63) == 63) atomicAdd(&a.lb.ctr->progress, 64ull);
          }
          __syncwarp();
          if (lvl == C - 1) {
            cnt += near_pairs<C>(a, mem, s0, s1);
            __syncwarp();
            continue;
          }
          const int32_t* B = a.dag.adj + __ldg(a.dag.row + v);
          const int nb = __ldg(a.dag.deg + v);
          const int m = dm_gpm::extend_intersect<32>(P + pos + 1, rem - 1, B, nb, base + (size_t)(lvl + 1) * a.dag_cap);
          __syncwarp();
          if (lane == 0) {
            N[lvl + 1] = m;
            Pos[lvl + 1] = 0;
          }
          __syncwarp();
          ++lvl;
        }
      }
      __syncwarp();
    }
    if (lane == 0) lb_done(a.lb, count);
  }
  // near_pairs returns the same value on every lane: count it once per warp
  if (lane == 0) {
    atomicAdd(&a.lb.ctr->count, cnt);
    atomicAdd(&a.lb.ctr->tasks, ntasks);
  }
}

template <int C>
static int launch_near(const NearArgs& a0, LaunchCtx& ctx, int* grid_out) {
  const int block = 32 * NEAR_WARPS;
  auto kern = near_clique_kernel<C>;
  static LaunchCache cache;
  int occ = 0;
  DM_CUDA(cached_occupancy(cache, kern, ctx.device, block, 0, &occ));
  if (occ < 1) return fail(DM_EINVAL, "near-clique kernel does not fit on an SM");
  int grid = ctx.num_sms * occ;
  if (ctx.threads > 0) grid = std::max(1, std::min(grid, (ctx.threads + block - 1) / block));
  if (grid * NEAR_WARPS > ctx.arena_warps) grid = std::max(1, ctx.arena_warps / NEAR_WARPS);
  NearArgs a = a0;
  a.lb.hungry_trigger = 0;  // no donation in this kernel
  kern<<<grid, block, 0, ctx.stream>>>(a);
  ctx.launches++;
  *grid_out = grid;
  DM_CUDA(cudaGetLastError());
  return DM_OK;
}

int near_clique_launch(const NearLaunch& L, LaunchCtx& ctx, int* grid) {
  NearArgs a;
  a.dag = L.dag;
  a.und = L.und;
  a.orig = L.orig;
  a.roots = L.roots;
  a.n_roots = L.n_roots;
  a.lb = LBArgs{L.ctr, reinterpret_cast<QHeader*>(L.queue),
                reinterpret_cast<QSlot*>(reinterpret_cast<char*>(L.queue) + sizeof(QHeader) * L.nq), L.qcap, 0, 0,
                (long long)ctx.donate_after_us * 1000ll, (long long)ctx.timeout_ms * 1000000ll, ctx.test_stall, 32,
                L.nq};
  a.arena = L.arena;
  a.dag_cap = L.dag_cap;
  a.und_cap = L.und_cap;
  switch (L.c) {
    case 2: return launch_near<2>(a, ctx, grid);
    case 3: return launch_near<3>(a, ctx, grid);
    case 4: return launch_near<4>(a, ctx, grid);
    case 5: return launch_near<5>(a, ctx, grid);
    case 6: return launch_near<6>(a, ctx, grid);
    case 7: return launch_near<7>(a, ctx, grid);
    case 8: return launch_near<8>(a, ctx, grid);
    case 9: return launch_near<9>(a, ctx, grid);
    case 10: return launch_near<10>(a, ctx, grid);
    case 11: return launch_near<11>(a, ctx, grid);
    default: return fail(DM_EINVAL, "near-clique queries take n in [4, 13]");
  }
}

size_t near_clique_warp_ints(int c, int dag_cap, int und_cap) { return (size_t)c * dag_cap + 2 * (size_t)und_cap; }

}  // namespace dmb
