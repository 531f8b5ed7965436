// k-clique enumeration for sm_100a: the per-task device code (bitmap and list paths).
//
// Semantics: the number of k-vertex cliques, each counted once, as the reference's clique
// driver computes (src/main/clique_PA.cu:9-32 with extend_clique, DuMatoGPU.cu:1194-1220:
// C_l = {u in N(v_l) : u > v_l} cap C_{l-1}, the leaf level adding |C_{k-2}| through
// aggregate_counter, DuMatoGPU.cu:1769-1771). The reference breaks symmetry by vertex id on
// the undirected graph; here the graph is oriented by (degree, id) rank, which counts the
// same cliques with out-degrees bounded by O(sqrt(m)).
//
// One persistent launch runs every root. A root's work is split into items that lanes (or
// warps) pull dynamically, and idle warps receive donated item ranges (lb.cuh):
//   bitmap path (out-degree d <= 64*NWMAX, NWMAX <= 4): the warp builds the local
//       adjacency bitmap of the root's out-neighbourhood L in shared memory (bit j of row i
//       set iff L[j] in N+(L[i])). Items are the local edges (c1, c2); a lane takes an item
//       and counts the (k-3)-cliques of row[c1] & row[c2] by its own DFS over 64-bit words:
//       extend = AND of two rows, compact = nothing (bit order is candidate order),
//       aggregate = popc at the last level.
//   list path (larger d, or DM_MODE_LIST): the reference's list structure. Items are the
//       first-level candidates c1; the warp extends sorted candidate lists level by level in
//       a per-warp global arena with dm_gpm::extend_intersect (a merge of lane slices, or a
//       probe of each candidate when the adjacency list is much longer) and counts the leaf
//       level with dm_gpm::intersect_count without writing it.
#pragma once

#include <climits>

#include "engine.hpp"
#include "gpm.cuh"
#include "lb.cuh"

namespace dmb {

template <int NW>
struct Bits {
  uint64_t w[NW];
};

template <int NW>
__device__ __forceinline__ int popc(const Bits<NW>& s) {
  int c = 0;
#pragma unroll
  for (int i = 0; i < NW; ++i) c += __popcll(s.w[i]);
  return c;
}

// Number of (D+1)-cliques inside the local vertex set S (rows: NW u64 words per row).
template <int D, int NW>
__device__ __forceinline__ unsigned long long count_rec(const Bits<NW>& S, const uint64_t* __restrict__ rows) {
  if constexpr (D == 0) {
    return (unsigned long long)popc(S);
  } else {
    unsigned long long sum = 0;
#pragma unroll
    for (int wi = 0; wi < NW; ++wi) {
      uint64_t bits = S.w[wi];
      while (bits) {
        const int b = __ffsll((long long)bits) - 1;
        bits &= bits - 1;
        const uint64_t* rc = rows + (wi * 64 + b) * NW;
        Bits<NW> T;
#pragma unroll
        for (int j = 0; j < NW; ++j) T.w[j] = (j < wi ? 0ull : (j == wi ? bits : S.w[j])) & rc[j];
        if constexpr (D == 1) {
          sum += (unsigned long long)popc(T);
        } else {
          if (popc(T) >= D) sum += count_rec<D - 1, NW>(T, rows);
        }
      }
    }
    return sum;
  }
}

// count_rec at the top of a long item, reporting progress to the load balancer's watched
// word every 16 subtrees: waiting warps treat a word that stops changing for the timeout as
// a lost wake-up, so an item that runs for seconds on one lane must keep it moving.
template <int D, int NW>
__device__ __forceinline__ unsigned long long count_rec_hb(const Bits<NW>& S, const uint64_t* __restrict__ rows,
                                                           unsigned long long* progress) {
  if constexpr (D < 3) {
    return count_rec<D, NW>(S, rows);
  } else {
    unsigned long long sum = 0;
    unsigned sub = 0;
#pragma unroll
    for (int wi = 0; wi < NW; ++wi) {
      uint64_t bits = S.w[wi];
      while (bits) {
        const int b = __ffsll((long long)bits) - 1;
        bits &= bits - 1;
        const uint64_t* rc = rows + (wi * 64 + b) * NW;
        Bits<NW> T;
#pragma unroll
        for (int j = 0; j < NW; ++j) T.w[j] = (j < wi ? 0ull : (j == wi ? bits : S.w[j])) & rc[j];
        if (popc(T) >= D) sum += count_rec<D - 1, NW>(T, rows);
        if ((++sub & 15) == 0) atomicAdd(progress, 1ull);
      }
    }
    return sum;
  }
}

// Position of the j-th (0-based) set bit of an NW-word row.
template <int NW>
__device__ __forceinline__ int select_bit(const uint64_t* row, int j) {
#pragma unroll
  for (int w = 0; w < NW; ++w) {
    const uint64_t x = row[w];
    const int pc = __popcll(x);
    if (j < pc) {
      const unsigned lo = (unsigned)x;
      const int pl = __popc(lo);
      if (j < pl) return w * 64 + (int)__fns(lo, 0, j + 1);
      return w * 64 + 32 + (int)__fns((unsigned)(x >> 32), 0, j - pl + 1);
    }
    j -= pc;
  }
  return -1;
}

// Shared memory of one warp for a launch whose bitmap roots need up to M words per row:
// rows | L | prefix of out-degrees | prefix of row popcounts | item range | list stack.
struct WarpLayout {
  int rows, L, P, E, range, don, busy, hn, heavy, n, pos, total;
};

constexpr int LIST_LEVELS = 16;  // list-path DFS levels kept per group (k <= 12)

__host__ __device__ constexpr WarpLayout warp_layout(int M) {
  WarpLayout w{};
  w.rows = 0;
  w.L = 512 * M * M;
  w.P = w.L + 4 * 64 * M;
  w.E = w.P + 4 * (64 * M + 1);
  w.range = (w.E + 4 * (64 * M + 1) + 7) / 8 * 8;
  w.don = w.range + 8;
  w.busy = w.don + 4;
  w.hn = w.busy + 4;
  w.heavy = w.hn + 4;  // 32 deferred heavy items
  w.n = (w.heavy + 4 * 32 + 7) / 8 * 8;  // list path: set sizes per level, 4 groups x 16 levels
  w.pos = w.n + 4 * 4 * LIST_LEVELS;       // list path: next member per level
  w.total = (w.pos + 4 * 4 * LIST_LEVELS + 15) / 16 * 16;
  return w;
}

struct CliqueArgs {
  GraphView g;
  const int32_t* roots;
  int n_roots;
  LBArgs lb;
  const int32_t* parts;         // optional per-root-entry part word (p | P << 16), else null
  int32_t* arena;               // list path: list_groups x K x arena_dcap ints per warp
  int arena_dcap;
  int list_vwarp;               // list path: lanes per group (8, 16 or 32)
  int list_threshold;           // roots with d > list_threshold take the list path
  unsigned long long* per_root; // optional: k-cliques found under each root (subtree logger)
};

// Loads L = N+(root) into shared memory and the exclusive prefix sum of the out-degrees
// of its members (sP[0..d]). Returns the total.
static __device__ __forceinline__ int load_root_list(const GraphView& g, int root, int d, int32_t* sL, int32_t* sP,
                                                     int32_t* sR) {
  const int lane = lane_id();
  const int32_t* L = g.adj + __ldg(g.row + root);
  int carry = 0;
  for (int i0 = 0; i0 < d; i0 += 32) {
    const int i = i0 + lane;
    int u = 0, du = 0;
    if (i < d) {
      u = __ldg(L + i);
      du = __ldg(g.deg + u);
      sR[i] = __ldg(g.row + u);
      sL[i] = u;
    }
    int s = du;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(FULL_MASK, s, o);
      if (lane >= o) s += y;
    }
    if (i < d) sP[i] = carry + s - du;
    carry += __shfl_sync(FULL_MASK, s, 31);
  }
  if (lane == 0) sP[d] = carry;
  __syncwarp();
  return carry;
}

// Local adjacency bitmap of L (rows zeroed by the caller): the (member, out-neighbour)
// pairs are flattened so the warp stays busy when rows are short; membership in L is a
// binary search in shared memory. Row starts come from shared memory (sR, filled with L), and
// each lane issues the loads of BUILD_UNROLL pairs before it uses any of them, so the
// adjacency loads of a lane overlap instead of forming one dependent chain per pair.
constexpr int BUILD_UNROLL = 4;

static __device__ __forceinline__ void build_local_rows(const int32_t* adj, const int32_t* sL, const int32_t* sP,
                                                        const int32_t* sR, int d, int total, uint32_t* rows,
                                                        int row_words) {
  const int lane = lane_id();
  const int32_t maxL = sL[d - 1];
  int i = 0;  // member owning pair f: the largest i with sP[i] <= f (f only grows per lane)
  for (int f0 = lane; f0 < total; f0 += 32 * BUILD_UNROLL) {
    int32_t x[BUILD_UNROLL];
    int own[BUILD_UNROLL];
#pragma unroll
    for (int u = 0; u < BUILD_UNROLL; ++u) {
      const int f = f0 + 32 * u;
      own[u] = -1;
      if (f < total) {
        while (sP[i + 1] <= f) ++i;
        own[u] = i;
        x[u] = __ldg(adj + sR[i] + (f - sP[i]));
      }
    }
#pragma unroll
    for (int u = 0; u < BUILD_UNROLL; ++u) {
      const int m = own[u];
      if (m >= 0 && x[u] <= maxL) {
        const int j = lower_bound(sL, m + 1, d, x[u]);
        if (j < d && sL[j] == x[u]) atomicOr(rows + m * row_words + (j >> 5), 1u << (j & 31));
      }
    }
  }
}

constexpr int HEAVY_BITS = 24;  // an item whose candidate set has this many members is
                                // run by the whole warp instead of one lane (k >= 6)
constexpr int HEAVY_SLOTS = 32;

// Counts the cliques of item `it` (a local edge c1 < c2, or a row c1 when k == 3) on one
// lane. For k >= 6 an item with a large candidate set is deferred to the warp instead
// (returns without counting) when a heavy slot is free.
template <int K, int NW>
__device__ __forceinline__ unsigned long long bitmap_item(int it, const uint64_t* rows, const int32_t* sE, int d,
                                                          int* hn, int* heavy, unsigned long long* progress) {
  if constexpr (K == 3) {
    Bits<NW> S;
#pragma unroll
    for (int w = 0; w < NW; ++w) S.w[w] = rows[it * NW + w];
    return (unsigned long long)popc(S);
  } else {
    const int c1 = lower_bound(sE, 0, d + 1, it + 1) - 1;
    const int c2 = select_bit<NW>(rows + c1 * NW, it - sE[c1]);
    Bits<NW> S;
#pragma unroll
    for (int w = 0; w < NW; ++w) S.w[w] = rows[c1 * NW + w] & rows[c2 * NW + w];
    if constexpr (K == 4) {
      return (unsigned long long)popc(S);
    } else {
      const int p = popc(S);
      if (p < K - 3) return 0;
      if constexpr (K >= 6) {
        if (p >= HEAVY_BITS && hn) {
          const int slot = atomicAdd(hn, 1);
          if (slot < HEAVY_SLOTS) {
            heavy[slot] = it;
            return 0;
          }
        }
      }
      return count_rec_hb<(K >= 5 ? K - 4 : 0), NW>(S, rows, progress);
    }
  }
}

// Warp-cooperative run of one heavy item: the third local vertex c3 is spread over the
// lanes (the j-th member of the candidate set goes to lane j mod 32).
template <int K, int NW>
__device__ __forceinline__ unsigned long long heavy_item(int it, const uint64_t* rows, const int32_t* sE, int d,
                                                         unsigned long long* progress) {
  const int lane = lane_id();
  const int c1 = lower_bound(sE, 0, d + 1, it + 1) - 1;
  const int c2 = select_bit<NW>(rows + c1 * NW, it - sE[c1]);
  Bits<NW> S;
#pragma unroll
  for (int w = 0; w < NW; ++w) S.w[w] = rows[c1 * NW + w] & rows[c2 * NW + w];
  unsigned long long sum = 0;
  int j = 0;
#pragma unroll
  for (int wi = 0; wi < NW; ++wi) {
    uint64_t bits = S.w[wi];
    while (bits) {
      const int b = __ffsll((long long)bits) - 1;
      bits &= bits - 1;
      if ((j++ & 31) != lane) continue;
      const uint64_t* rc = rows + (wi * 64 + b) * NW;
      Bits<NW> T;
#pragma unroll
      for (int w = 0; w < NW; ++w) T.w[w] = (w < wi ? 0ull : (w == wi ? bits : S.w[w])) & rc[w];
      if (popc(T) >= K - 4) sum += count_rec_hb<(K >= 6 ? K - 5 : 0), NW>(T, rows, progress);
    }
  }
  return sum;
}

// Bitmap path for one task. Returns the k-cliques counted by this lane.
template <int K, int NW, int M>
__device__ unsigned long long bitmap_task(const CliqueArgs& a, unsigned char* wsm, int root, int d, int b, int e) {
  constexpr WarpLayout LY = warp_layout(M);
  constexpr int RW = 2 * NW;
  const int lane = lane_id();
  uint32_t* rows32 = reinterpret_cast<uint32_t*>(wsm + LY.rows);
  int32_t* sL = reinterpret_cast<int32_t*>(wsm + LY.L);
  int32_t* sP = reinterpret_cast<int32_t*>(wsm + LY.P);
  int32_t* sE = reinterpret_cast<int32_t*>(wsm + LY.E);
  unsigned long long* range = reinterpret_cast<unsigned long long*>(wsm + LY.range);
  int* donations_left = reinterpret_cast<int*>(wsm + LY.don);
  int* busy = reinterpret_cast<int*>(wsm + LY.busy);
  int* hn = reinterpret_cast<int*>(wsm + LY.hn);
  int* heavy = reinterpret_cast<int*>(wsm + LY.heavy);
  const long long t_start = global_ns();
  for (int i = lane; i < d * RW; i += 32) rows32[i] = 0;
  // sE holds the members' row starts while the rows are built, the item prefix after
  const int total = load_root_list(a.g, root, d, sL, sP, sE);
  build_local_rows(a.g.adj, sL, sP, sE, d, total, rows32, RW);
  __syncwarp();
  const uint64_t* rows = reinterpret_cast<const uint64_t*>(rows32);
  int n_items;
  if constexpr (K >= 4) {
    // exclusive prefix of row popcounts: the items are the local edges
    int carry = 0;
    for (int i0 = 0; i0 < d; i0 += 32) {
      const int i = i0 + lane;
      int pc = 0;
      if (i < d) {
#pragma unroll
        for (int w = 0; w < NW; ++w) pc += __popcll(rows[i * NW + w]);
      }
      int s = pc;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(FULL_MASK, s, o);
        if (lane >= o) s += y;
      }
      if (i < d) sE[i] = carry + s - pc;
      carry += __shfl_sync(FULL_MASK, s, 31);
    }
    if (lane == 0) sE[d] = carry;
    n_items = carry;
  } else {
    n_items = d;
  }
  int lo, hi;
  task_range(b, e, n_items, lo, hi);
  if (lane == 0) {
    *range = pack_range(lo, hi);
    *donations_left = a.lb.max_donations;
    *busy = 0;
    *hn = 0;
  }
  __syncwarp();
  unsigned long long cnt = 0;
  unsigned done = 0;
  while (true) {
    const int it = range_take(range);
    if (it < 0) break;
    cnt += bitmap_item<K, NW>(it, rows, sE, d, hn, heavy, &a.lb.ctr->progress);
    if ((++done & 15) == 0) {
      int ob = 0, oe = 0;
      if (range_maybe_donate(a.lb, range, root, donations_left, t_start, busy, ob, oe)) {
        for (int j = ob; j < oe; ++j) cnt += bitmap_item<K, NW>(j, rows, sE, d, nullptr, nullptr, &a.lb.ctr->progress);
      }
      if ((done & 255) == 0) atomicAdd(&a.lb.ctr->progress, 256ull);
    }
  }
  __syncwarp();
  if constexpr (K >= 6) {
    const int nh = min(*hn, HEAVY_SLOTS);
    for (int h = 0; h < nh; ++h) {
      cnt += heavy_item<K, NW>(heavy[h], rows, sE, d, &a.lb.ctr->progress);
      if (lane == 0) atomicAdd(&a.lb.ctr->progress, 1ull);
    }
    __syncwarp();
  }
  return cnt;
}

// List path for one task. The warp's lanes form groups of W (the reference's virtual warps,
// src/DM_WCV/DuMatoGPU.cu:12-37, 8, 16 or 32 lanes): each group takes first-level
// candidates from the task's shared range and runs their DFS on its own stack and arena
// slice (warp_arena + group x K x arena_dcap; level l at l x arena_dcap). Returns this
// lane's share of the count; the whole warp enters and leaves together.
template <int K, int M, int W>
__device__ unsigned long long list_task_w(const CliqueArgs& a, unsigned char* wsm, int root, int d, int b, int e,
                                          int32_t* warp_arena) {
  constexpr WarpLayout LY = warp_layout(M);
  const int lane = lane_id();
  const int gl = lane & (W - 1), gi = lane / W;
  const unsigned gmask = dm_gpm::Group<W>::mask();
  unsigned long long* range = reinterpret_cast<unsigned long long*>(wsm + LY.range);
  int* donations_left = reinterpret_cast<int*>(wsm + LY.don);
  int* busy = reinterpret_cast<int*>(wsm + LY.busy);
  int* sN = reinterpret_cast<int*>(wsm + LY.n) + gi * LIST_LEVELS;
  int* sPos = reinterpret_cast<int*>(wsm + LY.pos) + gi * LIST_LEVELS;
  int32_t* my_arena = warp_arena + (size_t)gi * K * a.arena_dcap;
  const long long t_start = global_ns();
  const int32_t* L = a.g.adj + __ldg(a.g.row + root);
  int lo, hi;
  task_range(b, e, d, lo, hi);
  if (lane == 0) {
    *range = pack_range(lo, hi);
    *donations_left = a.lb.max_donations;
    *busy = 0;
  }
  __syncwarp();
  unsigned long long cnt = 0;
  int spill_b = 0, spill_e = 0;  // group leader: items split off when the queue was full
  while (true) {
    int it = -1;
    if (gl == 0) {
      if (spill_b < spill_e) {
        it = spill_b++;
      } else {
        it = range_take(range);
        int ob = 0, oe = 0;
        if (it >= 0 && range_maybe_donate(a.lb, range, root, donations_left, t_start, busy, ob, oe)) {
          spill_b = ob;
          spill_e = oe;
        }
      }
    }
    it = __shfl_sync(gmask, it, 0, W);
    if (it < 0) break;
    const int c = __ldg(L + it);
    const int32_t* A = L + it + 1;
    const int na = d - it - 1;
    if (na < K - 2) continue;
    const int32_t* B = a.g.adj + __ldg(a.g.row + c);
    const int nb = __ldg(a.g.deg + c);
    if constexpr (K == 3) {
      const int s = dm_gpm::intersect_count<W>(A, na, B, nb);
      if (gl == 0) cnt += (unsigned)s;
    } else {
      // C1 = A cap N+(c), written to level 1 of the group's arena
      const int m = dm_gpm::extend_intersect<W>(A, na, B, nb, my_arena + a.arena_dcap);
      __syncwarp(gmask);
      if (gl == 0) {
        sN[1] = m;
        sPos[1] = 0;
      }
      __syncwarp(gmask);
      int lvl = 1;
      while (lvl >= 1) {
        const int pos = sPos[lvl];
        const int rem = sN[lvl] - pos;
        if (rem - 1 < K - 2 - lvl) {
          --lvl;
          continue;
        }
        const int32_t* P = my_arena + (size_t)lvl * a.arena_dcap;
        const int v = P[pos];
        __syncwarp(gmask);
        if (gl == 0) {
          sPos[lvl] = pos + 1;
          if ((pos & 63) == 63) atomicAdd(&a.lb.ctr->progress, 64ull);
        }
        const int32_t* A2 = P + pos + 1;
        const int na2 = rem - 1;
        const int32_t* B2 = a.g.adj + __ldg(a.g.row + v);
        const int nb2 = __ldg(a.g.deg + v);
        if (lvl + 1 == K - 2) {
          const int s = dm_gpm::intersect_count<W>(A2, na2, B2, nb2);
          if (gl == 0) cnt += (unsigned)s;
        } else {
          const int m2 = dm_gpm::extend_intersect<W>(A2, na2, B2, nb2, my_arena + (size_t)(lvl + 1) * a.arena_dcap);
          __syncwarp(gmask);
          ++lvl;
          if (gl == 0) {
            sN[lvl] = m2;
            sPos[lvl] = 0;
          }
        }
        __syncwarp(gmask);
      }
    }
  }
  __syncwarp();
  return cnt;
}

template <int K, int M>
__device__ __forceinline__ unsigned long long list_task(const CliqueArgs& a, unsigned char* wsm, int root, int d,
                                                        int b, int e, int32_t* warp_arena) {
  switch (a.list_vwarp) {
    case 8: return list_task_w<K, M, 8>(a, wsm, root, d, b, e, warp_arena);
    case 16: return list_task_w<K, M, 16>(a, wsm, root, d, b, e, warp_arena);
    default: return list_task_w<K, M, 32>(a, wsm, root, d, b, e, warp_arena);
  }
}

// One root task: items [b, e) of root (task_range encoding), on the bitmap path when the
// out-degree d is at most a.list_threshold (local bitmaps of ceil(d/64) <= M words per row),
// else on the list path (needs `arena` with room for K lists of a.arena_dcap ids). Returns
// this lane's share of the k-cliques found.
template <int K, int M>
__device__ __forceinline__ unsigned long long clique_task(const CliqueArgs& a, unsigned char* wsm, int root, int b,
                                                          int e, int32_t* arena) {
  const int lane = lane_id();
  const int d = __ldg(a.g.deg + root);
  unsigned long long task_cnt = 0;
  if (e >= 0 && b >= e) {
    // empty donation: nothing to do
  } else if (K == 2) {
    if (lane == 0) task_cnt = (unsigned long long)d;
  } else if (d > a.list_threshold) {
    if (K > 3 && (!arena || d > a.arena_dcap)) {
      if (lane == 0) set_err(a.lb.ctr, ERR_ARENA_OVERFLOW);
    } else {
      task_cnt = list_task<K, M>(a, wsm, root, d, b, e, arena);
    }
  } else {
    const int nw = (d + 63) >> 6;
    if (nw <= 1) task_cnt = bitmap_task<K, 1, M>(a, wsm, root, d, b, e);
    else if (M >= 2 && nw == 2) task_cnt = bitmap_task<K, (M >= 2 ? 2 : 1), M>(a, wsm, root, d, b, e);
    else if (M >= 3 && nw == 3) task_cnt = bitmap_task<K, (M >= 3 ? 3 : 1), M>(a, wsm, root, d, b, e);
    else if (M >= 4 && nw == 4) task_cnt = bitmap_task<K, (M >= 4 ? 4 : 1), M>(a, wsm, root, d, b, e);
    else if (lane == 0) set_err(a.lb.ctr, ERR_BAD_TASK);
  }
  return task_cnt;
}

}  // namespace dmb
