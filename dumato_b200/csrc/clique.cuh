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
//       and counts the (k-3)-cliques of row[c1] & row[c2] by a depth-first walk over 64-bit
//       words that the warp's lanes step in lockstep (Walk, lockstep_items): extend = AND of
//       two rows, compact = nothing (bit order is candidate order), aggregate = popc at the
//       last level.
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

// Select the j-th set bit of a register bitset.
template <int NW>
__device__ __forceinline__ int select_bits(const Bits<NW>& S, int j) {
#pragma unroll
  for (int w = 0; w < NW; ++w) {
    const uint64_t x = S.w[w];
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

// Position of the k-th (0-based) set bit of a 64-bit word, without branches (a popcount
// halving search: the lanes of a warp stay together whatever their words).
__device__ __forceinline__ int select64(uint64_t v, int k) {
  const unsigned lo = (unsigned)v;
  const int c = __popc(lo);
  const bool up = k >= c;
  k -= up ? c : 0;
  unsigned w = up ? (unsigned)(v >> 32) : lo;
  int pos = up ? 32 : 0;
#pragma unroll
  for (int s = 16; s >= 1; s >>= 1) {
    const int cc = __popc(w & ((1u << s) - 1u));
    const bool u = k >= cc;
    k -= u ? cc : 0;
    w = u ? (w >> s) : w;
    pos += u ? s : 0;
  }
  return pos;
}

// First index i in [0, n) with a[i] >= x (n if none), for 1 <= n <= 2 * TOP, without
// branches: a fixed number of halving steps.
template <int TOP>
__device__ __forceinline__ int lower_bound_bl(const int32_t* a, int n, int32_t x) {
  static_assert(TOP > 0 && (TOP & (TOP - 1)) == 0, "the halving steps must be powers of two");
  int lo = 0;
#pragma unroll
  for (int h = TOP; h >= 1; h >>= 1) {
    const int idx = (lo + h < n ? lo + h : n) - 1;
    lo = (lo + h <= n && a[idx] < x) ? lo + h : lo;
  }
  return lo;
}

// The k-th (0-based) set bit of an NW-word row, without branches.
template <int NW>
__device__ __forceinline__ int select_row(const uint64_t* row, int k) {
  if constexpr (NW == 1) {
    return select64(row[0], k);
  } else {
    int base = 0;
    uint64_t word = row[0];
    bool found = false;
#pragma unroll
    for (int w = 0; w < NW; ++w) {
      const uint64_t v = row[w];
      const int pc = __popcll(v);
      const bool here = !found && k < pc;
      word = here ? v : word;
      base = here ? w * 64 : base;
      k -= (!found && !here) ? pc : 0;
      found = found || here;
    }
    return base + select64(word, k);
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

// The per-task words of a warp (shared memory).
struct TaskWords {
  unsigned long long* range;  // item (or position) range: next | end << 32
  int* don;                   // donations left to the task
  int* busy;                  // serialises donations
  int* hn;                    // deferred heavy items
  int* heavy;                 // their item indices
  uint64_t* stk = nullptr;    // the warp's walk stack (WalkR), where the kernel has one
};

// Per-lane clique counts by size (the fused count of every k up to K): c[s] = s-cliques.
template <int K>
struct Acc {
  unsigned long long c[K + 1];
};

// ---------------- lockstep walk ----------------
//
// A lane's share of a task is a depth-first walk over candidate sets, kept as an explicit
// stack of bitsets in registers, and each iteration of the warp's loop expands exactly one
// node on every lane that has one: pop the lowest member x of the top set and form
// T = (the rest of that set) & row[x]. All lanes run the same instructions on their own sets,
// so a warp costs about the largest lane's node count, where nested per-lane recursion costs,
// level by level, the sum of subtrees that the lanes reach at different loop positions. Lanes
// whose walk has ended take new items together, with one shared-memory atomic for all of
// them.
//
// Stack entry j holds the candidates for clique vertex LEV0 + j (vertices numbered from 1,
// the root first). Fused counts (MULTI): a set X formed for entry j adds |X| to c[LEV0 + j]
// and is expanded while LEV0 + j < K and |X| >= 2. One size K: |X| counts only at entry
// K - LEV0, and a set is kept only while it can still complete a K-clique. `live` has bit j
// set while entry j holds members.
constexpr int REFILL_MIN = 8;    // idle lanes that take new items while other lanes still walk
constexpr int CHECK_EVERY = 64;  // loop iterations between two donation checks (lane 0)

template <int K, int NW, bool MULTI, int LEV0>
struct Walk {
  static constexpr int D = K - LEV0 > 0 ? K - LEV0 : 1;
  Bits<NW> st[D];
  const uint64_t* rows = nullptr;  // the local bitmap rows of the walk's root
  int top = -1;
  unsigned live = 0u;

  // S: the candidates for vertex LEV0, rows: the root's local bitmap rows.
  __device__ __forceinline__ void start(const Bits<NW>& S, const uint64_t* root_rows, Acc<K>& acc,
                                        unsigned long long& cnt) {
    rows = root_rows;
    const int p = popc(S);
    if constexpr (MULTI) {
      acc.c[LEV0] += (unsigned long long)p;
      if constexpr (LEV0 < K) {
        if (p >= 2) {
          st[0] = S;
          top = 0;
          live = 1u;
        }
      }
    } else {
      if constexpr (LEV0 == K) {
        cnt += (unsigned long long)p;
      } else if (p >= K - LEV0 + 1) {
        st[0] = S;
        top = 0;
        live = 1u;
      }
    }
  }

  __device__ __forceinline__ void flush(Acc<K>&) {}

  // Expands one node of this lane's walk (top >= 0).
  __device__ __forceinline__ void step(Acc<K>& acc, unsigned long long& cnt) {
    if constexpr (LEV0 < K) {
      const int j = top;
      Bits<NW> cur;
#pragma unroll
      for (int q = 0; q < D; ++q)
        if (q == j) cur = st[q];
      int x = 0;
      bool found = false;
#pragma unroll
      for (int w = 0; w < NW; ++w) {
        if (!found && cur.w[w] != 0ull) {
          x = w * 64 + __ffsll((long long)cur.w[w]) - 1;
          cur.w[w] &= cur.w[w] - 1ull;
          found = true;
        }
      }
      const uint64_t* rx = rows + x * NW;
      Bits<NW> T;
#pragma unroll
      for (int w = 0; w < NW; ++w) T.w[w] = cur.w[w] & rx[w];
      const int pc = popc(T);
      bool push = false;
      if constexpr (MULTI) {
#pragma unroll
        for (int q = 0; q < D; ++q)
          if (q == j) acc.c[LEV0 + q + 1] += (unsigned long long)pc;
        push = LEV0 + j + 1 < K && pc >= 2;
      } else {
        if (LEV0 + j + 1 == K) cnt += (unsigned long long)pc;
        else push = pc >= K - LEV0 - j;
        // members left at this entry need K - LEV0 - j more vertices above them
        if (popc(cur) <= K - LEV0 - j) {
#pragma unroll
          for (int w = 0; w < NW; ++w) cur.w[w] = 0ull;
        }
      }
      uint64_t any = 0ull;
#pragma unroll
      for (int w = 0; w < NW; ++w) any |= cur.w[w];
#pragma unroll
      for (int q = 0; q < D; ++q)
        if (q == j) st[q] = cur;
      if (!any) live &= ~(1u << j);
      if (push) {
#pragma unroll
        for (int q = 1; q < D; ++q)
          if (q == j + 1) st[q] = T;
        live |= 1u << (j + 1);
        top = j + 1;
      } else if (!any) {
        top = live ? 31 - __clz((int)live) : -1;
      }
    }
  }
};

// Warp-lifetime state of the donation checks (lane 0): the hungry/queued counters loaded at
// the previous check, still in flight until the next one uses them, and the loop iterations
// run so far, across tasks.
struct CheckState {
  int hungry = 0;
  int queued = 0;
  unsigned iter = 0u;
};

// The walk as the index kernel runs it: the top set in registers, the entries below it in
// shared memory (stk: [entry][word][lane] u64 words of the warp, D - 1 entries), `live` bit j
// set while entry j holds members, and the fused counts in separate scalars. One step is
// branch-free: it reads the parent entry while the row of x loads and picks the next top set
// with selects, so a lane's choice between going down, staying and going up never splits the
// warp (a step is a chain of dependent operations: it costs the same for one lane or 32).
template <int K, int NW, bool MULTI, int LEV0>
struct WalkR {
  static constexpr int D = K - LEV0 > 0 ? K - LEV0 : 1;
  static_assert(!MULTI || D <= 4, "fused counts keep four level counters");
  uint64_t* stk = nullptr;
  const uint64_t* rows = nullptr;
  Bits<NW> cur;
  int top = -1;
  unsigned live = 0u;
  unsigned long long q0 = 0, q1 = 0, q2 = 0, q3 = 0;  // fused: counts at LEV0 + 1 + q

  // S: the candidates for vertex LEV0, root_rows: the root's local bitmap rows.
  __device__ __forceinline__ void start(const Bits<NW>& S, const uint64_t* root_rows, Acc<K>& acc,
                                        unsigned long long& cnt) {
    rows = root_rows;
    const int p = popc(S);
    bool go = false;
    if constexpr (MULTI) {
      acc.c[LEV0] += (unsigned long long)p;
      if constexpr (LEV0 < K) go = p >= 2;
    } else {
      if constexpr (LEV0 == K) cnt += (unsigned long long)p;
      else go = p >= K - LEV0 + 1;
    }
    if (go) {
      cur = S;
      top = 0;
      live = 0u;
    }
  }

  // Expands one node (top >= 0).
  __device__ __forceinline__ void step(Acc<K>& /*acc*/, unsigned long long& cnt) {
    if constexpr (LEV0 < K) {
      const int lane = lane_id();
      const int j = top;
      int x = 0;
      bool found = false;
      Bits<NW> rest;
#pragma unroll
      for (int w = 0; w < NW; ++w) {
        const uint64_t v = cur.w[w];
        const bool here = !found && v != 0ull;
        x = here ? w * 64 + __ffsll((long long)v) - 1 : x;
        rest.w[w] = here ? (v & (v - 1ull)) : v;
        found = found || here;
      }
      const unsigned below = live & ((1u << j) - 1u);
      const int tgt = below ? 31 - __clz((int)below) : -1;
      Bits<NW> par;
      if constexpr (D >= 2) {
        const int ti = tgt < 0 ? 0 : tgt;
#pragma unroll
        for (int w = 0; w < NW; ++w) par.w[w] = stk[(ti * NW + w) * 32 + lane];
      } else {
#pragma unroll
        for (int w = 0; w < NW; ++w) par.w[w] = 0ull;
      }
      Bits<NW> T;
#pragma unroll
      for (int w = 0; w < NW; ++w) T.w[w] = rest.w[w] & rows[x * NW + w];
      const int pc = popc(T);
      bool push;
      if constexpr (MULTI) {
        q0 += j == 0 ? (unsigned long long)pc : 0ull;
        if constexpr (D > 1) q1 += j == 1 ? (unsigned long long)pc : 0ull;
        if constexpr (D > 2) q2 += j == 2 ? (unsigned long long)pc : 0ull;
        if constexpr (D > 3) q3 += j == 3 ? (unsigned long long)pc : 0ull;
        push = LEV0 + j + 1 < K && pc >= 2;
      } else {
        cnt += LEV0 + j + 1 == K ? (unsigned long long)pc : 0ull;
        push = LEV0 + j + 1 < K && pc >= K - LEV0 - j;
        // members left at this entry need K - LEV0 - j more vertices above them
        const bool keep = popc(rest) > K - LEV0 - j;
#pragma unroll
        for (int w = 0; w < NW; ++w) rest.w[w] = keep ? rest.w[w] : 0ull;
      }
      uint64_t any = 0ull;
#pragma unroll
      for (int w = 0; w < NW; ++w) any |= rest.w[w];
      if constexpr (D >= 2) {
        if (push && any) {
#pragma unroll
          for (int w = 0; w < NW; ++w) stk[(j * NW + w) * 32 + lane] = rest.w[w];
        }
      }
#pragma unroll
      for (int w = 0; w < NW; ++w) cur.w[w] = push ? T.w[w] : (any ? rest.w[w] : par.w[w]);
      const unsigned live_up = tgt >= 0 ? (live & ~(1u << tgt)) : 0u;
      live = push ? (any ? (live | (1u << j)) : live) : (any ? live : live_up);
      top = push ? j + 1 : (any ? j : tgt);
    }
  }

  // Adds the fused counts of the steps taken to acc.
  __device__ __forceinline__ void flush(Acc<K>& acc) {
    if constexpr (MULTI && LEV0 < K) {
      acc.c[LEV0 + 1] += q0;
      if constexpr (D > 1) acc.c[LEV0 + 2] += q1;
      if constexpr (D > 2) acc.c[LEV0 + 3] += q2;
      if constexpr (D > 3) acc.c[LEV0 + 4] += q3;
      q0 = q1 = q2 = q3 = 0ull;
    }
  }
};

// Shared-memory words a warp's WalkR stack needs (entries below the top).
__host__ __device__ constexpr int walk_stack_words(int K, int NW, int LEV0) {
  return (K - LEV0 > 1 ? K - LEV0 - 1 : 0) * NW * 32;
}

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// The warp's loop over the items of tw.range: idle lanes take items (start_item(i) gives a
// lane item i), walking lanes expand one node each. Lane 0 decides on donations without a
// blocking load: from the counters it sampled at its previous check (loads that stay in
// flight meanwhile), the items it knows are left, and the task's age in SM clock cycles
// (two per nanosecond of donate_after_ns); it decides after every refill that leaves items in
// the range and every CHECK_EVERY iterations, where it also takes a new sample, and then
// range_split_donate splits the range. Items split off that no queue slot took are run after
// the range. Returns when every item is done.
// Lane 0: splits the rest of tw.range off as range_split_donate does when the sampled demand
// asks for it, `left` items remain and the task is old enough (or eager); items that no queue
// slot took are kept in [xb, xe).
__device__ __forceinline__ void lockstep_donate(const LBArgs& lb, const TaskWords& tw, CheckState& cs, int left,
                                                int need, int root, long long t_start, int cost_tail, int min_items,
                                                int level, const int* path, bool eager, int& xb, int& xe) {
  if (lb.hungry_trigger <= 0 || xe > xb || left < need) return;
  if (cs.hungry - cs.queued < lb.hungry_trigger) return;
  if (!eager && clock64() - t_start < 2ll * lb.donate_after_ns) return;
  int ob = 0, oe = 0;
  bool pushed = false;
  if (range_split_donate(lb, tw.range, root, tw.don, tw.busy, ob, oe, cost_tail, min_items, level, path, &pushed)) {
    xb = ob;
    xe = oe;
  }
  if (pushed) ++cs.queued;  // this demand is served
}

// `src(i, wk, acc, cnt)` (a functor with a force-inlined call operator, so that the walk's
// state stays in registers) starts item i on the calling lane.
template <int K, class WK, class Src>
__device__ __forceinline__ void lockstep_items(const LBArgs& lb, const TaskWords& tw, WK& wk, const Src& src,
                                               Acc<K>& acc, unsigned long long& cnt, int root,
                                               long long t_start, int cost_tail, int min_items, int level,
                                               const int* path, bool eager, CheckState& cs) {
  const int lane = lane_id();
  bool open = true;
  int xb = 0, xe = 0;  // lane 0: split-off items to run after the range
  const int need0 = min_items > 0 ? min_items : lb.min_split;
  const int need = need0 > 2 ? need0 : 2;
  while (true) {
    const unsigned idle = __ballot_sync(FULL_MASK, wk.top < 0);
    if (open && idle != 0u && (idle == FULL_MASK || __popc(idle) >= REFILL_MIN)) {
      const int leader = __ffs(idle) - 1;
      const int want = __popc(idle);
      unsigned long long old = 0ull;
      if (lane == leader) old = atomicAdd(tw.range, (unsigned long long)want);
      old = __shfl_sync(FULL_MASK, old, leader);
      const int next = (int)(unsigned)old, end = (int)(unsigned)(old >> 32);
      if (wk.top < 0) {
        const int my = next + __popc(idle & lanemask_lt());
        if (my < end) src(my, wk, acc, cnt);
      }
      if (next + want < end) {
        if (lane == 0)
          lockstep_donate(lb, tw, cs, end - next - want, need, root, t_start, cost_tail, min_items, level, path, eager,
                          xb, xe);
        __syncwarp();
      } else {
        const int has = __shfl_sync(FULL_MASK, xe > xb ? 1 : 0, 0);
        if (has) {
          const int b0 = __shfl_sync(FULL_MASK, xb, 0), e0 = __shfl_sync(FULL_MASK, xe, 0);
          if (lane == 0) {
            *tw.range = pack_range(b0, e0);
            xb = xe = 0;
          }
          __syncwarp();
        } else {
          open = false;
        }
      }
    }
    const unsigned walking = __ballot_sync(FULL_MASK, wk.top >= 0);
    if (walking == 0u) {
      if (!open) break;
      continue;
    }
    if (wk.top >= 0) wk.step(acc, cnt);
    if (++cs.iter % CHECK_EVERY == 0u) {
      if (lane == 0) {
        atomicAdd(&lb.ctr->progress, (unsigned long long)CHECK_EVERY);
        if (lb.hungry_trigger > 0) {
          if (open) {
            const unsigned long long r = *reinterpret_cast<volatile unsigned long long*>(tw.range);
            lockstep_donate(lb, tw, cs, (int)(unsigned)(r >> 32) - (int)(unsigned)r, need, root, t_start, cost_tail,
                            min_items, level, path, eager, xb, xe);
          }
          // read at the next check: the warp walks on while the loads complete
          cs.hungry = vload(&lb.ctr->hungry);
          cs.queued = vload(&lb.ctr->queued);
        }
      }
      __syncwarp();
    }
  }
  wk.flush(acc);
}

// Item sources. Local edges of one root: item i is the edge (c1, c2) with c1 found in the
// row prefix sE and c2 the matching bit of row c1; the walk starts at S = row[c1] & row[c2]
// (vertex 4). For K >= 6 an item with HEAVY_BITS or more candidates is deferred to the heavy
// list (run by the whole warp afterwards) while a slot is free.
template <int K, int NW, bool MULTI>
struct EdgeItems {
  const uint64_t* rows;
  const int32_t* sE;
  int d;
  int* hn;
  int* heavy;
  template <class WK>
  __device__ __forceinline__ void operator()(int i, WK& wk, Acc<K>& acc, unsigned long long& cnt) const {
    if constexpr (MULTI) acc.c[3] += 1ull;
    // d + 1 <= 64 * NW + 1 entries: powers of two up to 64, 128 or 256 cover them
    const int c1 = lower_bound_bl<(NW == 1 ? 64 : (NW == 2 ? 128 : 256))>(sE, d + 1, i + 1) - 1;
    const int c2 = select_row<NW>(rows + c1 * NW, i - sE[c1]);
    Bits<NW> S;
#pragma unroll
    for (int w = 0; w < NW; ++w) S.w[w] = rows[c1 * NW + w] & rows[c2 * NW + w];
    if constexpr (K >= 6) {
      const int p = popc(S);
      if (p >= HEAVY_BITS) {
        const int slot = atomicAdd(hn, 1);
        if (slot < HEAVY_SLOTS) {
          heavy[slot] = i;
          if constexpr (MULTI) acc.c[4] += (unsigned long long)p;
          return;
        }
      }
    }
    wk.start(S, rows, acc, cnt);
  }
};

// Positions of a heavy item's candidate set S: position j picks vertex 4, c3 = the j-th
// member of S, and the walk starts at S_{>c3} & row[c3] (vertex 5).
template <int K, int NW, bool MULTI>
struct PositionItems {
  const uint64_t* rows;
  Bits<NW> S;
  template <class WK>
  __device__ __forceinline__ void operator()(int j, WK& wk, Acc<K>& acc, unsigned long long& cnt) const {
    const int c3 = select_row<NW>(S.w, j);
    const int w3 = c3 >> 6;
    const uint64_t above = (c3 & 63) == 63 ? 0ull : (~0ull << ((c3 & 63) + 1));
    const uint64_t* rc = rows + c3 * NW;
    Bits<NW> T;
#pragma unroll
    for (int w = 0; w < NW; ++w) T.w[w] = (w < w3 ? 0ull : (w == w3 ? (S.w[w] & above) : S.w[w])) & rc[w];
    wk.start(T, rows, acc, cnt);
  }
};


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
  // the donation checks' first sample is loaded while the bitmaps are built
  CheckState cs;
  if (lane == 0 && a.lb.hungry_trigger > 0) {
    cs.hungry = vload(&a.lb.ctr->hungry);
    cs.queued = vload(&a.lb.ctr->queued);
  }
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
  if constexpr (K == 3) {
    // items are the rows: one popcount each, the lanes stay together
    const long long t_start = global_ns();
    unsigned done = 0;
    while (true) {
      const int it = range_take(range);
      if (it < 0) break;
      Bits<NW> S;
#pragma unroll
      for (int w = 0; w < NW; ++w) S.w[w] = rows[it * NW + w];
      cnt += (unsigned long long)popc(S);
      if ((++done & 15) == 0) {
        int ob = 0, oe = 0;
        if (range_maybe_donate(a.lb, range, root, donations_left, t_start, busy, ob, oe)) {
          for (int j = ob; j < oe; ++j) {
            Bits<NW> U;
#pragma unroll
            for (int w = 0; w < NW; ++w) U.w[w] = rows[j * NW + w];
            cnt += (unsigned long long)popc(U);
          }
        }
      }
    }
    __syncwarp();
    return cnt;
  } else {
    const TaskWords tw{range, donations_left, busy, hn, heavy};
    Acc<K> unused;
    Walk<K, NW, false, 4> wk;
    const EdgeItems<K, NW, false> items{rows, sE, d, hn, heavy};
    const long long t_cyc = clock64();
    lockstep_items<K>(a.lb, tw, wk, items, unused, cnt, root, t_cyc, 0, 0, 0, nullptr, false, cs);
    __syncwarp();
    if constexpr (K >= 6) {
      // heavy items: the members of S (clique vertex 4) are spread over the lanes; this
      // kernel takes no level-1 donations, so these ranges are never split
      const int nh = min(*hn, HEAVY_SLOTS);
      for (int h = 0; h < nh; ++h) {
        const int it = heavy[h];
        const int c1 = lower_bound(sE, 0, d + 1, it + 1) - 1;
        const int c2 = select_bit<NW>(rows + c1 * NW, it - sE[c1]);
        PositionItems<K, NW, false> pos{rows, {}};
#pragma unroll
        for (int w = 0; w < NW; ++w) pos.S.w[w] = rows[c1 * NW + w] & rows[c2 * NW + w];
        __syncwarp();
        if (lane == 0) *range = pack_range(0, popc(pos.S));
        __syncwarp();
        Walk<K, NW, false, 5> hw;
        lockstep_items<K>(a.lb, tw, hw, pos, unused, cnt, root, t_cyc, 0, INT_MAX, 0, nullptr, false, cs);
        __syncwarp();
      }
    }
    return cnt;
  }
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
