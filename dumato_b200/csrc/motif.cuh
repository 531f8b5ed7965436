// Motif enumeration for sm_100a: one task = (v0, range of second vertices) or a donated DFS
// prefix, run by a warp whose lanes form 32/W virtual warps ("groups") of W lanes.
//
// Semantics follow the reference's motif driver (src/main/motifs_DM_WCLB.cu:9-36): every
// connected induced k-subgraph is enumerated once, from its lowest-id vertex v0, along the one
// vertex order the reference's canonical filter accepts (extend(0,k), DuMatoGPU.cu:1702-1721;
// canonicalFilter2, 989-1012: an extension x whose first adjacent prefix vertex is v_src must
// exceed every prefix vertex after v_src), and classified through the quick code
// (forward_induce 846-869, aggregate_pattern 930-967) looked up in the dictionary.
//
// That filter makes the extension sets incremental. If E_t is the valid extension set of
// prefix (v_0..v_t) and w = v_{t+1} is taken from it, then
//     E_{t+1} = { e in E_t : e > w }  U  excl(w),
//     excl(w) = { x in N(w) : x > v0, x not in N(v_0) U .. U N(v_t) }
// (the inherited members keep their source, and the only new constraint is "> w"; the new
// members have w as their source). Every member carries its adjacency mask to the prefix
// (bit i = edge to v_i), so quick codes come from masks, not from the reference's per-leaf
// adjacency scans. The excluded set U_t = N(v_0..v_t) cap (v0, inf) is kept as disjoint
// sorted runs (run 0 = N(v0) above v0, run i = excl(v_i)). E_t is kept sorted by vertex id, so
// the inherited members are the suffix of E_t after w.
//
// Leaves are counted in bulk: at the last internal level, for each w the leaf masks of
// E_{k-2} are histogrammed without materialising it (inherited members: either a membership
// probe in N(w) each, or the suffix's mask counts corrected by the members of N(w) above w,
// whichever side is cheaper; excl(w): |N(w) above v0| - |N(w) cap U_t|, also from the
// cheaper side), then each non-empty mask bucket adds to one class counter.
//
// Virtual warps (the reference's DM_WCV variant, src/DM_WCV/DuMatoGPU.cu:12-37): with W < 32
// the groups of a warp take second vertices of the same task from its shared item range and
// run their subtrees independently, each with its own DFS state and arena; every collective
// uses the group's lane mask. Small extension sets (small graphs, low degree) keep more
// lanes busy this way.
//
// Load balancing (lb.cuh): idle warps get donated work, either a range of second vertices
// or, when one second vertex roots most of the work (a hub), a DFS prefix - the path to some
// level's extension set and a range of its members, which the receiver rebuilds by replaying
// the path (each level's set is a deterministic function of the path).
#pragma once

#include <climits>

#include "engine.hpp"
#include "gpm.cuh"
#include "lb.cuh"

namespace dmb {

constexpr int MOTIF_KMAX = 7;

__host__ __device__ constexpr int quick_off(int p) { return (p - 2) * (p + 1) / 2; }

// DFS state of one group.
struct alignas(16) MotifGroup {
  int n[MOTIF_KMAX];           // extension-set sizes per level
  int pos[MOTIF_KMAX];         // next member to expand per level
  int lim[MOTIF_KMAX];         // members [pos, lim) of a level are still this group's to expand
  int runn[MOTIF_KMAX];        // run sizes per level
  unsigned quick[MOTIF_KMAX];  // quick code of the prefix ending at level t
  int spill_lo, spill_hi;      // second vertices split off when the queue was full
  unsigned mh[64];             // leaf-mask histogram
  unsigned sh[32];             // masks of E_{k-3}[pos..n): the members still above the current vertex
};

// Task state shared by the groups of one warp.
struct alignas(16) MotifShared {
  unsigned long long range;    // second vertices not taken yet (pack_range)
  int donations_left;          // donation budget of the running task
  int busy;                    // serialises level-0 splits
};

template <int W>
__host__ __device__ constexpr size_t motif_warp_smem() {
  return sizeof(MotifShared) + sizeof(MotifGroup) * (32 / W);
}

// Everything a motif task needs besides its own (v0, range) or prefix.
struct MotifCtx {
  GraphView g;                 // undirected CSR, rows sorted
  LBArgs lb;
  const int32_t* q2c;          // quick code -> class
  int maxdeg;                  // bound on every degree in g (arena sizing)
  int arena_stride;            // int2 slots per group
  unsigned long long* per_root;  // optional: subgraphs found under each v0 (subtree logger)
  int bit_base;                // membership bitmaps index vertex x at bit x - bit_base
  int bit_words;               // 32-bit words per bitmap (0 = no bitmaps: binary searches only)
};

// Membership bitmaps of one group (2 x bit_words words in global memory, all zero between
// tasks): U holds U_t = N(v_0..v_t) above v0 for the levels materialised on the current path,
// E holds E_{k-3} (k = 3: E_0). They turn the leaf step and the exclusion test into one probe
// per neighbour instead of binary searches over the runs.
__device__ __forceinline__ bool bit_test(const uint32_t* b, int x) { return (b[x >> 5] >> (x & 31)) & 1u; }

template <int W>
__device__ __forceinline__ void bits_flip_ids(uint32_t* b, int base, const int32_t* ids, int n, bool set, int gl) {
  for (int i = gl; i < n; i += W) {
    const int x = __ldg(ids + i) - base;
    if (set) atomicOr(b + (x >> 5), 1u << (x & 31));
    else atomicAnd(b + (x >> 5), ~(1u << (x & 31)));
  }
}

template <int W>
__device__ __forceinline__ void bits_flip_list(uint32_t* b, int base, const int2* list, int n, bool set, int gl) {
  for (int i = gl; i < n; i += W) {
    const int x = list[i].x - base;
    if (set) atomicOr(b + (x >> 5), 1u << (x & 31));
    else atomicAnd(b + (x >> 5), ~(1u << (x & 31)));
  }
}

// int2 slots of one group's arena: extension levels 1..k-3 (level t holds at most
// (t+1) * maxdeg members) then runs 1..k-3 (at most maxdeg each).
__host__ __device__ inline size_t motif_group_stride(int k, int maxdeg) {
  size_t s = 0;
  for (int t = 1; t <= k - 3; ++t) s += (size_t)(t + 1) * maxdeg + 32;
  for (int t = 1; t <= k - 3; ++t) s += (size_t)maxdeg + 32;
  return s < 1 ? 1 : s;
}

// First index in [lo, hi) of an id-sorted (vertex, mask) list whose vertex is >= x.
__device__ __forceinline__ int lower_bound2(const int2* a, int lo, int hi, int32_t x) {
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (a[mid].x < x) lo = mid + 1; else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ int ilog2p1(int x) { return 32 - __clz(x | 1); }

// Membership of x in the disjoint sorted runs 0..t (run 0 is the CSR suffix of v0; run i >= 1
// starts at runs1 + (i - 1) * rstride).
__device__ __forceinline__ bool in_runs(int32_t x, const int32_t* run0, int n0, const int2* runs1, size_t rstride,
                                        const int* runn, int t) {
  if (contains(run0, n0, x)) return true;
  for (int i = 1; i <= t; ++i) {
    const int2* r = runs1 + (size_t)(i - 1) * rstride;
    const int nr = runn[i];
    const int j = lower_bound2(r, 0, nr, x);
    if (j < nr && r[j].x == x) return true;
  }
  return false;
}

// Adds the masks of list[lo, hi) to the group's 32-entry histogram h (aggregated per mask).
template <int W>
__device__ __forceinline__ void mask_hist(const int2* list, int lo, int hi, unsigned* h, int gl, unsigned gmask) {
  for (int i0 = lo; i0 < hi; i0 += W) {
    const int i = i0 + gl;
    const bool v = i < hi;
    dm_gpm::aggregate_pattern<W>(h, v ? list[i].y : 0, v);
  }
  __syncwarp(gmask);
}

// Flushes the group's leaf-mask histogram (masks below NMASK) into the class counters.
template <int W, int NMASK>
__device__ __forceinline__ void flush_masks(MotifGroup* sg, const int32_t* q2c, unsigned quick_p, int off,
                                            unsigned long long* hist, unsigned long long& task_cnt, int gl,
                                            unsigned gmask) {
  for (int m = gl; m < NMASK; m += W) {
    const unsigned c = sg->mh[m];
    if (c) {
      sg->mh[m] = 0;
      const int cls = __ldg(q2c + (quick_p + ((unsigned)m << off)));
      atomicAdd(hist + cls, (unsigned long long)c);
      task_cnt += c;
    }
  }
  __syncwarp(gmask);
}

// Group leader, between two expansions of a task whose lowest own level is `floor` (1 for an
// item task; L for a donated DFS prefix of level L) and whose deepest materialised level is
// t: when warps are hungry, hands the upper half of the shallowest level that still has
// unexpanded members to the queue. Level 0 is the task's second-vertex range (cost-aware
// split, shared by the groups); a level s >= 1 goes out as (root, s, path to E_s, position
// range), the path being the second vertex's index `it` and the index picked at each level
// 1..s-1.
__device__ __forceinline__ void motif_try_donate(const LBArgs& lb, MotifShared* ws, MotifGroup* sg, int v0,
                                                 int floor, int t, int it, int n0, long long t_start) {
  if (!lb_wants_donation(lb, &ws->donations_left, t_start)) return;
  if (floor == 1) {
    const unsigned long long cur = *reinterpret_cast<volatile unsigned long long*>(&ws->range);
    const int next = (int)(unsigned)cur, end = (int)(unsigned)(cur >> 32);
    if (end - next >= 2) {
      // inside a running item even two untaken second vertices are worth handing out
      if (sg->spill_lo >= sg->spill_hi) {
        int ob = 0, oe = 0;
        if (range_maybe_donate(lb, &ws->range, v0, &ws->donations_left, t_start, &ws->busy, ob, oe, n0, 2)) {
          // the queue was full: this group runs the split-off second vertices itself
          sg->spill_lo = ob;
          sg->spill_hi = oe;
        }
      }
      return;
    }
  }
  for (int s = floor; s <= t; ++s) {
    const int ps = sg->pos[s], lim = sg->lim[s];
    if (lim - ps >= 2) {
      // E_s is sorted by id: member i inherits the n - i - 1 members above it
      const int mid = split_mid(ps, lim, sg->n[s]);
      int path[QPATH];
      path[0] = it;
      for (int j = 1; j < s && j < QPATH; ++j) path[j] = sg->pos[j] - 1;
      if (lb_donate_deep(lb, v0, s, path, mid, lim)) {
        sg->lim[s] = mid;
        atomicSub(&ws->donations_left, 1);
      }
      return;
    }
  }
}

// Runs one task on the calling warp (all 32 lanes). level 0: second vertices [bb, ee) of v0
// (task_range encoding); level L >= 1: replay path[0..L-1], then expand positions [bb, ee) of
// E_L (group 0 only). Adds the task's subgraphs to hist (class counters in shared or global
// memory); nodes counts expansions (every
// lane of a group counts the same nodes; the caller keeps group leaders' counts only).
template <int K, int W>
__device__ __forceinline__ void motif_run_task(const MotifCtx& c, unsigned long long* hist, MotifShared* ws,
                                               MotifGroup* groups, int2* warp_arena, uint32_t* warp_bits, int v0,
                                               int bb, int ee, int level, const int* path,
                                               unsigned long long& nodes) {
  static_assert(W == 8 || W == 16 || W == 32, "virtual warp width must be 8, 16 or 32");
  const int lane = lane_id();
  const int gl = lane & (W - 1);
  const int gi = lane / W;
  const unsigned gmask = (W == 32) ? FULL_MASK : (((1u << W) - 1u) << (gi * W));
  const int gsrc = gi * W;  // the group leader's lane
  MotifGroup* sg = groups + gi;
  // level t (1..K-3): extension list E_t at ext_at(t); run t at run_at(t) (no pointer
  // tables, so nothing indexed dynamically lives in local memory)
  int2* const arena = warp_arena + (size_t)gi * c.arena_stride;
  const size_t md = (size_t)c.maxdeg;
  auto ext_at = [&](int t) -> int2* { return arena + md * (size_t)(t * (t + 1) / 2 - 1) + 32 * (size_t)(t - 1); };
  int2* const runs1 = ext_at(K - 2);
  const size_t rstride = md + 32;
  auto run_at = [&](int t) -> int2* { return runs1 + (size_t)(t - 1) * rstride; };
  // (k = 3 has a single level: setting and clearing E_0's bits per task costs more than the
  // binary searches it saves)
  const bool use_bits = K >= 4 && warp_bits != nullptr && c.bit_words > 0;
  uint32_t* const Ub = use_bits ? warp_bits + (size_t)gi * 2 * c.bit_words : nullptr;
  uint32_t* const Eb = use_bits ? Ub + c.bit_words : nullptr;
  int bdepth = 0;  // levels 1..bdepth have their run (and, at level k-3, E) bits set
  unsigned long long task_cnt = 0;
  const long long t_start = global_ns();
  // E_0 = run 0 = N(v0) above v0: a suffix of the sorted CSR row
  const int32_t* row0 = c.g.adj + __ldg(c.g.row + v0);
  const int deg0 = __ldg(c.g.deg + v0);
  const int s0 = lower_bound(row0, 0, deg0, v0 + 1);
  const int32_t* E0 = row0 + s0;
  const int n0 = deg0 - s0;
  const int floor = level > 0 ? level : 1;
  int lo = 0, hi = 0;
  if (level == 0) task_range(bb, ee, n0, lo, hi);
  __syncwarp();
  if (lane == 0) {
    ws->range = pack_range(lo, hi);
    ws->donations_left = c.lb.max_donations;
    ws->busy = 0;
  }
  if (gl == 0) {
    sg->quick[0] = 0;
    sg->spill_lo = sg->spill_hi = 0;
  }
  for (int m = gl; m < 64; m += W) sg->mh[m] = 0;
  if (use_bits) {
    bits_flip_ids<W>(Ub, c.bit_base, E0, n0, true, gl);
    if (K == 3) bits_flip_ids<W>(Eb, c.bit_base, E0, n0, true, gl);
  }
  __syncwarp();
  // drops the bits of levels from..bdepth (the group's lanes, then a group barrier)
  auto drop_levels = [&](int from) {
    for (int L = bdepth; L >= from; --L) {
      bits_flip_list<W>(Ub, c.bit_base, run_at(L), sg->runn[L], false, gl);
      if (L == K - 3) bits_flip_list<W>(Eb, c.bit_base, ext_at(L), sg->n[L], false, gl);
    }
    if (bdepth >= from) bdepth = from - 1;
    __syncwarp(gmask);
  };
  bool replay_item = level > 0 && gi == 0;
  while (true) {
    int it = 0;
    if (level > 0) {
      if (!replay_item) break;
      replay_item = false;
      it = path[0];
      if (it < 0 || it >= n0) {
        if (gl == 0) set_err(c.lb.ctr, ERR_BAD_TASK);
        break;
      }
    } else {
      if (gl == 0) {
        it = range_take(&ws->range);
        if (it < 0) {
          if (sg->spill_lo < sg->spill_hi) it = sg->spill_lo++;
        } else if (sg->spill_lo >= sg->spill_hi) {
          int ob = 0, oe = 0;
          if (range_maybe_donate(c.lb, &ws->range, v0, &ws->donations_left, t_start, &ws->busy, ob, oe, n0)) {
            sg->spill_lo = ob;
            sg->spill_hi = oe;
          }
        }
      }
      it = __shfl_sync(gmask, it, gsrc);
      if (it < 0) break;
    }
    // prefix (v0, w1); the members of E_0 after w1 are the inherited part
    int t = 0;
    int w = __ldg(E0 + it);
    int wmask = 1;
    bool bad = false;
    // depth-first over levels; level t's current vertex is w with mask wmask
    while (true) {
      // here the prefix is v_0..v_t plus w = v_{t+1}
      const int p = t + 1;  // position of w
      if (p > level) {
        // nodes at or above a donated prefix's level belong to the donor
        ++nodes;
        if (gl == 0 && (nodes & 255) == 0) atomicAdd(&c.lb.ctr->progress, 256ull);
      }
      unsigned quick_p = (t == 0) ? 0u : sg->quick[t];
      if (p >= 2) quick_p += ((unsigned)wmask & ((1u << p) - 1u)) << quick_off(p);
      const int32_t* Nw = c.g.adj + __ldg(c.g.row + w);
      const int dw = __ldg(c.g.deg + w);
      // inherited members: e in E_t with e > w. E_t is sorted by vertex id and w is its
      // member at position pos[t] - 1 (E_0: index it), so they are the suffix from there.
      const int2* Et = t == 0 ? nullptr : ext_at(t);
      const int nE = (t == 0) ? n0 : sg->n[t];
      const int startE = (t == 0) ? it + 1 : sg->pos[t];
      if (p == K - 2) {
        // leaves: histogram the masks of E_{p} without writing it
        const int leaf_off = quick_off(K - 1);
        const int n_inh = nE - startE;
        // a short row is scanned whole (members up to v0 skipped) instead of searched for v0
        const bool short_row = dw <= 2 * W;
        const int sw0b = short_row ? 0 : lower_bound(Nw, 0, dw, v0 + 1);
        int usize = n0;
        for (int i = 1; i <= t; ++i) usize += sg->runn[i];
        if (use_bits && dw - sw0b <= 4 * (n_inh + usize) + 128) {
          // one pass over N(w) above v0: a neighbour outside U_t is a new member of E_{p}
          // (excl(w)); a neighbour in E_t above w is an inherited member adjacent to w; the
          // inherited members not adjacent to w come from the suffix's mask counts
          if (t == 0) {
            if (gl == 0 && n_inh) atomicAdd(&sg->mh[1], (unsigned)n_inh);
          } else {
            for (int m = gl; m < (1 << (K - 2)); m += W) {
              const unsigned cm = sg->sh[m];
              if (cm) atomicAdd(&sg->mh[m], cm);
            }
          }
          __syncwarp(gmask);
          unsigned ex = 0;
          for (int i = sw0b + gl; i < dw; i += W) {
            const int32_t x = Nw[i];
            if (x <= v0) continue;
            const int xb = x - c.bit_base;
            if (!bit_test(Ub, xb)) {
              ++ex;
            } else if (x > w && bit_test(Eb, xb)) {
              const int em = (t == 0) ? 1 : Et[lower_bound2(Et, startE, nE, x)].y;
              atomicSub(&sg->mh[em], 1u);
              atomicAdd(&sg->mh[em | (1 << p)], 1u);
            }
          }
          for (int o = W / 2; o > 0; o >>= 1) ex += __shfl_xor_sync(gmask, ex, o);
          if (gl == 0 && ex) atomicAdd(&sg->mh[1 << p], ex);
          __syncwarp(gmask);
          flush_masks<W, (1 << (K - 1))>(sg, c.q2c, quick_p, leaf_off, hist, task_cnt, gl, gmask);
        } else {
        const int sw0 = short_row ? lower_bound(Nw, 0, dw, v0 + 1) : sw0b;
        const int above = dw - sw0;
        const int gt = lower_bound(Nw, 0, dw, w + 1);
        const int dgt = dw - gt;
        // probe each inherited member in N(w), or take the suffix's mask counts and move
        // the members found in N(w) above w (whichever side is cheaper)
        if ((long long)dgt * ilog2p1(n_inh) + (1 << (K - 2)) < (long long)n_inh * ilog2p1(dw)) {
          if (t == 0) {
            if (gl == 0 && n_inh) atomicAdd(&sg->mh[1], (unsigned)n_inh);
          } else {
            for (int m = gl; m < (1 << (K - 2)); m += W) {
              const unsigned cm = sg->sh[m];
              if (cm) atomicAdd(&sg->mh[m], cm);
            }
          }
          __syncwarp(gmask);
          for (int i = gt + gl; i < dw; i += W) {
            const int32_t x = Nw[i];
            int em = -1;
            if (t == 0) {
              const int j = lower_bound(E0, startE, n0, x);
              if (j < n0 && __ldg(E0 + j) == x) em = 1;
            } else {
              const int j = lower_bound2(Et, startE, nE, x);
              if (j < nE) {
                const int2 y = Et[j];
                if (y.x == x) em = y.y;
              }
            }
            if (em >= 0) {
              atomicSub(&sg->mh[em], 1u);
              atomicAdd(&sg->mh[em | (1 << p)], 1u);
            }
          }
        } else {
          for (int i = startE + gl; i < nE; i += W) {
            int ev, em;
            if (t == 0) {
              ev = __ldg(E0 + i);
              em = 1;
            } else {
              const int2 x = Et[i];
              ev = x.x;
              em = x.y;
            }
            const int m = em | (contains(Nw, dw, ev) ? (1 << p) : 0);
            atomicAdd(&sg->mh[m], 1u);
          }
        }
        // excl(w) = N(w) above v0 minus U_t
        unsigned inter = 0;
        if ((long long)usize <= (long long)above * (t + 1)) {
          // iterate U_t, probe N(w)
          for (int i = gl; i < n0; i += W) inter += contains(Nw, dw, __ldg(E0 + i)) ? 1u : 0u;
          for (int r = 1; r <= t; ++r) {
            const int2* R = run_at(r);
            const int nr = sg->runn[r];
            for (int i = gl; i < nr; i += W) inter += contains(Nw, dw, R[i].x) ? 1u : 0u;
          }
        } else {
          // iterate N(w) above v0, probe the runs
          for (int i = sw0 + gl; i < dw; i += W)
            inter += (use_bits ? bit_test(Ub, Nw[i] - c.bit_base)
                               : in_runs(Nw[i], E0, n0, runs1, rstride, sg->runn, t)) ? 1u : 0u;
        }
        for (int o = W / 2; o > 0; o >>= 1) inter += __shfl_xor_sync(gmask, inter, o);
        if (gl == 0) {
          const unsigned ex = (unsigned)above - inter;
          if (ex) atomicAdd(&sg->mh[1 << p], ex);
        }
        __syncwarp(gmask);
        flush_masks<W, (1 << (K - 1))>(sg, c.q2c, quick_p, leaf_off, hist, task_cnt, gl, gmask);
        }
      } else {
        // materialise E_{p} = inherited + excl(w), merged by vertex id; excl(w) is also run
        // p. Both parts are sorted and disjoint, so each member's place is its index in its
        // own part plus the number of smaller members of the other part.
        int2* Ep = ext_at(p);
        int2* Rp = run_at(p);
        if (use_bits) drop_levels(p);  // the previous member's sets at levels >= p
        const int sw0 = dw <= 2 * W ? 0 : lower_bound(Nw, 0, dw, v0 + 1);
        int rn = 0;
        for (int i0 = sw0; i0 < dw; i0 += W) {
          const int i = i0 + gl;
          int32_t x = 0;
          bool nw = false;
          if (i < dw && Nw[i] > v0) {
            x = Nw[i];
            nw = use_bits ? !bit_test(Ub, x - c.bit_base) : !in_runs(x, E0, n0, runs1, rstride, sg->runn, t);
          }
          const unsigned bal = __ballot_sync(gmask, nw) >> gsrc;
          if (nw) Rp[rn + __popc(bal & ((1u << gl) - 1u))] = make_int2(x, 0);
          rn += __popc(bal);
        }
        __syncwarp(gmask);
        for (int i = startE + gl; i < nE; i += W) {
          int ev, em;
          if (t == 0) {
            ev = __ldg(E0 + i);
            em = 1;
          } else {
            const int2 x = Et[i];
            ev = x.x;
            em = x.y;
          }
          if (contains(Nw, dw, ev)) em |= 1 << p;
          Ep[(i - startE) + lower_bound2(Rp, 0, rn, ev)] = make_int2(ev, em);
        }
        for (int j = gl; j < rn; j += W) {
          const int32_t x = Rp[j].x;
          const int cnt_lt = (t == 0) ? lower_bound(E0, 0, n0, x) : lower_bound2(Et, 0, nE, x);
          Ep[j + max(0, cnt_lt - startE)] = make_int2(x, 1 << p);
        }
        const int m = (nE - startE) + rn;
        __syncwarp(gmask);
        if (use_bits) {
          bits_flip_list<W>(Ub, c.bit_base, Rp, rn, true, gl);
          if (p == K - 3) bits_flip_list<W>(Eb, c.bit_base, Ep, m, true, gl);
          bdepth = p;
          __syncwarp(gmask);
        }
        if (p < level) {
          // replaying a donated prefix: the path fixes the member expanded at level p
          const int idx = (p < QPATH) ? path[p] : -1;
          if (idx < 0 || idx >= m) {
            if (gl == 0) set_err(c.lb.ctr, ERR_BAD_TASK);
            bad = true;
            break;
          }
          const int2 x = Ep[idx];
          if (gl == 0) {
            sg->n[p] = m;
            sg->pos[p] = idx + 1;
            sg->lim[p] = idx + 1;
            sg->runn[p] = rn;
            sg->quick[p] = quick_p;
          }
          __syncwarp(gmask);
          t = p;
          w = x.x;
          wmask = x.y;
          continue;
        }
        const int first_pos = p == level ? min(bb, m) : 0;
        if (gl == 0) {
          sg->n[p] = m;
          sg->pos[p] = first_pos;
          sg->lim[p] = p == level ? min(ee, m) : m;
          sg->runn[p] = rn;
          sg->quick[p] = quick_p;
        }
        if (p == K - 3) {
          for (int i = gl; i < 32; i += W) sg->sh[i] = 0;
          __syncwarp(gmask);
          mask_hist<W>(Ep, first_pos, m, sg->sh, gl, gmask);
        }
        __syncwarp(gmask);
        t = p;  // descend; pick the first member below
      }
      // give work away when warps are hungry (checked every 16 expansions)
      if (K >= 4 && (nodes & 15) == 0) {
        if (gl == 0) motif_try_donate(c.lb, ws, sg, v0, floor, t, it, n0, t_start);
        __syncwarp(gmask);
      }
      // next vertex: advance the deepest level that still has members
      bool found = false;
      while (t >= floor) {
        const int ps = sg->pos[t];
        if (ps < sg->lim[t]) {
          const int2 x = ext_at(t)[ps];
          __syncwarp(gmask);
          if (gl == 0) {
            sg->pos[t] = ps + 1;
            if (t == K - 3) sg->sh[x.y] -= 1u;
          }
          __syncwarp(gmask);
          w = x.x;
          wmask = x.y;
          found = true;
          break;
        }
        --t;
      }
      if (!found) break;
    }
    if (use_bits) drop_levels(1);
    if (bad) break;
  }
  if (use_bits) {
    bits_flip_ids<W>(Ub, c.bit_base, E0, n0, false, gl);
    if (K == 3) bits_flip_ids<W>(Eb, c.bit_base, E0, n0, false, gl);
  }
  __syncwarp();
  if (c.per_root) {
    const unsigned long long tsum = warp_sum_u64(task_cnt);
    if (lane == 0 && tsum) atomicAdd(c.per_root + v0, tsum);
  }
  if (lane == 0) lb_task_time(c.lb, t_start, v0);
}

}  // namespace dmb
