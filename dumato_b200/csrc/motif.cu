// Motif counting kernel for sm_100a: connected induced k-vertex subgraphs (k = 3..7) per
// canonical class.
//
// Semantics follow the reference's motif driver (src/main/motifs_DM_WCLB.cu:9-36): every
// connected induced subgraph is enumerated once, from its lowest-id vertex v0, along the one
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
// sorted runs (run 0 = N(v0) above v0, run i = excl(v_i)).
//
// Leaves are counted in bulk: at the last internal level, for each w the leaf masks of
// E_{k-2} are histogrammed without materialising it (inherited members: one membership
// probe in N(w) each; excl(w): |N(w) above v0| - |N(w) cap U_t|, counted from whichever side
// is cheaper), then each non-empty mask bucket adds to one class counter.
//
// Work is warp-cooperative: a task is (v0, range of second vertices); lane 0 takes items,
// the warp runs the subtree, and idle warps get donated work (lb.cuh): either a range of
// second vertices or, when one second vertex roots most of the work (a hub), a DFS prefix -
// the path to some level's extension set and a range of its members, which the receiver
// rebuilds by replaying the path (each level's set is a deterministic function of the path).
#include <algorithm>
#include <climits>
#include <string>

#include "engine.hpp"
#include "gpm.cuh"
#include "lb.cuh"

namespace dmb {

constexpr int MOTIF_WARPS = 8;
constexpr int MOTIF_KMAX = 7;

struct MotifArgs {
  GraphView g;                 // undirected CSR, original ids, rows sorted
  const int32_t* roots;
  int n_roots;
  LBArgs lb;
  int k;
  const int32_t* q2c;          // quick code -> class
  int n_classes;
  unsigned long long* hist;    // n_classes
  int2* arena;                 // per warp: extension levels 1..k-3 then runs 1..k-3
  int arena_stride;            // int2 slots per warp
  int maxdeg;
  unsigned long long* per_root;
  const int32_t* parts;        // optional per-root-entry part word (p | P << 16)
};

__host__ __device__ constexpr int quick_off(int p) { return (p - 2) * (p + 1) / 2; }

// Per-warp shared state.
struct alignas(16) MotifWarp {
  unsigned long long range;
  int donations_left;
  int busy;
  int n[MOTIF_KMAX];           // extension-set sizes per level
  int pos[MOTIF_KMAX];         // next member to expand per level
  int lim[MOTIF_KMAX];         // members [pos, lim) of a level are still this warp's to expand
  int runn[MOTIF_KMAX];        // run sizes per level
  unsigned quick[MOTIF_KMAX];  // quick code of the prefix ending at level t
  unsigned mh[64];             // leaf-mask histogram
  unsigned sh[32];             // masks of E_{k-3}[pos..n): the members still above the current vertex
};

// First index in [lo, hi) of an id-sorted (vertex, mask) list whose vertex is >= x.
__device__ __forceinline__ int lower_bound2(const int2* a, int lo, int hi, int32_t x) {
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (a[mid].x < x) lo = mid + 1; else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ int ilog2p1(int x) { return 32 - __clz(x | 1); }

// Adds the masks of list[lo, hi) to the warp's 32-entry histogram h (warp-aggregated).
__device__ __forceinline__ void mask_hist(const int2* list, int lo, int hi, unsigned* h) {
  for (int i0 = lo; i0 < hi; i0 += 32) {
    const int i = i0 + lane_id();
    const bool v = i < hi;
    const int m = v ? list[i].y : -1;
    const unsigned act = __ballot_sync(FULL_MASK, v);
    const unsigned same = __match_any_sync(FULL_MASK, m);
    if (v && (same & act & ((1u << lane_id()) - 1u)) == 0) atomicAdd(&h[m], (unsigned)__popc(same & act));
  }
  __syncwarp();
}

// Membership of x in the disjoint sorted runs 0..t (run 0 is the CSR suffix of v0).
__device__ __forceinline__ bool in_runs(int32_t x, const int32_t* run0, int n0, const int2* const* runs,
                                        const int* runn, int t) {
  if (contains(run0, n0, x)) return true;
  for (int i = 1; i <= t; ++i) {
    const int2* r = runs[i];
    int lo = 0, hi = runn[i];
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (r[mid].x < x) lo = mid + 1; else hi = mid;
    }
    if (lo < runn[i] && r[lo].x == x) return true;
  }
  return false;
}

// Lane 0, between two expansions of a task whose lowest own level is `floor` (1 for an item
// task; L for a donated DFS prefix of level L) and whose deepest materialised level is t:
// when warps are hungry, hands the upper half of the shallowest level that still has two
// unexpanded members to the queue. Level 0 is the task's second-vertex range (cost-aware
// split); a level s >= 1 goes out as (root, s, path to E_s, position range), the path being
// the second vertex's index `it` and the index picked at each level 1..s-1.
__device__ __forceinline__ void motif_try_donate(const LBArgs& lb, MotifWarp* sw, int v0, int floor, int t, int it,
                                                 int n0, long long t_start) {
  if (!lb_wants_donation(lb, &sw->donations_left, t_start)) return;
  if (floor == 1) {
    const unsigned long long cur = sw->range;
    const int next = (int)(unsigned)cur, end = (int)(unsigned)(cur >> 32);
    if (end - next >= 2) {
      const int mid = split_mid(next, end, n0);
      if (lb_donate_deep(lb, v0, 0, nullptr, mid, end)) {
        sw->range = pack_range(next, mid);
        sw->donations_left -= 1;
      }
      return;
    }
  }
  for (int s = floor; s <= t; ++s) {
    const int ps = sw->pos[s], lim = sw->lim[s];
    if (lim - ps >= 2) {
      // E_s is sorted by id: member i inherits the n - i - 1 members above it
      const int mid = split_mid(ps, lim, sw->n[s]);
      int path[QPATH];
      path[0] = it;
      for (int j = 1; j < s && j < QPATH; ++j) path[j] = sw->pos[j] - 1;
      if (lb_donate_deep(lb, v0, s, path, mid, lim)) {
        sw->lim[s] = mid;
        sw->donations_left -= 1;
      }
      return;
    }
  }
}

// Flushes the warp's leaf-mask histogram into the block's class counters.
__device__ __forceinline__ void flush_masks(MotifWarp* sw, const MotifArgs& a, unsigned quick_p, int off,
                                            unsigned long long* bhist, unsigned long long& task_cnt) {
  const int lane = lane_id();
  for (int m = lane; m < 64; m += 32) {
    const unsigned c = sw->mh[m];
    if (c) {
      sw->mh[m] = 0;
      const int cls = __ldg(a.q2c + (quick_p + ((unsigned)m << off)));
      atomicAdd(bhist + cls, (unsigned long long)c);
      task_cnt += c;
    }
  }
  __syncwarp();
}

template <int K>
__global__ void __launch_bounds__(32 * MOTIF_WARPS) motif_kernel(MotifArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  unsigned long long* bhist = reinterpret_cast<unsigned long long*>(smem);
  MotifWarp* swall = reinterpret_cast<MotifWarp*>(bhist + ((a.n_classes + 1) & ~1));
  const int lane = lane_id();
  const int wib = warp_in_block();
  MotifWarp* sw = swall + wib;
  for (int c = threadIdx.x; c < a.n_classes; c += blockDim.x) bhist[c] = 0;
  for (int m = lane; m < 64; m += 32) sw->mh[m] = 0;
  __syncthreads();
  const size_t gw = (size_t)blockIdx.x * MOTIF_WARPS + wib;
  const int total_warps = gridDim.x * MOTIF_WARPS;
  int2* arena = a.arena + gw * (size_t)a.arena_stride;
  // level t (1..K-3): extension list E_t at ext[t]; run t at runs[t]
  const int2* ext_c[MOTIF_KMAX];
  const int2* runs_c[MOTIF_KMAX];
  int2* ext[MOTIF_KMAX];
  int2* runs[MOTIF_KMAX];
  {
    size_t off = 0;
    for (int t = 1; t <= K - 3; ++t) {
      ext[t] = arena + off;
      off += (size_t)(t + 1) * a.maxdeg + 32;
    }
    for (int t = 1; t <= K - 3; ++t) {
      runs[t] = arena + off;
      off += (size_t)a.maxdeg + 32;
    }
    for (int t = 0; t < MOTIF_KMAX; ++t) {
      ext_c[t] = (t >= 1 && t <= K - 3) ? ext[t] : nullptr;
      runs_c[t] = (t >= 1 && t <= K - 3) ? runs[t] : nullptr;
    }
  }
  unsigned long long ntasks = 0, nodes = 0;
  while (true) {
    int first = 0, count = 0, b = 0, e = -1, ok = 0, level = 0;
    int path[QPATH];
    for (int j = 0; j < QPATH; ++j) path[j] = 0;
    bool donated = false;
    if (lane == 0) ok = lb_next(a.lb, a.n_roots, total_warps, first, count, b, e, donated, level, path) ? 1 : 0;
    ok = __shfl_sync(FULL_MASK, ok, 0);
    if (!ok) break;
    first = __shfl_sync(FULL_MASK, first, 0);
    count = __shfl_sync(FULL_MASK, count, 0);
    b = __shfl_sync(FULL_MASK, b, 0);
    e = __shfl_sync(FULL_MASK, e, 0);
    level = __shfl_sync(FULL_MASK, level, 0);
    for (int j = 0; j < K - 3 && j < QPATH; ++j) path[j] = __shfl_sync(FULL_MASK, path[j], 0);
    donated = __shfl_sync(FULL_MASK, donated ? 1 : 0, 0) != 0;
    // a donated DFS prefix names a level that this k has
    if (level < 0 || level > K - 3) {
      if (lane == 0) {
        set_err(a.lb.ctr, ERR_BAD_TASK);
        lb_done(a.lb, count);
      }
      break;
    }
    for (int ti = 0; ti < count; ++ti) {
      const int v0 = donated ? first : __ldg(a.roots + first + ti);
      int bb = b, ee = e;
      if (!donated && a.parts) part_bounds(__ldg(a.parts + first + ti), bb, ee);
      ++ntasks;
      unsigned long long task_cnt = 0;
      const long long t_start = global_ns();
      // E_0 = run 0 = N(v0) above v0: a suffix of the sorted CSR row
      const int32_t* row0 = a.g.adj + __ldg(a.g.row + v0);
      const int deg0 = __ldg(a.g.deg + v0);
      const int s0 = lower_bound(row0, 0, deg0, v0 + 1);
      const int32_t* E0 = row0 + s0;
      const int n0 = deg0 - s0;
      // level >= 1: replay the path down to E_level, then expand positions [b, e) there
      const int floor = level > 0 ? level : 1;
      int lo, hi;
      if (level > 0) {
        lo = 0;
        hi = 0;
      } else {
        task_range(bb, ee, n0, lo, hi);
      }
      if (lane == 0) {
        sw->range = pack_range(lo, hi);
        sw->donations_left = a.lb.max_donations;
        sw->busy = 0;
        sw->quick[0] = 0;
      }
      __syncwarp();
      bool replay_item = level > 0;
      while (true) {
        int it = 0;
        if (replay_item) {
          it = path[0];
          replay_item = false;
          if (it < 0 || it >= n0) {
            if (lane == 0) set_err(a.lb.ctr, ERR_BAD_TASK);
            break;
          }
        } else if (level > 0) {
          break;
        } else {
          if (lane == 0) {
            it = range_take(&sw->range);
            int ob = 0, oe = 0;
            if (it >= 0 &&
                range_maybe_donate(a.lb, &sw->range, v0, &sw->donations_left, t_start, &sw->busy, ob, oe, n0)) {
              // lane 0 is the only taker, so the split can be undone
              const unsigned long long cur = *reinterpret_cast<volatile unsigned long long*>(&sw->range);
              sw->range = (cur & 0xffffffffull) | ((unsigned long long)(unsigned)oe << 32);
            }
          }
          it = __shfl_sync(FULL_MASK, it, 0);
          if (it < 0) break;
        }
        // prefix (v0, w1); the members of E_0 after w1 are the inherited part
        int t = 0;
        int w = __ldg(E0 + it);
        int wmask = 1;
        int src_lo = it + 1;  // level 0: inherited members are E0[it+1 ..]
        bool bad = false;
        // depth-first over levels; level t's current vertex is w with mask wmask
        while (true) {
          // here the prefix is v_0..v_t plus w = v_{t+1}
          const int p = t + 1;  // position of w
          if (p > level) {
            // nodes at or above a donated prefix's level belong to the donor
            ++nodes;
            if (lane == 0 && (nodes & 255) == 0) atomicAdd(&a.lb.ctr->progress, 256ull);
          }
          unsigned quick_p = (t == 0) ? 0u : sw->quick[t];
          if (p >= 2) quick_p += ((unsigned)wmask & ((1u << p) - 1u)) << quick_off(p);
          const int32_t* Nw = a.g.adj + __ldg(a.g.row + w);
          const int dw = __ldg(a.g.deg + w);
          // inherited members: e in E_t with e > w. E_t is sorted by vertex id and w is its
          // member at position pos[t] - 1 (E_0: index it), so they are the suffix from there.
          const int2* Et = (t == 0) ? nullptr : ext_c[t];
          const int nE = (t == 0) ? n0 : sw->n[t];
          const int startE = (t == 0) ? src_lo : sw->pos[t];
          if (p == K - 2) {
            // leaves: histogram the masks of E_{p} without writing it
            const int leaf_off = quick_off(K - 1);
            const int n_inh = nE - startE;
            const int gt = lower_bound(Nw, 0, dw, w + 1);
            const int dgt = dw - gt;
            // probe each inherited member in N(w), or take the suffix's mask counts and
            // move the members found in N(w) above w (whichever side is cheaper)
            if ((long long)dgt * ilog2p1(n_inh) + (1 << (K - 2)) < (long long)n_inh * ilog2p1(dw)) {
              if (t == 0) {
                if (lane == 0 && n_inh) atomicAdd(&sw->mh[1], (unsigned)n_inh);
              } else if (lane < (1 << (K - 2))) {
                const unsigned c = sw->sh[lane];
                if (c) atomicAdd(&sw->mh[lane], c);
              }
              __syncwarp();
              for (int i = gt + lane; i < dw; i += 32) {
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
                  atomicSub(&sw->mh[em], 1u);
                  atomicAdd(&sw->mh[em | (1 << p)], 1u);
                }
              }
            } else {
              for (int i = startE + lane; i < nE; i += 32) {
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
                atomicAdd(&sw->mh[m], 1u);
              }
            }
            // excl(w) = N(w) above v0 minus U_t
            const int sw0 = lower_bound(Nw, 0, dw, v0 + 1);
            const int above = dw - sw0;
            int usize = n0;
            for (int i = 1; i <= t; ++i) usize += sw->runn[i];
            unsigned inter = 0;
            if ((long long)usize <= (long long)above * (t + 1)) {
              // iterate U_t, probe N(w)
              for (int i = lane; i < n0; i += 32) inter += contains(Nw, dw, __ldg(E0 + i)) ? 1u : 0u;
              for (int r = 1; r <= t; ++r) {
                const int2* R = runs_c[r];
                const int nr = sw->runn[r];
                for (int i = lane; i < nr; i += 32) inter += contains(Nw, dw, R[i].x) ? 1u : 0u;
              }
            } else {
              // iterate N(w) above v0, probe the runs
              for (int i = sw0 + lane; i < dw; i += 32)
                inter += in_runs(Nw[i], E0, n0, runs_c, sw->runn, t) ? 1u : 0u;
            }
            for (int o = 16; o > 0; o >>= 1) inter += __shfl_xor_sync(FULL_MASK, inter, o);
            if (lane == 0) {
              const unsigned ex = (unsigned)above - inter;
              if (ex) atomicAdd(&sw->mh[1 << p], ex);
            }
            __syncwarp();
            flush_masks(sw, a, quick_p, leaf_off, bhist, task_cnt);
          } else {
            // materialise E_{p} = inherited + excl(w), merged by vertex id; excl(w) is also
            // run p. Both parts are sorted and disjoint, so each member's place is its index
            // in its own part plus the number of smaller members of the other part.
            int2* Ep = ext[p];
            int2* Rp = runs[p];
            const int sw0 = lower_bound(Nw, 0, dw, v0 + 1);
            int rn = 0;
            for (int i0 = sw0; i0 < dw; i0 += 32) {
              const int i = i0 + lane;
              int32_t x = 0;
              bool nw = false;
              if (i < dw) {
                x = Nw[i];
                nw = !in_runs(x, E0, n0, runs_c, sw->runn, t);
              }
              const unsigned bal = __ballot_sync(FULL_MASK, nw);
              if (nw) Rp[rn + __popc(bal & ((1u << lane) - 1u))] = make_int2(x, 0);
              rn += __popc(bal);
            }
            __syncwarp();
            for (int i = startE + lane; i < nE; i += 32) {
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
            for (int j = lane; j < rn; j += 32) {
              const int32_t x = Rp[j].x;
              const int c = (t == 0) ? lower_bound(E0, 0, n0, x) : lower_bound2(Et, 0, nE, x);
              Ep[j + max(0, c - startE)] = make_int2(x, 1 << p);
            }
            const int m = (nE - startE) + rn;
            __syncwarp();
            if (p < level) {
              // replaying a donated prefix: the path fixes the member expanded at level p
              const int idx = (p < QPATH) ? path[p] : -1;
              if (idx < 0 || idx >= m) {
                if (lane == 0) set_err(a.lb.ctr, ERR_BAD_TASK);
                bad = true;
                break;
              }
              const int2 x = Ep[idx];
              if (lane == 0) {
                sw->n[p] = m;
                sw->pos[p] = idx + 1;
                sw->lim[p] = idx + 1;
                sw->runn[p] = rn;
                sw->quick[p] = quick_p;
              }
              __syncwarp();
              t = p;
              w = x.x;
              wmask = x.y;
              continue;
            }
            const int first_pos = p == level ? min(b, m) : 0;
            if (lane == 0) {
              sw->n[p] = m;
              sw->pos[p] = first_pos;
              sw->lim[p] = p == level ? min(e, m) : m;
              sw->runn[p] = rn;
              sw->quick[p] = quick_p;
            }
            if (p == K - 3) {
              sw->sh[lane] = 0;
              __syncwarp();
              mask_hist(Ep, first_pos, m, sw->sh);
            }
            __syncwarp();
            t = p;  // descend; pick the first member below
          }
          // give work away when warps are hungry (checked every 16 expansions)
          if ((nodes & 15) == 0 && K >= 4) {
            if (lane == 0) motif_try_donate(a.lb, sw, v0, floor, t, it, n0, t_start);
            __syncwarp();
          }
          // next vertex: advance the deepest level that still has members
          bool found = false;
          while (t >= floor) {
            const int ps = sw->pos[t];
            if (ps < sw->lim[t]) {
              const int2 x = ext_c[t][ps];
              __syncwarp();
              if (lane == 0) {
                sw->pos[t] = ps + 1;
                if (t == K - 3) sw->sh[x.y] -= 1u;
              }
              __syncwarp();
              w = x.x;
              wmask = x.y;
              found = true;
              break;
            }
            --t;
          }
          if (!found) break;
        }
        if (bad) break;
      }
      if (a.per_root) {
        const unsigned long long tsum = warp_sum_u64(task_cnt);
        if (lane == 0 && tsum) atomicAdd(a.per_root + v0, tsum);
      }
      __syncwarp();
      if (lane == 0) lb_task_time(a.lb, t_start, v0);
    }
    if (lane == 0) lb_done(a.lb, count);
  }
  nodes = warp_sum_u64(nodes);
  if (lane == 0) {
    atomicAdd(&a.lb.ctr->tasks, ntasks);
    atomicAdd(&a.lb.ctr->nodes, nodes);
  }
  __syncthreads();
  for (int c = threadIdx.x; c < a.n_classes; c += blockDim.x)
    if (bhist[c]) atomicAdd(a.hist + c, bhist[c]);
}

size_t motif_arena_stride(int k, int maxdeg) {
  size_t s = 0;
  for (int t = 1; t <= k - 3; ++t) s += (size_t)(t + 1) * maxdeg + 32;
  for (int t = 1; t <= k - 3; ++t) s += (size_t)maxdeg + 32;
  return s < 1 ? 1 : s;
}

template <int K>
static int launch_motif(MotifArgs a, LaunchCtx& ctx, int* grid_out) {
  const int block = 32 * MOTIF_WARPS;
  const size_t smem = sizeof(unsigned long long) * ((a.n_classes + 1) & ~1) + sizeof(MotifWarp) * MOTIF_WARPS;
  auto kern = motif_kernel<K>;
  DM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int occ = 0;
  DM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, block, smem));
  if (occ < 1) return fail(DM_EINVAL, "motif kernel does not fit on an SM");
  int grid = ctx.num_sms * occ;
  if (ctx.threads > 0) grid = std::max(1, std::min(grid, (ctx.threads + block - 1) / block));
  if (grid * MOTIF_WARPS > ctx.arena_warps) grid = std::max(1, ctx.arena_warps / MOTIF_WARPS);
  const int warps = grid * MOTIF_WARPS;
  a.lb.hungry_trigger = ctx.threshold >= 100 ? 0 : std::max(1, (ctx.threshold * warps + 99) / 100);
  kern<<<grid, block, smem, ctx.stream>>>(a);
  ctx.launches++;
  *grid_out = grid;
  DM_CUDA(cudaGetLastError());
  return DM_OK;
}

int motif_launch(const MotifLaunch& L, LaunchCtx& ctx, int* grid) {
  MotifArgs a;
  a.g = L.g;
  a.roots = L.roots;
  a.n_roots = L.n_roots;
  a.lb = LBArgs{L.ctr, reinterpret_cast<QHeader*>(L.queue),
                reinterpret_cast<QSlot*>(reinterpret_cast<char*>(L.queue) + sizeof(QHeader) * L.nq), L.qcap, 0,
                L.max_donations, (long long)ctx.donate_after_us * 1000ll, (long long)ctx.timeout_ms * 1000000ll,
                ctx.test_stall, 4, L.nq};
  a.k = L.k;
  a.q2c = L.q2c;
  a.n_classes = L.n_classes;
  a.hist = L.hist;
  a.arena = reinterpret_cast<int2*>(L.arena);
  a.arena_stride = (int)motif_arena_stride(L.k, L.maxdeg);
  a.maxdeg = L.maxdeg;
  a.per_root = L.per_root;
  a.parts = L.parts;
  switch (L.k) {
    case 3: return launch_motif<3>(a, ctx, grid);
    case 4: return launch_motif<4>(a, ctx, grid);
    case 5: return launch_motif<5>(a, ctx, grid);
    case 6: return launch_motif<6>(a, ctx, grid);
    case 7: return launch_motif<7>(a, ctx, grid);
    default: return fail(DM_EINVAL, "motif k must be in [3, 7]");
  }
}

}  // namespace dmb
