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
// the warp runs the subtree, and idle warps get donated item ranges (lb.cuh).
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
struct MotifWarp {
  unsigned long long range;
  int donations_left;
  int busy;
  int n[MOTIF_KMAX];           // extension-set sizes per level
  int pos[MOTIF_KMAX];         // next member to expand per level
  int runn[MOTIF_KMAX];        // run sizes per level
  unsigned quick[MOTIF_KMAX];  // quick code of the prefix ending at level t
  unsigned mh[64];             // leaf-mask histogram
};

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
    int first = 0, count = 0, b = 0, e = -1, ok = 0;
    bool donated = false;
    if (lane == 0) ok = lb_next(a.lb, a.n_roots, total_warps, first, count, b, e, donated) ? 1 : 0;
    ok = __shfl_sync(FULL_MASK, ok, 0);
    if (!ok) break;
    first = __shfl_sync(FULL_MASK, first, 0);
    count = __shfl_sync(FULL_MASK, count, 0);
    b = __shfl_sync(FULL_MASK, b, 0);
    e = __shfl_sync(FULL_MASK, e, 0);
    donated = __shfl_sync(FULL_MASK, donated ? 1 : 0, 0) != 0;
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
      int lo, hi;
      task_range(bb, ee, n0, lo, hi);
      if (lane == 0) {
        sw->range = pack_range(lo, hi);
        sw->donations_left = a.lb.max_donations;
        sw->busy = 0;
        sw->quick[0] = 0;
      }
      __syncwarp();
      while (true) {
        int it = 0;
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
        // prefix (v0, w1); the members of E_0 after w1 are the inherited part
        int t = 0;
        int w = __ldg(E0 + it);
        int wmask = 1;
        int src_lo = it + 1;  // level 0: inherited members are E0[it+1 ..]
        // depth-first over levels; level t's current vertex is w with mask wmask
        while (true) {
          // here the prefix is v_0..v_t plus w = v_{t+1}
          ++nodes;
          if (lane == 0 && (nodes & 255) == 0) atomicAdd(&a.lb.ctr->progress, 256ull);
          const int p = t + 1;  // position of w
          unsigned quick_p = (t == 0) ? 0u : sw->quick[t];
          if (p >= 2) quick_p += ((unsigned)wmask & ((1u << p) - 1u)) << quick_off(p);
          const int32_t* Nw = a.g.adj + __ldg(a.g.row + w);
          const int dw = __ldg(a.g.deg + w);
          // inherited members: e in E_t with e > w
          const int2* Et = (t == 0) ? nullptr : ext_c[t];
          const int nE = (t == 0) ? n0 : sw->n[t];
          const int startE = (t == 0) ? src_lo : 0;
          if (p == K - 2) {
            // leaves: histogram the masks of E_{p} without writing it
            const int leaf_off = quick_off(K - 1);
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
              if (ev > w) {
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
                inter += in_runs(__ldg(Nw + i), E0, n0, runs_c, sw->runn, t) ? 1u : 0u;
            }
            for (int o = 16; o > 0; o >>= 1) inter += __shfl_xor_sync(FULL_MASK, inter, o);
            if (lane == 0) {
              const unsigned ex = (unsigned)above - inter;
              if (ex) atomicAdd(&sw->mh[1 << p], ex);
            }
            __syncwarp();
            flush_masks(sw, a, quick_p, leaf_off, bhist, task_cnt);
          } else {
            // materialise E_{p} = inherited + excl(w); excl(w) also becomes run p
            int2* Ep = ext[p];
            int2* Rp = runs[p];
            int m = 0;
            for (int i0 = startE; i0 < nE; i0 += 32) {
              const int i = i0 + lane;
              int ev = 0, em = 0;
              bool keep = false;
              if (i < nE) {
                if (t == 0) {
                  ev = __ldg(E0 + i);
                  em = 1;
                } else {
                  const int2 x = Et[i];
                  ev = x.x;
                  em = x.y;
                }
                keep = ev > w;
                if (keep && contains(Nw, dw, ev)) em |= 1 << p;
              }
              const unsigned bal = __ballot_sync(FULL_MASK, keep);
              if (keep) Ep[m + __popc(bal & ((1u << lane) - 1u))] = make_int2(ev, em);
              m += __popc(bal);
            }
            const int sw0 = lower_bound(Nw, 0, dw, v0 + 1);
            int rn = 0;
            for (int i0 = sw0; i0 < dw; i0 += 32) {
              const int i = i0 + lane;
              int32_t x = 0;
              bool nw = false;
              if (i < dw) {
                x = __ldg(Nw + i);
                nw = !in_runs(x, E0, n0, runs_c, sw->runn, t);
              }
              const unsigned bal = __ballot_sync(FULL_MASK, nw);
              if (nw) {
                const int q = __popc(bal & ((1u << lane) - 1u));
                Rp[rn + q] = make_int2(x, 0);
                Ep[m + q] = make_int2(x, 1 << p);
              }
              rn += __popc(bal);
              m += __popc(bal);
            }
            __syncwarp();
            if (lane == 0) {
              sw->n[p] = m;
              sw->pos[p] = 0;
              sw->runn[p] = rn;
              sw->quick[p] = quick_p;
            }
            __syncwarp();
            t = p;  // descend; pick the first member below
          }
          // next vertex: advance the deepest level that still has members
          bool found = false;
          while (t >= 1) {
            const int ps = sw->pos[t];
            if (ps < sw->n[t]) {
              const int2 x = ext_c[t][ps];
              __syncwarp();
              if (lane == 0) sw->pos[t] = ps + 1;
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
