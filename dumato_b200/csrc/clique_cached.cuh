// k-clique counting on a per-graph local-bitmap index (sm_100a).
//
// The bitmap path of clique.cuh rebuilds, for every root r, the local adjacency bitmap of
// L = N+(r) (bit j of row i set iff L[j] in N+(L[i])) from the CSR: a chain of dependent
// loads (row starts, member rows) and a shared-memory search per (member, neighbour) pair,
// repeated for every k. Here those bitmaps are built once per device copy of the graph
// (index_build_kernel, 16-byte vector loads of the padded adjacency rows) and kept as the
// clique index: one block of d x ceil(d/64) u64 words per root with 2 <= d <= 256, each
// block starting on a 16-byte boundary. A counting launch then only stages a root's block
// into shared memory (plain 16-byte loads, or one bulk asynchronous copy per block) and
// runs the DFS, which is the reference's extend_clique / aggregate_counter loop
// (src/main/DuMatoGPU.cu:1194-1220, 1769-1771) as AND + popc over the rows.
//
// Task structure (one warp per task):
//   chunk tasks: entries of the root list; the warp stages as many of their blocks as fit
//       in one round of loads, then counts them one after the other. The first CHUNK_MAX x T
//       entries (T warps) are dealt statically and interleaved - warp w takes w, w + T, ... -
//       so the heaviest roots of the descending order start on different warps and no cursor
//       atomics are needed; the rest is claimed from the cursor in runs. Completions of the
//       static entries are settled once per block, later ones once per warp when it runs out
//       of work, and the final sums once per block: a launch issues few global atomics on the
//       shared words.
//   level-0 donations: (root, item range) as in clique.cuh.
//   level-1 donations (k >= 6): (root, item, range of positions in the item's candidate
//       set S = row[c1] & row[c2]): the positions choose the third local vertex c3, so a
//       heavy item is split across warps below the first level - the reference's donation
//       of (id[0..t], lastExt(t)) prefixes at a target level t (DuMatoCPU.cu:463-539).
#pragma once

#include "clique.cuh"

namespace dmb {

constexpr int INDEX_MAX_WORDS = 4;  // rows of up to INDEX_MAX_DEGREE = 256 bits

// 16-byte units of a root's block: d rows of ceil(d/64) u64 words, rounded up to two words.
__device__ __forceinline__ uint32_t index_block_units(int d) {
  const int nw = (d + 63) >> 6;
  return (uint32_t)((d * nw + 1) >> 1);
}

// ---------------- index build ----------------

// Loads L = N+(root) into sL, the members' row starts into sR, and the exclusive prefix of
// the members' 16-byte chunk counts (ceil(deg/4)) into sC[0..d]. Returns the chunk total.
static __device__ __forceinline__ int load_root_chunks(const GraphView& g, int root, int d, int32_t* sL,
                                                       int32_t* sC, int32_t* sR) {
  const int lane = lane_id();
  const int32_t* L = g.adj + __ldg(g.row + root);
  int carry = 0;
  for (int i0 = 0; i0 < d; i0 += 32) {
    const int i = i0 + lane;
    int ch = 0;
    if (i < d) {
      const int u = __ldg(L + i);
      ch = (__ldg(g.deg + u) + 3) >> 2;
      sR[i] = __ldg(g.row + u);
      sL[i] = u;
    }
    int s = ch;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(FULL_MASK, s, o);
      if (lane >= o) s += y;
    }
    if (i < d) sC[i] = carry + s - ch;
    carry += __shfl_sync(FULL_MASK, s, 31);
  }
  if (lane == 0) sC[d] = carry;
  __syncwarp();
  return carry;
}

// Sets the local rows from 16-byte chunks of the members' padded adjacency rows (every row
// starts on 16 bytes and is padded with INT32_MAX, which lies above every member): each
// lane issues INDEX_UNROLL int4 loads before it uses any of them, and tests each of the four
// neighbours for membership in L by a binary search over the members after the owner (the
// DAG only points upwards in rank).
constexpr int INDEX_UNROLL = 4;

template <int M>
static __device__ __forceinline__ void build_rows_v4(const int32_t* adj, const int32_t* sL, const int32_t* sC,
                                                     const int32_t* sR, int d, int total, uint32_t* rows,
                                                     int row_words) {
  const int lane = lane_id();
  const int32_t maxL = sL[d - 1];
  int i = 0;
  for (int f0 = lane; f0 < total; f0 += 32 * INDEX_UNROLL) {
    int4 x[INDEX_UNROLL];
    int own[INDEX_UNROLL];
#pragma unroll
    for (int u = 0; u < INDEX_UNROLL; ++u) {
      const int f = f0 + 32 * u;
      own[u] = -1;
      if (f < total) {
        while (sC[i + 1] <= f) ++i;
        own[u] = i;
        x[u] = ldg4(adj + sR[i] + 4 * (f - sC[i]));
      }
    }
#pragma unroll
    for (int u = 0; u < INDEX_UNROLL; ++u) {
      const int m = own[u];
      if (m < 0) continue;
      const int32_t v[4] = {x[u].x, x[u].y, x[u].z, x[u].w};
      // a binary search over the members above m (out-neighbours rank above m): most of these
      // ranges are short, so it beats a fixed-length branch-free search here (measured: 32 µs
      // against 38 µs per build on chunglu18k)
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        if (v[c] > maxL) continue;
        const int j = lower_bound(sL, m + 1, d, v[c]);
        if (j < d && sL[j] == v[c]) atomicOr(rows + m * row_words + (j >> 5), 1u << (j & 31));
      }
    }
  }
}

// One warp per listed root (grid-stride): builds the root's rows in shared memory and
// stores the block. Shared memory per warp: warp_layout(M).
template <int M>
__global__ void __launch_bounds__(256) index_build_kernel(GraphView g, const int32_t* __restrict__ roots, int n,
                                                          uint4* __restrict__ blocks,
                                                          const uint32_t* __restrict__ boff) {
  extern __shared__ __align__(16) unsigned char smem[];
  constexpr WarpLayout LY = warp_layout(M);
  const int lane = lane_id();
  unsigned char* wsm = smem + (size_t)LY.total * warp_in_block();
  uint32_t* rows32 = reinterpret_cast<uint32_t*>(wsm + LY.rows);
  int32_t* sL = reinterpret_cast<int32_t*>(wsm + LY.L);
  int32_t* sC = reinterpret_cast<int32_t*>(wsm + LY.P);
  int32_t* sR = reinterpret_cast<int32_t*>(wsm + LY.E);
  const int gw = blockIdx.x * (blockDim.x >> 5) + warp_in_block();
  const int tw = gridDim.x * (blockDim.x >> 5);
  for (int t = gw; t < n; t += tw) {
    const int root = __ldg(roots + t);
    const int d = __ldg(g.deg + root);
    const int nw = (d + 63) >> 6;
    const int units = (int)index_block_units(d);
    for (int i = lane; i < units * 4; i += 32) rows32[i] = 0;
    const int total = load_root_chunks(g, root, d, sL, sC, sR);
    build_rows_v4<M>(g.adj, sL, sC, sR, d, total, rows32, 2 * nw);
    __syncwarp();
    const uint4* src = reinterpret_cast<const uint4*>(rows32);
    uint4* dst = blocks + __ldg(boff + root);
    for (int u = lane; u < units; u += 32) dst[u] = src[u];
    __syncwarp();
  }
}

// ---------------- counting on the index ----------------

__host__ __device__ constexpr int stage_words(int M) { return M == 1 ? 512 : 1024; }
constexpr int CHUNK_MAX = 16;     // roots claimed together
constexpr int SMALL_ITEMS = 64;   // roots with at most this many local edges are batched
constexpr int SMALL_WORDS = 512;  // ... from staging rounds of at most this many words
constexpr int SMALL_ARRAYS = 4;   // batched entries: item offset, first word, out-degree, root

// Shared memory of one warp: staged blocks | item prefix of the current root | task state |
// bulk-copy barrier. At least warp_layout(M).total bytes, so that the list path (roots above
// 256 out-neighbours), which keeps its state at warp_layout(M)'s offsets, can share it.
struct CachedWarp {
  int stage, E, bat, stk, range, don, busy, hn, heavy, mbar, total;
};

__host__ __device__ constexpr CachedWarp cached_layout(int M) {
  CachedWarp w{};
  w.stage = 0;
  w.E = 8 * stage_words(M);
  // item prefix: of one root's rows, or of up to SMALL_WORDS staged words when small roots
  // are batched
  w.bat = w.E + 4 * (SMALL_WORDS + 1);
  w.stk = (w.bat + 4 * SMALL_ARRAYS * (CHUNK_MAX + 1) + 15) / 16 * 16;
  w.range = w.stk + 8 * walk_stack_words(INDEX_MAX_K, M, 4);
  w.don = w.range + 8;
  w.busy = w.don + 4;
  w.hn = w.busy + 4;
  w.heavy = w.hn + 4;
  w.mbar = (w.heavy + 4 * HEAVY_SLOTS + 7) / 8 * 8;
  const int own = (w.mbar + 8 + 15) / 16 * 16;
  const int list = warp_layout(M).total;
  w.total = own > list ? own : list;
  return w;
}

struct CachedArgs {
  CliqueArgs c;                // graph (rank-space DAG), LB, per-root log, list-path arena
  const RootDesc* desc;        // task list (c.n_roots entries)
  const uint4* blocks;         // the clique index
  const uint32_t* boff;        // block offset per root (rank space), for donated tasks
  int static_chunk;            // entries per warp dealt statically (at most CHUNK_MAX)
  int n_static;                // entries [0, n_static) are dealt statically, warp w taking
                               // w, w + T, w + 2T, ... (T warps): the heaviest entries of a
                               // descending order land on different warps; the cursor starts
                               // at n_static
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Bulk asynchronous copy of `bytes` (a multiple of 16, both addresses 16-byte aligned) from
// global to this CTA's shared memory, completing on the mbarrier.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* mbar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(mbar))
      : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* mbar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(mbar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

__device__ __forceinline__ void mbar_expect(uint64_t* mbar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(mbar)), "r"(bytes)
               : "memory");
}

// Waits for the barrier's phase `parity` to complete; gives up after a bounded number of
// polls (returns false).
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, unsigned parity) {
  for (int it = 0; it < (1 << 22); ++it) {
    unsigned done = 0;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(mbar)), "r"(parity)
        : "memory");
    if (done) return true;
    if (it > 64) __nanosleep(64);
  }
  return false;
}

// Level-1 task: positions [lo, hi) (hi < 0: to the end) of the candidate set S of item
// `it` (the root, c1 and c2 are clique vertices 1..3) choose vertex 4, c3; each lane walks
// S_{>c3} & row[c3], the candidates for vertex 5, for the positions it takes. While warps
// are hungry the upper part of the positions left is donated as (root, level 1, path = {it},
// range).
template <int K, int NW, bool MULTI>
__device__ __forceinline__ unsigned long long heavy_walk(const CachedArgs& a, const TaskWords& tw, const uint64_t* rows,
                                                         const Bits<NW>& S, int root, int it, int lo, int hi,
                                                         bool eager, Acc<K>& acc, CheckState& cs) {
  const int lane = lane_id();
  const int p = popc(S);
  const int end = hi < 0 ? p : min(hi, p);
  __syncwarp();
  if (lane == 0) {
    *tw.range = pack_range(lo, end);
    *tw.don = a.c.lb.max_donations;
    *tw.busy = 0;
  }
  __syncwarp();
  const long long t_start = lane == 0 ? clock64() : 0;  // SM clock cycles
  const int path[1] = {it};
  unsigned long long cnt = 0;
  WalkR<K, NW, MULTI, 5> wk;
  wk.stk = tw.stk;
  const PositionItems<K, NW, MULTI> pos{rows, S};
  lockstep_items<K>(a.c.lb, tw, wk, pos, acc, cnt, root, t_start, p, 2, 1, path, eager, cs);
  __syncwarp();
  return cnt;
}

// heavy_walk of item `it` of a root whose row prefix is sE.
template <int K, int NW, bool MULTI>
__device__ __forceinline__ unsigned long long heavy_run(const CachedArgs& a, const TaskWords& tw, const uint64_t* rows,
                                                        const int32_t* sE, int d, int root, int it, int lo, int hi,
                                                        bool eager, Acc<K>& acc, CheckState& cs) {
  const int c1 = lower_bound(sE, 0, d + 1, it + 1) - 1;
  const int c2 = select_bit<NW>(rows + c1 * NW, it - sE[c1]);
  Bits<NW> S;
#pragma unroll
  for (int w = 0; w < NW; ++w) S.w[w] = rows[c1 * NW + w] & rows[c2 * NW + w];
  return heavy_walk<K, NW, MULTI>(a, tw, rows, S, root, it, lo, hi, eager, acc, cs);
}

// Counts one root's task from its staged rows: level 0 runs items [b, e) (task_range
// encoding; items are the local edges, or the rows when k == 3), level 1 runs positions
// [b, e) of item `it`'s candidate set. Returns this lane's share.
template <int K, int NW, bool MULTI>
__device__ __forceinline__ unsigned long long staged_run(const CachedArgs& a, const TaskWords& tw,
                                                         const uint64_t* rows, int32_t* sE, int root, int d, int b,
                                                         int e, int level, int it, bool eager, Acc<K>& acc,
                                                         CheckState& cs) {
  const int lane = lane_id();
  int n_items;
  if constexpr (K >= 4) {
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
        const int y = __shfl_up_sync(FULL_MASK, s, o);
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
  __syncwarp();
  if constexpr (K >= 6) {
    if (level == 1) return heavy_run<K, NW, MULTI>(a, tw, rows, sE, d, root, it, b, e, eager, acc, cs);
  }
  int lo, hi;
  task_range(b, e, n_items, lo, hi);
  if (lane == 0) {
    *tw.range = pack_range(lo, hi);
    *tw.don = a.c.lb.max_donations;
    *tw.busy = 0;
    *tw.hn = 0;
  }
  __syncwarp();
  unsigned long long cnt = 0;
  if constexpr (K == 3) {
    // items are the rows: one popcount each, the lanes stay together
    const long long t_start = global_ns();
    unsigned done = 0;
    int x;
    while ((x = range_take(tw.range)) >= 0) {
      Bits<NW> S;
#pragma unroll
      for (int w = 0; w < NW; ++w) S.w[w] = rows[x * NW + w];
      cnt += (unsigned long long)popc(S);
      if ((++done & 15) == 0) {
        int ob = 0, oe = 0;
        if (range_maybe_donate(a.c.lb, tw.range, root, tw.don, t_start, tw.busy, ob, oe, 0, 0, 0, nullptr, eager)) {
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
    WalkR<K, NW, MULTI, 4> wk;
    wk.stk = tw.stk;
    const EdgeItems<K, NW, MULTI> items{rows, sE, d, tw.hn, tw.heavy};
    const long long t_cyc = lane == 0 ? clock64() : 0;
    lockstep_items<K>(a.c.lb, tw, wk, items, acc, cnt, root, t_cyc, 0, 0, 0, nullptr, eager, cs);
    __syncwarp();
    if constexpr (K >= 6) {
      const int nh = min(*tw.hn, HEAVY_SLOTS);
      for (int h = 0; h < nh; ++h) {
        const int hit = tw.heavy[h];
        cnt += heavy_run<K, NW, MULTI>(a, tw, rows, sE, d, root, hit, 0, -1, eager, acc, cs);
      }
    }
    return cnt;
  }
}

// Items of the batched small roots of a staging round (small_batch): item g belongs to the
// entry j with sO[j] <= g < sO[j + 1]; it is that entry's item e = g - sO[j], whose row c1
// is the word r of the entry with E[r] <= E[sB[j]] + e < E[r + 1].
template <int K, bool MULTI>
struct BatchItems {
  const uint64_t* srows;
  const int32_t* E;
  const int32_t* bat;  // sO | sB | sD | sR, CHUNK_MAX + 1 each
  int ne;
  int* hn;
  int* heavy;
  __device__ __forceinline__ void locate(int g, int& j, int& e, int& b0, Bits<1>& S) const {
    const int32_t* sO = bat;
    const int32_t* sB = bat + (CHUNK_MAX + 1);
    const int32_t* sD = bat + 2 * (CHUNK_MAX + 1);
    j = lower_bound_bl<16>(sO, ne + 1, g + 1) - 1;
    e = g - sO[j];
    b0 = sB[j];
    const int target = E[b0] + e;
    const int r = b0 + lower_bound_bl<64>(E + b0, sD[j] + 1, target + 1) - 1;
    const int c2 = select64(srows[r], target - E[r]);
    S.w[0] = srows[r] & srows[b0 + c2];
  }
  template <class WK>
  __device__ __forceinline__ void operator()(int g, WK& wk, Acc<K>& acc, unsigned long long& cnt) const {
    int j, e, b0;
    Bits<1> S;
    locate(g, j, e, b0, S);
    if constexpr (MULTI) acc.c[3] += 1ull;
    if constexpr (K >= 6) {
      const int p = popc(S);
      if (p >= HEAVY_BITS) {
        const int slot = atomicAdd(hn, 1);
        if (slot < HEAVY_SLOTS) {
          heavy[slot] = g;
          if constexpr (MULTI) acc.c[4] += (unsigned long long)p;
          return;
        }
      }
    }
    wk.start(S, srows + b0, acc, cnt);
  }
};

// Small roots of a staging round counted together. Entries [i0, i1) of the round are staged
// (lane i holds entry i); those with rows of one word, a whole root (no part or donated range)
// and at most SMALL_ITEMS local edges form one item space: the exclusive prefix E of the
// popcounts of every staged word gives each entry's items, an entry's items follow the
// items of the batched entries before it, and a lane maps item g to its entry (a search over
// the entries' item offsets), its row c1 (a search over E within the entry) and c2 (a bit
// select). One lockstep walk then covers all of them, so a root of a few items costs a few
// lanes of one refill rather than a pass of the whole warp. The combined range is not
// donated (a donation names one root); heavy items still donate their positions (level 1).
// Returns the mask of the entries counted here.
template <int K, bool MULTI>
__device__ __forceinline__ unsigned small_batch(const CachedArgs& a, const TaskWords& tw, const uint64_t* srows,
                                                int32_t* E, int32_t* bat, int i0, int i1, int root, int d,
                                                uint32_t units, uint32_t rspos, int part, Acc<K>& acc,
                                                unsigned long long& cnt, CheckState& cs) {
  const int lane = lane_id();
  const bool in_round = lane >= i0 && lane < i1;
  const bool cand = in_round && units > 0 && d >= 2 && d <= 64 && (part & ~PART_EAGER) == 0;
  if (__popc(__ballot_sync(FULL_MASK, cand)) < 2) return 0u;
  // E over the round's staged words
  const int W = (int)(2u * __shfl_sync(FULL_MASK, rspos + units, i1 - 1));
  if (W > SMALL_WORDS) return 0u;
  int carry = 0;
  for (int w0 = 0; w0 < W; w0 += 32) {
    const int w = w0 + lane;
    const int pc = w < W ? __popcll(srows[w]) : 0;
    int s = pc;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(FULL_MASK, s, o);
      if (lane >= o) s += y;
    }
    if (w < W) E[w] = carry + s - pc;
    carry += __shfl_sync(FULL_MASK, s, 31);
  }
  if (lane == 0) E[W] = carry;
  __syncwarp();
  const int base = (int)(2u * rspos);
  const int n_items = cand ? E[base + d] - E[base] : 0;
  const bool small = cand && n_items <= SMALL_ITEMS;
  const unsigned done = __ballot_sync(FULL_MASK, small);
  if (__popc(done) < 2) return 0u;
  // item offsets of the batched entries (others hold no items), relative to i0
  const int mine = small ? n_items : 0;
  int s = mine;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(FULL_MASK, s, o);
    if (lane >= o) s += y;
  }
  const int before = s - mine - __shfl_sync(FULL_MASK, s - mine, i0);  // exclusive, from entry i0
  const int total = __shfl_sync(FULL_MASK, s, i1 - 1) - __shfl_sync(FULL_MASK, s - mine, i0);
  const int ne = i1 - i0;
  int32_t* sO = bat;
  int32_t* sB = bat + (CHUNK_MAX + 1);
  int32_t* sD = bat + 2 * (CHUNK_MAX + 1);
  int32_t* sR = bat + 3 * (CHUNK_MAX + 1);
  if (in_round) {
    sO[lane - i0] = before;
    sB[lane - i0] = base;
    sD[lane - i0] = d;
    sR[lane - i0] = root;
  }
  if (lane == 0) {
    sO[ne] = total;
    *tw.range = pack_range(0, total);
    *tw.don = a.c.lb.max_donations;
    *tw.busy = 0;
    *tw.hn = 0;
  }
  __syncwarp();
  if (total > 0) {
    WalkR<K, 1, MULTI, 4> wk;
    wk.stk = tw.stk;
    const BatchItems<K, MULTI> items{srows, E, bat, ne, tw.hn, tw.heavy};
    const long long t_cyc = lane == 0 ? clock64() : 0;
    lockstep_items<K>(a.c.lb, tw, wk, items, acc, cnt, 0, t_cyc, 0, INT_MAX, 0, nullptr, false, cs);
    __syncwarp();
    if constexpr (K >= 6) {
      const int nh = min(*tw.hn, HEAVY_SLOTS);
      for (int h = 0; h < nh; ++h) {
        int j, e, b0;
        Bits<1> S;
        items.locate(tw.heavy[h], j, e, b0, S);
        cnt += heavy_walk<K, 1, MULTI>(a, tw, srows + b0, S, sR[j], e, 0, -1, false, acc, cs);
      }
    }
  }
  __syncwarp();
  return done;
}

template <int K, int M, bool MULTI>
__device__ __forceinline__ unsigned long long staged_dispatch(const CachedArgs& a, const TaskWords& tw,
                                                              const uint64_t* rows, int32_t* sE, int root, int d,
                                                              int b, int e, int level, int it, bool eager,
                                                              Acc<K>& acc, CheckState& cs) {
  const int nw = (d + 63) >> 6;
  if (nw <= 1) return staged_run<K, 1, MULTI>(a, tw, rows, sE, root, d, b, e, level, it, eager, acc, cs);
  if constexpr (M >= 2)
    if (nw == 2) return staged_run<K, 2, MULTI>(a, tw, rows, sE, root, d, b, e, level, it, eager, acc, cs);
  if constexpr (M >= 3)
    if (nw == 3) return staged_run<K, 3, MULTI>(a, tw, rows, sE, root, d, b, e, level, it, eager, acc, cs);
  if constexpr (M >= 4)
    if (nw == 4) return staged_run<K, 4, MULTI>(a, tw, rows, sE, root, d, b, e, level, it, eager, acc, cs);
  if (lane_id() == 0) set_err(a.c.lb.ctr, ERR_BAD_TASK);
  return 0;
}

// Stages blocks [i0, i1) of the chunk (lane i of the warp holds entry i's offset `off`
// and its staging position `spos`, both in 16-byte units) into the warp's staging area.
// TMA: one bulk asynchronous copy per block, issued by lane 0, completing on the warp's
// mbarrier (phase `*phase`, flipped here). Else: 16-byte loads, INDEX_UNROLL per lane in
// flight. Returns false if the bounded wait on the barrier gave up.
template <bool TMA>
__device__ __forceinline__ bool stage_blocks(const uint4* blocks, uint4* stage, uint64_t* mbar, unsigned* phase,
                                             int i0, int i1, uint32_t off, uint32_t spos, uint32_t units) {
  const int lane = lane_id();
  const uint32_t total = __shfl_sync(FULL_MASK, spos + units, i1 - 1) - __shfl_sync(FULL_MASK, spos, i0);
  const uint32_t base = __shfl_sync(FULL_MASK, spos, i0);
  if constexpr (TMA) {
    // the generic-proxy reads of the previous round are done before the async proxy writes
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncwarp();
    if (lane == 0) mbar_expect(mbar, total * 16u);
    __syncwarp();
    if (lane >= i0 && lane < i1 && units > 0) bulk_g2s(stage + (spos - base), blocks + off, units * 16u, mbar);
    const bool ok = mbar_wait(mbar, *phase);
    *phase ^= 1u;
    return ok;
  } else {
    __syncwarp();
    // warp-uniform loop: every lane takes part in the shuffles that name each unit's block
    for (uint32_t u0 = 0; u0 < total; u0 += 32 * INDEX_UNROLL) {
      uint32_t src[INDEX_UNROLL];
#pragma unroll
      for (int q = 0; q < INDEX_UNROLL; ++q) src[q] = 0;
      for (int i = i0; i < i1; ++i) {
        const uint32_t si = __shfl_sync(FULL_MASK, spos, i) - base;
        const uint32_t oi = __shfl_sync(FULL_MASK, off, i);
#pragma unroll
        for (int q = 0; q < INDEX_UNROLL; ++q) {
          const uint32_t u = u0 + lane + 32 * q;
          if (u >= si) src[q] = oi + (u - si);  // the last block starting at or before u
        }
      }
      uint4 v[INDEX_UNROLL];
#pragma unroll
      for (int q = 0; q < INDEX_UNROLL; ++q) {
        const uint32_t u = u0 + lane + 32 * q;
        if (u < total) v[q] = __ldg(blocks + src[q]);
      }
#pragma unroll
      for (int q = 0; q < INDEX_UNROLL; ++q) {
        const uint32_t u = u0 + lane + 32 * q;
        if (u < total) stage[u] = v[q];
      }
    }
    __syncwarp();
    return true;
  }
}

// Blocks per SM the register budget is sized for: the index kernel of rows up to 64 bits
// keeps four blocks (the shared-memory limit), wider rows two.
template <int M>
constexpr int cached_min_blocks() { return M == 1 ? 2 : 2; }

template <int K, int M, bool TMA, bool MULTI>
__global__ void __launch_bounds__(256, cached_min_blocks<M>()) clique_cached_kernel(const __grid_constant__ CachedArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  constexpr CachedWarp LY = cached_layout(M);
  constexpr uint32_t STAGE_UNITS = stage_words(M) / 2;
  const int lane = lane_id();
  unsigned char* wsm = smem + (size_t)LY.total * warp_in_block();
  uint4* stage = reinterpret_cast<uint4*>(wsm + LY.stage);
  const uint64_t* srows = reinterpret_cast<const uint64_t*>(wsm + LY.stage);
  int32_t* sE = reinterpret_cast<int32_t*>(wsm + LY.E);
  int32_t* sBat = reinterpret_cast<int32_t*>(wsm + LY.bat);
  uint64_t* mbar = reinterpret_cast<uint64_t*>(wsm + LY.mbar);
  TaskWords tw{reinterpret_cast<unsigned long long*>(wsm + LY.range), reinterpret_cast<int*>(wsm + LY.don),
               reinterpret_cast<int*>(wsm + LY.busy), reinterpret_cast<int*>(wsm + LY.hn),
               reinterpret_cast<int*>(wsm + LY.heavy), reinterpret_cast<uint64_t*>(wsm + LY.stk)};
  if constexpr (TMA) {
    if (lane == 0) mbar_init(mbar);
    __syncwarp();
  }
  unsigned phase = 0;
  const int gw = blockIdx.x * (blockDim.x >> 5) + warp_in_block();
  const int total_warps = gridDim.x * (blockDim.x >> 5);
  // per-block sums, flushed by one thread at exit (few global atomics per launch):
  // [0] cliques, [1] tasks, [2] idle polls, [3] waiting ns; and the block's static entries
  // finished, subtracted from `pending` by the last of its warps to finish its static chunk
  __shared__ unsigned long long blk_sum[4];
  __shared__ unsigned long long blk_k[16];  // fused counts by clique size
  __shared__ int blk_static_done, blk_warps_done;
  if (threadIdx.x < 4) blk_sum[threadIdx.x] = 0ull;
  if (MULTI && threadIdx.x < 16) blk_k[threadIdx.x] = 0ull;
  if (threadIdx.x == 0) {
    blk_static_done = 0;
    blk_warps_done = 0;
  }
  __syncthreads();
  unsigned long long idle[2] = {0ull, 0ull};
  CheckState cs;
  Acc<K> acc;
#pragma unroll
  for (int j = 0; j <= K; ++j) acc.c[j] = 0ull;
  int32_t* my_arena =
      a.c.arena ? a.c.arena + (size_t)gw * (32 / a.c.list_vwarp) * K * a.c.arena_dcap : nullptr;
  unsigned long long cnt = 0, ntasks = 0;
  int unflushed = 0;  // lane 0: finished chunk entries not yet subtracted from pending
  bool first_claim = true;
  while (true) {
    int first = 0, count = 0, b = 0, e = -1, ok = 0, level = 0;
    int path[QPATH];
#pragma unroll
    for (int j = 0; j < QPATH; ++j) path[j] = 0;
    bool donated = false;
    const bool is_static = first_claim;
    if (lane == 0) {
      if (is_static) {
        first = gw;
        count = gw < a.n_static ? (a.n_static - gw + total_warps - 1) / total_warps : 0;
        ok = 1;
      } else {
        ok = lb_next(a.c.lb, a.c.n_roots, total_warps, first, count, b, e, donated, level, path, &unflushed, idle)
                 ? 1 : 0;
      }
    }
    first_claim = false;
    ok = __shfl_sync(FULL_MASK, ok, 0);
    if (!ok) break;
    first = __shfl_sync(FULL_MASK, first, 0);
    count = __shfl_sync(FULL_MASK, count, 0);
    b = __shfl_sync(FULL_MASK, b, 0);
    e = __shfl_sync(FULL_MASK, e, 0);
    level = __shfl_sync(FULL_MASK, level, 0);
    const int it1 = __shfl_sync(FULL_MASK, level > 0 ? path[0] : 0, 0);
    donated = __shfl_sync(FULL_MASK, donated ? 1 : 0, 0) != 0;
    if (donated && (level < 0 || level > 1 || (level == 1 && K < 6))) {
      if (lane == 0) {
        set_err(a.c.lb.ctr, ERR_BAD_TASK);
        lb_done(a.c.lb, 1);
      }
      break;
    }
    // the chunk's entries, one per lane (a donated task is one entry)
    int root = 0, d = 0, part = 0;
    uint32_t off = INDEX_NONE;
    if (lane < count) {
      if (donated) {
        root = first;
        d = __ldg(a.c.g.deg + root);
        off = d >= 2 && d <= 64 * INDEX_MAX_WORDS ? __ldg(a.boff + root) : INDEX_NONE;
      } else {
        const RootDesc rd = a.desc[is_static ? first + lane * total_warps : first + lane];
        root = rd.root;
        d = rd.d;
        off = rd.off;
        part = rd.part;
      }
    }
    const uint32_t units = off != INDEX_NONE && d <= 64 * M ? index_block_units(d) : 0u;
    uint32_t spos = units;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(FULL_MASK, spos, o);
      if (lane >= o) spos += y;
    }
    spos -= units;  // exclusive prefix in 16-byte units
    int i0 = 0;
    while (i0 < count) {
      // the entries from i0 whose blocks fit in one staging round (at least one does)
      const uint32_t start = __shfl_sync(FULL_MASK, spos, i0);
      const unsigned fit = __ballot_sync(FULL_MASK, lane >= i0 && lane < count && spos + units - start <= STAGE_UNITS);
      int i1 = i0 + 1;
      while (i1 < count && ((fit >> i1) & 1u)) ++i1;
      const uint32_t rspos = spos - start;
      if (__shfl_sync(FULL_MASK, rspos + units, i1 - 1) > 0) {
        if (!stage_blocks<TMA>(a.blocks, stage, mbar, &phase, i0, i1, off, rspos, units)) {
          if (lane == 0) set_err(a.c.lb.ctr, ERR_TIMEOUT);
        }
      }
      unsigned batched = 0u;
      if constexpr (K >= 4) {
        if (!donated && !a.c.per_root) {
          batched = small_batch<K, MULTI>(a, tw, srows, sE, sBat, i0, i1, root, d, units, rspos, part, acc, cnt, cs);
          ntasks += __popc(batched);
        }
      }
      for (int i = i0; i < i1; ++i) {
        if ((batched >> i) & 1u) continue;
        const int r = __shfl_sync(FULL_MASK, root, i);
        const int di = __shfl_sync(FULL_MASK, d, i);
        const uint32_t ui = __shfl_sync(FULL_MASK, units, i);
        const uint32_t si = __shfl_sync(FULL_MASK, rspos, i);
        int bb = b, ee = e;
        const int pw = donated ? 0 : __shfl_sync(FULL_MASK, part, i);
        if (!donated) part_bounds(pw, bb, ee);
        const bool eager = (pw & PART_EAGER) != 0;
        ++ntasks;
        unsigned long long tc = 0;
        if (bb >= 0 && ee >= 0 && bb >= ee) {
          // empty donation
        } else if (K == 2) {
          if (lane == 0) tc = (unsigned long long)di;
        } else if (ui > 0) {
          tc = staged_dispatch<K, M, MULTI>(a, tw, srows + 2 * si, sE, r, di, bb, ee, level, it1, eager, acc, cs);
        } else if (MULTI && di > a.c.list_threshold) {
          if (lane == 0) set_err(a.c.lb.ctr, ERR_BAD_TASK);  // the fused count runs on the index only
        } else if (di > a.c.list_threshold) {
          if (K > 3 && (!my_arena || di > a.c.arena_dcap)) {
            if (lane == 0) set_err(a.c.lb.ctr, ERR_ARENA_OVERFLOW);
          } else {
            tc = list_task<K, M>(a.c, wsm, r, di, bb, ee, my_arena);
          }
        }
        cnt += tc;
        if (a.c.per_root) {
          const unsigned long long ts = warp_sum_u64(tc);
          if (lane == 0 && ts) atomicAdd(a.c.per_root + r, ts);
        }
        __syncwarp();
      }
      i0 = i1;
    }
    if (lane == 0) {
      if (donated) {
        lb_done(a.c.lb, 1);
      } else if (is_static) {
        // the block's last warp to finish its static chunk settles the whole block's
        atomicAdd(&blk_static_done, count);
        if (atomicAdd(&blk_warps_done, 1) == (int)(blockDim.x >> 5) - 1) {
          __threadfence_block();
          const int done = atomicAdd(&blk_static_done, 0);
          if (done) lb_done(a.c.lb, done);
        }
      } else {
        unflushed += count;
      }
    }
  }
  if (lane == 0 && unflushed) lb_done(a.c.lb, unflushed);
  if constexpr (MULTI) {
#pragma unroll
    for (int j = 3; j <= K; ++j) {
      const unsigned long long v = warp_sum_u64(acc.c[j]);
      if (lane == 0 && v) atomicAdd(&blk_k[j], v);
    }
    cnt = acc.c[K];
  }
  cnt = warp_sum_u64(cnt);
  if (lane == 0) {
    atomicAdd(&blk_sum[0], cnt);
    atomicAdd(&blk_sum[1], ntasks);
    atomicAdd(&blk_sum[2], idle[0]);
    atomicAdd(&blk_sum[3], idle[1]);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (blk_sum[0]) atomicAdd(&a.c.lb.ctr->count, blk_sum[0]);
    atomicAdd(&a.c.lb.ctr->tasks, blk_sum[1]);
    if (blk_sum[2]) atomicAdd(&a.c.lb.ctr->idle_polls, blk_sum[2]);
    if (blk_sum[3]) atomicAdd(&a.c.lb.ctr->hungry_ns, blk_sum[3]);
    if constexpr (MULTI) {
      for (int j = 3; j <= K; ++j)
        if (blk_k[j]) atomicAdd(&a.c.lb.ctr->count_k[j], blk_k[j]);
    }
  }
}

}  // namespace dmb
