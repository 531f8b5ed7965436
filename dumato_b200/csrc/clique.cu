// k-clique counting kernels for sm_100a.
//
// Semantics: the number of k-vertex cliques, each counted once, as the reference's clique
// driver computes (src/main/clique_PA.cu:9-32 with extend_clique, DuMatoGPU.cu:1194-1220:
// C_l = {u in N(v_l) : u > v_l} cap C_{l-1}, the leaf level adding |C_{k-2}|,
// aggregate_counter DuMatoGPU.cu:1769-1771). The reference breaks symmetry by vertex id on
// the undirected graph; here the graph is oriented by (degree, id) rank, which counts the
// same set of cliques with out-degrees bounded by O(sqrt(m)).
//
// Three execution modes, chosen per root by its out-degree d (all produce exact counts):
//   thread mode (d <= 128): the warp turns the root's out-neighbourhood into a local
//       adjacency bitmap in shared memory (row c = out-neighbours of the c-th neighbour,
//       as a d-bit set); each lane then runs its own DFS over 64-bit (or 128-bit) sets.
//       extend = AND of two rows, compact = nothing (bit order is the candidate order),
//       aggregate = popc at the last level.
//   warp mode (128 < d <= 2048): same local bitmap in global scratch, one 32-bit word per
//       lane (two for d > 1024), warp-cooperative DFS with ballot-based candidate pops.
//   list mode (any d): the reference's list structure - per-level sorted candidate lists in
//       a per-warp global arena, extended by binary-search intersection and ballot
//       compaction (DuMatoGPU.cu:317-328 write), the leaf level counted without writing.
#include <climits>
#include <cstdio>
#include <string>

#include "engine.hpp"
#include "gpm.cuh"

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

// Shared-memory bytes one warp needs in thread mode.
template <int NW>
__host__ __device__ constexpr size_t thread_warp_smem() {
  return sizeof(uint32_t) * (64 * NW) * (2 * NW) + sizeof(int32_t) * (2 * 64 * NW + 4);
}

// Builds the local adjacency bitmap of the root's out-neighbourhood L[0..d):
// bit j of row i is set iff L[j] is an out-neighbour of L[i]. The work is flattened over
// all (i, neighbour) pairs so a warp stays busy when rows are short; membership in L is a
// binary search in shared memory. Rows are zeroed by the caller.
__device__ __forceinline__ void build_local_rows(const GraphView& g, const int32_t* sL, const int32_t* sP, int d,
                                                 int total, uint32_t* rows, int row_words) {
  const int lane = lane_id();
  const int32_t maxL = sL[d - 1];
  for (int f = lane; f < total; f += 32) {
    int i = lower_bound(sP, 0, d + 1, f + 1) - 1;  // largest i with sP[i] <= f
    const int u = sL[i];
    const int32_t x = __ldg(g.adj + __ldg(g.row + u) + (f - sP[i]));
    if (x <= maxL) {
      int j = lower_bound(sL, i + 1, d, x);
      if (j < d && sL[j] == x) {
        uint32_t* w = rows + (size_t)i * row_words + (j >> 5);
        atomicOr(w, 1u << (j & 31));
      }
    }
  }
}

// Loads L = N+(root) into shared memory and the exclusive prefix sum of the out-degrees
// of its members (sP[0..d]). Returns the total.
__device__ __forceinline__ int load_root_list(const GraphView& g, int root, int d, int32_t* sL, int32_t* sP) {
  const int lane = lane_id();
  const int32_t* L = g.adj + __ldg(g.row + root);
  int carry = 0;
  for (int i0 = 0; i0 < d; i0 += 32) {
    const int i = i0 + lane;
    int u = 0, du = 0;
    if (i < d) {
      u = __ldg(L + i);
      du = __ldg(g.deg + u);
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

template <int K, int NW>
__global__ void __launch_bounds__(256) clique_thread_kernel(GraphView g, const int32_t* __restrict__ tasks,
                                                            int n_tasks, DevCounters* ctr, int slot) {
  constexpr int DCAP = 64 * NW;
  constexpr int RW = 2 * NW;
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = lane_id();
  unsigned char* base = smem + thread_warp_smem<NW>() * warp_in_block();
  uint32_t* rows = reinterpret_cast<uint32_t*>(base);
  int32_t* sL = reinterpret_cast<int32_t*>(rows + DCAP * RW);
  int32_t* sP = sL + DCAP;
  int* sNext = sP + DCAP + 1;
  unsigned long long cnt = 0, ntasks = 0;
  while (true) {
    int t = 0;
    if (lane == 0) t = atomicAdd(&ctr->cursor[slot], 1);
    t = __shfl_sync(FULL_MASK, t, 0);
    if (t >= n_tasks) break;
    ++ntasks;
    const int root = __ldg(tasks + t);
    const int d = __ldg(g.deg + root);
    if constexpr (K == 2) {
      if (lane == 0) cnt += (unsigned long long)d;
      continue;
    }
    for (int i = lane; i < d * RW; i += 32) rows[i] = 0;
    const int total = load_root_list(g, root, d, sL, sP);
    if (lane == 0) *sNext = 32;
    build_local_rows(g, sL, sP, d, total, rows, RW);
    __syncwarp();
    const uint64_t* rows64 = reinterpret_cast<const uint64_t*>(rows);
    int c1 = lane;
    while (c1 < d) {
      Bits<NW> S;
#pragma unroll
      for (int j = 0; j < NW; ++j) S.w[j] = rows64[c1 * NW + j];
      if (K == 3) cnt += (unsigned long long)popc(S);
      else if (popc(S) >= K - 3) cnt += count_rec<(K >= 4 ? K - 3 : 0), NW>(S, rows64);
      c1 = atomicAdd(sNext, 1);
    }
    __syncwarp();
  }
  cnt = warp_sum_u64(cnt);
  if (lane == 0) {
    atomicAdd(&ctr->count, cnt);
    atomicAdd(&ctr->tasks, ntasks);
  }
}

// ---------------- warp mode ----------------

// Number of (D+1)-cliques inside a warp-distributed set (lane holds words lane, lane+32).
template <int D>
__device__ __forceinline__ unsigned long long wcount(uint32_t a, uint32_t b, const uint32_t* __restrict__ rows,
                                                     int W) {
  const int lane = lane_id();
  if constexpr (D == 0) {
    return (unsigned long long)(__popc(a) + __popc(b));
  } else {
    unsigned long long sum = 0;
    while (true) {
      unsigned nz = __ballot_sync(FULL_MASK, a != 0);
      int c;
      if (nz) {
        const int owner = __ffs(nz) - 1;
        int bit = 0;
        if (lane == owner) {
          bit = __ffs(a) - 1;
          a &= a - 1;
        }
        c = owner * 32 + __shfl_sync(FULL_MASK, bit, owner);
      } else {
        unsigned nz2 = __ballot_sync(FULL_MASK, b != 0);
        if (!nz2) break;
        const int owner = __ffs(nz2) - 1;
        int bit = 0;
        if (lane == owner) {
          bit = __ffs(b) - 1;
          b &= b - 1;
        }
        c = (owner + 32) * 32 + __shfl_sync(FULL_MASK, bit, owner);
      }
      const uint32_t* rc = rows + (size_t)c * W;
      const uint32_t ta = a & (lane < W ? __ldcg(rc + lane) : 0u);
      const uint32_t tb = b & (lane + 32 < W ? __ldcg(rc + lane + 32) : 0u);
      if constexpr (D == 1) {
        sum += (unsigned long long)(__popc(ta) + __popc(tb));
      } else {
        if (__any_sync(FULL_MASK, (ta | tb) != 0)) sum += wcount<D - 1>(ta, tb, rows, W);
      }
    }
    return sum;
  }
}

constexpr int WARP_MODE_DMAX = 2048;
constexpr int WARP_MODE_WARPS = 4;  // warps per block

template <int K>
__global__ void __launch_bounds__(32 * WARP_MODE_WARPS) clique_warp_kernel(GraphView g, const int32_t* __restrict__ tasks,
                                                                          int n_tasks, DevCounters* ctr, int slot,
                                                                          uint32_t* scratch, int dcap) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = lane_id();
  const int wib = warp_in_block();
  int32_t* sL = reinterpret_cast<int32_t*>(smem) + (size_t)wib * (2 * WARP_MODE_DMAX + 4);
  int32_t* sP = sL + WARP_MODE_DMAX;
  const size_t gw = (size_t)blockIdx.x * WARP_MODE_WARPS + wib;
  const int Wmax = (dcap + 31) / 32;
  uint32_t* rows = scratch + gw * (size_t)dcap * Wmax;
  unsigned long long cnt = 0, ntasks = 0;
  while (true) {
    int t = 0;
    if (lane == 0) t = atomicAdd(&ctr->cursor[slot], 1);
    t = __shfl_sync(FULL_MASK, t, 0);
    if (t >= n_tasks) break;
    ++ntasks;
    const int root = __ldg(tasks + t);
    const int d = __ldg(g.deg + root);
    if (d > dcap || d > WARP_MODE_DMAX) {
      if (lane == 0) atomicCAS(&ctr->err, 0, ERR_BAD_TASK);
      continue;
    }
    const int W = (d + 31) / 32;
    for (int i = lane; i < d * W; i += 32) rows[i] = 0;
    const int total = load_root_list(g, root, d, sL, sP);
    __syncwarp();
    __threadfence_block();
    build_local_rows(g, sL, sP, d, total, rows, W);
    __syncwarp();
    __threadfence_block();
    for (int c1 = 0; c1 < d; ++c1) {
      const uint32_t* rc = rows + (size_t)c1 * W;
      uint32_t a = lane < W ? __ldcg(rc + lane) : 0u;
      uint32_t b = lane + 32 < W ? __ldcg(rc + lane + 32) : 0u;
      if (K == 3) cnt += (unsigned long long)(__popc(a) + __popc(b));
      else if (__any_sync(FULL_MASK, (a | b) != 0)) cnt += wcount<(K >= 4 ? K - 3 : 0)>(a, b, rows, W);
    }
    __syncwarp();
  }
  cnt = warp_sum_u64(cnt);
  if (lane == 0) {
    atomicAdd(&ctr->count, cnt);
    atomicAdd(&ctr->tasks, ntasks);
  }
}

// ---------------- list mode ----------------

constexpr int LIST_WARPS = 8;

template <int K>
__global__ void __launch_bounds__(32 * LIST_WARPS) clique_list_kernel(GraphView g, const int32_t* __restrict__ tasks,
                                                                     int n_tasks, DevCounters* ctr, int slot,
                                                                     int32_t* arena, int dcap) {
  __shared__ const int32_t* sPtr[LIST_WARPS][K];
  __shared__ int sN[LIST_WARPS][K];
  __shared__ int sPos[LIST_WARPS][K];
  const int lane = lane_id();
  const int wib = warp_in_block();
  const size_t gw = (size_t)blockIdx.x * LIST_WARPS + wib;
  int32_t* my = arena + gw * (size_t)K * dcap;
  unsigned long long cnt = 0, ntasks = 0, nodes = 0;
  while (true) {
    int t = 0;
    if (lane == 0) t = atomicAdd(&ctr->cursor[slot], 1);
    t = __shfl_sync(FULL_MASK, t, 0);
    if (t >= n_tasks) break;
    ++ntasks;
    const int root = __ldg(tasks + t);
    const int d = __ldg(g.deg + root);
    if (K == 2) {
      if (lane == 0) cnt += (unsigned long long)d;
      continue;
    }
    if (d > dcap) {
      if (lane == 0) atomicCAS(&ctr->err, 0, ERR_ARENA_OVERFLOW);
      continue;
    }
    if (lane == 0) {
      sPtr[wib][0] = g.adj + g.row[root];
      sN[wib][0] = d;
      sPos[wib][0] = 0;
    }
    __syncwarp();
    int lvl = 0;
    while (lvl >= 0) {
      const int pos = sPos[wib][lvl];
      const int rem = sN[wib][lvl] - pos;
      if (rem - 1 < K - 2 - lvl) {
        --lvl;
        continue;
      }
      const int32_t* P = sPtr[wib][lvl];
      const int c = P[pos];
      __syncwarp();
      if (lane == 0) sPos[wib][lvl] = pos + 1;
      // extend: candidates after c intersected with N+(c)
      const int32_t* A = P + pos + 1;
      const int na = rem - 1;
      const int32_t* B = g.adj + __ldg(g.row + c);
      const int nb = __ldg(g.deg + c);
      ++nodes;
      if (lvl + 1 == K - 2) {
        unsigned s = 0;
        for (int i = lane; i < na; i += 32) s += contains(B, nb, A[i]) ? 1u : 0u;
        cnt += s;
      } else {
        int32_t* out = my + (size_t)(lvl + 1) * dcap;
        int m = 0;
        for (int i0 = 0; i0 < na; i0 += 32) {
          const int i = i0 + lane;
          const int32_t x = i < na ? A[i] : 0;
          const bool ok = i < na && contains(B, nb, x);
          m += compact(out, m, x, ok);
        }
        __syncwarp();
        ++lvl;
        if (lane == 0) {
          sPtr[wib][lvl] = out;
          sN[wib][lvl] = m;
          sPos[wib][lvl] = 0;
        }
      }
      __syncwarp();
    }
  }
  cnt = warp_sum_u64(cnt);
  if (lane == 0) {
    atomicAdd(&ctr->count, cnt);
    atomicAdd(&ctr->tasks, ntasks);
    atomicAdd(&ctr->nodes, nodes);
  }
}

// ---------------- host launchers ----------------

template <typename Kern>
static int grid_for(Kern kern, int block, size_t smem, const LaunchCtx& ctx, int* grid) {
  int occ = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, block, smem);
  if (e != cudaSuccess) return fail(DM_ECUDA, std::string("occupancy query failed: ") + cudaGetErrorString(e));
  if (occ < 1) return fail(DM_EINVAL, "kernel does not fit on an SM with the requested block size");
  *grid = ctx.num_sms * occ;
  if (ctx.threads > 0 && ctx.block > 0) {
    // the reference's (threads, blockSize) pair maps onto the persistent grid
    int want = (ctx.threads + block - 1) / block;
    *grid = want < 1 ? 1 : want;
  }
  return DM_OK;
}

template <int K, int NW>
static int launch_thread(const GraphView& g, const int32_t* tasks, int n, DevCounters* ctr, int slot, LaunchCtx& ctx) {
  if (n == 0) return DM_OK;
  const int block = 256;
  const size_t smem = thread_warp_smem<NW>() * (block / 32);
  auto kern = clique_thread_kernel<K, NW>;
  if (smem > 48 * 1024) DM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int grid = 0;
  int rc = grid_for(kern, block, smem, ctx, &grid);
  if (rc) return rc;
  kern<<<grid, block, smem, ctx.stream>>>(g, tasks, n, ctr, slot);
  ctx.launches++;
  DM_CUDA(cudaGetLastError());
  return DM_OK;
}

template <int K>
static int launch_warp(const GraphView& g, const int32_t* tasks, int n, DevCounters* ctr, int slot, LaunchCtx& ctx,
                       void* scratch, size_t bytes, int dcap) {
  if (n == 0) return DM_OK;
  const int block = 32 * WARP_MODE_WARPS;
  auto kern = clique_warp_kernel<K>;
  const size_t smem = sizeof(int32_t) * (2 * WARP_MODE_DMAX + 4) * WARP_MODE_WARPS;
  DM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int grid = 0;
  int rc = grid_for(kern, block, smem, ctx, &grid);
  if (rc) return rc;
  const size_t per_warp = (size_t)dcap * ((dcap + 31) / 32) * sizeof(uint32_t);
  const size_t max_warps = bytes / per_warp;
  if ((size_t)grid * WARP_MODE_WARPS > max_warps) grid = (int)(max_warps / WARP_MODE_WARPS);
  if (grid < 1) return fail(DM_ENOMEM, "warp-mode scratch too small");
  kern<<<grid, block, smem, ctx.stream>>>(g, tasks, n, ctr, slot, reinterpret_cast<uint32_t*>(scratch), dcap);
  ctx.launches++;
  DM_CUDA(cudaGetLastError());
  return DM_OK;
}

template <int K>
static int launch_list(const GraphView& g, const int32_t* tasks, int n, DevCounters* ctr, int slot, LaunchCtx& ctx,
                       void* scratch, size_t bytes, int dcap) {
  if (n == 0) return DM_OK;
  const int block = 32 * LIST_WARPS;
  auto kern = clique_list_kernel<K>;
  int grid = 0;
  int rc = grid_for(kern, block, 0, ctx, &grid);
  if (rc) return rc;
  const size_t per_warp = (size_t)K * dcap * sizeof(int32_t);
  const size_t max_warps = bytes / per_warp;
  if ((size_t)grid * LIST_WARPS > max_warps) grid = (int)(max_warps / LIST_WARPS);
  if (grid < 1) return fail(DM_ENOMEM, "list-mode arena too small");
  kern<<<grid, block, 0, ctx.stream>>>(g, tasks, n, ctr, slot, reinterpret_cast<int32_t*>(scratch), dcap);
  ctx.launches++;
  DM_CUDA(cudaGetLastError());
  return DM_OK;
}

static size_t list_bytes(const CliqueTasks& t, int k, const LaunchCtx& ctx) {
  if (!t.n_list) return 0;
  size_t warps = (size_t)ctx.num_sms * 8 * LIST_WARPS;
  return warps * (size_t)k * (t.max_list_deg + 4) * sizeof(int32_t);
}

static size_t warp_bytes(const CliqueTasks& t, const LaunchCtx& ctx) {
  if (!t.n_warp) return 0;
  const int dcap = t.max_warp_deg;
  size_t per_warp = (size_t)dcap * ((dcap + 31) / 32) * sizeof(uint32_t);
  size_t warps = (size_t)ctx.num_sms * 4 * WARP_MODE_WARPS;
  return warps * per_warp;
}

size_t clique_scratch_bytes(const CliqueTasks& t, int k, const LaunchCtx& ctx) {
  size_t a = list_bytes(t, k, ctx), b = warp_bytes(t, ctx);
  return a > b ? a : b;
}

template <int K>
static int run_k(const GraphView& g, const CliqueTasks& t, DevCounters* ctr, LaunchCtx& ctx, void* scratch,
                 size_t bytes) {
  int rc = DM_OK;
  // heaviest first: list roots, warp-mode roots, then the bulk in thread mode
  if (!rc) rc = launch_list<K>(g, t.d_list, t.n_list, ctr, 0, ctx, scratch, bytes, t.max_list_deg + 4);
  if (!rc) rc = launch_warp<K>(g, t.d_warp, t.n_warp, ctr, 1, ctx, scratch, bytes, t.max_warp_deg);
  if (!rc) rc = launch_thread<K, 2>(g, t.d_thread2, t.n_thread2, ctr, 2, ctx);
  if (!rc) rc = launch_thread<K, 1>(g, t.d_thread1, t.n_thread1, ctr, 3, ctx);
  return rc;
}

int clique_launch(const GraphView& g, int k, const CliqueTasks& t, DevCounters* ctr, LaunchCtx& ctx, void* scratch,
                  size_t bytes, dm_stats* st) {
  (void)st;
  switch (k) {
    case 2: return run_k<2>(g, t, ctr, ctx, scratch, bytes);
    case 3: return run_k<3>(g, t, ctr, ctx, scratch, bytes);
    case 4: return run_k<4>(g, t, ctr, ctx, scratch, bytes);
    case 5: return run_k<5>(g, t, ctr, ctx, scratch, bytes);
    case 6: return run_k<6>(g, t, ctr, ctx, scratch, bytes);
    case 7: return run_k<7>(g, t, ctr, ctx, scratch, bytes);
    case 8: return run_k<8>(g, t, ctr, ctx, scratch, bytes);
    case 9: return run_k<9>(g, t, ctr, ctx, scratch, bytes);
    case 10: return run_k<10>(g, t, ctr, ctx, scratch, bytes);
    case 11: return run_k<11>(g, t, ctr, ctx, scratch, bytes);
    case 12: return run_k<12>(g, t, ctr, ctx, scratch, bytes);
    default: return fail(DM_EINVAL, "k must be in [2, 12]");
  }
}

}  // namespace dmb
