// Motif counting kernel for sm_100a: connected induced k-vertex subgraphs (k = 3..7) per
// canonical class, one persistent launch over all roots. The enumeration itself (semantics,
// extension sets, bulk leaf counting, virtual warps, donation) is motif_run_task in
// motif.cuh; this file holds the single-graph kernel and its launcher.
#include <algorithm>
#include <climits>
#include <string>

#include "motif.cuh"

namespace dmb {

constexpr int MOTIF_WARPS = 8;

struct MotifArgs {
  MotifCtx c;                  // graph, LB, dictionary, arena layout
  const int32_t* roots;
  int n_roots;
  int n_classes;
  unsigned long long* hist;    // n_classes
  int2* arena;                 // per warp: 32/W group arenas of c.arena_stride int2
  uint32_t* bits;              // per warp: 32/W groups x 2 membership bitmaps of c.bit_words (or null)
  const int32_t* parts;        // optional per-root-entry part word (p | P << 16)
  int bits_smem;               // the bitmaps live in shared memory (zeroed at launch), not in `bits`
};

// Shared-memory budget of one block's membership bitmaps; larger graphs keep them in global
// memory.
constexpr size_t MOTIF_SMEM_BITS_MAX = 64 * 1024;

template <int K, int W>
__global__ void __launch_bounds__(32 * MOTIF_WARPS, 4) motif_kernel(const __grid_constant__ MotifArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  unsigned long long* bhist = reinterpret_cast<unsigned long long*>(smem);
  unsigned char* wbase = smem + sizeof(unsigned long long) * ((a.n_classes + 1) & ~1);
  const int lane = lane_id();
  const int wib = warp_in_block();
  MotifShared* ws = reinterpret_cast<MotifShared*>(wbase + motif_warp_smem<W>() * wib);
  MotifGroup* groups = reinterpret_cast<MotifGroup*>(ws + 1);
  const MotifCtx& c = a.c;
  const size_t warp_bit_words = (size_t)c.bit_words * 2 * (32 / W);
  uint32_t* sbits = reinterpret_cast<uint32_t*>(wbase + motif_warp_smem<W>() * MOTIF_WARPS);
  for (int cl = threadIdx.x; cl < a.n_classes; cl += blockDim.x) bhist[cl] = 0;
  if (a.bits_smem)
    for (size_t i = threadIdx.x; i < warp_bit_words * MOTIF_WARPS; i += blockDim.x) sbits[i] = 0u;
  __syncthreads();
  const size_t gw = (size_t)blockIdx.x * MOTIF_WARPS + wib;
  const int total_warps = gridDim.x * MOTIF_WARPS;
  int2* warp_arena = a.arena + gw * (size_t)c.arena_stride * (32 / W);
  uint32_t* warp_bits = a.bits_smem ? sbits + wib * warp_bit_words
                                    : (a.bits ? a.bits + gw * warp_bit_words : nullptr);
  unsigned long long ntasks = 0, nodes = 0;
  while (true) {
    int first = 0, count = 0, b = 0, e = -1, ok = 0, level = 0;
    int path[QPATH];
    for (int j = 0; j < QPATH; ++j) path[j] = 0;
    bool donated = false;
    if (lane == 0) ok = lb_next(c.lb, a.n_roots, total_warps, first, count, b, e, donated, level, path) ? 1 : 0;
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
        set_err(c.lb.ctr, ERR_BAD_TASK);
        lb_done(c.lb, count);
      }
      break;
    }
    for (int ti = 0; ti < count; ++ti) {
      const int v0 = donated ? first : __ldg(a.roots + first + ti);
      int bb = b, ee = e;
      if (!donated && a.parts) part_bounds(__ldg(a.parts + first + ti), bb, ee);
      ++ntasks;
      // block-level class counters, added to the global ones at exit
      motif_run_task<K, W>(c, bhist, ws, groups, warp_arena, warp_bits, v0, bb, ee, level, path, nodes);
    }
    if (lane == 0) lb_done(c.lb, count);
  }
  // every lane of a group counted the group's nodes: keep the leaders' counts
  nodes = warp_sum_u64((lane & (W - 1)) == 0 ? nodes : 0ull);
  if (lane == 0) {
    atomicAdd(&c.lb.ctr->tasks, ntasks);
    atomicAdd(&c.lb.ctr->nodes, nodes);
  }
  __syncthreads();
  for (int cl = threadIdx.x; cl < a.n_classes; cl += blockDim.x)
    if (bhist[cl]) atomicAdd(a.hist + cl, bhist[cl]);
}

size_t motif_arena_stride(int k, int maxdeg, int vwarp) {
  const int w = (vwarp == 8 || vwarp == 16) ? vwarp : 32;
  return motif_group_stride(k, maxdeg) * (size_t)(32 / w);
}

template <int K, int W>
static int launch_motif(MotifArgs a, LaunchCtx& ctx, int* grid_out) {
  const int block = 32 * MOTIF_WARPS;
  const size_t bits_bytes = (size_t)a.c.bit_words * 2 * (32 / W) * sizeof(uint32_t) * MOTIF_WARPS;
  a.bits_smem = a.bits && a.c.bit_words > 0 && bits_bytes <= MOTIF_SMEM_BITS_MAX ? 1 : 0;
  const size_t smem = sizeof(unsigned long long) * ((a.n_classes + 1) & ~1) +
                      motif_warp_smem<W>() * MOTIF_WARPS + (a.bits_smem ? bits_bytes : 0);
  auto kern = motif_kernel<K, W>;
  static LaunchCache cache;
  int occ = 0;
  DM_CUDA(cached_occupancy(cache, kern, ctx.device, block, smem, &occ));
  if (occ < 1) return fail(DM_EINVAL, "motif kernel does not fit on an SM");
  int grid = ctx.num_sms * occ;
  if (ctx.threads > 0) grid = std::max(1, std::min(grid, (ctx.threads + block - 1) / block));
  if (grid * MOTIF_WARPS > ctx.arena_warps) grid = std::max(1, ctx.arena_warps / MOTIF_WARPS);
  const int warps = grid * MOTIF_WARPS;
  a.c.lb.hungry_trigger = ctx.threshold >= 100 ? 0 : std::max(1, (ctx.threshold * warps + 99) / 100);
  kern<<<grid, block, smem, ctx.stream>>>(a);
  ctx.launches++;
  *grid_out = grid;
  DM_CUDA(cudaGetLastError());
  return DM_OK;
}

template <int K>
static int launch_motif_w(const MotifArgs& a, int vwarp, LaunchCtx& ctx, int* grid) {
  switch (vwarp) {
    case 8: return launch_motif<K, 8>(a, ctx, grid);
    case 16: return launch_motif<K, 16>(a, ctx, grid);
    default: return launch_motif<K, 32>(a, ctx, grid);
  }
}

int motif_launch(const MotifLaunch& L, LaunchCtx& ctx, int* grid) {
  MotifArgs a;
  a.c.g = L.g;
  a.c.lb = LBArgs{L.ctr, reinterpret_cast<QHeader*>(L.queue),
                  reinterpret_cast<QSlot*>(reinterpret_cast<char*>(L.queue) + sizeof(QHeader) * L.nq), L.qcap, 0,
                  L.max_donations, (long long)ctx.donate_after_us * 1000ll, (long long)ctx.timeout_ms * 1000000ll,
                  ctx.test_stall, 4, L.nq};
  a.c.q2c = L.q2c;
  a.c.maxdeg = L.maxdeg;
  a.c.arena_stride = (int)motif_group_stride(L.k, L.maxdeg);
  a.c.per_root = L.per_root;
  a.c.bit_base = 0;
  a.c.bit_words = L.bits ? L.bit_words : 0;
  a.bits = L.bits;
  a.roots = L.roots;
  a.n_roots = L.n_roots;
  a.n_classes = L.n_classes;
  a.hist = L.hist;
  a.arena = reinterpret_cast<int2*>(L.arena);
  a.parts = L.parts;
  a.bits_smem = 0;
  const int w = (L.vwarp == 8 || L.vwarp == 16) ? L.vwarp : 32;
  switch (L.k) {
    case 3: return launch_motif_w<3>(a, w, ctx, grid);
    case 4: return launch_motif_w<4>(a, w, ctx, grid);
    case 5: return launch_motif_w<5>(a, w, ctx, grid);
    case 6: return launch_motif_w<6>(a, w, ctx, grid);
    case 7: return launch_motif_w<7>(a, w, ctx, grid);
    default: return fail(DM_EINVAL, "motif k must be in [3, 7]");
  }
}

}  // namespace dmb
