// Batched mining: many (graph, query) pairs in one persistent launch.
//
// The graphs are laid out as one disjoint union in HBM: query q's graph occupies global
// vertex ids [vbase[q], vbase[q+1]), its rows hold global ids, and each query keeps the
// representation its path needs (clique queries: the degree-ordered DAG in rank space;
// motif queries: the undirected sorted CSR). The task list is every query's roots, ordered
// by a per-root cost estimate across the whole batch, so the heavy roots of all queries
// start first. A task (or a donated range or DFS prefix) is just a global vertex id, so the
// load balancer of the single-graph kernels (lb.cuh) works unchanged: the warp that takes
// a task finds its query by binary search over vbase and runs the query's path from its
// descriptor (clique bitmap/list tasks from clique.cuh, motif tasks with the query's
// virtual-warp width from motif.cuh), with the query's donation trigger.
//
// The launch (counter reset, output clear, the kernel and the read-back of results and
// counters) is captured once into a CUDA graph; dm_batch_run replays it.
//
// Autotuning chooses per query: the virtual-warp width of motif queries (8/16/32), the
// donation threshold, and list vs bitmap intersection for cliques - from a cost model of
// the graph, or by timing each candidate on the query alone.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "clique.cuh"
#include "motif.cuh"

namespace dmb {

struct BatchQuery {
  int kind, k, vbase, nv;
  int trigger;          // hungry_trigger for this query's donations (0 = never donate)
  int list_threshold;   // cliques: roots with out-degree above this take the list path
  int vwarp;            // motifs: virtual-warp width
  int maxdeg;           // degree bound of the query's rows (arena layout)
  int arena_stride;     // motifs: int2 slots per group
  int arena_dcap;       // cliques: list capacity per level
  int n_classes;
  int bit_words;        // motifs: membership bitmap words (0 = none)
  const int32_t* q2c;   // motifs: quick code -> class
  unsigned long long* out;  // count (cliques) or class counters (motifs)
  // the task contexts of this query, built on the host: the kernel passes references into
  // this table, so no per-task copy of the load-balancer arguments lands in local memory
  CliqueArgs cargs;
  MotifCtx mctx;
};

struct BatchArgs {
  GraphView g;                 // union graph
  const int32_t* roots;
  int n_roots;
  LBArgs lb;                   // hungry_trigger / min_split are set per task from the query
  const BatchQuery* queries;
  const int32_t* vbase;        // n_queries + 1, ascending
  int n_queries;
  unsigned char* arena;
  size_t arena_bytes;          // per warp
  uint32_t* bits;              // motif membership bitmaps (zero between runs), or null
  size_t bits_words;           // per warp
};

constexpr int BATCH_WARPS = 8;
constexpr int BATCH_CLIQUE_KMAX = 6;
constexpr int BATCH_MOTIF_KMAX = 5;
// bitmap rows of up to 2 words: clique roots with out-degree up to 128 take the bitmap path,
// larger ones the list path. The per-warp shared memory then stays small enough for four
// blocks per SM (the motif paths, which dominate mixed batches, are latency-bound and want
// the resident warps).
constexpr int BATCH_M = 2;

template <int M>
__host__ __device__ constexpr size_t batch_warp_smem() {
  const size_t a = (size_t)warp_layout(M).total, b = motif_warp_smem<8>();
  return ((a > b ? a : b) + 15) / 16 * 16;
}

// The query whose vertex range holds v: the last q with vbase[q] <= v.
__device__ __forceinline__ int batch_find_query(const int32_t* vbase, int n, int v) {
  int lo = 0, hi = n;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(vbase + mid) <= v) lo = mid; else hi = mid;
  }
  return lo;
}

template <int K, int M>
__device__ unsigned long long batch_clique(const BatchArgs& a, const BatchQuery& q, unsigned char* wsm,
                                           int32_t* arena, int root, int b, int e) {
  return clique_task<K, M>(q.cargs, wsm, root, b, e, arena);
}

template <int K, int W>
__device__ void batch_motif(const BatchArgs& a, const BatchQuery& q, unsigned char* wsm, int2* arena,
                            uint32_t* bits, int v0, int b, int e, int level, const int* path,
                            unsigned long long& nodes) {
  MotifShared* ws = reinterpret_cast<MotifShared*>(wsm);
  MotifGroup* groups = reinterpret_cast<MotifGroup*>(ws + 1);
  unsigned long long tn = 0;
  motif_run_task<K, W>(q.mctx, q.out, ws, groups, arena, bits, v0, b, e, level, path, tn);
  // every lane of a group counted the group's nodes: keep the leaders' counts
  if ((lane_id() & (W - 1)) == 0) nodes += tn;
}

template <int K>
__device__ void batch_motif_w(const BatchArgs& a, const BatchQuery& q, unsigned char* wsm, int2* arena,
                              uint32_t* bits, int v0, int b, int e, int level, const int* path,
                              unsigned long long& nodes) {
  if (q.vwarp == 8) batch_motif<K, 8>(a, q, wsm, arena, bits, v0, b, e, level, path, nodes);
  else if (q.vwarp == 16) batch_motif<K, 16>(a, q, wsm, arena, bits, v0, b, e, level, path, nodes);
  else batch_motif<K, 32>(a, q, wsm, arena, bits, v0, b, e, level, path, nodes);
}

__global__ void batch_reset(DevCounters* c, int n_roots) {
  int* w = reinterpret_cast<int*>(c);
  for (int i = threadIdx.x; i < (int)(sizeof(DevCounters) / sizeof(int)); i += blockDim.x) w[i] = 0;
  __syncthreads();
  if (threadIdx.x == 0) c->pending = n_roots;
}

template <int M>
__global__ void __launch_bounds__(32 * BATCH_WARPS, 4) batch_kernel(const __grid_constant__ BatchArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = lane_id();
  const int wib = warp_in_block();
  unsigned char* wsm = smem + batch_warp_smem<M>() * wib;
  const size_t gw = (size_t)blockIdx.x * BATCH_WARPS + wib;
  const int total_warps = gridDim.x * BATCH_WARPS;
  unsigned char* warp_arena = a.arena + gw * a.arena_bytes;
  uint32_t* warp_bits = a.bits ? a.bits + gw * a.bits_words : nullptr;
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
    for (int j = 0; j < BATCH_MOTIF_KMAX - 3; ++j) path[j] = __shfl_sync(FULL_MASK, path[j], 0);
    donated = __shfl_sync(FULL_MASK, donated ? 1 : 0, 0) != 0;
    for (int ti = 0; ti < count; ++ti) {
      const int root = donated ? first : __ldg(a.roots + first + ti);
      ++ntasks;
      const BatchQuery& q = a.queries[batch_find_query(a.vbase, a.n_queries, root)];
      const int kind = q.kind, k = q.k;
      if (kind == DM_QUERY_CLIQUE) {
        unsigned long long c = 0;
        int32_t* arena = reinterpret_cast<int32_t*>(warp_arena);
        if (level != 0) {
          if (lane == 0) set_err(a.lb.ctr, ERR_BAD_TASK);
        } else {
          switch (k) {
            case 2: c = batch_clique<2, M>(a, q, wsm, arena, root, b, e); break;
            case 3: c = batch_clique<3, M>(a, q, wsm, arena, root, b, e); break;
            case 4: c = batch_clique<4, M>(a, q, wsm, arena, root, b, e); break;
            case 5: c = batch_clique<5, M>(a, q, wsm, arena, root, b, e); break;
            case 6: c = batch_clique<6, M>(a, q, wsm, arena, root, b, e); break;
            default:
              if (lane == 0) set_err(a.lb.ctr, ERR_BAD_TASK);
          }
        }
        c = warp_sum_u64(c);
        if (lane == 0 && c) atomicAdd(q.out, c);
        __syncwarp();
      } else {
        int2* arena = reinterpret_cast<int2*>(warp_arena);
        if (level < 0 || level > k - 3) {
          if (lane == 0) set_err(a.lb.ctr, ERR_BAD_TASK);
        } else {
          switch (k) {
            case 3: batch_motif_w<3>(a, q, wsm, arena, warp_bits, root, b, e, level, path, nodes); break;
            case 4: batch_motif_w<4>(a, q, wsm, arena, warp_bits, root, b, e, level, path, nodes); break;
            case 5: batch_motif_w<5>(a, q, wsm, arena, warp_bits, root, b, e, level, path, nodes); break;
            default:
              if (lane == 0) set_err(a.lb.ctr, ERR_BAD_TASK);
          }
        }
        __syncwarp();
      }
    }
    if (lane == 0) lb_done(a.lb, count);
  }
  nodes = warp_sum_u64(nodes);
  if (lane == 0) {
    atomicAdd(&a.lb.ctr->tasks, ntasks);
    atomicAdd(&a.lb.ctr->nodes, nodes);
  }
}

template <int M>
static int batch_configure(int num_sms, int threads, int* grid_out, size_t* smem_out) {
  const size_t smem = batch_warp_smem<M>() * BATCH_WARPS;
  auto kern = batch_kernel<M>;
  DM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int occ = 0;
  DM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, 32 * BATCH_WARPS, smem));
  if (occ < 1) return fail(DM_EINVAL, "batch kernel does not fit on an SM");
  int grid = num_sms * occ;
  if (threads > 0) grid = std::max(1, std::min(grid, (threads + 32 * BATCH_WARPS - 1) / (32 * BATCH_WARPS)));
  *grid_out = grid;
  *smem_out = smem;
  return DM_OK;
}

template <int M>
static int batch_launch(const BatchArgs& a, int grid, size_t smem, cudaStream_t st) {
  batch_kernel<M><<<grid, 32 * BATCH_WARPS, smem, st>>>(a);
  DM_CUDA(cudaGetLastError());
  return DM_OK;
}

}  // namespace dmb

using namespace dmb;

struct dm_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  int num_sms = 0;
  int n_queries = 0;
  std::vector<dm_query_tuning> tuning;
  int64_t n_results = 0;
  int n_roots = 0;
  int grid = 0;
  size_t smem = 0;
  // device
  int32_t *d_row = nullptr, *d_deg = nullptr, *d_adj = nullptr;
  int32_t* d_roots = nullptr;
  int32_t* d_vbase = nullptr;
  BatchQuery* d_desc = nullptr;
  unsigned long long* d_out = nullptr;
  DevCounters* d_ctr = nullptr;
  void* d_queue = nullptr;
  unsigned char* d_arena = nullptr;
  uint32_t* d_bits = nullptr;
  size_t bits_bytes = 0;
  std::map<uint64_t, int32_t*> d_q2c;  // per dictionary uid
  unsigned long long* h_out = nullptr;  // pinned
  DevCounters* h_ctr = nullptr;         // pinned
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  BatchArgs args{};
};

namespace {

void batch_release(dm_batch* b) {
  if (!b) return;
  int cur = 0;
  if (cudaGetDevice(&cur) == cudaSuccess) {
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    cudaFree(b->d_row);
    cudaFree(b->d_deg);
    cudaFree(b->d_adj);
    cudaFree(b->d_roots);
    cudaFree(b->d_vbase);
    cudaFree(b->d_desc);
    cudaFree(b->d_out);
    cudaFree(b->d_ctr);
    cudaFree(b->d_queue);
    cudaFree(b->d_arena);
    cudaFree(b->d_bits);
    for (auto& kv : b->d_q2c) cudaFree(kv.second);
    if (b->h_out) cudaFreeHost(b->h_out);
    if (b->h_ctr) cudaFreeHost(b->h_ctr);
    if (b->e0) cudaEventDestroy(b->e0);
    if (b->e1) cudaEventDestroy(b->e1);
    if (b->stream) cudaStreamDestroy(b->stream);
    cudaSetDevice(cur);
  }
  cudaGetLastError();
  delete b;
}

// Per-root cost estimates of the cost model (arbitrary units, comparable across queries):
// a clique root with out-degree d costs about d^(k-2) set operations of length d; a motif
// root v0 with u members above it and degree g about u * g^(k-2).
double clique_root_cost(int d, int k) { return std::pow((double)d + 1.0, (double)std::max(1, k - 2)) * (d + 1.0); }
double motif_root_cost(int up, int deg, int k) { return (double)up * std::pow((double)deg + 1.0, (double)(k - 2)); }

int upper_count(const dm_graph* g, int32_t v) {
  const int32_t* s = g->adj.data() + g->row[v];
  const int32_t* e = g->adj.data() + g->row[v + 1];
  return (int)(e - std::upper_bound(s, e, v));
}

// Times one candidate setting of a query alone (kernel time of its single-graph launch).
int time_candidate(const dm_query& q, const dm_opts& base, int vwarp, int threshold, int mode, double* ms) {
  dm_opts o = base;
  o.vwarp = vwarp;
  o.threshold = threshold;
  o.mode = mode;
  dm_stats st;
  double best = 1e300;
  for (int rep = 0; rep < 2; ++rep) {  // the first run also uploads the graph
    int rc;
    if (q.kind == DM_QUERY_CLIQUE) {
      uint64_t c = 0;
      rc = dm_count_cliques(q.graph, q.k, &o, &c, &st);
    } else {
      std::vector<uint64_t> h((size_t)q.dict->n_classes);
      rc = dm_count_motifs(q.graph, q.k, q.dict, &o, h.data(), &st);
    }
    if (rc) return rc;
    if (rep > 0) best = std::min(best, st.kernel_ms);
  }
  *ms = best;
  return DM_OK;
}

int fail_release(dm_batch* b, int rc) {
  batch_release(b);
  return rc;
}

}  // namespace

extern "C" {

int dm_batch_create(const dm_query* queries, int32_t n, const dm_opts* opts, int32_t autotune, dm_batch** out) {
  if (!out || n < 0 || (n > 0 && !queries)) return fail(DM_EINVAL, "dm_batch_create: bad arguments");
  if (autotune != DM_AUTOTUNE_MODEL && autotune != DM_AUTOTUNE_MEASURE)
    return fail(DM_EINVAL, "dm_batch_create: autotune must be DM_AUTOTUNE_MODEL or DM_AUTOTUNE_MEASURE");
  *out = nullptr;
  int rc = check_opts(opts);
  if (rc) return rc;
  for (int32_t i = 0; i < n; ++i) {
    const dm_query& q = queries[i];
    const std::string at = " (query " + std::to_string(i) + ")";
    if (!q.graph) return fail(DM_EINVAL, "dm_batch_create: no graph" + at);
    if (q.kind == DM_QUERY_CLIQUE) {
      if (q.k < 2 || q.k > BATCH_CLIQUE_KMAX) return fail(DM_EINVAL, "dm_batch_create: clique k must be in [2, 6]" + at);
    } else if (q.kind == DM_QUERY_MOTIF) {
      if (q.k < 3 || q.k > BATCH_MOTIF_KMAX) return fail(DM_EINVAL, "dm_batch_create: motif k must be in [3, 5]" + at);
      if (!q.dict || q.dict->k != q.k) return fail(DM_EINVAL, "dm_batch_create: a motif query needs the k-vertex dictionary" + at);
    } else {
      return fail(DM_EINVAL, "dm_batch_create: unknown query kind" + at);
    }
    if (q.vwarp != 0 && q.vwarp != 8 && q.vwarp != 16 && q.vwarp != 32)
      return fail(DM_EINVAL, "dm_batch_create: vwarp must be 0, 8, 16 or 32" + at);
    if (q.mode < 0 || q.mode > 2) return fail(DM_EINVAL, "dm_batch_create: mode out of range" + at);
  }
  LaunchCtx ctx;
  if ((rc = select_device(opts, ctx))) return rc;
  dm_opts base{};
  if (opts) base = *opts;
  base.struct_size = sizeof(dm_opts);
  base.device = ctx.device;
  base.stream = 0;
  base.scheduler = DM_SCHED_PLAIN;
  base.world_size = 0;
  base.subtree_counts = nullptr;
  base.predictor = nullptr;

  auto* b = new dm_batch;
  b->device = ctx.device;
  b->num_sms = ctx.num_sms;
  b->n_queries = n;
  b->tuning.assign((size_t)n, dm_query_tuning{});
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
    b->stream = nullptr;
    return fail_release(b, fail(DM_ECUDA, "dm_batch_create: cannot create a stream"));
  }

  // ---- host layout of the union graph, roots and descriptors ----
  std::vector<int32_t> vbase((size_t)n + 1, 0);
  std::vector<int32_t> hrow, pdeg, padj;
  std::vector<std::pair<double, int32_t>> roots;  // (cost, global id)
  std::vector<BatchQuery> desc((size_t)n);
  std::vector<double> qcost((size_t)n, 0.0);
  int64_t total_v = 0;
  for (int32_t i = 0; i < n; ++i) {
    const dm_query& q = queries[i];
    dm_graph* g = q.graph;
    std::lock_guard<std::mutex> lk(g->mu);
    if (total_v + g->n >= INT32_MAX)
      return fail_release(b, fail(DM_EOVERFLOW, "dm_batch_create: the union graph exceeds 32-bit vertex ids"));
    vbase[i] = (int32_t)total_v;
    const bool clique = q.kind == DM_QUERY_CLIQUE;
    if (clique) ensure_oriented(g);
    const std::vector<int64_t>& row = clique ? g->orow : g->row;
    const std::vector<int32_t>& adj = clique ? g->oadj : g->adj;
    int maxd = 0;
    for (int32_t v = 0; v < g->n; ++v) {
      const int64_t d = row[v + 1] - row[v];
      maxd = std::max<int>(maxd, (int)d);
      if ((int64_t)padj.size() + d + 4 >= (int64_t)INT32_MAX)
        return fail_release(b, fail(DM_EOVERFLOW, "dm_batch_create: the union adjacency exceeds 32-bit offsets"));
      // rows start on 16-byte boundaries and are padded with INT32_MAX
      hrow.push_back((int32_t)padj.size());
      pdeg.push_back((int32_t)d);
      for (int64_t e = row[v]; e < row[v + 1]; ++e) padj.push_back(adj[e] + (int32_t)total_v);
      while (padj.size() % 4) padj.push_back(INT32_MAX);
      double c = 0;
      if (clique) {
        if (d >= q.k - 1) {
          c = clique_root_cost((int)d, q.k);
          roots.emplace_back(c, (int32_t)(total_v + v));
        }
      } else {
        const int up = upper_count(g, v);
        if (up > 0) {
          c = motif_root_cost(up, (int)d, q.k);
          roots.emplace_back(c, (int32_t)(total_v + v));
        }
      }
      qcost[i] += c;
    }
    BatchQuery& d = desc[i];
    std::memset(&d, 0, sizeof(d));
    d.kind = q.kind;
    d.k = q.k;
    d.vbase = (int32_t)total_v;
    d.nv = g->n;
    d.maxdeg = std::max(maxd, 1);
    d.n_classes = clique ? 1 : q.dict->n_classes;
    total_v += g->n;
  }
  vbase[n] = (int32_t)total_v;

  // ---- autotuning ----
  int64_t off = 0;
  for (int32_t i = 0; i < n; ++i) {
    const dm_query& q = queries[i];
    BatchQuery& d = desc[i];
    dm_query_tuning& t = b->tuning[i];
    const bool clique = q.kind == DM_QUERY_CLIQUE;
    t.est_cost = qcost[i];
    // cost model: bitmap intersection wherever a root's out-neighbourhood fits the bitmap
    // rows (the list path takes the larger roots); narrow groups only pay off when the
    // extension sets are tiny (k = 3 on a sparse graph); every query donates on demand
    // (threshold 0): donation is demand-limited, so it costs nothing while no warp is
    // hungry, and a per-root estimate that is too low must not leave a heavy root unsplit
    int vw = 32, thr = 0, mode = clique ? DM_MODE_AUTO : DM_MODE_LIST;
    if (!clique) {
      const double mean_deg = q.graph->n ? 2.0 * (double)q.graph->m / q.graph->n : 0.0;
      if (q.k == 3 && mean_deg <= 16.0) vw = 16;
    }
    if (autotune == DM_AUTOTUNE_MEASURE) {
      const std::vector<int> vws = clique ? std::vector<int>{32} : std::vector<int>{8, 16, 32};
      const std::vector<int> modes = clique ? std::vector<int>{DM_MODE_AUTO, DM_MODE_LIST} : std::vector<int>{DM_MODE_AUTO};
      double best = 1e300;
      for (int cv : vws)
        for (int cm : modes)
          for (int ct : {0, 100}) {
            double ms = 0;
            if ((rc = time_candidate(q, base, cv, ct, cm, &ms))) return fail_release(b, rc);
            if (ms < best) {
              best = ms;
              vw = cv;
              thr = ct;
              mode = clique ? cm : DM_MODE_LIST;
            }
          }
      t.tune_ms = best;
    }
    // explicit per-query settings win
    if (q.vwarp) vw = q.vwarp;
    if (q.threshold >= 0) thr = q.threshold;
    if (clique && q.mode != DM_MODE_AUTO) mode = q.mode;
    if (clique) vw = 32;
    t.vwarp = vw;
    t.threshold = thr;
    t.mode = (clique && mode != DM_MODE_LIST) ? DM_MODE_BITMAP : DM_MODE_LIST;
    t.n_results = d.n_classes;
    t.result_offset = off;
    off += d.n_classes;
    d.vwarp = vw;
    d.trigger = thr;  // converted to a warp count once the grid is known
    if (clique) {
      d.list_threshold = mode == DM_MODE_LIST ? -1 : 64 * BATCH_M;
      d.arena_dcap = d.maxdeg + 4;
    } else {
      d.arena_stride = (int)motif_group_stride(q.k, d.maxdeg);
      d.bit_words = motif_bit_words(d.nv);
    }
  }
  b->n_results = off;

  // ---- device buffers ----
  std::stable_sort(roots.begin(), roots.end(),
                   [](const std::pair<double, int32_t>& x, const std::pair<double, int32_t>& y) { return x.first > y.first; });
  b->n_roots = (int)roots.size();
  std::vector<int32_t> hroots(roots.size());
  for (size_t i = 0; i < roots.size(); ++i) hroots[i] = roots[i].second;
  if (padj.empty()) padj.assign(4, INT32_MAX);
  auto upload = [&](void** dst, const void* src, size_t bytes) -> int {
    DM_CUDA(cudaMalloc(dst, std::max<size_t>(bytes, 16)));
    if (bytes) DM_CUDA(cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, b->stream));
    return DM_OK;
  };
  if ((rc = upload(reinterpret_cast<void**>(&b->d_row), hrow.data(), sizeof(int32_t) * hrow.size())) ||
      (rc = upload(reinterpret_cast<void**>(&b->d_deg), pdeg.data(), sizeof(int32_t) * pdeg.size())) ||
      (rc = upload(reinterpret_cast<void**>(&b->d_adj), padj.data(), sizeof(int32_t) * padj.size())) ||
      (rc = upload(reinterpret_cast<void**>(&b->d_roots), hroots.data(), sizeof(int32_t) * hroots.size())) ||
      (rc = upload(reinterpret_cast<void**>(&b->d_vbase), vbase.data(), sizeof(int32_t) * vbase.size())))
    return fail_release(b, rc);
  const size_t out_bytes = sizeof(unsigned long long) * (size_t)std::max<int64_t>(b->n_results, 1);
  cudaError_t ce = cudaMalloc(&b->d_out, out_bytes);
  if (ce == cudaSuccess) ce = cudaMallocHost(&b->h_out, out_bytes);
  if (ce == cudaSuccess) ce = cudaMalloc(&b->d_ctr, sizeof(DevCounters));
  if (ce == cudaSuccess) ce = cudaMallocHost(&b->h_ctr, sizeof(DevCounters));
  if (ce == cudaSuccess)
    ce = cudaMalloc(&b->d_queue, sizeof(QHeader) * QUEUE_SHARDS + (size_t)QUEUE_SHARDS * QUEUE_SHARD_SLOTS * sizeof(QSlot));
  if (ce == cudaSuccess) ce = cudaEventCreate(&b->e0);
  if (ce == cudaSuccess) ce = cudaEventCreate(&b->e1);
  if (ce != cudaSuccess) return fail_release(b, fail(DM_ECUDA, std::string("dm_batch_create: ") + cudaGetErrorString(ce)));
  if ((rc = queue_init_launch(b->d_queue, QUEUE_SHARDS, QUEUE_SHARD_SLOTS, b->stream))) return fail_release(b, rc);
  for (int32_t i = 0; i < n; ++i) {
    const dm_query& q = queries[i];
    desc[i].out = b->d_out + b->tuning[i].result_offset;
    if (q.kind == DM_QUERY_MOTIF) {
      auto it = b->d_q2c.find(q.dict->uid);
      if (it == b->d_q2c.end()) {
        int32_t* p = nullptr;
        if ((rc = upload(reinterpret_cast<void**>(&p), q.dict->quick_to_class.data(),
                         sizeof(int32_t) * q.dict->quick_to_class.size())))
          return fail_release(b, rc);
        it = b->d_q2c.emplace(q.dict->uid, p).first;
      }
      desc[i].q2c = it->second;
    }
  }
  if ((rc = batch_configure<BATCH_M>(ctx.num_sms, ctx.threads, &b->grid, &b->smem))) return fail_release(b, rc);
  // per-warp arena: the largest need over the queries (clique list path: k lists; motif:
  // 32/W group arenas)
  size_t arena_bytes = 256;
  for (int32_t i = 0; i < n; ++i) {
    const BatchQuery& d = desc[i];
    size_t need = 0;
    if (d.kind == DM_QUERY_CLIQUE) {
      if (d.maxdeg > d.list_threshold && d.k > 3) need = (size_t)d.k * d.arena_dcap * sizeof(int32_t);
    } else {
      need = motif_group_stride(d.k, d.maxdeg) * (size_t)(32 / d.vwarp) * sizeof(int2);
    }
    arena_bytes = std::max(arena_bytes, (need + 255) / 256 * 256);
  }
  const size_t budget = (size_t)8 << 30;
  const size_t warps_fit = std::max<size_t>(BATCH_WARPS, budget / arena_bytes);
  b->grid = std::max(1, std::min(b->grid, (int)(warps_fit / BATCH_WARPS)));
  const int warps = b->grid * BATCH_WARPS;
  // a threshold is a percentage of the warps (>= 100: this query never donates)
  for (int32_t i = 0; i < n; ++i) {
    const int thr = desc[i].trigger;
    desc[i].trigger = thr >= 100 ? 0 : std::max(1, (thr * warps + 99) / 100);
  }
  ce = cudaMalloc(&b->d_arena, arena_bytes * (size_t)warps);
  if (ce != cudaSuccess)
    return fail_release(b, fail(DM_ECUDA, std::string("dm_batch_create: arena: ") + cudaGetErrorString(ce)));
  // membership bitmaps of the motif queries: per warp, 32/W groups x 2 bitmaps over the
  // largest motif graph (zeroed here; every task leaves them zero)
  size_t bits_words = 0;
  for (int32_t i = 0; i < n; ++i)
    if (desc[i].kind == DM_QUERY_MOTIF)
      bits_words = std::max(bits_words, (size_t)desc[i].bit_words * 2 * (32 / desc[i].vwarp));
  if (bits_words && bits_words * sizeof(uint32_t) * (size_t)warps <= ((size_t)2 << 30)) {
    b->bits_bytes = bits_words * sizeof(uint32_t) * (size_t)warps;
    ce = cudaMalloc(&b->d_bits, b->bits_bytes);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(b->d_bits, 0, b->bits_bytes, b->stream);
    if (ce != cudaSuccess)
      return fail_release(b, fail(DM_ECUDA, std::string("dm_batch_create: bitmaps: ") + cudaGetErrorString(ce)));
  }
  BatchArgs& a = b->args;
  a.g = GraphView{b->d_row, b->d_deg, b->d_adj, (int32_t)total_v};
  a.roots = b->d_roots;
  a.n_roots = b->n_roots;
  a.lb = LBArgs{b->d_ctr, reinterpret_cast<QHeader*>(b->d_queue),
                reinterpret_cast<QSlot*>(reinterpret_cast<char*>(b->d_queue) + sizeof(QHeader) * QUEUE_SHARDS),
                QUEUE_SHARD_SLOTS, 0, ctx.donations_per_warp, (long long)ctx.donate_after_us * 1000ll,
                (long long)ctx.timeout_ms * 1000000ll, ctx.test_stall, 32, QUEUE_SHARDS};
  a.vbase = b->d_vbase;
  a.n_queries = n;
  a.arena = b->d_arena;
  a.arena_bytes = arena_bytes;
  a.bits = b->d_bits;
  a.bits_words = bits_words;
  // per-query task contexts (the query's donation trigger and split granularity)
  for (int32_t i = 0; i < n; ++i) {
    BatchQuery& d = desc[i];
    std::memset(&d.cargs, 0, sizeof(d.cargs));
    std::memset(&d.mctx, 0, sizeof(d.mctx));
    if (d.kind == DM_QUERY_CLIQUE) {
      d.cargs.g = a.g;
      d.cargs.lb = a.lb;
      d.cargs.lb.hungry_trigger = d.trigger;
      d.cargs.lb.min_split = 32;
      d.cargs.arena_dcap = d.arena_dcap;
      d.cargs.list_vwarp = 32;  // the batch arena holds one list stack per warp
      d.cargs.list_threshold = d.list_threshold;
    } else {
      d.mctx.g = a.g;
      d.mctx.lb = a.lb;
      d.mctx.lb.hungry_trigger = d.trigger;
      d.mctx.lb.min_split = 4;
      d.mctx.q2c = d.q2c;
      d.mctx.maxdeg = d.maxdeg;
      d.mctx.arena_stride = d.arena_stride;
      d.mctx.bit_base = d.vbase;
      d.mctx.bit_words = b->d_bits ? d.bit_words : 0;
    }
  }
  if ((rc = upload(reinterpret_cast<void**>(&b->d_desc), desc.data(), sizeof(BatchQuery) * desc.size())))
    return fail_release(b, rc);
  a.queries = b->d_desc;
  DM_CUDA(cudaStreamSynchronize(b->stream));

  // ---- capture: reset, clear, launch, read back ----
  ce = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
  if (ce != cudaSuccess)
    return fail_release(b, fail(DM_ECUDA, std::string("dm_batch_create: capture: ") + cudaGetErrorString(ce)));
  batch_reset<<<1, 128, 0, b->stream>>>(b->d_ctr, b->n_roots);
  cudaMemsetAsync(b->d_out, 0, out_bytes, b->stream);
  if (b->n_roots > 0) rc = batch_launch<BATCH_M>(a, b->grid, b->smem, b->stream);
  cudaMemcpyAsync(b->h_out, b->d_out, out_bytes, cudaMemcpyDeviceToHost, b->stream);
  cudaMemcpyAsync(b->h_ctr, b->d_ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost, b->stream);
  ce = cudaStreamEndCapture(b->stream, &b->graph);
  if (rc || ce != cudaSuccess)
    return fail_release(b, rc ? rc : fail(DM_ECUDA, std::string("dm_batch_create: capture: ") + cudaGetErrorString(ce)));
  ce = cudaGraphInstantiate(&b->exec, b->graph, 0);
  if (ce != cudaSuccess)
    return fail_release(b, fail(DM_ECUDA, std::string("dm_batch_create: instantiate: ") + cudaGetErrorString(ce)));
  *out = b;
  return DM_OK;
}

int64_t dm_batch_num_results(const dm_batch* b) { return b ? b->n_results : 0; }

int dm_batch_tuning(const dm_batch* b, int32_t query, dm_query_tuning* out) {
  if (!b || !out || query < 0 || query >= b->n_queries) return fail(DM_EINVAL, "dm_batch_tuning: bad arguments");
  *out = b->tuning[query];
  return DM_OK;
}

int dm_batch_run(dm_batch* b, uint64_t* results, int64_t n_results, dm_stats* st) {
  if (!b || (b->n_results > 0 && !results)) return fail(DM_EINVAL, "dm_batch_run: bad arguments");
  if (n_results < b->n_results)
    return fail(DM_EINVAL, "dm_batch_run: results has room for fewer than dm_batch_num_results words");
  DM_CUDA(cudaSetDevice(b->device));
  DM_CUDA(cudaEventRecord(b->e0, b->stream));
  DM_CUDA(cudaGraphLaunch(b->exec, b->stream));
  DM_CUDA(cudaEventRecord(b->e1, b->stream));
  DM_CUDA(cudaStreamSynchronize(b->stream));
  const DevCounters h = *b->h_ctr;
  if (h.err) {
    // a failed launch can leave donations queued: empty the queue for the next run
    queue_init_launch(b->d_queue, QUEUE_SHARDS, QUEUE_SHARD_SLOTS, b->stream);
    if (b->d_bits) cudaMemsetAsync(b->d_bits, 0, b->bits_bytes, b->stream);
    cudaStreamSynchronize(b->stream);
    return fail(kernel_status(h.err), "batch kernel reported error " + std::to_string(h.err));
  }
  if (b->n_results) std::memcpy(results, b->h_out, sizeof(uint64_t) * (size_t)b->n_results);
  if (st) {
    float ms = 0;
    cudaEventElapsedTime(&ms, b->e0, b->e1);
    std::memset(st, 0, sizeof(*st));
    st->kernel_ms = ms;
    st->tasks = h.tasks;
    st->donations = h.donations;
    st->idle_polls = h.idle_polls;
    st->nodes = h.nodes;
    st->mode_used = DM_MODE_AUTO;
    st->vwarp_used = 0;
    st->grid = b->grid;
    st->block = 32 * BATCH_WARPS;
    st->kernel_launches = b->n_roots > 0 ? 1 : 0;
    const double warp_ns = (double)b->grid * BATCH_WARPS * (double)ms * 1e6;
    st->idle_warp_fraction = warp_ns > 0 ? std::min(1.0, (double)h.hungry_ns / warp_ns) : 0.0;
    st->max_task_ms = (double)h.max_task_ns * 1e-6;
    st->max_task_root = h.max_task_root;
    st->prefix_donations = (int32_t)std::min<unsigned long long>(h.prefix_donations, INT32_MAX);
  }
  return DM_OK;
}

void dm_batch_free(dm_batch* b) { batch_release(b); }

}  // extern "C"
