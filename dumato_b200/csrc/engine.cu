// C ABI entry points for counting, device graph residency and per-call workspaces.
//
// One call = one counting job on one device: the graph's CSR is uploaded once per device
// (padded rows, 16-byte aligned), the root tasks are ordered and split by execution mode,
// the kernels run on the caller's stream (or the library's own), and the u64 results are
// read back. This replaces the reference's DuMatoCPU set-up / runKernel / waitKernel /
// copyResult sequence (src/main/DuMatoCPU.cu:13-30, 204-276, 316-326, 419-423), whose
// per-warp DataGPU state is replaced by on-chip stacks and a small scratch arena.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "engine.hpp"

namespace dmb {

const char* cuda_err_str(cudaError_t e) { return cudaGetErrorString(e); }

// Per-(graph, device) workspace, reused across calls.
struct Workspace {
  DevCounters* d_ctr = nullptr;
  int32_t* d_tasks = nullptr;
  size_t tasks_cap = 0;
  void* d_scratch = nullptr;
  size_t scratch_cap = 0;
  unsigned long long* d_hist = nullptr;
  size_t hist_cap = 0;
  int32_t* d_q2c = nullptr;
  size_t q2c_cap = 0;
  const void* q2c_owner = nullptr;  // dictionary whose table is resident
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

struct DeviceSlot {
  DeviceGraph dg;
  Workspace ws;
};

static std::mutex g_dev_mu;
static std::map<int, cudaStream_t> g_streams;
static std::map<int, int> g_sms;

static int select_device(const dm_opts* o, LaunchCtx& ctx) {
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    cudaGetLastError();
    return fail(DM_ENODEVICE, std::string("no usable CUDA device: ") + cudaGetErrorString(e));
  }
  int dev = (o && o->device >= 0) ? o->device : -1;
  if (dev < 0) DM_CUDA(cudaGetDevice(&dev));
  if (dev >= count) return fail(DM_EINVAL, "device ordinal out of range");
  DM_CUDA(cudaSetDevice(dev));
  ctx.device = dev;
  std::lock_guard<std::mutex> lk(g_dev_mu);
  if (!g_sms.count(dev)) {
    int sms = 0;
    DM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    g_sms[dev] = sms;
  }
  ctx.num_sms = g_sms[dev];
  if (o && o->stream) {
    ctx.stream = reinterpret_cast<cudaStream_t>(o->stream);
  } else {
    if (!g_streams.count(dev)) {
      cudaStream_t s;
      DM_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
      g_streams[dev] = s;
    }
    ctx.stream = g_streams[dev];
  }
  if (o) {
    ctx.timeout_ms = o->timeout_ms > 0 ? o->timeout_ms : 2000;
    ctx.threads = o->threads;
    ctx.block = o->block_size;
    ctx.vwarp = o->vwarp;
    ctx.threshold = o->threshold > 0 ? o->threshold : 100;
    ctx.donations_per_warp = o->donations_per_warp > 0 ? o->donations_per_warp : 16;
  }
  return DM_OK;
}

static DeviceSlot* slot_for(dm_graph* g, int dev) {
  for (auto* p : g->dev)
    if (p->device == dev) return reinterpret_cast<DeviceSlot*>(p);
  auto* s = new DeviceSlot();
  s->dg.device = dev;
  g->dev.push_back(&s->dg);
  return s;
}

// Pads rows to multiples of 4 ints (16 bytes) filled with INT32_MAX.
static int upload_csr(const std::vector<int64_t>& row, const std::vector<int32_t>& adj, int32_t n, int32_t** d_row,
                      int32_t** d_deg, int32_t** d_adj, cudaStream_t st) {
  std::vector<int32_t> prow(n), pdeg(n);
  int64_t total = 0;
  for (int32_t v = 0; v < n; ++v) {
    int64_t d = row[v + 1] - row[v];
    prow[v] = (int32_t)total;
    pdeg[v] = (int32_t)d;
    total += (d + 3) & ~3ll;
    if (total >= INT32_MAX) return fail(DM_EOVERFLOW, "padded adjacency exceeds 32-bit offsets");
  }
  std::vector<int32_t> padj((size_t)std::max<int64_t>(total, 4), INT32_MAX);
  for (int32_t v = 0; v < n; ++v) std::memcpy(padj.data() + prow[v], adj.data() + row[v], sizeof(int32_t) * pdeg[v]);
  DM_CUDA(cudaMalloc(d_row, sizeof(int32_t) * std::max(n, 1)));
  DM_CUDA(cudaMalloc(d_deg, sizeof(int32_t) * std::max(n, 1)));
  DM_CUDA(cudaMalloc(d_adj, sizeof(int32_t) * padj.size()));
  if (n) {
    DM_CUDA(cudaMemcpyAsync(*d_row, prow.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, st));
    DM_CUDA(cudaMemcpyAsync(*d_deg, pdeg.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, st));
  }
  DM_CUDA(cudaMemcpyAsync(*d_adj, padj.data(), sizeof(int32_t) * padj.size(), cudaMemcpyHostToDevice, st));
  DM_CUDA(cudaStreamSynchronize(st));
  return DM_OK;
}

static int ensure_ws_bytes(void** p, size_t* cap, size_t want) {
  if (*cap >= want) return DM_OK;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  size_t alloc = want + want / 4 + 256;
  DM_CUDA(cudaMalloc(p, alloc));
  *cap = alloc;
  return DM_OK;
}

static int prepare_ws(Workspace& ws) {
  if (!ws.d_ctr) DM_CUDA(cudaMalloc(&ws.d_ctr, sizeof(DevCounters)));
  if (!ws.ev0) {
    DM_CUDA(cudaEventCreate(&ws.ev0));
    DM_CUDA(cudaEventCreate(&ws.ev1));
  }
  return DM_OK;
}

void release_device_graphs(dm_graph* g) {
  for (auto* p : g->dev) {
    auto* s = reinterpret_cast<DeviceSlot*>(p);
    int cur = 0;
    if (cudaGetDevice(&cur) == cudaSuccess) {
      cudaSetDevice(s->dg.device);
      cudaFree(s->dg.d_row);
      cudaFree(s->dg.d_deg);
      cudaFree(s->dg.d_adj);
      cudaFree(s->dg.d_orow);
      cudaFree(s->dg.d_odeg);
      cudaFree(s->dg.d_oadj);
      cudaFree(s->ws.d_ctr);
      cudaFree(s->ws.d_tasks);
      cudaFree(s->ws.d_scratch);
      cudaFree(s->ws.d_hist);
      cudaFree(s->ws.d_q2c);
      if (s->ws.ev0) cudaEventDestroy(s->ws.ev0);
      if (s->ws.ev1) cudaEventDestroy(s->ws.ev1);
      cudaSetDevice(cur);
    }
    cudaGetLastError();
    delete s;
  }
  g->dev.clear();
}

static int check_opts(const dm_opts* o) {
  if (!o) return DM_OK;
  if (o->struct_size != 0 && o->struct_size != (int32_t)sizeof(dm_opts))
    return fail(DM_EINVAL, "dm_opts.struct_size does not match this library");
  if (o->mode < 0 || o->mode > 2) return fail(DM_EINVAL, "dm_opts.mode out of range");
  if (o->scheduler < 0 || o->scheduler > 2) return fail(DM_EINVAL, "dm_opts.scheduler out of range");
  if (o->vwarp != 0 && o->vwarp != 8 && o->vwarp != 16 && o->vwarp != 32)
    return fail(DM_EINVAL, "dm_opts.vwarp must be 0, 8, 16 or 32");
  if (o->world_size > 1 && (o->rank < 0 || o->rank >= o->world_size)) return fail(DM_EINVAL, "dm_opts.rank out of range");
  if (o->block_size < 0 || o->threads < 0) return fail(DM_EINVAL, "negative threads / block_size");
  if (o->block_size && (o->block_size % 32 || o->block_size > 1024))
    return fail(DM_EINVAL, "block_size must be a multiple of 32 up to 1024");
  if (o->scheduler == DM_SCHED_LEARNED && !o->predictor) return fail(DM_EINVAL, "learned scheduler needs a predictor");
  return DM_OK;
}

// Root order (shared by both engines): plain = descending degree (heaviest first), id =
// ascending vertex id (the reference's round-robin striping order, DuMatoCPU.cu:126-135),
// learned = descending predicted cost. The shard keeps every world_size-th task.
int predictor_order(const void* predictor, dm_graph* g, int k, bool clique, std::vector<int32_t>& roots);

static int order_roots(dm_graph* g, const dm_opts* o, int k, bool clique, std::vector<int32_t>& roots) {
  const int sched = o ? o->scheduler : DM_SCHED_PLAIN;
  if (sched == DM_SCHED_LEARNED) {
    int rc = predictor_order(o->predictor, g, k, clique, roots);
    if (rc) return rc;
  } else if (sched == DM_SCHED_ID) {
    if (clique) std::sort(roots.begin(), roots.end(), [&](int32_t a, int32_t b) { return a < b; });
  } else {
    if (clique) {
      std::stable_sort(roots.begin(), roots.end(), [&](int32_t a, int32_t b) {
        return g->orow[a + 1] - g->orow[a] > g->orow[b + 1] - g->orow[b];
      });
    } else {
      std::stable_sort(roots.begin(), roots.end(), [&](int32_t a, int32_t b) {
        return g->row[a + 1] - g->row[a] > g->row[b + 1] - g->row[b];
      });
    }
  }
  if (o && o->world_size > 1) {
    std::vector<int32_t> mine;
    for (size_t i = o->rank; i < roots.size(); i += o->world_size) mine.push_back(roots[i]);
    roots.swap(mine);
  }
  return DM_OK;
}

}  // namespace dmb

using namespace dmb;

extern "C" {

int dm_device_count(void) {
  int c = 0;
  if (cudaGetDeviceCount(&c) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return c;
}

int dm_graph_release_device(dm_graph* g) {
  if (!g) return fail(DM_EINVAL, "null graph");
  std::lock_guard<std::mutex> lk(g->mu);
  release_device_graphs(g);
  return DM_OK;
}

int dm_count_cliques(dm_graph* g, int32_t k, const dm_opts* o, uint64_t* count, dm_stats* st) {
  if (!g || !count) return fail(DM_EINVAL, "dm_count_cliques: null argument");
  if (k < 2 || k > 12) return fail(DM_EINVAL, "dm_count_cliques: k must be in [2, 12]");
  int rc = check_opts(o);
  if (rc) return rc;
  LaunchCtx ctx;
  rc = select_device(o, ctx);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(g->mu);
  ensure_oriented(g);
  DeviceSlot* s = slot_for(g, ctx.device);
  Workspace& ws = s->ws;
  if ((rc = prepare_ws(ws))) return rc;
  DM_CUDA(cudaEventRecord(ws.ev0, ctx.stream));
  if (!s->dg.has_oriented) {
    rc = upload_csr(g->orow, g->oadj, g->n, &s->dg.d_orow, &s->dg.d_odeg, &s->dg.d_oadj, ctx.stream);
    if (rc) return rc;
    s->dg.has_oriented = true;
  }
  // tasks: roots with at least k-1 out-neighbours
  const int need = k - 1;
  std::vector<int32_t> roots;
  roots.reserve(g->n);
  for (int32_t r = 0; r < g->n; ++r)
    if (g->orow[r + 1] - g->orow[r] >= need) roots.push_back(r);
  if ((rc = order_roots(g, o, k, true, roots))) return rc;
  const int mode = o ? o->mode : DM_MODE_AUTO;
  std::vector<int32_t> t1, t2, tw, tl;
  int max_w = 0, max_l = 0;
  for (int32_t r : roots) {
    const int d = (int)(g->orow[r + 1] - g->orow[r]);
    if (mode == DM_MODE_LIST || d > 2048) {
      tl.push_back(r);
      max_l = std::max(max_l, d);
    } else if (d > 128) {
      tw.push_back(r);
      max_w = std::max(max_w, d);
    } else if (d > 64) {
      t2.push_back(r);
    } else {
      t1.push_back(r);
    }
  }
  std::vector<int32_t> all;
  all.reserve(roots.size());
  all.insert(all.end(), tl.begin(), tl.end());
  all.insert(all.end(), tw.begin(), tw.end());
  all.insert(all.end(), t2.begin(), t2.end());
  all.insert(all.end(), t1.begin(), t1.end());
  if ((rc = ensure_ws_bytes(reinterpret_cast<void**>(&ws.d_tasks), &ws.tasks_cap, sizeof(int32_t) * (all.size() + 1))))
    return rc;
  if (!all.empty())
    DM_CUDA(cudaMemcpyAsync(ws.d_tasks, all.data(), sizeof(int32_t) * all.size(), cudaMemcpyHostToDevice, ctx.stream));
  CliqueTasks t;
  t.d_list = ws.d_tasks;
  t.n_list = (int)tl.size();
  t.d_warp = t.d_list + t.n_list;
  t.n_warp = (int)tw.size();
  t.d_thread2 = t.d_warp + t.n_warp;
  t.n_thread2 = (int)t2.size();
  t.d_thread1 = t.d_thread2 + t.n_thread2;
  t.n_thread1 = (int)t1.size();
  t.max_warp_deg = max_w;
  t.max_list_deg = max_l;
  const size_t sb = clique_scratch_bytes(t, k, ctx);
  if (sb && (rc = ensure_ws_bytes(&ws.d_scratch, &ws.scratch_cap, sb))) return rc;
  DM_CUDA(cudaMemsetAsync(ws.d_ctr, 0, sizeof(DevCounters), ctx.stream));
  cudaEvent_t k0, k1;
  DM_CUDA(cudaEventCreate(&k0));
  DM_CUDA(cudaEventCreate(&k1));
  DM_CUDA(cudaEventRecord(k0, ctx.stream));
  GraphView view{s->dg.d_orow, s->dg.d_odeg, s->dg.d_oadj, g->n};
  rc = clique_launch(view, k, t, ws.d_ctr, ctx, ws.d_scratch, ws.scratch_cap, st);
  if (rc) {
    cudaEventDestroy(k0);
    cudaEventDestroy(k1);
    return rc;
  }
  DM_CUDA(cudaEventRecord(k1, ctx.stream));
  DevCounters h;
  DM_CUDA(cudaMemcpyAsync(&h, ws.d_ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost, ctx.stream));
  DM_CUDA(cudaStreamSynchronize(ctx.stream));
  float kms = 0, pms = 0;
  cudaEventElapsedTime(&kms, k0, k1);
  cudaEventElapsedTime(&pms, ws.ev0, k0);
  cudaEventDestroy(k0);
  cudaEventDestroy(k1);
  if (h.err) return fail(h.err == ERR_TIMEOUT ? DM_ETIMEOUT : DM_EOVERFLOW,
                         "clique kernel reported error " + std::to_string(h.err));
  *count = h.count;
  if (st) {
    std::memset(st, 0, sizeof(*st));
    st->kernel_ms = kms;
    st->prep_ms = pms;
    st->tasks = h.tasks;
    st->donations = h.donations;
    st->idle_polls = h.idle_polls;
    st->nodes = h.nodes;
    st->mode_used = tl.size() == roots.size() && !roots.empty() ? DM_MODE_LIST : DM_MODE_BITMAP;
    st->block = 256;
    st->kernel_launches = ctx.launches;
  }
  return DM_OK;
}

}  // extern "C"
