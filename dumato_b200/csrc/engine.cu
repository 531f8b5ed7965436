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
#include <atomic>
#include <chrono>
#include <climits>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "engine.hpp"
#include "lb.cuh"

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
  uint64_t q2c_uid = 0;             // dictionary whose table is resident
  void* d_queue = nullptr;          // donation queue, ready flags kept zero between calls
  int qcap = 0;
  unsigned long long* d_per_root = nullptr;
  size_t per_root_cap = 0;
  int32_t* d_parts = nullptr;       // scheduler part words, parallel to the task list
  size_t parts_cap = 0;
  uint32_t* d_bits = nullptr;       // motif membership bitmaps, all zero between calls
  size_t bits_cap = 0;
  RootDesc* d_desc = nullptr;       // task list of a call on the clique index
  size_t desc_cap = 0;
  // learned schedule: MLP parameters, scratch and output task list
  float* d_params = nullptr;
  size_t params_cap = 0;
  uint64_t params_uid = 0, params_version = 0;  // the predictor version held in d_params
  int* h_hdr = nullptr;                          // pinned pair for the schedule's header
  void* d_sched = nullptr;
  size_t sched_cap = 0;
  int32_t* d_sroots = nullptr;
  size_t sroots_cap = 0;
  int32_t* d_sparts = nullptr;
  size_t sparts_cap = 0;
  RootDesc* d_sdesc = nullptr;
  size_t sdesc_cap = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, k0 = nullptr, k1 = nullptr;
  DevCounters* h_init = nullptr;    // pinned: a call's initial counters (asynchronous upload)
  DevCounters* h_out = nullptr;     // pinned: the counters read back after the kernel
};


// Empty state: every shard's positions at 0, slot j of a shard carrying sequence j.
__global__ void queue_init_kernel(QHeader* h, QSlot* q, int nq, int cap) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nq) {
    h[i].write_pos = 0;
    h[i].read_pos = 0;
  }
  if (i < nq * cap) {
    q[i].seq = (unsigned)(i % cap);
    q[i].root = q[i].begin = q[i].end = q[i].level = 0;
  }
}

int queue_init_launch(void* queue, int nq, int cap, cudaStream_t st) {
  QHeader* h = reinterpret_cast<QHeader*>(queue);
  QSlot* q = reinterpret_cast<QSlot*>(reinterpret_cast<char*>(queue) + sizeof(QHeader) * nq);
  queue_init_kernel<<<(nq * cap + 255) / 256, 256, 0, st>>>(h, q, nq, cap);
  DM_CUDA(cudaGetLastError());
  return DM_OK;
}

static int init_queue(Workspace& ws, cudaStream_t st) {
  QHeader* h = reinterpret_cast<QHeader*>(ws.d_queue);
  QSlot* q = reinterpret_cast<QSlot*>(reinterpret_cast<char*>(ws.d_queue) + sizeof(QHeader) * QUEUE_SHARDS);
  queue_init_kernel<<<(QUEUE_SHARDS * ws.qcap + 255) / 256, 256, 0, st>>>(h, q, QUEUE_SHARDS, ws.qcap);
  DM_CUDA(cudaGetLastError());
  return DM_OK;
}

struct DeviceSlot {
  DeviceGraph dg;
  Workspace ws;
  // roots (rank space) in descending out-degree order, resident on the device; the roots
  // eligible for k-cliques (out-degree >= k-1) are a prefix of it
  int32_t* d_deg_order = nullptr;
  // motif roots (vertices with a neighbour above them) by descending upper degree
  int32_t* d_up_order = nullptr;
  int n_up = 0;
  // clique index: the local bitmaps of every root with 2 <= out-degree <= 256, built on the
  // first clique call that can use it and kept with the device copy of the graph
  int index_state = 0;              // 0 not built, 1 built, -1 over the memory budget
  void* d_blocks = nullptr;
  uint32_t* d_boff = nullptr;
  size_t index_bytes = 0;
  void* d_image = nullptr;          // the graph's clique image (host_clique_image) on this device
  uint32_t* d_boff_img = nullptr;   // its index block offsets
  RootDesc* d_desc_img = nullptr;   // its plain task list
  RootDesc* d_desc_deg = nullptr;   // task list of the descending-degree order (index counting)
  // learned scheduler inputs on the device: base features per engine (0 = motifs, 1 =
  // cliques) by original id, and the rank -> original id map of the DAG
  float* d_feat[2] = {nullptr, nullptr};
  int32_t* d_orig = nullptr;
};

static std::mutex g_dev_mu;
static std::map<int, cudaStream_t> g_streams;
static std::map<int, int> g_sms;

int select_device(const dm_opts* o, LaunchCtx& ctx) {
  // the device count is fixed for the process once it is known (a failed query is retried)
  static std::atomic<int> known_count{0};
  int count = known_count.load(std::memory_order_relaxed);
  if (count == 0) {
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
      cudaGetLastError();
      return fail(DM_ENODEVICE, std::string("no usable CUDA device: ") + cudaGetErrorString(e));
    }
    known_count.store(count, std::memory_order_relaxed);
  }
  int cur = -1;
  DM_CUDA(cudaGetDevice(&cur));
  int dev = (o && o->device >= 0) ? o->device : cur;
  if (dev >= count) return fail(DM_EINVAL, "device ordinal out of range");
  if (dev != cur) DM_CUDA(cudaSetDevice(dev));
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
    ctx.timeout_ms = o->timeout_ms > 0 ? o->timeout_ms : 30000;
    ctx.threads = o->threads;
    ctx.block = o->block_size;
    ctx.vwarp = o->vwarp;
    ctx.threshold = o->threshold > 0 ? o->threshold : 0;
    ctx.donations_per_warp = o->donations_per_warp > 0 ? o->donations_per_warp : 64;
    ctx.test_stall = (o->test_flags & DM_TEST_STALL_AT_EXIT) ? 1 : 0;
    if (o->test_flags & DM_TEST_EAGER_DONATION) ctx.donate_after_us = 0;
  }
  return DM_OK;
}

// Access-policy window for one call (DM_FLAG_L2_PERSIST): the hottest device array of the
// call (the clique index, else the adjacency) is marked persisting on the call's stream, with
// the context's persisting set-aside raised to cover it. Everything is put back when the
// guard goes out of scope, after the call's stream has been synchronised: the window is
// removed, persisting lines return to normal, and the previous set-aside is restored.
struct L2Window {
  bool active = false;
  size_t prev_limit = 0;
  cudaStream_t st = nullptr;
  size_t window_bytes = 0;

  int begin(int dev, cudaStream_t stream, const void* base, size_t bytes) {
    int max_persist = 0, max_window = 0;
    DM_CUDA(cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, dev));
    DM_CUDA(cudaDeviceGetAttribute(&max_window, cudaDevAttrMaxAccessPolicyWindowSize, dev));
    if (max_persist <= 0 || max_window <= 0 || !base || bytes == 0) return DM_OK;
    DM_CUDA(cudaDeviceGetLimit(&prev_limit, cudaLimitPersistingL2CacheSize));
    const size_t want = std::min(bytes, (size_t)max_persist);
    DM_CUDA(cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, want));
    active = true;
    st = stream;
    cudaStreamAttrValue v{};
    v.accessPolicyWindow.base_ptr = const_cast<void*>(base);
    v.accessPolicyWindow.num_bytes = std::min(bytes, (size_t)max_window);
    v.accessPolicyWindow.hitRatio = std::min(1.0f, (float)want / (float)v.accessPolicyWindow.num_bytes);
    v.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
    v.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
    window_bytes = v.accessPolicyWindow.num_bytes;
    DM_CUDA(cudaStreamSetAttribute(stream, cudaStreamAttributeAccessPolicyWindow, &v));
    return DM_OK;
  }

  ~L2Window() {
    if (!active) return;
    cudaStreamAttrValue v{};
    v.accessPolicyWindow.num_bytes = 0;
    v.accessPolicyWindow.hitRatio = 0.f;
    v.accessPolicyWindow.hitProp = cudaAccessPropertyNormal;
    v.accessPolicyWindow.missProp = cudaAccessPropertyNormal;
    cudaStreamSetAttribute(st, cudaStreamAttributeAccessPolicyWindow, &v);
    cudaCtxResetPersistingL2Cache();
    cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, prev_limit);
    cudaGetLastError();
  }
};

// Live reports (dm_opts.report): while a counting kernel runs, a library thread copies the
// call's counter block every report_ms on a stream of its own (non-blocking, so the copy
// runs beside the kernel) into pinned memory and hands a dm_report to the caller's
// function. The thread stops after the call's stream has been synchronised.
static std::map<int, cudaStream_t> g_report_streams;

class Reporter {
 public:
  int start(const dm_opts* o, int dev, const DevCounters* ctr, int warps, int64_t roots) {
    if (!o || !o->report || o->report_ms <= 0) return DM_OK;
    {
      std::lock_guard<std::mutex> lk(g_dev_mu);
      if (!g_report_streams.count(dev)) {
        cudaStream_t s;
        DM_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        g_report_streams[dev] = s;
      }
      st_ = g_report_streams[dev];
    }
    DM_CUDA(cudaMallocHost(&snap_, sizeof(DevCounters)));
    fn_ = o->report;
    user_ = o->report_user;
    ms_ = o->report_ms;
    dev_ = dev;
    ctr_ = ctr;
    warps_ = warps;
    roots_ = roots;
    t0_ = std::chrono::steady_clock::now();
    th_ = std::thread([this] { run(); });
    return DM_OK;
  }
  ~Reporter() { stop(); }
  void stop() {
    if (th_.joinable()) {
      done_ = true;
      th_.join();
    }
    if (snap_) cudaFreeHost(snap_);
    snap_ = nullptr;
  }

 private:
  void run() {
    cudaSetDevice(dev_);
    while (!done_) {
      std::this_thread::sleep_for(std::chrono::milliseconds(ms_));
      if (done_) break;
      if (cudaMemcpyAsync(snap_, ctr_, sizeof(DevCounters), cudaMemcpyDeviceToHost, st_) != cudaSuccess ||
          cudaStreamSynchronize(st_) != cudaSuccess) {
        cudaGetLastError();
        break;
      }
      dm_report r{};
      r.elapsed_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0_).count();
      r.warps = warps_;
      r.hungry_warps = std::max(0, std::min(warps_, snap_->hungry));
      r.roots_claimed = std::min<int64_t>(roots_, snap_->cursor);
      r.roots_total = roots_;
      r.pending = snap_->pending;
      r.donations = snap_->donations;
      r.progress = snap_->progress;
      fn_(&r, user_);
    }
  }
  std::thread th_;
  std::atomic<bool> done_{false};
  DevCounters* snap_ = nullptr;
  const DevCounters* ctr_ = nullptr;
  cudaStream_t st_ = nullptr;
  dm_report_fn fn_ = nullptr;
  void* user_ = nullptr;
  int ms_ = 0, dev_ = 0, warps_ = 0;
  int64_t roots_ = 0;
  std::chrono::steady_clock::time_point t0_;
};

// Workspaces of released graphs, per device, handed to the next graph that needs one on that
// device. A graph's own device memory is its CSR copies and root orders; the scratch, the
// donation queue, the counters and the events are not tied to a graph, and allocating and
// freeing them costs milliseconds per call that re-uploads a graph.
static std::map<int, std::vector<Workspace>> g_ws_pool;
constexpr size_t WS_POOL_MAX = 4;

static void free_workspace(Workspace& w) {
  cudaFree(w.d_ctr);
  cudaFree(w.d_tasks);
  cudaFree(w.d_scratch);
  cudaFree(w.d_hist);
  cudaFree(w.d_q2c);
  cudaFree(w.d_queue);
  cudaFree(w.d_per_root);
  cudaFree(w.d_parts);
  cudaFree(w.d_bits);
  cudaFree(w.d_desc);
  cudaFree(w.d_params);
  cudaFree(w.d_sched);
  cudaFree(w.d_sroots);
  cudaFree(w.d_sparts);
  cudaFree(w.d_sdesc);
  if (w.ev0) cudaEventDestroy(w.ev0);
  if (w.ev1) cudaEventDestroy(w.ev1);
  if (w.k0) cudaEventDestroy(w.k0);
  if (w.k1) cudaEventDestroy(w.k1);
  if (w.h_init) cudaFreeHost(w.h_init);
  if (w.h_hdr) cudaFreeHost(w.h_hdr);
  if (w.h_out) cudaFreeHost(w.h_out);
  w = Workspace();
}

static DeviceSlot* slot_for(dm_graph* g, int dev) {
  for (auto* p : g->dev)
    if (p->device == dev) return reinterpret_cast<DeviceSlot*>(p);
  auto* s = new DeviceSlot();
  {
    std::lock_guard<std::mutex> lk(g_dev_mu);
    auto& pool = g_ws_pool[dev];
    if (!pool.empty()) {
      s->ws = pool.back();
      pool.pop_back();
    }
  }
  s->dg.device = dev;
  g->dev.push_back(&s->dg);
  return s;
}

// Device buffers owned by graphs (CSR copies, root orders, the clique index) go back to a
// per-device pool when a graph's device copy is released, and the next upload of the same
// or another graph takes them from there (best fit, at most twice the size asked for), so
// re-uploading a graph costs copies, not cudaMalloc/cudaFree. The pool holds at most 4 GB.
static std::mutex g_buf_mu;
static std::map<void*, size_t> g_buf_size;
static std::map<int, std::multimap<size_t, void*>> g_buf_pool;
static size_t g_buf_pooled = 0;
constexpr size_t BUF_POOL_MAX = (size_t)4 << 30;

static cudaError_t gbuf_alloc(void** p, size_t bytes) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  bytes = (std::max<size_t>(bytes, 256) + 255) / 256 * 256;
  std::lock_guard<std::mutex> lk(g_buf_mu);
  auto& pool = g_buf_pool[dev];
  auto it = pool.lower_bound(bytes);
  if (it != pool.end() && it->first <= 2 * bytes) {
    *p = it->second;
    g_buf_pooled -= it->first;
    pool.erase(it);
    return cudaSuccess;
  }
  e = cudaMalloc(p, bytes);
  if (e == cudaSuccess) g_buf_size[*p] = bytes;
  return e;
}

static void gbuf_free(void* p, int dev) {
  if (!p) return;
  std::lock_guard<std::mutex> lk(g_buf_mu);
  auto it = g_buf_size.find(p);
  if (it != g_buf_size.end() && g_buf_pooled + it->second <= BUF_POOL_MAX) {
    g_buf_pool[dev].insert({it->second, p});
    g_buf_pooled += it->second;
    return;
  }
  if (it != g_buf_size.end()) g_buf_size.erase(it);
  cudaFree(p);
}

// Registers a host array of the graph with the driver once (page-locked), so uploads from it
// are asynchronous DMA; the arrays are never resized afterwards and are unregistered when the
// graph is freed.
static void pin_host(dm_graph* g, const void* p, size_t bytes) {
  if (!p || !bytes) return;
  if (std::find(g->pinned.begin(), g->pinned.end(), p) != g->pinned.end()) return;
  if (cudaHostRegister(const_cast<void*>(p), bytes, cudaHostRegisterPortable) == cudaSuccess)
    g->pinned.push_back(const_cast<void*>(p));
  else
    cudaGetLastError();
}

void unpin_host_arrays(dm_graph* g) {
  for (void* p : g->pinned) cudaHostUnregister(p);
  g->pinned.clear();
  cudaGetLastError();
}

// Pads rows to multiples of 4 ints (16 bytes) filled with INT32_MAX; the padded layout is
// built on the first upload of a graph and kept (page-locked) with it.
static int host_pad_csr(const std::vector<int64_t>& row, const std::vector<int32_t>& adj, int32_t n,
                        std::vector<int32_t>& prow, std::vector<int32_t>& pdeg, std::vector<int32_t>& padj) {
  if (padj.empty()) {
    prow.assign(n, 0);
    pdeg.assign(n, 0);
    int64_t total = 0;
    for (int32_t v = 0; v < n; ++v) {
      int64_t d = row[v + 1] - row[v];
      prow[v] = (int32_t)total;
      pdeg[v] = (int32_t)d;
      total += (d + 3) & ~3ll;
      if (total >= INT32_MAX) {
        prow.clear();
        pdeg.clear();
        return fail(DM_EOVERFLOW, "padded adjacency exceeds 32-bit offsets");
      }
    }
    padj.assign((size_t)std::max<int64_t>(total, 4), INT32_MAX);
    for (int32_t v = 0; v < n; ++v) std::memcpy(padj.data() + prow[v], adj.data() + row[v], sizeof(int32_t) * pdeg[v]);
  }
  return DM_OK;
}

static int upload_csr(dm_graph* g, const std::vector<int64_t>& row, const std::vector<int32_t>& adj, int32_t n,
                      std::vector<int32_t>& prow, std::vector<int32_t>& pdeg, std::vector<int32_t>& padj,
                      int32_t** d_row, int32_t** d_deg, int32_t** d_adj, cudaStream_t st) {
  if (padj.empty()) {
    int rc = host_pad_csr(row, adj, n, prow, pdeg, padj);
    if (rc) return rc;
    pin_host(g, prow.data(), sizeof(int32_t) * prow.size());
    pin_host(g, pdeg.data(), sizeof(int32_t) * pdeg.size());
    pin_host(g, padj.data(), sizeof(int32_t) * padj.size());
  }
  // the three buffers are published together: a failure frees what was allocated
  int32_t *r = nullptr, *d = nullptr, *a = nullptr;
  int dev = 0;
  cudaGetDevice(&dev);
  cudaError_t e = gbuf_alloc(reinterpret_cast<void**>(&r), sizeof(int32_t) * std::max(n, 1));
  if (e == cudaSuccess) e = gbuf_alloc(reinterpret_cast<void**>(&d), sizeof(int32_t) * std::max(n, 1));
  if (e == cudaSuccess) e = gbuf_alloc(reinterpret_cast<void**>(&a), sizeof(int32_t) * padj.size());
  if (e == cudaSuccess && n) e = cudaMemcpyAsync(r, prow.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && n) e = cudaMemcpyAsync(d, pdeg.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(a, padj.data(), sizeof(int32_t) * padj.size(), cudaMemcpyHostToDevice, st);
  // (the host arrays live as long as the graph: no synchronisation is needed here)
  if (e != cudaSuccess) {
    gbuf_free(r, dev);
    gbuf_free(d, dev);
    gbuf_free(a, dev);
    return fail(e == cudaErrorMemoryAllocation ? DM_ENOMEM : DM_ECUDA,
                std::string("graph upload failed: ") + cudaGetErrorString(e));
  }
  *d_row = r;
  *d_deg = d;
  *d_adj = a;
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

static int prepare_ws(Workspace& ws, cudaStream_t st) {
  if (!ws.d_ctr) DM_CUDA(cudaMalloc(&ws.d_ctr, sizeof(DevCounters)));
  if (!ws.h_init) DM_CUDA(cudaMallocHost(&ws.h_init, sizeof(DevCounters)));
  if (!ws.h_out) DM_CUDA(cudaMallocHost(&ws.h_out, sizeof(DevCounters)));
  if (!ws.ev0) {
    DM_CUDA(cudaEventCreate(&ws.ev0));
    DM_CUDA(cudaEventCreate(&ws.ev1));
    DM_CUDA(cudaEventCreate(&ws.k0));
    DM_CUDA(cudaEventCreate(&ws.k1));
  }
  if (!ws.d_queue) {
    DM_CUDA(cudaMalloc(&ws.d_queue,
                       sizeof(QHeader) * QUEUE_SHARDS + (size_t)QUEUE_SHARDS * QUEUE_SHARD_SLOTS * sizeof(QSlot)));
    ws.qcap = QUEUE_SHARD_SLOTS;
    int rc = init_queue(ws, st);
    if (rc) return rc;
  }
  return DM_OK;
}

// Initial counters: every root task is pending until a warp finishes it; the root cursor
// starts after the entries dealt statically.
// (pinned source: the copy is asynchronous; the previous call's copies have completed, since
// every call ends by synchronising its stream)
static int init_counters(Workspace& ws, int n_roots, cudaStream_t st, int cursor = 0) {
  DevCounters* h = ws.h_init;
  std::memset(h, 0, sizeof(DevCounters));
  h->pending = n_roots;
  h->cursor = cursor;
  DM_CUDA(cudaMemcpyAsync(ws.d_ctr, h, sizeof(DevCounters), cudaMemcpyHostToDevice, st));
  return DM_OK;
}

// A call that ended in an error may leave tasks in the queue: start the next one clean.
static int reset_queue(Workspace& ws, const DevCounters& h, cudaStream_t st) {
  if (h.err) return init_queue(ws, st);
  return DM_OK;
}

void release_device_graphs(dm_graph* g) {
  for (auto* p : g->dev) {
    auto* s = reinterpret_cast<DeviceSlot*>(p);
    int cur = 0;
    if (cudaGetDevice(&cur) == cudaSuccess) {
      cudaSetDevice(s->dg.device);
      const int dv = s->dg.device;
      if (s->d_image) {
        // the oriented CSR, the root order and the index tables live in the image
        gbuf_free(s->d_image, dv);
        s->d_image = nullptr;
        s->dg.d_orow = s->dg.d_odeg = s->dg.d_oadj = nullptr;
        s->d_deg_order = nullptr;
        if (s->d_boff == s->d_boff_img) s->d_boff = nullptr;
        if (s->d_desc_deg == s->d_desc_img) s->d_desc_deg = nullptr;
      }
      for (void* p : {(void*)s->dg.d_row, (void*)s->dg.d_deg, (void*)s->dg.d_adj, (void*)s->dg.d_orow,
                      (void*)s->dg.d_odeg, (void*)s->dg.d_oadj, (void*)s->d_deg_order, (void*)s->d_up_order,
                      s->d_blocks, (void*)s->d_boff, (void*)s->d_desc_deg, (void*)s->d_feat[0], (void*)s->d_feat[1],
                      (void*)s->d_orig})
        gbuf_free(p, dv);
      {
        std::lock_guard<std::mutex> lk(g_dev_mu);
        auto& pool = g_ws_pool[s->dg.device];
        if (s->ws.d_queue && pool.size() < WS_POOL_MAX) {
          pool.push_back(s->ws);
          s->ws = Workspace();
        }
      }
      free_workspace(s->ws);

      cudaSetDevice(cur);
    }
    cudaGetLastError();
    delete s;
  }
  g->dev.clear();
}

static int upload_parts(Workspace& ws, const std::vector<int32_t>& parts, cudaStream_t st, const int32_t** out) {
  *out = nullptr;
  if (parts.empty()) return DM_OK;
  int rc = ensure_ws_bytes(reinterpret_cast<void**>(&ws.d_parts), &ws.parts_cap, sizeof(int32_t) * parts.size());
  if (rc) return rc;
  DM_CUDA(cudaMemcpyAsync(ws.d_parts, parts.data(), sizeof(int32_t) * parts.size(), cudaMemcpyHostToDevice, st));
  *out = ws.d_parts;
  return DM_OK;
}

int check_opts(const dm_opts* o) {
  if (!o) return DM_OK;
  if (o->struct_size != 0 && o->struct_size != (int32_t)sizeof(dm_opts))
    return fail(DM_EINVAL, "dm_opts.struct_size does not match this library");
  if (o->mode < 0 || o->mode > 3) return fail(DM_EINVAL, "dm_opts.mode out of range");
  if (o->staging < 0 || o->staging > 2) return fail(DM_EINVAL, "dm_opts.staging out of range");
  if (o->flags & ~DM_FLAG_L2_PERSIST) return fail(DM_EINVAL, "dm_opts.flags has unknown bits");
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

// Descending out-degree order of all roots: computed once per graph (host), uploaded once
// per device copy.
static void host_deg_order(dm_graph* g) {
  const int32_t n = g->n;
  if (g->deg_order.size() != (size_t)n || g->cnt_ge.empty()) {
    const int maxd = g->max_out_degree;
    std::vector<int64_t> cnt((size_t)maxd + 2, 0);
    for (int32_t r = 0; r < n; ++r) cnt[g->orow[r + 1] - g->orow[r]]++;
    g->cnt_ge.assign((size_t)maxd + 2, 0);
    for (int d = maxd; d >= 0; --d) g->cnt_ge[d] = g->cnt_ge[d + 1] + cnt[d];
    // counting sort by descending degree, stable in rank
    std::vector<int64_t> pos((size_t)maxd + 2, 0);
    for (int d = 0; d <= maxd; ++d) pos[d] = g->cnt_ge[d + 1];
    g->deg_order.assign(n, 0);
    for (int32_t r = 0; r < n; ++r) g->deg_order[pos[g->orow[r + 1] - g->orow[r]]++] = r;
  }
}

static int ensure_deg_order(dm_graph* g, DeviceSlot* s, cudaStream_t st) {
  if (s->d_deg_order) return DM_OK;
  const int32_t n = g->n;
  host_deg_order(g);
  pin_host(g, g->deg_order.data(), sizeof(int32_t) * g->deg_order.size());
  DM_CUDA(gbuf_alloc(reinterpret_cast<void**>(&s->d_deg_order), sizeof(int32_t) * std::max(n, 1)));
  if (n)
    DM_CUDA(cudaMemcpyAsync(s->d_deg_order, g->deg_order.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, st));
  return DM_OK;
}

// Entries of a root in the plain task list of the index: about d^2 / 256 for 20 to 64
// out-neighbours (its local edges, the items, number up to d(d-1)/2), else 1. Wider roots
// stay whole: their heavy items already split below the first level (level-1 donations), and
// parts would stage their large blocks once per part (measured on an R-MAT graph with roots
// of 106-171 out-neighbours: 7-cliques 70 ms whole, 79 ms in 16 parts; roots of 48-59
// out-neighbours on another R-MAT graph: 173 µs whole, 129 µs in parts).
static int split_parts(int d) { return d < 20 || d > 64 ? 1 : std::max(1, (d * d + 128) / 256); }

static RootDesc root_desc(const dm_graph* g, const DeviceSlot* /*s*/, int32_t r, int32_t part) {
  return RootDesc{r, (int32_t)(g->orow[r + 1] - g->orow[r]), g->idx_boff.empty() ? INDEX_NONE : g->idx_boff[r],
                  part};
}

// Builds the clique index of this device copy (once): host block offsets, the device
// blocks (index_build_kernel over the roots with 2 <= out-degree <= 256), and the task list
// of the descending-degree order. Graphs whose index would exceed min(8 GB, a quarter of
// the free device memory) keep rebuilding bitmaps per launch instead (index_state -1).
static void host_index_tables(dm_graph* g) {
  const int32_t n = g->n;
  if (g->idx_boff.size() != (size_t)n) {
    // block offsets and the task list of the descending-degree order, once per graph
    std::vector<uint32_t> boff((size_t)n, INDEX_NONE);
    uint64_t total = 0;
    int max_d = 0;
    for (int32_t r = 0; r < n; ++r) {
      const int d = (int)(g->orow[r + 1] - g->orow[r]);
      if (d >= 2 && d <= INDEX_MAX_DEGREE) {
        boff[r] = total < INDEX_NONE ? (uint32_t)total : INDEX_NONE;
        total += index_block_units_host(d);
        max_d = std::max(max_d, d);
      }
    }
    g->idx_boff.swap(boff);
    g->idx_units = total;
    g->idx_maxd = max_d;
    // roots of 32 or more out-neighbours enter the list as split_parts(d) entries, each for
    // an even share of the root's items: the warps dealt those entries start on the heaviest
    // roots together instead of one warp walking each of them alone
    g->idx_desc.clear();
    g->idx_desc.reserve((size_t)4 * n);
    for (int32_t i = 0; i < n; ++i) {
      const int32_t r = g->deg_order[i];
      const int P = split_parts((int)(g->orow[r + 1] - g->orow[r]));
      for (int q = 0; q < P; ++q) {
        const RootDesc rd = root_desc(g, nullptr, r, P > 1 ? (q | (P << 16)) : 0);
        const int32_t* w = reinterpret_cast<const int32_t*>(&rd);
        g->idx_desc.insert(g->idx_desc.end(), w, w + 4);
      }
    }
    g->idx_extra = (int32_t)(g->idx_desc.size() / 4 - (size_t)n);
  }
}

// The clique path's host arrays in one page-locked image, so that a device copy of the graph
// is one host-to-device copy: the padded oriented CSR (row starts, degrees, rows), the
// descending-degree order, the index block offsets and the plain task list, each starting
// on 256 bytes. Built once per graph; the separate padded CSR and task list are dropped.
// (One copy of the 1.57 MB of chunglu18k took 38 µs, seven copies of its parts 67 µs.)
static int host_clique_image(dm_graph* g) {
  if (!g->img.empty()) return DM_OK;
  int rc = host_pad_csr(g->orow, g->oadj, g->n, g->pad_row[1], g->pad_deg[1], g->pad_adj[1]);
  if (rc) return rc;
  host_deg_order(g);
  host_index_tables(g);
  const size_t n = (size_t)std::max(g->n, 1);
  const size_t sizes[6] = {4 * n, 4 * n, 4 * g->pad_adj[1].size(), 4 * n, 4 * n,
                           std::max<size_t>(4 * g->idx_desc.size(), 16)};
  size_t off = 0;
  for (int i = 0; i < 6; ++i) {
    g->img_off[i] = off;
    off += (sizes[i] + 255) / 256 * 256;
  }
  std::vector<uint8_t> img(off, 0);
  const int32_t nn = g->n;
  if (nn) {
    std::memcpy(img.data() + g->img_off[0], g->pad_row[1].data(), 4 * (size_t)nn);
    std::memcpy(img.data() + g->img_off[1], g->pad_deg[1].data(), 4 * (size_t)nn);
    std::memcpy(img.data() + g->img_off[3], g->deg_order.data(), 4 * (size_t)nn);
    std::memcpy(img.data() + g->img_off[4], g->idx_boff.data(), 4 * (size_t)nn);
  }
  std::memcpy(img.data() + g->img_off[2], g->pad_adj[1].data(), 4 * g->pad_adj[1].size());
  if (!g->idx_desc.empty()) std::memcpy(img.data() + g->img_off[5], g->idx_desc.data(), 4 * g->idx_desc.size());
  g->img_adj_ints = g->pad_adj[1].size();
  g->img.swap(img);
  pin_host(g, g->img.data(), g->img.size());
  std::vector<int32_t>().swap(g->pad_row[1]);
  std::vector<int32_t>().swap(g->pad_deg[1]);
  std::vector<int32_t>().swap(g->pad_adj[1]);
  std::vector<int32_t>().swap(g->idx_desc);
  return DM_OK;
}

// The oriented CSR, the root order and the index tables of a new device copy, from the
// image in one copy (the buffer returns to the pool when the copy is released).
static int upload_clique_image(dm_graph* g, DeviceSlot* s, cudaStream_t st) {
  int rc = host_clique_image(g);
  if (rc) return rc;
  void* base = nullptr;
  cudaError_t e = gbuf_alloc(&base, g->img.size());
  if (e == cudaSuccess) e = cudaMemcpyAsync(base, g->img.data(), g->img.size(), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) {
    int dev = 0;
    cudaGetDevice(&dev);
    gbuf_free(base, dev);
    return fail(e == cudaErrorMemoryAllocation ? DM_ENOMEM : DM_ECUDA,
                std::string("graph upload failed: ") + cudaGetErrorString(e));
  }
  char* b = static_cast<char*>(base);
  s->d_image = base;
  s->dg.d_orow = reinterpret_cast<int32_t*>(b + g->img_off[0]);
  s->dg.d_odeg = reinterpret_cast<int32_t*>(b + g->img_off[1]);
  s->dg.d_oadj = reinterpret_cast<int32_t*>(b + g->img_off[2]);
  s->d_deg_order = reinterpret_cast<int32_t*>(b + g->img_off[3]);
  s->d_boff_img = reinterpret_cast<uint32_t*>(b + g->img_off[4]);
  s->d_desc_img = reinterpret_cast<RootDesc*>(b + g->img_off[5]);
  s->dg.has_oriented = true;
  return DM_OK;
}

static int ensure_index(dm_graph* g, DeviceSlot* s, LaunchCtx& ctx) {
  if (s->index_state != 0) return DM_OK;
  const int32_t n = g->n;
  host_index_tables(g);
  const uint64_t total = g->idx_units;
  const size_t bytes = (size_t)total * 16;
  bool fits = total < INDEX_NONE;
  if (fits && bytes > ((size_t)256 << 20)) {
    size_t free_b = 0, tot_b = 0;
    DM_CUDA(cudaMemGetInfo(&free_b, &tot_b));
    fits = bytes <= std::min<size_t>((size_t)8 << 30, free_b / 4);
  }
  if (!fits) {
    s->index_state = -1;
    return DM_OK;
  }
  if (!s->d_image) return fail(DM_EINTERNAL, "clique index: the graph's image is not on the device");
  // the block offsets and the task list came with the image
  uint32_t* d_boff = s->d_boff_img;
  RootDesc* desc = s->d_desc_img;
  void* blocks = nullptr;
  cudaError_t e = gbuf_alloc(&blocks, std::max<size_t>(bytes, 16));
  if (e != cudaSuccess) {
    cudaGetLastError();
    s->index_state = -1;  // no room: per-launch bitmaps
    return DM_OK;
  }
  s->d_blocks = blocks;
  s->d_boff = d_boff;
  s->d_desc_deg = desc;
  s->index_bytes = bytes;
  s->index_state = 1;
  // roots with out-degree in [2, 256] are a contiguous range of the descending-degree order
  const int64_t lo = INDEX_MAX_DEGREE + 1 < (int64_t)g->cnt_ge.size() ? g->cnt_ge[INDEX_MAX_DEGREE + 1] : 0;
  const int64_t hi = 2 < (int64_t)g->cnt_ge.size() ? g->cnt_ge[2] : 0;
  const GraphView gv{s->dg.d_orow, s->dg.d_odeg, s->dg.d_oadj, n};
  return clique_index_build(gv, s->d_deg_order + lo, (int)(hi - lo), blocks, d_boff,
                            std::max(1, (std::min(INDEX_MAX_DEGREE, g->idx_maxd) + 63) / 64), ctx);
}

// Root order (shared by both engines): plain = descending degree (heaviest first), id =
// ascending vertex id (the reference's round-robin striping order, DuMatoCPU.cu:126-135),
// learned = descending predicted cost. The shard keeps every world_size-th task.
int predictor_schedule(const void* pv, dm_graph* g, int k, bool clique, int total_warps, std::vector<int32_t>& roots,
                       std::vector<int32_t>& parts);
int ensure_features(dm_graph* g, bool clique);
void predictor_key(const void* pv, uint64_t* uid, uint64_t* version);

// rank -> original id map of the DAG on the device (once per device copy)
static int ensure_orig(dm_graph* g, DeviceSlot* s, LaunchCtx& ctx) {
  if (s->d_orig) return DM_OK;
  std::vector<int32_t> inv(std::max(g->n, 1));
  for (int32_t v = 0; v < g->n; ++v) inv[g->rank[v]] = v;
  DM_CUDA(gbuf_alloc(reinterpret_cast<void**>(&s->d_orig), sizeof(int32_t) * inv.size()));
  DM_CUDA(cudaMemcpyAsync(s->d_orig, inv.data(), sizeof(int32_t) * inv.size(), cudaMemcpyHostToDevice, ctx.stream));
  DM_CUDA(cudaStreamSynchronize(ctx.stream));
  return DM_OK;
}

// Runs the learned schedule on the device for the input entries in_roots[0..n_in) (device
// pointer; rank space for cliques) and points *roots / *parts (and *desc for cliques on the
// index) at the workspace's output task list of *n entries.
static int learned_device(dm_graph* g, DeviceSlot* s, const dm_opts* o, int k, bool clique, const int32_t* in_roots,
                          int n_in, LaunchCtx& ctx, const int32_t** roots, const int32_t** parts,
                          const RootDesc** desc, int* n) {
  Workspace& ws = s->ws;
  const int eng = clique ? 1 : 0;
  int rc;
  if (!s->d_feat[eng]) {
    const auto& F = g->feat[eng];
    if (F.empty()) return fail(DM_EINVAL, "predictor features were not prepared");
    DM_CUDA(gbuf_alloc(reinterpret_cast<void**>(&s->d_feat[eng]), sizeof(float) * F.size()));
    DM_CUDA(cudaMemcpyAsync(s->d_feat[eng], F.data(), sizeof(float) * F.size(), cudaMemcpyHostToDevice, ctx.stream));
  }
  if (clique && (rc = ensure_orig(g, s, ctx))) return rc;
  const int warps = ctx.num_sms * 32;
  const int cap = learned_schedule_cap(n_in, warps);
  if ((rc = ensure_ws_bytes(reinterpret_cast<void**>(&ws.d_params), &ws.params_cap,
                            sizeof(float) * predictor_num_params())) ||
      (rc = ensure_ws_bytes(&ws.d_sched, &ws.sched_cap, learned_schedule_scratch_bytes(n_in))) ||
      (rc = ensure_ws_bytes(reinterpret_cast<void**>(&ws.d_sroots), &ws.sroots_cap, sizeof(int32_t) * cap)) ||
      (rc = ensure_ws_bytes(reinterpret_cast<void**>(&ws.d_sparts), &ws.sparts_cap, sizeof(int32_t) * cap)))
    return rc;
  const bool with_desc = clique && s->index_state == 1;
  if (with_desc &&
      (rc = ensure_ws_bytes(reinterpret_cast<void**>(&ws.d_sdesc), &ws.sdesc_cap, sizeof(RootDesc) * cap)))
    return rc;
  if (!ws.h_hdr) DM_CUDA(cudaMallocHost(&ws.h_hdr, 2 * sizeof(int)));
  uint64_t uid = 0, version = 0;
  predictor_key(o->predictor, &uid, &version);
  SchedIO io;
  io.feat = s->d_feat[eng];
  io.params = ws.d_params;
  io.params_current = uid != 0 && ws.params_uid == uid && ws.params_version == version;
  io.h_hdr = ws.h_hdr;
  io.roots = in_roots;
  io.orig = clique ? s->d_orig : nullptr;
  io.n_in = n_in;
  io.k = k;
  io.warps = warps;
  io.cap = cap;
  io.scratch = ws.d_sched;
  io.out_roots = ws.d_sroots;
  io.out_parts = ws.d_sparts;
  io.out_desc = with_desc ? ws.d_sdesc : nullptr;
  io.odeg = s->dg.d_odeg;
  io.boff = with_desc ? s->d_boff : nullptr;
  ws.params_uid = 0;  // until the call has written this version's parameters
  if ((rc = learned_schedule_device(o->predictor, io, ctx, n))) return rc;
  ws.params_uid = uid;
  ws.params_version = version;
  *roots = ws.d_sroots;
  *parts = ws.d_sparts;
  if (desc) *desc = with_desc ? ws.d_sdesc : nullptr;
  return DM_OK;
}

static int order_roots(dm_graph* g, const dm_opts* o, int k, bool clique, int total_warps,
                       std::vector<int32_t>& roots, std::vector<int32_t>& parts) {
  const int sched = o ? o->scheduler : DM_SCHED_PLAIN;
  parts.clear();
  if (sched == DM_SCHED_ID) {
    if (clique) {
      // rank space -> ascending original id
      std::vector<int32_t> inv(g->n);
      for (int32_t v = 0; v < g->n; ++v) inv[g->rank[v]] = v;
      std::sort(roots.begin(), roots.end(), [&](int32_t a, int32_t b) { return inv[a] < inv[b]; });
    } else {
      std::sort(roots.begin(), roots.end());
    }
  } else {
    if (clique) {
      std::stable_sort(roots.begin(), roots.end(), [&](int32_t a, int32_t b) {
        return g->orow[a + 1] - g->orow[a] > g->orow[b + 1] - g->orow[b];
      });
    } else {
      auto upper = [&](int32_t v) {
        const int32_t* b = g->adj.data() + g->row[v];
        const int32_t* e = g->adj.data() + g->row[v + 1];
        return e - std::upper_bound(b, e, v);
      };
      std::stable_sort(roots.begin(), roots.end(), [&](int32_t a, int32_t b) { return upper(a) > upper(b); });
    }
  }
  if (o && o->world_size > 1) {
    std::vector<int32_t> mine;
    for (size_t i = o->rank; i < roots.size(); i += o->world_size) mine.push_back(roots[i]);
    roots.swap(mine);
  }
  // the learned schedule reorders and splits the shard of the plain order
  if (sched == DM_SCHED_LEARNED) return predictor_schedule(o->predictor, g, k, clique, total_warps, roots, parts);
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

// One clique count (upto == nullptr) or the fused count of every size 3..k into upto[0..k-3].
// Returns 1, having counted nothing, when the fused walk cannot run on this graph and call
// (no clique index, roots above 256 out-neighbours, a per-launch or list mode, or a subtree
// log), so that the caller counts size by size instead.
static int count_cliques_impl(dm_graph* g, int32_t k, const dm_opts* o, uint64_t* count, dm_stats* st,
                              uint64_t* upto) {
  if (!g || !count) return fail(DM_EINVAL, "dm_count_cliques: null argument");
  if (k < 2 || k > 12) return fail(DM_EINVAL, "dm_count_cliques: k must be in [2, 12]");
  int rc = check_opts(o);
  if (rc) return rc;
  LaunchCtx ctx;
  rc = select_device(o, ctx);
  if (rc) return rc;
  if (o && o->scheduler == DM_SCHED_LEARNED && (rc = ensure_features(g, true))) return rc;
  std::lock_guard<std::mutex> lk(g->mu);
  ensure_oriented(g);
  DeviceSlot* s = slot_for(g, ctx.device);
  Workspace& ws = s->ws;
  if ((rc = prepare_ws(ws, ctx.stream))) return rc;
  DM_CUDA(cudaEventRecord(ws.ev0, ctx.stream));
  if (!s->dg.has_oriented && (rc = upload_clique_image(g, s, ctx.stream))) return rc;
  // tasks: roots (rank space) with at least k-1 out-neighbours
  const int need = upto ? 2 : k - 1;  // a fused count starts from every root with a local edge
  const int sched = o ? o->scheduler : DM_SCHED_PLAIN;
  const int world = (o && o->world_size > 1) ? o->world_size : 1;
  if ((rc = ensure_deg_order(g, s, ctx.stream))) return rc;
  const int mode = o ? o->mode : DM_MODE_AUTO;
  const bool want_index = (mode == DM_MODE_AUTO || mode == DM_MODE_BITMAP) && k >= 3 && k <= INDEX_MAX_K;
  if (want_index && (rc = ensure_index(g, s, ctx))) return rc;
  std::vector<int32_t> roots, parts;
  const int32_t* d_roots = nullptr;
  const RootDesc* d_desc = nullptr;
  int n_roots = 0, max_d = 0;
  if (sched == DM_SCHED_PLAIN && world == 1) {
    // the eligible roots are a prefix of the cached descending-degree order
    n_roots = need <= g->max_out_degree ? (int)g->cnt_ge[need] : 0;
    d_roots = s->d_deg_order;
    d_desc = s->d_desc_deg;
    max_d = n_roots ? (int)(g->orow[g->deg_order[0] + 1] - g->orow[g->deg_order[0]]) : 0;
  }
  const int32_t* d_parts = nullptr;
  if (d_roots) {
  } else if (sched == DM_SCHED_LEARNED) {
    // the plain order (this shard of it), reordered and split by the schedule on the device
    const int32_t* in = s->d_deg_order;
    int n_in = need <= g->max_out_degree ? (int)g->cnt_ge[need] : 0;
    if (n_in) max_d = (int)(g->orow[g->deg_order[0] + 1] - g->orow[g->deg_order[0]]);
    if (world > 1) {
      dm_opts po = *o;
      po.scheduler = DM_SCHED_PLAIN;
      for (int32_t r = 0; r < g->n; ++r)
        if (g->orow[r + 1] - g->orow[r] >= need) roots.push_back(r);
      if ((rc = order_roots(g, &po, k, true, ctx.num_sms * 32, roots, parts))) return rc;
      max_d = roots.empty() ? 0 : (int)(g->orow[roots[0] + 1] - g->orow[roots[0]]);
      if ((rc = ensure_ws_bytes(reinterpret_cast<void**>(&ws.d_tasks), &ws.tasks_cap,
                                sizeof(int32_t) * (roots.size() + 1))))
        return rc;
      if (!roots.empty())
        DM_CUDA(cudaMemcpyAsync(ws.d_tasks, roots.data(), sizeof(int32_t) * roots.size(), cudaMemcpyHostToDevice,
                                ctx.stream));
      in = ws.d_tasks;
      n_in = (int)roots.size();
    }
    if ((rc = learned_device(g, s, o, k, true, in, n_in, ctx, &d_roots, &d_parts, &d_desc, &n_roots))) return rc;
  } else {
    roots.reserve(g->n);
    for (int32_t r = 0; r < g->n; ++r)
      if (g->orow[r + 1] - g->orow[r] >= need) roots.push_back(r);
    if ((rc = order_roots(g, o, k, true, ctx.num_sms * 32, roots, parts))) return rc;
    for (int32_t r : roots) max_d = std::max(max_d, (int)(g->orow[r + 1] - g->orow[r]));
    n_roots = (int)roots.size();
    {
      if ((rc = upload_parts(ws, parts, ctx.stream, &d_parts))) return rc;
      if (s->index_state == 1) {
        std::vector<RootDesc> hd(roots.size());
        for (size_t i = 0; i < roots.size(); ++i) hd[i] = root_desc(g, s, roots[i], parts.empty() ? 0 : parts[i]);
        if ((rc = ensure_ws_bytes(reinterpret_cast<void**>(&ws.d_desc), &ws.desc_cap,
                                  sizeof(RootDesc) * (hd.size() + 1))))
          return rc;
        if (!hd.empty())
          DM_CUDA(cudaMemcpyAsync(ws.d_desc, hd.data(), sizeof(RootDesc) * hd.size(), cudaMemcpyHostToDevice,
                                  ctx.stream));
        d_desc = ws.d_desc;
      }
    }
  }
  const bool use_index = want_index && s->index_state == 1 && d_desc != nullptr;
  // the plain task list on the index holds the parts of the split roots too (they lead it)
  if (use_index && d_desc == s->d_desc_deg && n_roots > 0) n_roots += g->idx_extra;
  if (upto && (!use_index || max_d > INDEX_MAX_DEGREE || (o && o->subtree_counts))) return 1;
  CliqueLaunch L;
  L.k = k;
  if (mode == DM_MODE_LIST) {
    L.nwmax = 1;
    L.list_threshold = -1;
  } else {
    L.nwmax = std::min(4, std::max(1, (std::min(max_d, 256) + 63) / 64));
    L.list_threshold = 64 * L.nwmax;
  }
  const bool need_arena = max_d > L.list_threshold && k > 3;
  if (!d_roots) {
    if ((rc = ensure_ws_bytes(reinterpret_cast<void**>(&ws.d_tasks), &ws.tasks_cap,
                              sizeof(int32_t) * (roots.size() + 1))))
      return rc;
    if (!roots.empty())
      DM_CUDA(cudaMemcpyAsync(ws.d_tasks, roots.data(), sizeof(int32_t) * roots.size(), cudaMemcpyHostToDevice,
                              ctx.stream));
    d_roots = ws.d_tasks;
  }
  // list path: virtual-warp groups of 8, 16 or 32 lanes (32 unless dm_opts.vwarp says otherwise)
  L.list_vwarp = (ctx.vwarp == 8 || ctx.vwarp == 16) ? ctx.vwarp : 32;
  if (need_arena) {
    L.arena_dcap = max_d + 4;
    const size_t per_warp = (size_t)(32 / L.list_vwarp) * k * L.arena_dcap * sizeof(int32_t);
    const size_t budget = (size_t)8 << 30;
    ctx.arena_warps = (int)std::min<size_t>((size_t)clique_max_warps(ctx.num_sms), std::max<size_t>(8, budget / per_warp));
    if ((rc = ensure_ws_bytes(&ws.d_scratch, &ws.scratch_cap, per_warp * ctx.arena_warps))) return rc;
    L.arena = reinterpret_cast<int32_t*>(ws.d_scratch);
  }
  const bool want_log = o && o->subtree_counts;
  if (want_log) {
    if ((rc = ensure_ws_bytes(reinterpret_cast<void**>(&ws.d_per_root), &ws.per_root_cap,
                              sizeof(unsigned long long) * std::max(g->n, 1))))
      return rc;
    DM_CUDA(cudaMemsetAsync(ws.d_per_root, 0, sizeof(unsigned long long) * std::max(g->n, 1), ctx.stream));
    L.per_root = ws.d_per_root;
  }
  L.g = GraphView{s->dg.d_orow, s->dg.d_odeg, s->dg.d_oadj, g->n};
  L.roots = d_roots;
  L.parts = d_parts;
  L.n_roots = n_roots;
  L.ctr = ws.d_ctr;
  L.queue = ws.d_queue;
  L.qcap = ws.qcap;
  L.nq = QUEUE_SHARDS;
  L.max_donations = ctx.donations_per_warp;
  int grid = 0, cursor = 0;
  if (use_index) {
    // a root's block is staged in one round trip, so tasks are short: a task may donate
    // after 2 us instead of 20
    ctx.donate_after_us = std::min(ctx.donate_after_us, 2);
    L.multi = upto != nullptr;
    L.desc = d_desc;
    L.blocks = s->d_blocks;
    L.boff = s->d_boff;
    L.tma = !(o && o->staging == DM_STAGE_LOADS);
    if (n_roots > 0) {
      if ((rc = clique_cached_grid(L, ctx, &grid))) return rc;
      // every warp starts on static entries of the list (w, w + T, ...): no cursor atomics
      // while the first CHUNK_MAX x T entries are counted
      const int warps = grid * 8;
      L.static_chunk = std::max(1, std::min(16, (n_roots + warps - 1) / std::max(warps, 1)));
      L.n_static = (int)std::min<int64_t>(n_roots, (int64_t)warps * L.static_chunk);
      cursor = L.n_static;
    }
  }
  if ((rc = init_counters(ws, n_roots, ctx.stream, cursor))) return rc;
  L2Window l2;
  if (o && (o->flags & DM_FLAG_L2_PERSIST)) {
    if (use_index) rc = l2.begin(ctx.device, ctx.stream, s->d_blocks, s->index_bytes);
    else rc = l2.begin(ctx.device, ctx.stream, s->dg.d_oadj, sizeof(int32_t) * g->img_adj_ints);
    if (rc) return rc;
  }
  DM_CUDA(cudaEventRecord(ws.k0, ctx.stream));
  Reporter reporter;
  if (n_roots > 0) {
    rc = use_index ? clique_cached_launch(L, ctx, grid) : clique_launch(L, ctx, &grid);
    if (rc) return rc;
    if ((rc = reporter.start(o, ctx.device, ws.d_ctr, grid * 8, n_roots))) return rc;
  }
  DM_CUDA(cudaEventRecord(ws.k1, ctx.stream));
  DM_CUDA(cudaMemcpyAsync(ws.h_out, ws.d_ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost, ctx.stream));
  std::vector<unsigned long long> per_rank;
  if (want_log) {
    per_rank.resize(g->n);
    if (g->n)
      DM_CUDA(cudaMemcpyAsync(per_rank.data(), ws.d_per_root, sizeof(unsigned long long) * g->n, cudaMemcpyDeviceToHost,
                              ctx.stream));
  }
  DM_CUDA(cudaStreamSynchronize(ctx.stream));
  const DevCounters h = *ws.h_out;
  if ((rc = reset_queue(ws, h, ctx.stream))) return rc;
  float kms = 0, pms = 0;
  cudaEventElapsedTime(&kms, ws.k0, ws.k1);
  cudaEventElapsedTime(&pms, ws.ev0, ws.k0);
  if (h.err)
    return fail(kernel_status(h.err),
                "clique kernel reported error " + std::to_string(h.err));
  *count = h.count;
  if (upto) {
    for (int j = 3; j <= k; ++j) upto[j - 3] = h.count_k[j];
    *count = h.count_k[k];
  }
  if (want_log)
    for (int32_t v = 0; v < g->n; ++v) o->subtree_counts[v] = per_rank[g->rank[v]];
  if (st) {
    std::memset(st, 0, sizeof(*st));
    st->kernel_ms = kms;
    st->prep_ms = pms;
    st->tasks = h.tasks;
    st->donations = h.donations;
    st->idle_polls = h.idle_polls;
    st->nodes = h.nodes;
    st->mode_used = mode == DM_MODE_LIST ? DM_MODE_LIST : (use_index ? DM_MODE_BITMAP : DM_MODE_REBUILD);
    st->vwarp_used = L.list_vwarp;
    st->grid = grid;
    st->block = 256;
    st->kernel_launches = ctx.launches;
    const double warp_ns = (double)grid * 8.0 * (double)kms * 1e6;
    st->idle_warp_fraction = warp_ns > 0 ? std::min(1.0, (double)h.hungry_ns / warp_ns) : 0.0;
    st->max_task_ms = (double)h.max_task_ns * 1e-6;
    st->max_task_root = h.max_task_root;
    st->prefix_donations = (int32_t)std::min<unsigned long long>(h.prefix_donations, INT32_MAX);
  }
  return DM_OK;
}

int dm_count_cliques(dm_graph* g, int32_t k, const dm_opts* o, uint64_t* count, dm_stats* st) {
  return count_cliques_impl(g, k, o, count, st, nullptr);
}

int dm_count_cliques_upto(dm_graph* g, int32_t kmax, const dm_opts* o, uint64_t* counts, dm_stats* st) {
  if (!g || !counts) return fail(DM_EINVAL, "dm_count_cliques_upto: null argument");
  if (kmax < 4 || kmax > INDEX_MAX_K) return fail(DM_EINVAL, "dm_count_cliques_upto: kmax must be in [4, 8]");
  uint64_t top = 0;
  int rc = count_cliques_impl(g, kmax, o, &top, st, counts);
  if (rc != 1) return rc;
  // one launch per size
  dm_stats sum{}, one{};
  for (int k = 3; k <= kmax; ++k) {
    if ((rc = count_cliques_impl(g, k, o, &counts[k - 3], st ? &one : nullptr, nullptr))) return rc;
    if (st) {
      if (k == 3) sum = one;
      else {
        sum.kernel_ms += one.kernel_ms;
        sum.prep_ms += one.prep_ms;
        sum.tasks += one.tasks;
        sum.donations += one.donations;
        sum.idle_polls += one.idle_polls;
        sum.kernel_launches += one.kernel_launches;
        sum.prefix_donations += one.prefix_donations;
        sum.max_task_ms = std::max(sum.max_task_ms, one.max_task_ms);
      }
    }
  }
  if (st) *st = sum;
  return DM_OK;
}

int dm_count_near_cliques(dm_graph* g, int32_t n, const dm_opts* o, uint64_t* count, dm_stats* st) {
  if (!g || !count) return fail(DM_EINVAL, "dm_count_near_cliques: null argument");
  if (n < 4 || n > 13) return fail(DM_EINVAL, "dm_count_near_cliques: n must be in [4, 13]");
  int rc = check_opts(o);
  if (rc) return rc;
  LaunchCtx ctx;
  rc = select_device(o, ctx);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(g->mu);
  ensure_oriented(g);
  DeviceSlot* s = slot_for(g, ctx.device);
  Workspace& ws = s->ws;
  if ((rc = prepare_ws(ws, ctx.stream))) return rc;
  DM_CUDA(cudaEventRecord(ws.ev0, ctx.stream));
  if (!s->dg.has_oriented && (rc = upload_clique_image(g, s, ctx.stream))) return rc;
  if (!s->dg.has_undirected) {
    rc = upload_csr(g, g->row, g->adj, g->n, g->pad_row[0], g->pad_deg[0], g->pad_adj[0], &s->dg.d_row, &s->dg.d_deg,
                    &s->dg.d_adj, ctx.stream);
    if (rc) return rc;
    s->dg.has_undirected = true;
  }
  if ((rc = ensure_deg_order(g, s, ctx.stream)) || (rc = ensure_orig(g, s, ctx))) return rc;
  const int c = n - 2;
  const int need = c - 1;  // out-neighbours a root needs to start a c-clique
  const int world = (o && o->world_size > 1) ? o->world_size : 1;
  int n_roots = need <= g->max_out_degree ? (int)g->cnt_ge[need] : 0;
  const int32_t* d_roots = s->d_deg_order;
  if (world > 1) {
    std::vector<int32_t> mine;
    for (int i = o->rank; i < n_roots; i += world) mine.push_back(g->deg_order[i]);
    if ((rc = ensure_ws_bytes(reinterpret_cast<void**>(&ws.d_tasks), &ws.tasks_cap,
                              sizeof(int32_t) * (mine.size() + 1))))
      return rc;
    if (!mine.empty())
      DM_CUDA(cudaMemcpyAsync(ws.d_tasks, mine.data(), sizeof(int32_t) * mine.size(), cudaMemcpyHostToDevice,
                              ctx.stream));
    d_roots = ws.d_tasks;
    n_roots = (int)mine.size();
  }
  NearLaunch L;
  L.dag = GraphView{s->dg.d_orow, s->dg.d_odeg, s->dg.d_oadj, g->n};
  L.und = GraphView{s->dg.d_row, s->dg.d_deg, s->dg.d_adj, g->n};
  L.orig = s->d_orig;
  L.roots = d_roots;
  L.n_roots = n_roots;
  L.c = c;
  L.ctr = ws.d_ctr;
  L.queue = ws.d_queue;
  L.qcap = ws.qcap;
  L.nq = QUEUE_SHARDS;
  L.dag_cap = g->max_out_degree + 4;
  L.und_cap = g->max_degree + 4;
  const size_t per_warp = near_clique_warp_ints(c, L.dag_cap, L.und_cap) * sizeof(int32_t);
  ctx.arena_warps = (int)std::min<size_t>((size_t)ctx.num_sms * 64, std::max<size_t>(8, ((size_t)8 << 30) / per_warp));
  if ((rc = ensure_ws_bytes(&ws.d_scratch, &ws.scratch_cap, per_warp * ctx.arena_warps))) return rc;
  L.arena = reinterpret_cast<int32_t*>(ws.d_scratch);
  if ((rc = init_counters(ws, n_roots, ctx.stream))) return rc;
  DM_CUDA(cudaEventRecord(ws.k0, ctx.stream));
  int grid = 0;
  Reporter reporter;
  if (n_roots > 0) {
    if ((rc = near_clique_launch(L, ctx, &grid))) return rc;
    if ((rc = reporter.start(o, ctx.device, ws.d_ctr, grid * 8, n_roots))) return rc;
  }
  DM_CUDA(cudaEventRecord(ws.k1, ctx.stream));
  DM_CUDA(cudaMemcpyAsync(ws.h_out, ws.d_ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost, ctx.stream));
  DM_CUDA(cudaStreamSynchronize(ctx.stream));
  const DevCounters h = *ws.h_out;
  if ((rc = reset_queue(ws, h, ctx.stream))) return rc;
  float kms = 0, pms = 0;
  cudaEventElapsedTime(&kms, ws.k0, ws.k1);
  cudaEventElapsedTime(&pms, ws.ev0, ws.k0);
  if (h.err) return fail(kernel_status(h.err), "near-clique kernel reported error " + std::to_string(h.err));
  *count = h.count;
  if (st) {
    std::memset(st, 0, sizeof(*st));
    st->kernel_ms = kms;
    st->prep_ms = pms;
    st->tasks = h.tasks;
    st->idle_polls = h.idle_polls;
    st->mode_used = DM_MODE_LIST;
    st->vwarp_used = 32;
    st->grid = grid;
    st->block = 256;
    st->kernel_launches = ctx.launches;
    const double warp_ns = (double)grid * 8.0 * (double)kms * 1e6;
    st->idle_warp_fraction = warp_ns > 0 ? std::min(1.0, (double)h.hungry_ns / warp_ns) : 0.0;
  }
  return DM_OK;
}

int dm_count_motifs(dm_graph* g, int32_t k, const dm_dictionary* dict, const dm_opts* o, uint64_t* class_counts,
                    dm_stats* st) {
  if (!g || !dict || !class_counts) return fail(DM_EINVAL, "dm_count_motifs: null argument");
  if (k < 3 || k > 7) return fail(DM_EINVAL, "dm_count_motifs: k must be in [3, 7]");
  if (dict->k != k) return fail(DM_EINVAL, "dm_count_motifs: dictionary was built for another k");
  int rc = check_opts(o);
  if (rc) return rc;
  LaunchCtx ctx;
  rc = select_device(o, ctx);
  if (rc) return rc;
  if (o && o->scheduler == DM_SCHED_LEARNED && (rc = ensure_features(g, false))) return rc;
  std::lock_guard<std::mutex> lk(g->mu);
  DeviceSlot* s = slot_for(g, ctx.device);
  Workspace& ws = s->ws;
  if ((rc = prepare_ws(ws, ctx.stream))) return rc;
  DM_CUDA(cudaEventRecord(ws.ev0, ctx.stream));
  if (!s->dg.has_undirected) {
    rc = upload_csr(g, g->row, g->adj, g->n, g->pad_row[0], g->pad_deg[0], g->pad_adj[0], &s->dg.d_row,
                    &s->dg.d_deg, &s->dg.d_adj, ctx.stream);
    if (rc) return rc;
    s->dg.has_undirected = true;
  }
  auto upper = [&](int32_t v) {
    const int32_t* b = g->adj.data() + g->row[v];
    const int32_t* e = g->adj.data() + g->row[v + 1];
    return (int)(e - std::upper_bound(b, e, v));
  };
  const int sched = o ? o->scheduler : DM_SCHED_PLAIN;
  const int world = (o && o->world_size > 1) ? o->world_size : 1;
  const int32_t* d_roots = nullptr;
  int n_roots = 0;
  if (!s->d_up_order) {
    std::vector<int32_t>& order = g->up_order;
    if (order.empty()) {
      for (int32_t v = 0; v < g->n; ++v)
        if (upper(v) > 0) order.push_back(v);
      std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return upper(a) > upper(b); });
      pin_host(g, order.data(), sizeof(int32_t) * order.size());
    }
    DM_CUDA(gbuf_alloc(reinterpret_cast<void**>(&s->d_up_order), sizeof(int32_t) * std::max<size_t>(order.size(), 1)));
    if (!order.empty())
      DM_CUDA(cudaMemcpyAsync(s->d_up_order, order.data(), sizeof(int32_t) * order.size(), cudaMemcpyHostToDevice,
                              ctx.stream));
    s->n_up = (int)order.size();
  }
  std::vector<int32_t> roots, parts;
  const int32_t* d_parts_cached = nullptr;
  if (sched == DM_SCHED_PLAIN && world == 1) {
    d_roots = s->d_up_order;
    n_roots = s->n_up;
  } else if (sched == DM_SCHED_LEARNED) {
    // the plain order (this shard of it), reordered and split by the schedule on the device
    const int32_t* in = s->d_up_order;
    int n_in = s->n_up;
    if (world > 1) {
      dm_opts po = *o;
      po.scheduler = DM_SCHED_PLAIN;
      for (int32_t v = 0; v < g->n; ++v)
        if (upper(v) > 0) roots.push_back(v);
      if ((rc = order_roots(g, &po, k, false, ctx.num_sms * 32, roots, parts))) return rc;
      if ((rc = ensure_ws_bytes(reinterpret_cast<void**>(&ws.d_tasks), &ws.tasks_cap,
                                sizeof(int32_t) * (roots.size() + 1))))
        return rc;
      if (!roots.empty())
        DM_CUDA(cudaMemcpyAsync(ws.d_tasks, roots.data(), sizeof(int32_t) * roots.size(), cudaMemcpyHostToDevice,
                                ctx.stream));
      in = ws.d_tasks;
      n_in = (int)roots.size();
    }
    if ((rc = learned_device(g, s, o, k, false, in, n_in, ctx, &d_roots, &d_parts_cached, nullptr, &n_roots)))
      return rc;
  } else {
    for (int32_t v = 0; v < g->n; ++v)
      if (upper(v) > 0) roots.push_back(v);
    if ((rc = order_roots(g, o, k, false, ctx.num_sms * 32, roots, parts))) return rc;
    n_roots = (int)roots.size();
    {
      if ((rc = ensure_ws_bytes(reinterpret_cast<void**>(&ws.d_tasks), &ws.tasks_cap,
                                sizeof(int32_t) * (roots.size() + 1))))
        return rc;
      if (!roots.empty())
        DM_CUDA(cudaMemcpyAsync(ws.d_tasks, roots.data(), sizeof(int32_t) * roots.size(), cudaMemcpyHostToDevice,
                                ctx.stream));
      d_roots = ws.d_tasks;
    }
  }
  // dictionary table
  if (ws.q2c_uid != dict->uid) {
    if ((rc = ensure_ws_bytes(reinterpret_cast<void**>(&ws.d_q2c), &ws.q2c_cap, sizeof(int32_t) * dict->n_quicks)))
      return rc;
    DM_CUDA(cudaMemcpyAsync(ws.d_q2c, dict->quick_to_class.data(), sizeof(int32_t) * dict->n_quicks,
                            cudaMemcpyHostToDevice, ctx.stream));
    ws.q2c_uid = dict->uid;
  }
  if ((rc = ensure_ws_bytes(reinterpret_cast<void**>(&ws.d_hist), &ws.hist_cap,
                            sizeof(unsigned long long) * dict->n_classes)))
    return rc;
  DM_CUDA(cudaMemsetAsync(ws.d_hist, 0, sizeof(unsigned long long) * dict->n_classes, ctx.stream));
  // arena: extension levels and runs per warp
  const int maxdeg = std::max(g->max_degree, 1);
  const int vwarp = (ctx.vwarp == 8 || ctx.vwarp == 16) ? ctx.vwarp : 32;
  const size_t per_warp = motif_arena_stride(k, maxdeg, vwarp) * sizeof(int2);
  const size_t budget = (size_t)8 << 30;
  ctx.arena_warps = (int)std::min<size_t>((size_t)ctx.num_sms * 64, std::max<size_t>(8, budget / per_warp));
  if ((rc = ensure_ws_bytes(&ws.d_scratch, &ws.scratch_cap, per_warp * ctx.arena_warps))) return rc;
  // membership bitmaps (2 per group, zero between calls; skipped past 2 GB)
  const int bit_words = motif_bit_words(g->n);
  const size_t bits_bytes = (size_t)bit_words * 2 * (32 / vwarp) * sizeof(uint32_t) * ctx.arena_warps;
  uint32_t* d_bits = nullptr;
  if (bits_bytes <= ((size_t)2 << 30)) {
    if (ws.bits_cap < bits_bytes) {
      cudaFree(ws.d_bits);
      ws.d_bits = nullptr;
      ws.bits_cap = 0;
      DM_CUDA(cudaMalloc(&ws.d_bits, bits_bytes));
      DM_CUDA(cudaMemsetAsync(ws.d_bits, 0, bits_bytes, ctx.stream));
      ws.bits_cap = bits_bytes;
    }
    d_bits = ws.d_bits;
  }
  const bool want_log = o && o->subtree_counts;
  if (want_log) {
    if ((rc = ensure_ws_bytes(reinterpret_cast<void**>(&ws.d_per_root), &ws.per_root_cap,
                              sizeof(unsigned long long) * std::max(g->n, 1))))
      return rc;
    DM_CUDA(cudaMemsetAsync(ws.d_per_root, 0, sizeof(unsigned long long) * std::max(g->n, 1), ctx.stream));
  }
  if ((rc = init_counters(ws, n_roots, ctx.stream))) return rc;
  const int32_t* d_parts = d_parts_cached;
  if (!d_parts && (rc = upload_parts(ws, parts, ctx.stream, &d_parts))) return rc;
  MotifLaunch L;
  L.parts = d_parts;
  L.g = GraphView{s->dg.d_row, s->dg.d_deg, s->dg.d_adj, g->n};
  L.k = k;
  L.roots = d_roots;
  L.n_roots = n_roots;
  L.ctr = ws.d_ctr;
  L.queue = ws.d_queue;
  L.qcap = ws.qcap;
  L.nq = QUEUE_SHARDS;
  L.max_donations = ctx.donations_per_warp;
  L.q2c = ws.d_q2c;
  L.n_classes = dict->n_classes;
  L.hist = ws.d_hist;
  L.arena = ws.d_scratch;
  L.maxdeg = maxdeg;
  L.per_root = want_log ? ws.d_per_root : nullptr;
  L.vwarp = vwarp;
  L.bits = d_bits;
  L.bit_words = bit_words;
  L2Window l2;
  if (o && (o->flags & DM_FLAG_L2_PERSIST) &&
      (rc = l2.begin(ctx.device, ctx.stream, s->dg.d_adj, sizeof(int32_t) * g->pad_adj[0].size())))
    return rc;
  DM_CUDA(cudaEventRecord(ws.k0, ctx.stream));
  int grid = 0;
  Reporter reporter;
  if (n_roots > 0) {
    rc = motif_launch(L, ctx, &grid);
    if (rc) return rc;
    if ((rc = reporter.start(o, ctx.device, ws.d_ctr, grid * 8, n_roots))) return rc;
  }
  DM_CUDA(cudaEventRecord(ws.k1, ctx.stream));
  DM_CUDA(cudaMemcpyAsync(ws.h_out, ws.d_ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost, ctx.stream));
  DM_CUDA(cudaMemcpyAsync(class_counts, ws.d_hist, sizeof(unsigned long long) * dict->n_classes,
                          cudaMemcpyDeviceToHost, ctx.stream));
  if (want_log && g->n)
    DM_CUDA(cudaMemcpyAsync(o->subtree_counts, ws.d_per_root, sizeof(unsigned long long) * g->n,
                            cudaMemcpyDeviceToHost, ctx.stream));
  DM_CUDA(cudaStreamSynchronize(ctx.stream));
  const DevCounters h = *ws.h_out;
  if (h.err && d_bits) {
    // a failed launch can leave bits set: clear them for the next call
    DM_CUDA(cudaMemsetAsync(ws.d_bits, 0, ws.bits_cap, ctx.stream));
    DM_CUDA(cudaStreamSynchronize(ctx.stream));
  }
  if ((rc = reset_queue(ws, h, ctx.stream))) return rc;
  float kms = 0, pms = 0;
  cudaEventElapsedTime(&kms, ws.k0, ws.k1);
  cudaEventElapsedTime(&pms, ws.ev0, ws.k0);
  if (h.err)
    return fail(kernel_status(h.err),
                "motif kernel reported error " + std::to_string(h.err));
  if (st) {
    std::memset(st, 0, sizeof(*st));
    st->kernel_ms = kms;
    st->prep_ms = pms;
    st->tasks = h.tasks;
    st->donations = h.donations;
    st->idle_polls = h.idle_polls;
    st->nodes = h.nodes;
    st->mode_used = DM_MODE_LIST;
    st->vwarp_used = vwarp;
    st->grid = grid;
    st->block = 256;
    st->kernel_launches = ctx.launches;
    const double warp_ns = (double)grid * 8.0 * (double)kms * 1e6;
    st->idle_warp_fraction = warp_ns > 0 ? std::min(1.0, (double)h.hungry_ns / warp_ns) : 0.0;
    st->max_task_ms = (double)h.max_task_ns * 1e-6;
    st->max_task_root = h.max_task_root;
    st->prefix_donations = (int32_t)std::min<unsigned long long>(h.prefix_donations, INT32_MAX);
  }
  return DM_OK;
}

int dm_plan_roots(dm_graph* g, int32_t k, int32_t clique, const dm_opts* o, int32_t* out_roots, int32_t* out_parts,
                  int64_t cap, int64_t* n_out) {
  if (!g || !n_out || (cap > 0 && (!out_roots || !out_parts))) return fail(DM_EINVAL, "dm_plan_roots: bad arguments");
  if (k < 2 || k > 12 || (!clique && (k < 3 || k > 7))) return fail(DM_EINVAL, "dm_plan_roots: k out of range");
  int rc = check_opts(o);
  if (rc) return rc;
  if (o && o->scheduler == DM_SCHED_LEARNED && (rc = ensure_features(g, clique != 0))) return rc;
  std::lock_guard<std::mutex> lk(g->mu);
  ensure_oriented(g);
  std::vector<int32_t> roots, parts;
  if (clique) {
    for (int32_t r = 0; r < g->n; ++r)
      if (g->orow[r + 1] - g->orow[r] >= k - 1) roots.push_back(r);
  } else {
    for (int32_t v = 0; v < g->n; ++v) {
      const int32_t* b = g->adj.data() + g->row[v];
      const int32_t* e = g->adj.data() + g->row[v + 1];
      if (e - std::upper_bound(b, e, v) > 0) roots.push_back(v);
    }
  }
  int sms = 148;
  if ((rc = order_roots(g, o, k, clique != 0, sms * 32, roots, parts))) return rc;
  if (clique) {
    std::vector<int32_t> inv(g->n);
    for (int32_t v = 0; v < g->n; ++v) inv[g->rank[v]] = v;
    for (auto& r : roots) r = inv[r];
  }
  *n_out = (int64_t)roots.size();
  for (int64_t i = 0; i < std::min<int64_t>(cap, (int64_t)roots.size()); ++i) {
    out_roots[i] = roots[i];
    out_parts[i] = parts.empty() ? 0 : parts[i];
  }
  return DM_OK;
}

}  // extern "C"
