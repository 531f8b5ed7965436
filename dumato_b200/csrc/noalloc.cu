// k-clique counting for callers that cannot allocate GPU memory.
//
// Some callers cannot call cudaMalloc: code running inside another framework's memory
// pool or an allocator-free runtime, a process whose device memory is fully reserved up
// front, or a hook that must not change the device's allocation state. For them,
// dm_count_cliques_noalloc runs the same clique kernel as dm_count_cliques on a DAG the
// caller already holds in device memory, and takes its scratch (per-call counters and the
// donation queue of the load balancer) from one fixed array compiled into this library.
//
// The array below is a file-scope __device__ variable: every GPU that loads the library
// holds NOALLOC_SCRATCH_BYTES of it until the process exits. In host code its name is
// only a host-side stand-in for the device object; handing that name to a kernel would
// fault, or silently use the wrong memory where the GPU can reach host memory. The device
// address is obtained once per device with cudaGetSymbolAddress (with that device current)
// and that address is what the kernel receives.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "engine.hpp"
#include "lb.cuh"

namespace dmb {

// Donation-queue slots held by the fixed scratch (64 bytes each).
constexpr int NOALLOC_QUEUE_SLOTS = 4096;
// Largest out-degree the fixed scratch supports: roots up to this size run on the bitmap
// path, which needs no per-warp arena.
constexpr int NOALLOC_MAX_OUT_DEGREE = 256;
constexpr size_t NOALLOC_COUNTERS_BYTES = (sizeof(DevCounters) + 255) / 256 * 256;
constexpr size_t NOALLOC_SCRATCH_BYTES =
    NOALLOC_COUNTERS_BYTES + sizeof(QHeader) + sizeof(QSlot) * (size_t)NOALLOC_QUEUE_SLOTS;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

constexpr int NOALLOC_MAX_DEVICES = 64;
static std::mutex g_noalloc_mu;
static void* g_noalloc_ptr[NOALLOC_MAX_DEVICES];  // device address of the scratch, per device

__global__ void noalloc_queue_init(QHeader* h, QSlot* q, int cap) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) {
    h->write_pos = 0;
    h->read_pos = 0;
  }
  if (i < cap) {
    q[i].seq = (unsigned)i;
    q[i].root = q[i].begin = q[i].end = q[i].level = 0;
  }
}

// The counters start every call at zero, with every root pending.
__global__ void noalloc_reset_counters(DevCounters* c, int n_roots) {
  int* w = reinterpret_cast<int*>(c);
  for (int i = threadIdx.x; i < (int)(sizeof(DevCounters) / sizeof(int)); i += blockDim.x) w[i] = 0;
  __syncthreads();
  if (threadIdx.x == 0) c->pending = n_roots;
}

// Set-up, once per device with that device current: resolve the scratch's device address
// and put its queue in the empty state.
static int noalloc_scratch(int dev, cudaStream_t st, void** out) {
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return fail(DM_EINVAL, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return fail(DM_ECUDA, std::string("cudaGetSymbolAddress of the fixed scratch failed: ") + cudaGetErrorString(e));
    char* base = reinterpret_cast<char*>(p);
    QHeader* h = reinterpret_cast<QHeader*>(base + NOALLOC_COUNTERS_BYTES);
    QSlot* q = reinterpret_cast<QSlot*>(base + NOALLOC_COUNTERS_BYTES + sizeof(QHeader));
    noalloc_queue_init<<<(NOALLOC_QUEUE_SLOTS + 255) / 256, 256, 0, st>>>(h, q, NOALLOC_QUEUE_SLOTS);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(DM_ECUDA, std::string("scratch set-up failed: ") + cudaGetErrorString(e));
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return DM_OK;
}

}  // namespace dmb

using namespace dmb;

extern "C" int dm_count_cliques_noalloc(const int32_t* d_row, const int32_t* d_deg, const int32_t* d_adj,
                                        int32_t n_vertices, const int32_t* d_roots, int32_t n_roots,
                                        int32_t max_out_degree, int32_t k, uint64_t stream, uint64_t* count) {
  if (!count || n_vertices < 0 || n_roots < 0) return fail(DM_EINVAL, "dm_count_cliques_noalloc: bad arguments");
  if (n_roots > 0 && (!d_row || !d_deg || !d_adj || !d_roots))
    return fail(DM_EINVAL, "dm_count_cliques_noalloc: null device array");
  if (k < 2 || k > 12) return fail(DM_EINVAL, "dm_count_cliques_noalloc: k must be in [2, 12]");
  if (max_out_degree < 0 || max_out_degree > NOALLOC_MAX_OUT_DEGREE)
    return fail(DM_EINVAL, "dm_count_cliques_noalloc: max_out_degree " + std::to_string(max_out_degree) +
                               " exceeds the fixed-scratch limit of " + std::to_string(NOALLOC_MAX_OUT_DEGREE) +
                               " (use dm_count_cliques)");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(DM_ENODEVICE, "no usable CUDA device");
  }
  int dev = 0;
  DM_CUDA(cudaGetDevice(&dev));
  LaunchCtx ctx;
  ctx.device = dev;
  ctx.stream = reinterpret_cast<cudaStream_t>(stream);
  DM_CUDA(cudaDeviceGetAttribute(&ctx.num_sms, cudaDevAttrMultiProcessorCount, dev));
  void* scratch = nullptr;
  int rc = noalloc_scratch(dev, ctx.stream, &scratch);
  if (rc) return rc;
  char* base = reinterpret_cast<char*>(scratch);
  DevCounters* ctr = reinterpret_cast<DevCounters*>(base);
  noalloc_reset_counters<<<1, 128, 0, ctx.stream>>>(ctr, n_roots);
  DM_CUDA(cudaGetLastError());
  int grid = 0;
  if (n_roots > 0) {
    CliqueLaunch L;
    L.g = GraphView{d_row, d_deg, d_adj, n_vertices};
    L.k = k;
    L.roots = d_roots;
    L.n_roots = n_roots;
    L.ctr = ctr;
    L.queue = base + NOALLOC_COUNTERS_BYTES;
    L.qcap = NOALLOC_QUEUE_SLOTS;
    L.max_donations = ctx.donations_per_warp;
    L.nwmax = std::min(4, std::max(1, (max_out_degree + 63) / 64));
    L.list_threshold = 64 * L.nwmax;
    rc = clique_launch(L, ctx, &grid);
    if (rc) return rc;
  }
  DevCounters h;
  DM_CUDA(cudaMemcpyAsync(&h, ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost, ctx.stream));
  DM_CUDA(cudaStreamSynchronize(ctx.stream));
  if (h.err) {
    // a failed call can leave donations queued: empty the queue for the next call
    QHeader* qh = reinterpret_cast<QHeader*>(base + NOALLOC_COUNTERS_BYTES);
    QSlot* q = reinterpret_cast<QSlot*>(base + NOALLOC_COUNTERS_BYTES + sizeof(QHeader));
    noalloc_queue_init<<<(NOALLOC_QUEUE_SLOTS + 255) / 256, 256, 0, ctx.stream>>>(qh, q, NOALLOC_QUEUE_SLOTS);
    cudaStreamSynchronize(ctx.stream);
    return fail(h.err == ERR_TIMEOUT ? DM_ETIMEOUT : DM_EOVERFLOW,
                "clique kernel reported error " + std::to_string(h.err) +
                    (h.err == ERR_ARENA_OVERFLOW ? " (a root's out-degree exceeds max_out_degree)" : ""));
  }
  *count = h.count;
  return DM_OK;
}
