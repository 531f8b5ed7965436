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
// fault, or silently use the wrong memory where the GPU can reach host memory. Every call
// resolves the device address with cudaGetSymbolAddress (on the current device, in the
// current context) and hands that address to the kernels; nothing about the array is
// cached on the host. Whether the donation queue inside it is in its empty state is also
// kept on the device, in a tag word that the set-up kernel checks at the start of every
// call: a context that was reset or re-created loads the module again with the array
// zeroed, so the tag is missing and the queue is rebuilt there.
#include <cuda_runtime.h>

#include <algorithm>
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
constexpr size_t NOALLOC_TAG_BYTES = 256;
constexpr size_t NOALLOC_SCRATCH_BYTES =
    NOALLOC_COUNTERS_BYTES + NOALLOC_TAG_BYTES + sizeof(QHeader) + sizeof(QSlot) * (size_t)NOALLOC_QUEUE_SLOTS;
// Tag word value meaning "the queue below is in its empty state".
constexpr unsigned NOALLOC_QUEUE_READY = 0x51554555u;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

struct NoallocParts {
  DevCounters* ctr;
  unsigned* tag;
  QHeader* qh;
  QSlot* q;
};

static NoallocParts noalloc_parts(void* base) {
  char* b = reinterpret_cast<char*>(base);
  NoallocParts p;
  p.ctr = reinterpret_cast<DevCounters*>(b);
  p.tag = reinterpret_cast<unsigned*>(b + NOALLOC_COUNTERS_BYTES);
  p.qh = reinterpret_cast<QHeader*>(b + NOALLOC_COUNTERS_BYTES + NOALLOC_TAG_BYTES);
  p.q = reinterpret_cast<QSlot*>(b + NOALLOC_COUNTERS_BYTES + NOALLOC_TAG_BYTES + sizeof(QHeader));
  return p;
}

// Start of every call (one block): zero the counters with every root pending, and put the
// queue in its empty state unless the tag says it already is (the kernels leave it empty
// after a call that raised no error; a call that raised one clears the tag).
__global__ void __launch_bounds__(1024) noalloc_setup(NoallocParts p, int n_roots, int cap) {
  __shared__ int rebuild;
  if (threadIdx.x == 0) rebuild = *reinterpret_cast<volatile unsigned*>(p.tag) != NOALLOC_QUEUE_READY;
  int* w = reinterpret_cast<int*>(p.ctr);
  for (int i = threadIdx.x; i < (int)(sizeof(DevCounters) / sizeof(int)); i += blockDim.x) w[i] = 0;
  __syncthreads();
  if (rebuild) {
    if (threadIdx.x == 0) {
      p.qh->write_pos = 0;
      p.qh->read_pos = 0;
    }
    for (int i = threadIdx.x; i < cap; i += blockDim.x) {
      p.q[i].seq = (unsigned)i;
      p.q[i].root = p.q[i].begin = p.q[i].end = p.q[i].level = 0;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    p.ctr->pending = n_roots;
    if (rebuild) *p.tag = NOALLOC_QUEUE_READY;
  }
}

// After a call whose kernel raised an error: donations may be left in the queue, so the
// next call's set-up rebuilds it.
__global__ void noalloc_invalidate(unsigned* tag) { *tag = 0u; }

// Device address of the fixed scratch in the current context.
static int noalloc_scratch(void** out) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p)
    return fail(DM_ECUDA, std::string("cudaGetSymbolAddress of the fixed scratch failed: ") + cudaGetErrorString(e));
  *out = p;
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
  int rc = noalloc_scratch(&scratch);
  if (rc) return rc;
  const NoallocParts parts = noalloc_parts(scratch);
  noalloc_setup<<<1, 1024, 0, ctx.stream>>>(parts, n_roots, NOALLOC_QUEUE_SLOTS);
  DM_CUDA(cudaGetLastError());
  int grid = 0;
  if (n_roots > 0) {
    CliqueLaunch L;
    L.g = GraphView{d_row, d_deg, d_adj, n_vertices};
    L.k = k;
    L.roots = d_roots;
    L.n_roots = n_roots;
    L.ctr = parts.ctr;
    L.queue = parts.qh;
    L.qcap = NOALLOC_QUEUE_SLOTS;
    L.nq = 1;
    L.max_donations = ctx.donations_per_warp;
    L.nwmax = std::min(4, std::max(1, (max_out_degree + 63) / 64));
    L.list_threshold = 64 * L.nwmax;
    rc = clique_launch(L, ctx, &grid);
    if (rc) return rc;
  }
  DevCounters h;
  DM_CUDA(cudaMemcpyAsync(&h, parts.ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost, ctx.stream));
  DM_CUDA(cudaStreamSynchronize(ctx.stream));
  if (h.err) {
    noalloc_invalidate<<<1, 1, 0, ctx.stream>>>(parts.tag);
    cudaStreamSynchronize(ctx.stream);
    return fail(kernel_status(h.err),
                "clique kernel reported error " + std::to_string(h.err) +
                    (h.err == ERR_ARENA_OVERFLOW ? " (a root's out-degree exceeds max_out_degree)" : ""));
  }
  *count = h.count;
  return DM_OK;
}
