// Internal launch interfaces between the C ABI (engine.cu) and the kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "dm_internal.hpp"

namespace dmb {

// Per-call device counters and load-balancer state. One instance lives in device memory
// for each call; the host initialises it (pending = number of root tasks). Words that
// busy and hungry warps hit concurrently sit on separate 128-byte lines.
struct alignas(128) DevCounters {
  int cursor;                    // root cursor
  int pad0[31];
  int pending;                   // roots + donated tasks not finished yet
  int pad1[31];
  int hungry;                    // warps waiting for work
  int pad2[31];
  unsigned long long progress;   // work finished (batched), watched by waiting warps
  unsigned long long pad3[15];
  int queued;                    // donated tasks in the queue
  int pad4[31];
  unsigned long long count;      // clique total
  unsigned long long nodes;      // DFS nodes expanded
  unsigned long long tasks;      // tasks executed (roots + donated ranges)
  unsigned long long donations;  // donated ranges
  unsigned long long idle_polls; // polls of the donation queue by hungry warps
  unsigned long long hungry_ns;  // time warps spent waiting for work, summed over warps
  unsigned long long max_task_ns;  // longest single task
  unsigned long long prefix_donations;  // donated DFS prefixes (a level >= 1 extension set)
  unsigned long long count_k[16];  // fused counts: cliques of every size up to k
  int max_task_root;             // its root (best effort under races)
  int test_gate;                 // never written by the library (failure-path tests)
  int err;                       // first error code raised by a kernel (0 = none)
  int err_info;
};

constexpr int ERR_ARENA_OVERFLOW = 1;
constexpr int ERR_TIMEOUT = 2;
constexpr int ERR_BAD_TASK = 3;

// Status of a call whose kernel raised device error word `err` (non-zero): a bounded wait
// that gave up is DM_ETIMEOUT, an exceeded capacity bound DM_EOVERFLOW, and a task the
// kernel could not place (its own bookkeeping disagreeing with the graph) DM_EINTERNAL.
inline int kernel_status(int err) {
  return err == ERR_TIMEOUT ? DM_ETIMEOUT : (err == ERR_ARENA_OVERFLOW ? DM_EOVERFLOW : DM_EINTERNAL);
}

struct GraphView {
  const int32_t* row;   // padded row starts
  const int32_t* deg;
  const int32_t* adj;
  int32_t n;
};

struct LaunchCtx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int num_sms = 148;
  int launches = 0;
  int timeout_ms = 30000;
  int threads = 0;       // requested total threads (reference argv[3]); 0 = persistent default
  int block = 0;         // requested block size (reference argv[4]); 0 = kernel default
  int vwarp = 0;
  int threshold = 0;     // donation trigger (hungry-warp percentage); >= 100 = off
  int donations_per_warp = 16;
  int arena_warps = 0;   // warps the list arena has room for
  int donate_after_us = 20;  // a task donates only after running this long
  int test_stall = 0;        // DM_TEST_STALL_AT_EXIT
};

// Clique index (clique_cached.cuh): the local adjacency bitmap of every root r of the DAG
// with 2 <= d = |N+(r)| <= 256, as d rows of ceil(d/64) u64 words, the block starting on a
// 16-byte boundary (offset in 16-byte units; INDEX_NONE for roots without a block).
constexpr uint32_t INDEX_NONE = 0xffffffffu;
constexpr int INDEX_MAX_DEGREE = 256;
constexpr int INDEX_MAX_K = 8;  // larger k rebuild the bitmaps per launch

inline uint32_t index_block_units_host(int d) {
  const int nw = (d + 63) >> 6;
  return (uint32_t)((d * nw + 1) >> 1);
}

// One entry of a counting launch's task list on the index: root (rank space), out-degree,
// block offset (16-byte units, or INDEX_NONE) and scheduler part word (p | P << 16, 0 = whole).
struct RootDesc {
  int32_t root;
  int32_t d;
  uint32_t off;
  int32_t part;
};

// Scheduler part words: p | P << 16 (part p of P; 0 = the whole root), plus PART_EAGER when
// the learned scheduler predicts the task to be heavy, so that it donates without waiting
// for the minimum task age.
constexpr int PART_EAGER = 1 << 30;

// The learned schedule on the device (predictor.cu): inputs, scratch and outputs.
struct SchedIO {
  const float* feat = nullptr;       // n x 6 base features by original id
  float* params = nullptr;           // MLP parameters on the device
  bool params_current = false;       // params already hold this predictor's version
  int* h_hdr = nullptr;              // pinned: the schedule's task count and error flag
  const int32_t* roots = nullptr;    // n_in input entries
  const int32_t* orig = nullptr;     // rank -> original id (cliques), else null
  int n_in = 0, k = 0, warps = 1, cap = 0;
  void* scratch = nullptr;           // learned_schedule_scratch_bytes(n_in)
  int32_t* out_roots = nullptr;      // cap
  int32_t* out_parts = nullptr;      // cap
  RootDesc* out_desc = nullptr;      // cap or null
  const int32_t* odeg = nullptr;     // rank-space out-degrees (out_desc)
  const uint32_t* boff = nullptr;    // index block offsets (out_desc), or null
};
int learned_schedule_device(const void* predictor, const SchedIO& io, LaunchCtx& ctx, int* n_out);
size_t learned_schedule_scratch_bytes(int n_in);
inline int learned_schedule_cap(int n_in, int warps) { return n_in + 4 * warps + 64; }
int predictor_num_params();

// Clique engine (clique.cu).
struct CliqueLaunch {
  GraphView g;                   // degree-ordered DAG in rank space
  int k = 0;
  const int32_t* roots = nullptr;  // ordered root ranks
  int n_roots = 0;
  DevCounters* ctr = nullptr;
  void* queue = nullptr;         // donation queue: nq headers + nq * qcap slots (lb.cuh)
  int qcap = 0;                  // slots per shard
  int nq = 1;                    // shards
  int max_donations = 16;        // per task
  int32_t* arena = nullptr;      // list path: (32 / list_vwarp) x k x arena_dcap ints per warp
  int arena_dcap = 0;
  int list_vwarp = 32;           // list path: lanes per group (8, 16 or 32)
  int list_threshold = 256;
  int nwmax = 1;
  unsigned long long* per_root = nullptr;
  const int32_t* parts = nullptr;   // per root entry: p | P << 16 (0 = whole root)
  // counting on the clique index (clique_cached_*), else the per-launch bitmap build
  const RootDesc* desc = nullptr;   // task list (n_roots entries)
  const void* blocks = nullptr;     // the index (16-byte units)
  const uint32_t* boff = nullptr;   // block offset per root
  int static_chunk = 1;             // warp w starts with entries [w * static_chunk, +static_chunk)
  int n_static = 0;                 // entries dealt statically; the root cursor starts here
  bool tma = true;                  // stage blocks by bulk asynchronous copies (else 16-byte loads)
  bool multi = false;               // fused: count every clique size up to k (count_k)
};
int clique_launch(const CliqueLaunch& L, LaunchCtx& ctx, int* grid);
int clique_max_warps(int num_sms);
// Grid of the index-counting kernel for this launch (occupancy, requested threads, arena).
int clique_cached_grid(const CliqueLaunch& L, LaunchCtx& ctx, int* grid);
// Counting on the index with that grid (L.static_chunk / L.n_static set for it).
int clique_cached_launch(const CliqueLaunch& L, LaunchCtx& ctx, int grid);
// Builds the index blocks of roots[0..n) (rank space, 2 <= out-degree <= 64 * m).
int clique_index_build(const GraphView& g, const int32_t* roots, int n, void* blocks, const uint32_t* boff, int m,
                       LaunchCtx& ctx);

// Pattern-aware queries q4..q13 (near_clique.cu): (n-2)-cliques and their common neighbours.
struct NearLaunch {
  GraphView dag;                   // rank space
  GraphView und;                   // undirected, original ids
  const int32_t* orig = nullptr;   // rank -> original id
  const int32_t* roots = nullptr;
  int n_roots = 0;
  int c = 2;                       // clique size n - 2
  DevCounters* ctr = nullptr;
  void* queue = nullptr;
  int qcap = 0;
  int nq = 1;
  int32_t* arena = nullptr;        // near_clique_warp_ints ints per warp
  int dag_cap = 0, und_cap = 0;
};
int near_clique_launch(const NearLaunch& L, LaunchCtx& ctx, int* grid);
size_t near_clique_warp_ints(int c, int dag_cap, int und_cap);

// Motif engine (motif.cu).
struct MotifLaunch {
  GraphView g;                   // undirected CSR, original ids
  int k = 0;
  const int32_t* roots = nullptr;
  int n_roots = 0;
  DevCounters* ctr = nullptr;
  void* queue = nullptr;
  int qcap = 0;
  int nq = 1;
  int max_donations = 16;
  const int32_t* q2c = nullptr;
  int n_classes = 0;
  unsigned long long* hist = nullptr;
  void* arena = nullptr;
  int maxdeg = 0;
  unsigned long long* per_root = nullptr;
  const int32_t* parts = nullptr;
  int vwarp = 32;                // virtual-warp width: 8, 16 or 32
  uint32_t* bits = nullptr;      // per warp: 32/vwarp x 2 zeroed bitmaps of bit_words words (or null)
  int bit_words = 0;
};
// 32-bit words of one membership bitmap over n vertices.
inline int motif_bit_words(int n) { return (n + 31) / 32 + 1; }
int motif_launch(const MotifLaunch& L, LaunchCtx& ctx, int* grid);
size_t motif_arena_stride(int k, int maxdeg, int vwarp);  // int2 slots per warp

const char* cuda_err_str(cudaError_t e);

// Launch configuration of one kernel, settled once per device: the dynamic shared-memory
// attribute is set and the resident blocks per SM are queried on the first launch only, so
// a call spends no driver time on them afterwards.
constexpr int LAUNCH_CACHE_DEVICES = 64;
struct LaunchCache {
  int smem[LAUNCH_CACHE_DEVICES] = {};
  int occ[LAUNCH_CACHE_DEVICES] = {};
};
template <typename Kern>
inline cudaError_t cached_occupancy(LaunchCache& c, Kern kern, int device, int block, size_t smem, int* occ) {
  if (device >= 0 && device < LAUNCH_CACHE_DEVICES && c.occ[device] > 0 && c.smem[device] == (int)smem) {
    *occ = c.occ[device];
    return cudaSuccess;
  }
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, kern, block, smem);
  if (e == cudaSuccess && device >= 0 && device < LAUNCH_CACHE_DEVICES) {
    c.smem[device] = (int)smem;
    c.occ[device] = *occ;
  }
  return e;
}

// Host helpers shared by the entry points (engine.cu).
int select_device(const dm_opts* o, LaunchCtx& ctx);   // device, stream and options -> ctx
int check_opts(const dm_opts* o);
int queue_init_launch(void* queue, int nq, int cap, cudaStream_t st);  // empty donation queue
constexpr int QUEUE_SHARDS = 64;        // donation-queue shards of a workspace
constexpr int QUEUE_SHARD_SLOTS = 2048; // slots per shard

}  // namespace dmb

#define DM_CUDA(call)                                                              \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess)                                                         \
      return ::dmb::fail(DM_ECUDA, std::string(#call " failed: ") + cudaGetErrorString(e_)); \
  } while (0)
