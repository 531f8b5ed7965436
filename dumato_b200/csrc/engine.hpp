// Internal launch interfaces between the C ABI (engine.cu) and the kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "dm_internal.hpp"

namespace dmb {

// Per-call device counters. One instance lives in device memory for each call.
struct DevCounters {
  unsigned long long count;      // clique total
  unsigned long long nodes;      // DFS nodes expanded
  unsigned long long tasks;      // tasks executed
  unsigned long long donations;  // donated work items
  unsigned long long idle_polls;
  int cursor[8];                 // task cursors (one per kernel)
  int err;                       // first error code raised by a kernel (0 = none)
  int err_info;
  int pad[6];
};

constexpr int ERR_ARENA_OVERFLOW = 1;
constexpr int ERR_TIMEOUT = 2;
constexpr int ERR_BAD_TASK = 3;

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
  int timeout_ms = 2000;
  int threads = 0;       // requested total threads (reference argv[3]); 0 = persistent default
  int block = 0;         // requested block size (reference argv[4]); 0 = kernel default
  int vwarp = 0;
  int threshold = 100;   // donation trigger (idle percentage); >= 100 = off
  int donations_per_warp = 16;
};

// Clique engine (clique.cu). tasks_* are device arrays of root ranks.
struct CliqueTasks {
  int32_t* d_thread1 = nullptr; int n_thread1 = 0;   // out-degree <= 64
  int32_t* d_thread2 = nullptr; int n_thread2 = 0;   // 64 < out-degree <= 128
  int32_t* d_warp = nullptr; int n_warp = 0;         // 128 < out-degree <= 2048
  int32_t* d_list = nullptr; int n_list = 0;         // list-mode roots
  int max_warp_deg = 0;
  int max_list_deg = 0;
};

int clique_launch(const GraphView& dag, int k, const CliqueTasks& t, DevCounters* d_ctr, LaunchCtx& ctx,
                  void* d_scratch, size_t scratch_bytes, dm_stats* st);
size_t clique_scratch_bytes(const CliqueTasks& t, int k, const LaunchCtx& ctx);

// Motif engine (motif.cu).
struct MotifPlan {
  int k = 0;
  int n_classes = 0;
  const int32_t* d_q2c = nullptr;        // quick -> class
  unsigned long long* d_hist = nullptr;  // n_classes
  int32_t* d_tasks = nullptr;            // roots
  int n_tasks = 0;
  int max_deg = 0;
};

int motif_launch(const GraphView& g, const MotifPlan& p, DevCounters* d_ctr, LaunchCtx& ctx, void* d_scratch,
                 size_t scratch_bytes, dm_stats* st);
size_t motif_scratch_bytes(const MotifPlan& p, const LaunchCtx& ctx, int* warps_out);

const char* cuda_err_str(cudaError_t e);

}  // namespace dmb

#define DM_CUDA(call)                                                              \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess)                                                         \
      return ::dmb::fail(DM_ECUDA, std::string(#call " failed: ") + cudaGetErrorString(e_)); \
  } while (0)
