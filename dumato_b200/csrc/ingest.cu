// Edgelist ingest and CSR build on the GPU: parse, deduplicate, symmetrise and orient.
//
// The reference reads its edgelists on the host into a std::map of std::set adjacency
// (src/main/Graph.cpp:17-75) and builds the CSR from it (src/main/DuMatoCPU.cu:94-108),
// which dominates its end-to-end time on large graphs. Here the file's bytes are copied to
// the device once and every step after that runs there:
//   1. comments: byte i lies in a comment when the last '#' or '%' at or before it comes
//      after the last newline at or before it (two inclusive max-scans of positions);
//   2. tokens: a digit outside a comment whose predecessor is not a digit starts a token;
//      an exclusive scan of those starts numbers the tokens, and each start parses its id;
//      a '-' or any byte other than a digit, blank, tab, CR, LF or ',' outside a comment is
//      a format error, as is an id above INT32_MAX - 1 or an odd number of ids (the host
//      reader's rules, dm_graph_load_edgelist);
//   3. pairs (2j, 2j+1): self-loops are counted and dropped, the others become u < v keys,
//      sorted and deduplicated (cub radix sort + unique);
//   4. symmetric CSR: both directions of every edge, sorted, give rows sorted ascending;
//   5. degree order: vertices sorted by (degree, id) give the ranks, and the arcs
//      rank(u) -> rank(v) for rank(u) < rank(v), sorted, give the oriented CSR.
// The results are copied into the graph's host arrays, exactly as the host reader builds
// them, so every other entry point works on the graph unchanged.
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_reduce.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>

#include <algorithm>
#include <climits>
#include <cstdio>
#include <string>
#include <vector>

#include "engine.hpp"

namespace dmb {

constexpr int INGEST_ERR_NEGATIVE = 1;
constexpr int INGEST_ERR_CHAR = 2;
constexpr int INGEST_ERR_RANGE = 4;

__device__ __forceinline__ bool is_digit(char c) { return c >= '0' && c <= '9'; }

__global__ void ingest_mark_kernel(const char* __restrict__ B, int64_t n, int32_t* __restrict__ nl,
                                   int32_t* __restrict__ cm) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const char c = B[i];
  nl[i] = c == '\n' ? (int32_t)i : -1;
  cm[i] = (c == '#' || c == '%') ? (int32_t)i : -1;
}

__global__ void ingest_token_kernel(const char* __restrict__ B, int64_t n, const int32_t* __restrict__ nl,
                                    const int32_t* __restrict__ cm, int32_t* __restrict__ start,
                                    int* __restrict__ err) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const char c = B[i];
  const bool comment = cm[i] > nl[i];
  int s = 0;
  if (!comment) {
    if (is_digit(c)) {
      s = (i == 0 || !is_digit(B[i - 1])) ? 1 : 0;
    } else if (!(c == ' ' || c == '\t' || c == '\r' || c == '\n' || c == ',')) {
      atomicOr(err, c == '-' ? INGEST_ERR_NEGATIVE : INGEST_ERR_CHAR);
    }
  }
  start[i] = s;
}

__global__ void ingest_parse_kernel(const char* __restrict__ B, int64_t n, const int32_t* __restrict__ start,
                                    const int32_t* __restrict__ index, int32_t* __restrict__ tok,
                                    int* __restrict__ err) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !start[i]) return;
  int64_t x = 0;
  for (int64_t j = i; j < n && is_digit(B[j]); ++j) {
    x = x * 10 + (B[j] - '0');
    if (x > INT32_MAX - 1) {
      atomicOr(err, INGEST_ERR_RANGE);
      return;
    }
  }
  tok[index[i]] = (int32_t)x;
}

// pair j -> (u < v) key, or a self-loop; the largest id of the pair
__global__ void ingest_pair_kernel(const int32_t* __restrict__ tok, int64_t pairs, uint64_t* __restrict__ keys,
                                   char* __restrict__ keep, int32_t* __restrict__ pair_max) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= pairs) return;
  const uint32_t u = (uint32_t)tok[2 * j], v = (uint32_t)tok[2 * j + 1];
  const uint32_t a = u < v ? u : v, b = u < v ? v : u;
  keys[j] = ((uint64_t)a << 32) | b;
  keep[j] = u != v ? 1 : 0;
  pair_max[j] = (int32_t)b;
}

// both directions of every edge, and the degrees
__global__ void ingest_sym_kernel(const uint64_t* __restrict__ edges, int64_t m, uint64_t* __restrict__ both,
                                  int32_t* __restrict__ deg) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= m) return;
  const uint64_t k = edges[e];
  const uint32_t u = (uint32_t)(k >> 32), v = (uint32_t)k;
  both[2 * e] = k;
  both[2 * e + 1] = ((uint64_t)v << 32) | u;
  atomicAdd(deg + u, 1);
  atomicAdd(deg + v, 1);
}

__global__ void ingest_low_kernel(const uint64_t* __restrict__ k, int64_t n, int32_t* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (int32_t)(uint32_t)k[i];
}

__global__ void ingest_rank_key_kernel(const int32_t* __restrict__ deg, int32_t n, uint64_t* __restrict__ key) {
  const int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < n) key[v] = ((uint64_t)(uint32_t)deg[v] << 32) | (uint32_t)v;
}

__global__ void ingest_rank_kernel(const uint64_t* __restrict__ sorted, int32_t n, int32_t* __restrict__ rank) {
  const int32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < n) rank[(uint32_t)sorted[r]] = r;
}

__global__ void ingest_arc_kernel(const uint64_t* __restrict__ edges, int64_t m, const int32_t* __restrict__ rank,
                                  uint64_t* __restrict__ arcs, int32_t* __restrict__ odeg) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= m) return;
  const uint64_t k = edges[e];
  const uint32_t ru = (uint32_t)rank[(uint32_t)(k >> 32)], rv = (uint32_t)rank[(uint32_t)k];
  const uint32_t a = ru < rv ? ru : rv, b = ru < rv ? rv : ru;
  arcs[e] = ((uint64_t)a << 32) | b;
  atomicAdd(odeg + a, 1);
}

__global__ void ingest_widen_kernel(const int32_t* __restrict__ deg, int32_t n, int64_t* __restrict__ out) {
  const int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < n) out[v] = deg[v];
  if (v == n) out[n] = 0;
}

namespace {

// Device buffers of one ingest; everything is freed when it goes out of scope.
struct DevBufs {
  std::vector<void*> ptrs;
  template <typename T>
  T* get(size_t count) {
    void* p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) return nullptr;
    ptrs.push_back(p);
    return reinterpret_cast<T*>(p);
  }
  ~DevBufs() {
    for (void* p : ptrs) cudaFree(p);
  }
};

unsigned blocks_for(int64_t n) { return (unsigned)std::max<int64_t>(1, (n + 255) / 256); }

}  // namespace

#define ING_ALLOC(var, T, count)                                        \
  T* var = bufs.get<T>(count);                                          \
  if (!var) {                                                           \
    cudaGetLastError();                                                 \
    return fail(DM_ENOMEM, "device allocation failed during ingest");   \
  }

// cub temporary storage: query, allocate, run
#define ING_CUB(call_with_tmp)                                          \
  do {                                                                  \
    void* d_tmp = nullptr;                                              \
    size_t tmp_bytes = 0;                                               \
    DM_CUDA(call_with_tmp);                                             \
    d_tmp = bufs.get<char>(tmp_bytes);                                  \
    if (!d_tmp) return fail(DM_ENOMEM, "device allocation failed during ingest"); \
    DM_CUDA(call_with_tmp);                                             \
  } while (0)

int ingest_edgelist_device(const char* path, const dm_opts* o, dm_graph** out, double* ms) {
  LaunchCtx ctx;
  int rc = select_device(o, ctx);
  if (rc) return rc;
  FILE* fp = std::fopen(path, "rb");
  if (!fp) return fail(DM_EIO, std::string("cannot open edgelist ") + path);
  std::fseek(fp, 0, SEEK_END);
  const long size = std::ftell(fp);
  std::fseek(fp, 0, SEEK_SET);
  if (size < 0 || size >= (long)INT32_MAX) {
    std::fclose(fp);
    return fail(DM_EINVAL, "device ingest takes files below 2 GiB (use dm_graph_load_edgelist)");
  }
  std::vector<char> host((size_t)size + 1);
  const size_t got = std::fread(host.data(), 1, (size_t)size, fp);
  std::fclose(fp);
  const int64_t N = (int64_t)got;
  cudaStream_t st = ctx.stream;
  cudaEvent_t e0, e1;
  DM_CUDA(cudaEventCreate(&e0));
  DM_CUDA(cudaEventCreate(&e1));
  DM_CUDA(cudaEventRecord(e0, st));
  DevBufs bufs;
  ING_ALLOC(dB, char, N);
  ING_ALLOC(dErr, int, 1);
  DM_CUDA(cudaMemsetAsync(dErr, 0, sizeof(int), st));
  if (N) DM_CUDA(cudaMemcpyAsync(dB, host.data(), (size_t)N, cudaMemcpyHostToDevice, st));
  // 1-2: comments, token starts, token numbers, ids
  ING_ALLOC(dNl, int32_t, N);
  ING_ALLOC(dCm, int32_t, N);
  ING_ALLOC(dStart, int32_t, N + 1);
  ING_ALLOC(dIdx, int32_t, N + 1);
  int32_t T = 0;
  if (N) {
    ingest_mark_kernel<<<blocks_for(N), 256, 0, st>>>(dB, N, dNl, dCm);
    ING_CUB(cub::DeviceScan::InclusiveScan(d_tmp, tmp_bytes, dNl, dNl, cub::Max(), (int)N, st));
    ING_CUB(cub::DeviceScan::InclusiveScan(d_tmp, tmp_bytes, dCm, dCm, cub::Max(), (int)N, st));
    ingest_token_kernel<<<blocks_for(N), 256, 0, st>>>(dB, N, dNl, dCm, dStart, dErr);
    DM_CUDA(cudaMemsetAsync(dStart + N, 0, sizeof(int32_t), st));
    ING_CUB(cub::DeviceScan::ExclusiveSum(d_tmp, tmp_bytes, dStart, dIdx, (int)N + 1, st));
    DM_CUDA(cudaMemcpyAsync(&T, dIdx + N, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    DM_CUDA(cudaStreamSynchronize(st));
  }
  int herr = 0;
  DM_CUDA(cudaMemcpy(&herr, dErr, sizeof(int), cudaMemcpyDeviceToHost));
  if (herr & INGEST_ERR_NEGATIVE) return fail(DM_EFORMAT, std::string("negative vertex id in ") + path);
  if (herr & INGEST_ERR_CHAR) return fail(DM_EFORMAT, std::string("non-integer token in ") + path);
  ING_ALLOC(dTok, int32_t, T);
  if (T) ingest_parse_kernel<<<blocks_for(N), 256, 0, st>>>(dB, N, dStart, dIdx, dTok, dErr);
  DM_CUDA(cudaMemcpyAsync(&herr, dErr, sizeof(int), cudaMemcpyDeviceToHost, st));
  DM_CUDA(cudaStreamSynchronize(st));
  if (herr & INGEST_ERR_RANGE) return fail(DM_EFORMAT, std::string("vertex id out of int32 range in ") + path);
  if (T % 2) return fail(DM_EFORMAT, std::string("odd number of ids in ") + path);
  const int64_t P = T / 2;
  // 3: pairs -> sorted unique u < v keys
  ING_ALLOC(dKeys, uint64_t, P);
  ING_ALLOC(dKeep, char, P);
  ING_ALLOC(dPMax, int32_t, P);
  ING_ALLOC(dSel, uint64_t, P);
  ING_ALLOC(dNSel, int32_t, 1);
  ING_ALLOC(dMax, int32_t, 1);
  int32_t maxid = -1, nsel = 0;
  if (P) {
    ingest_pair_kernel<<<blocks_for(P), 256, 0, st>>>(dTok, P, dKeys, dKeep, dPMax);
    ING_CUB(cub::DeviceReduce::Max(d_tmp, tmp_bytes, dPMax, dMax, (int)P, st));
    ING_CUB(cub::DeviceSelect::Flagged(d_tmp, tmp_bytes, dKeys, dKeep, dSel, dNSel, (int)P, st));
    DM_CUDA(cudaMemcpyAsync(&maxid, dMax, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    DM_CUDA(cudaMemcpyAsync(&nsel, dNSel, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    DM_CUDA(cudaStreamSynchronize(st));
  }
  const int32_t n = maxid + 1;
  const int64_t loops = P - nsel;
  ING_ALLOC(dSorted, uint64_t, nsel);
  ING_ALLOC(dEdges, uint64_t, nsel);
  int32_t m32 = 0;
  if (nsel) {
    ING_CUB(cub::DeviceRadixSort::SortKeys(d_tmp, tmp_bytes, dSel, dSorted, (int)nsel, 0, 64, st));
    ING_CUB(cub::DeviceSelect::Unique(d_tmp, tmp_bytes, dSorted, dEdges, dNSel, (int)nsel, st));
    DM_CUDA(cudaMemcpyAsync(&m32, dNSel, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    DM_CUDA(cudaStreamSynchronize(st));
  }
  const int64_t m = m32;
  if (m * 2 >= (int64_t)INT32_MAX) return fail(DM_EOVERFLOW, "graph has too many edges for 32-bit device offsets");
  // 4: symmetric CSR
  ING_ALLOC(dBoth, uint64_t, 2 * m);
  ING_ALLOC(dBothS, uint64_t, 2 * m);
  ING_ALLOC(dDeg, int32_t, n);
  ING_ALLOC(dRow, int64_t, (int64_t)n + 1);
  ING_ALLOC(dRowS, int64_t, (int64_t)n + 1);
  ING_ALLOC(dAdj, int32_t, 2 * m);
  DM_CUDA(cudaMemsetAsync(dDeg, 0, sizeof(int32_t) * std::max(n, 1), st));
  if (m) {
    ingest_sym_kernel<<<blocks_for(m), 256, 0, st>>>(dEdges, m, dBoth, dDeg);
    ING_CUB(cub::DeviceRadixSort::SortKeys(d_tmp, tmp_bytes, dBoth, dBothS, (int)(2 * m), 0, 64, st));
    ingest_low_kernel<<<blocks_for(2 * m), 256, 0, st>>>(dBothS, 2 * m, dAdj);
  }
  if (n) {
    ingest_widen_kernel<<<blocks_for((int64_t)n + 1), 256, 0, st>>>(dDeg, n, dRow);
    ING_CUB(cub::DeviceScan::ExclusiveSum(d_tmp, tmp_bytes, dRow, dRowS, n + 1, st));
  }
  // 5: degree order and the oriented CSR
  ING_ALLOC(dRk, uint64_t, n);
  ING_ALLOC(dRkS, uint64_t, n);
  ING_ALLOC(dRank, int32_t, n);
  ING_ALLOC(dArcs, uint64_t, m);
  ING_ALLOC(dArcsS, uint64_t, m);
  ING_ALLOC(dODeg, int32_t, n);
  ING_ALLOC(dORow, int64_t, (int64_t)n + 1);
  ING_ALLOC(dORowS, int64_t, (int64_t)n + 1);
  ING_ALLOC(dOAdj, int32_t, m);
  ING_ALLOC(dMaxD, int32_t, 2);
  int32_t maxd[2] = {0, 0};
  if (n) {
    ingest_rank_key_kernel<<<blocks_for(n), 256, 0, st>>>(dDeg, n, dRk);
    ING_CUB(cub::DeviceRadixSort::SortKeys(d_tmp, tmp_bytes, dRk, dRkS, n, 0, 64, st));
    ingest_rank_kernel<<<blocks_for(n), 256, 0, st>>>(dRkS, n, dRank);
    DM_CUDA(cudaMemsetAsync(dODeg, 0, sizeof(int32_t) * n, st));
    if (m) {
      ingest_arc_kernel<<<blocks_for(m), 256, 0, st>>>(dEdges, m, dRank, dArcs, dODeg);
      ING_CUB(cub::DeviceRadixSort::SortKeys(d_tmp, tmp_bytes, dArcs, dArcsS, (int)m, 0, 64, st));
      ingest_low_kernel<<<blocks_for(m), 256, 0, st>>>(dArcsS, m, dOAdj);
    }
    ingest_widen_kernel<<<blocks_for((int64_t)n + 1), 256, 0, st>>>(dODeg, n, dORow);
    ING_CUB(cub::DeviceScan::ExclusiveSum(d_tmp, tmp_bytes, dORow, dORowS, n + 1, st));
    ING_CUB(cub::DeviceReduce::Max(d_tmp, tmp_bytes, dDeg, dMaxD, n, st));
    ING_CUB(cub::DeviceReduce::Max(d_tmp, tmp_bytes, dODeg, dMaxD + 1, n, st));
    DM_CUDA(cudaMemcpyAsync(maxd, dMaxD, sizeof(int32_t) * 2, cudaMemcpyDeviceToHost, st));
  }
  DM_CUDA(cudaGetLastError());
  // results into the host graph
  dm_graph* g = new (std::nothrow) dm_graph();
  if (!g) return fail(DM_ENOMEM, "out of host memory");
  g->n = std::max(n, 0);
  g->m = m;
  g->self_loops = loops;
  g->input_pairs = P;
  g->row.assign((size_t)g->n + 1, 0);
  g->adj.resize((size_t)(2 * m));
  g->rank.resize((size_t)g->n);
  g->orow.assign((size_t)g->n + 1, 0);
  g->oadj.resize((size_t)m);
  cudaError_t e = cudaSuccess;
  if (g->n) {
    e = cudaMemcpyAsync(g->row.data(), dRowS, sizeof(int64_t) * (g->n + 1), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(g->rank.data(), dRank, sizeof(int32_t) * g->n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(g->orow.data(), dORowS, sizeof(int64_t) * (g->n + 1), cudaMemcpyDeviceToHost, st);
  }
  if (e == cudaSuccess && m)
    e = cudaMemcpyAsync(g->adj.data(), dAdj, sizeof(int32_t) * 2 * m, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess && m)
    e = cudaMemcpyAsync(g->oadj.data(), dOAdj, sizeof(int32_t) * m, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaEventRecord(e1, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    delete g;
    return fail(DM_ECUDA, std::string("device ingest failed: ") + cudaGetErrorString(e));
  }
  float t = 0;
  cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (ms) *ms = t;
  g->max_degree = maxd[0];
  g->max_out_degree = maxd[1];
  g->oriented_built = true;
  *out = g;
  return DM_OK;
}

}  // namespace dmb

extern "C" int dm_graph_load_edgelist_device(const char* path, const dm_opts* o, dm_graph** out, double* device_ms) {
  if (!path || !out) return dmb::fail(DM_EINVAL, "dm_graph_load_edgelist_device: null argument");
  int rc = dmb::check_opts(o);
  if (rc) return rc;
  return dmb::ingest_edgelist_device(path, o, out, device_ms);
}
