// Learned work predictor and the learned scheduler (no counterpart in the reference).
//
// A small MLP (8 features -> 32 -> 32 -> 1, FP32, ReLU) predicts log(1 + subtree size) of a
// root task, where the subtree size is the number of subgraphs the task counts (the log the
// plain engine writes through dm_opts.subtree_counts). Training, gradients and inference
// are this file's own CUDA kernels: a per-sample forward/backward whose activations stay in
// shared memory, a per-parameter reduction over each block's samples, and an Adam step.
//
// Features of root v for a k query (all FP32):
//   f0 log1p(deg v)            f1 log1p(core number of v)
//   f2 log1p(|C_0|)            candidate-set size: out-degree in the degree-ordered DAG for
//                              cliques, neighbours above v for motifs
//   f3 k / 8                   f4 (k - 2) / 8: DFS depth below a root task
//   f5 log1p(DAG out-degree)   f6 log1p(2-hop size: sum over C_0 of DAG out-degrees for
//                              cliques, of degrees for motifs)
//   f7 log1p(triangles whose lowest-ranked vertex is v)
//
// The learned scheduler orders root tasks by predicted cost (longest first) and splits a
// root whose predicted cost exceeds the per-warp share into P parts up front, so heavy
// subtrees start on several warps at once instead of waiting for reactive donation.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "engine.hpp"

// MLP geometry
constexpr int MLP_F = 8, MLP_H = 32;
constexpr int OFF_W1 = 0;                       // [H][F]
constexpr int OFF_B1 = OFF_W1 + MLP_H * MLP_F;  // [H]
constexpr int OFF_W2 = OFF_B1 + MLP_H;          // [H][H] (row = output unit)
constexpr int OFF_B2 = OFF_W2 + MLP_H * MLP_H;  // [H]
constexpr int OFF_W3 = OFF_B2 + MLP_H;          // [H]
constexpr int OFF_B3 = OFF_W3 + MLP_H;          // [1]
constexpr int MLP_NP = OFF_B3 + 1;              // 1377

struct dm_predictor {
  int device = -1;
  uint64_t uid = 0;           // identity for schedule caches
  uint64_t version = 0;       // bumped whenever the parameters change
  std::vector<float> params;  // host copy (authoritative between calls)
  uint64_t seed = 0;
  int steps = 0;
  std::vector<float> adam_m, adam_v;
};

namespace dmb {

static std::atomic<uint64_t> g_pred_uid{1};

// (identity, parameter version) of a predictor, the key of cached learned schedules.
void predictor_key(const void* pv, uint64_t* uid, uint64_t* version) {
  const dm_predictor* p = reinterpret_cast<const dm_predictor*>(pv);
  *uid = p->uid;
  *version = p->version;
}

// MLP forward of one feature row, parameters in shared memory.
__device__ __forceinline__ float mlp_eval(const float* sp, const float* x) {
  float h1[MLP_H];
#pragma unroll
  for (int h = 0; h < MLP_H; ++h) {
    float a = sp[OFF_B1 + h];
#pragma unroll
    for (int f = 0; f < MLP_F; ++f) a = fmaf(sp[OFF_W1 + h * MLP_F + f], x[f], a);
    h1[h] = fmaxf(a, 0.f);
  }
  float out = sp[OFF_B3];
  for (int h = 0; h < MLP_H; ++h) {
    float a = sp[OFF_B2 + h];
#pragma unroll
    for (int j = 0; j < MLP_H; ++j) a = fmaf(sp[OFF_W2 + h * MLP_H + j], h1[j], a);
    out = fmaf(sp[OFF_W3 + h], fmaxf(a, 0.f), out);
  }
  return out;
}

__global__ void mlp_forward_kernel(const float* __restrict__ P, const float* __restrict__ X, int n,
                                   float* __restrict__ y) {
  __shared__ float sp[MLP_NP];
  for (int i = threadIdx.x; i < MLP_NP; i += blockDim.x) sp[i] = P[i];
  __syncthreads();
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  float x[MLP_F];
#pragma unroll
  for (int f = 0; f < MLP_F; ++f) x[f] = X[(size_t)s * MLP_F + f];
  y[s] = mlp_eval(sp, x);
}

// Gradients of mean squared error over the samples idx[0..n) (or 0..n when idx is null).
// One block takes TB samples: each thread runs one sample forward and back to the
// pre-activation gradients, keeping inputs, activations and those gradients in shared
// memory; then the block reduces every parameter's gradient over its samples and adds it
// to `grad` (zeroed by the caller) with one atomic per parameter. loss_sum receives the sum
// of squared errors.
constexpr int TB = 128;
constexpr int ROW = MLP_F + 4 * MLP_H + 1;  // x | h1 | h2 | dz1 | dz2 | dy

__global__ void __launch_bounds__(TB) mlp_backward_kernel(const float* __restrict__ P, const float* __restrict__ X,
                                                          const float* __restrict__ T, const int* __restrict__ idx,
                                                          int n, float inv_n, float* __restrict__ grad,
                                                          float* __restrict__ loss_sum) {
  extern __shared__ float sm[];
  float* sp = sm;               // MLP_NP
  float* rows = sm + MLP_NP + 3;  // TB x ROW
  for (int i = threadIdx.x; i < MLP_NP; i += blockDim.x) sp[i] = P[i];
  __syncthreads();
  const int t = blockIdx.x * TB + threadIdx.x;
  float* r = rows + threadIdx.x * ROW;
  float* rx = r;
  float* rh1 = r + MLP_F;
  float* rh2 = rh1 + MLP_H;
  float* rd1 = rh2 + MLP_H;
  float* rd2 = rd1 + MLP_H;
  float sq = 0.f;
  if (t < n) {
    const int s = idx ? idx[t] : t;
#pragma unroll
    for (int f = 0; f < MLP_F; ++f) rx[f] = X[(size_t)s * MLP_F + f];
    for (int h = 0; h < MLP_H; ++h) {
      float a = sp[OFF_B1 + h];
#pragma unroll
      for (int f = 0; f < MLP_F; ++f) a = fmaf(sp[OFF_W1 + h * MLP_F + f], rx[f], a);
      rh1[h] = fmaxf(a, 0.f);
    }
    float out = sp[OFF_B3];
    for (int h = 0; h < MLP_H; ++h) {
      float a = sp[OFF_B2 + h];
      for (int j = 0; j < MLP_H; ++j) a = fmaf(sp[OFF_W2 + h * MLP_H + j], rh1[j], a);
      rh2[h] = fmaxf(a, 0.f);
      out = fmaf(sp[OFF_W3 + h], rh2[h], out);
    }
    const float err = out - T[s];
    sq = err * err;
    const float dy = 2.f * err * inv_n;
    r[ROW - 1] = dy;
    for (int h = 0; h < MLP_H; ++h) rd2[h] = rh2[h] > 0.f ? dy * sp[OFF_W3 + h] : 0.f;
    for (int j = 0; j < MLP_H; ++j) {
      float a = 0.f;
      for (int h = 0; h < MLP_H; ++h) a = fmaf(rd2[h], sp[OFF_W2 + h * MLP_H + j], a);
      rd1[j] = rh1[j] > 0.f ? a : 0.f;
    }
  } else {
    for (int i = 0; i < ROW; ++i) r[i] = 0.f;
  }
  for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
  if ((threadIdx.x & 31) == 0 && sq != 0.f) atomicAdd(loss_sum, sq);
  __syncthreads();
  // per-parameter reductions over the block's samples
  for (int i = threadIdx.x; i < MLP_NP; i += blockDim.x) {
    float acc = 0.f;
    if (i < OFF_B1) {  // W1[h][f] = sum dz1[h] x[f]
      const int h = i / MLP_F, f = i % MLP_F;
      for (int q = 0; q < TB; ++q) acc = fmaf(rows[q * ROW + MLP_F + 2 * MLP_H + h], rows[q * ROW + f], acc);
    } else if (i < OFF_W2) {  // b1[h] = sum dz1[h]
      const int h = i - OFF_B1;
      for (int q = 0; q < TB; ++q) acc += rows[q * ROW + MLP_F + 2 * MLP_H + h];
    } else if (i < OFF_B2) {  // W2[h][j] = sum dz2[h] h1[j]
      const int h = (i - OFF_W2) / MLP_H, j = (i - OFF_W2) % MLP_H;
      for (int q = 0; q < TB; ++q)
        acc = fmaf(rows[q * ROW + MLP_F + 3 * MLP_H + h], rows[q * ROW + MLP_F + j], acc);
    } else if (i < OFF_W3) {  // b2[h] = sum dz2[h]
      const int h = i - OFF_B2;
      for (int q = 0; q < TB; ++q) acc += rows[q * ROW + MLP_F + 3 * MLP_H + h];
    } else if (i < OFF_B3) {  // W3[h] = sum dy h2[h]
      const int h = i - OFF_W3;
      for (int q = 0; q < TB; ++q) acc = fmaf(rows[q * ROW + ROW - 1], rows[q * ROW + MLP_F + MLP_H + h], acc);
    } else {  // b3 = sum dy
      for (int q = 0; q < TB; ++q) acc += rows[q * ROW + ROW - 1];
    }
    if (acc != 0.f) atomicAdd(grad + i, acc);
  }
}

constexpr size_t BACKWARD_SMEM = sizeof(float) * (MLP_NP + 3 + TB * ROW);

__global__ void adam_kernel(float* __restrict__ P, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= MLP_NP) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  P[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

static int pred_device(int* dev) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return fail(DM_ENODEVICE, "no usable CUDA device");
  }
  DM_CUDA(cudaGetDevice(dev));
  return DM_OK;
}

// Batagelj-Zaversnik core decomposition, O(m).
static std::vector<int32_t> core_numbers(const dm_graph* g) {
  const int32_t n = g->n;
  std::vector<int32_t> deg(n), bin(g->max_degree + 2, 0), pos(n), vert(n);
  for (int32_t v = 0; v < n; ++v) {
    deg[v] = (int32_t)(g->row[v + 1] - g->row[v]);
    bin[deg[v]]++;
  }
  int32_t start = 0;
  for (int d = 0; d <= g->max_degree; ++d) {
    const int32_t num = bin[d];
    bin[d] = start;
    start += num;
  }
  for (int32_t v = 0; v < n; ++v) {
    pos[v] = bin[deg[v]];
    vert[pos[v]] = v;
    bin[deg[v]]++;
  }
  for (int d = g->max_degree; d >= 1; --d) bin[d] = bin[d - 1];
  bin[0] = 0;
  for (int32_t i = 0; i < n; ++i) {
    const int32_t v = vert[i];
    for (int64_t e = g->row[v]; e < g->row[v + 1]; ++e) {
      const int32_t u = g->adj[e];
      if (deg[u] > deg[v]) {
        const int32_t du = deg[u], pu = pos[u], pw = bin[du], w = vert[pw];
        if (u != w) {
          pos[u] = pw;
          vert[pu] = w;
          pos[w] = pu;
          vert[pw] = u;
        }
        bin[du]++;
        deg[u]--;
      }
    }
  }
  return deg;
}

constexpr int BASE_F = 6;  // f0 f1 f2 f5 f6 f7 per vertex; f3, f4 depend on k only

// Caches the k-independent features of every vertex. Counts triangles with the clique
// engine, so it must be called without the graph's mutex held.
int ensure_features(dm_graph* g, bool clique) {
  {
    std::lock_guard<std::mutex> lk(g->mu);
    ensure_oriented(g);
    if (!g->feat[clique ? 1 : 0].empty()) return DM_OK;
  }
  const int32_t n = g->n;
  std::vector<int32_t> core = core_numbers(g);
  // triangles per lowest-ranked vertex, counted by the clique engine (k = 3 subtree log)
  std::vector<uint64_t> tri(n, 0);
  {
    dm_opts o{};
    o.struct_size = sizeof(dm_opts);
    o.device = -1;
    o.subtree_counts = tri.data();
    uint64_t total = 0;
    int rc = dm_count_cliques(g, 3, &o, &total, nullptr);
    if (rc) return rc;
  }
  std::vector<float> F((size_t)n * BASE_F, 0.f);
  for (int32_t v = 0; v < n; ++v) {
    const int32_t deg = (int32_t)(g->row[v + 1] - g->row[v]);
    const int32_t r = g->rank[v];
    const int32_t outd = (int32_t)(g->orow[r + 1] - g->orow[r]);
    int32_t c0 = 0;
    double hop2 = 0;
    if (clique) {
      // C_0 = out-neighbours in the DAG; 2-hop size = their out-degrees
      c0 = outd;
      for (int64_t e = g->orow[r]; e < g->orow[r + 1]; ++e) {
        const int32_t ur = g->oadj[e];
        hop2 += (double)(g->orow[ur + 1] - g->orow[ur]);
      }
    } else {
      // C_0 = neighbours above v; 2-hop size = their degrees
      const int32_t* b = g->adj.data() + g->row[v];
      const int32_t* e = g->adj.data() + g->row[v + 1];
      const int32_t* s = std::upper_bound(b, e, v);
      c0 = (int32_t)(e - s);
      for (const int32_t* p = s; p < e; ++p) hop2 += (double)(g->row[*p + 1] - g->row[*p]);
    }
    float* x = F.data() + (size_t)v * BASE_F;
    x[0] = std::log1p((float)deg);
    x[1] = std::log1p((float)core[v]);
    x[2] = std::log1p((float)c0);
    x[3] = std::log1p((float)outd);
    x[4] = std::log1p((float)hop2);
    x[5] = std::log1p((float)tri[v]);
  }
  std::lock_guard<std::mutex> lk(g->mu);
  g->feat[clique ? 1 : 0].swap(F);
  return DM_OK;
}

// Full 8-feature row of vertex v for a k query from the cached base features.
static void feature_row(const dm_graph* g, bool clique, int k, int32_t v, float* x) {
  const float* b = g->feat[clique ? 1 : 0].data() + (size_t)v * BASE_F;
  x[0] = b[0];
  x[1] = b[1];
  x[2] = b[2];
  x[3] = k / 8.f;
  x[4] = (k - 2) / 8.f;
  x[5] = b[3];
  x[6] = b[4];
  x[7] = b[5];
}

static uint64_t g_pred_seed_mix(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// Runs inference for n feature rows on the current device.
static int predict_rows(const dm_predictor* p, const float* X, int64_t n, float* y) {
  if (n == 0) return DM_OK;
  float *dP = nullptr, *dX = nullptr, *dY = nullptr;
  DM_CUDA(cudaMalloc(&dP, sizeof(float) * MLP_NP));
  DM_CUDA(cudaMalloc(&dX, sizeof(float) * n * MLP_F));
  DM_CUDA(cudaMalloc(&dY, sizeof(float) * n));
  cudaMemcpy(dP, p->params.data(), sizeof(float) * MLP_NP, cudaMemcpyHostToDevice);
  cudaMemcpy(dX, X, sizeof(float) * n * MLP_F, cudaMemcpyHostToDevice);
  mlp_forward_kernel<<<(unsigned)((n + 255) / 256), 256>>>(dP, dX, (int)n, dY);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(y, dY, sizeof(float) * n, cudaMemcpyDeviceToHost);
  cudaFree(dP);
  cudaFree(dX);
  cudaFree(dY);
  if (e != cudaSuccess) return fail(DM_ECUDA, std::string("predictor inference failed: ") + cudaGetErrorString(e));
  return DM_OK;
}

// ---------------- the learned schedule on the device ----------------
//
// For the n_in root entries of a launch (the plain order, or one shard of it): the feature
// row of each root is assembled from the cached per-vertex base features, the MLP predicts
// log(1 + subtree size), and
//   cost = expm1(prediction) and a descending log-cost bucket (1/64 per bucket);
//   P = parts of the root: 1, or min(64, ceil(4 cost / share)) when the cost exceeds one
//       warp's share (total cost / warps);
//   the entries are written longest-first by a counting sort over the buckets (order inside
//   a bucket is arbitrary), each root as P consecutive entries (p | P << 16), flagged
//   PART_EAGER when its predicted cost is above EAGER_SHARE x share, so that the counting
//   kernel donates from it without waiting for the minimum task age.
// No allocation per call: the scratch lives in the caller's workspace.
constexpr int SCHED_BINS = 2048;
constexpr float EAGER_SHARE = 0.25f;

struct SchedArgs {
  const float* feat;        // n x BASE_F base features by original id
  const float* params;      // MLP_NP
  const int32_t* roots;     // n_in entries: rank space (cliques) or vertex ids (motifs)
  const int32_t* orig;      // rank -> original id (cliques), else null
  int n_in, k, warps, cap;
  float* cost;              // n_in
  int* bin;                 // n_in
  int* nparts;              // n_in
  double* total;            // 1
  unsigned* bins;           // SCHED_BINS
  int* n_out;               // 1
  int* err;                 // 1 (set when the output capacity would be exceeded)
  int32_t* out_roots;       // cap
  int32_t* out_parts;       // cap
  RootDesc* out_desc;       // cap, or null (cliques on the index)
  const int32_t* odeg;      // rank-space out-degrees (out_desc)
  const uint32_t* boff;     // index block offsets (out_desc)
};

__global__ void __launch_bounds__(256) sched_predict_kernel(SchedArgs a) {
  __shared__ float sp[MLP_NP];
  __shared__ double red[8];
  for (int i = threadIdx.x; i < MLP_NP; i += blockDim.x) sp[i] = a.params[i];
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double c = 0.0;
  if (i < a.n_in) {
    const int32_t r = a.roots[i];
    const int32_t v = a.orig ? a.orig[r] : r;
    const float* b = a.feat + (size_t)v * BASE_F;
    const float x[MLP_F] = {b[0], b[1], b[2], a.k / 8.f, (a.k - 2) / 8.f, b[3], b[4], b[5]};
    const float y = fminf(fmaxf(mlp_eval(sp, x), 0.f), 40.f);
    c = (double)expm1f(y);
    a.cost[i] = (float)c;
    a.bin[i] = SCHED_BINS - 1 - min(SCHED_BINS - 1, (int)(y * 64.f));
  }
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    atomicAdd(a.total, t);
  }
}

__global__ void __launch_bounds__(256) sched_parts_kernel(SchedArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n_in) return;
  const double share = *a.total / (double)max(1, a.warps);
  const double c = (double)a.cost[i];
  int P = 1;
  if (share > 0 && c > share) P = (int)fmin(64.0, ceil(4.0 * c / share));
  a.nparts[i] = P;
  atomicAdd(a.bins + a.bin[i], (unsigned)P);
}

// Exclusive scan of the bucket counts (one block of 1024 threads, two buckets per thread).
__global__ void __launch_bounds__(1024) sched_scan_kernel(SchedArgs a) {
  __shared__ unsigned part[1024];
  const int t = threadIdx.x;
  const unsigned c0 = a.bins[2 * t], c1 = a.bins[2 * t + 1];
  part[t] = c0 + c1;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    const unsigned y = t >= o ? part[t - o] : 0u;
    __syncthreads();
    part[t] += y;
    __syncthreads();
  }
  const unsigned excl = part[t] - (c0 + c1);
  a.bins[2 * t] = excl;
  a.bins[2 * t + 1] = excl + c0;
  if (t == 1023) *a.n_out = (int)part[t];
}

__global__ void __launch_bounds__(256) sched_scatter_kernel(SchedArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n_in) return;
  const int P = a.nparts[i];
  const unsigned pos = atomicAdd(a.bins + a.bin[i], (unsigned)P);
  if ((long long)pos + P > a.cap) {
    atomicExch(a.err, 1);
    return;
  }
  const int32_t r = a.roots[i];
  const double share = *a.total / (double)max(1, a.warps);
  const int eager = share > 0 && (double)a.cost[i] > EAGER_SHARE * share ? PART_EAGER : 0;
  for (int q = 0; q < P; ++q) {
    const int32_t pw = (P > 1 ? (q | (P << 16)) : 0) | eager;
    a.out_roots[pos + q] = r;
    a.out_parts[pos + q] = pw;
    if (a.out_desc) a.out_desc[pos + q] = RootDesc{r, a.odeg[r], a.boff ? a.boff[r] : INDEX_NONE, pw};
  }
}

// Runs the schedule of `in` (device root entries) on ctx.stream into the scratch `w`, and
// returns the number of output entries (a 4-byte read-back). Output capacity: n_in + 4 x
// warps + 64 entries (the parts of the roots above one share sum to at most 4 x warps +
// their count).
int learned_schedule_device(const void* pv, const SchedIO& io, LaunchCtx& ctx, int* n_out) {
  const dm_predictor* p = reinterpret_cast<const dm_predictor*>(pv);
  SchedArgs a;
  a.feat = io.feat;
  a.params = io.params;
  a.roots = io.roots;
  a.orig = io.orig;
  a.n_in = io.n_in;
  a.k = io.k;
  a.warps = io.warps;
  a.cap = io.cap;
  char* w = reinterpret_cast<char*>(io.scratch);
  auto take = [&](size_t bytes) {
    char* q = w;
    w += (bytes + 255) / 256 * 256;
    return q;
  };
  a.total = reinterpret_cast<double*>(take(sizeof(double)));
  a.n_out = reinterpret_cast<int*>(take(sizeof(int)));
  a.err = reinterpret_cast<int*>(take(sizeof(int)));
  a.bins = reinterpret_cast<unsigned*>(take(sizeof(unsigned) * SCHED_BINS));
  a.cost = reinterpret_cast<float*>(take(sizeof(float) * std::max(io.n_in, 1)));
  a.bin = reinterpret_cast<int*>(take(sizeof(int) * std::max(io.n_in, 1)));
  a.nparts = reinterpret_cast<int*>(take(sizeof(int) * std::max(io.n_in, 1)));
  a.out_roots = io.out_roots;
  a.out_parts = io.out_parts;
  a.out_desc = io.out_desc;
  a.odeg = io.odeg;
  a.boff = io.boff;
  // the scratch header (total, n_out, err, bins) starts at zero
  DM_CUDA(cudaMemsetAsync(io.scratch, 0, (size_t)(reinterpret_cast<char*>(a.cost) - reinterpret_cast<char*>(io.scratch)),
                          ctx.stream));
  if (!io.params_current)
    DM_CUDA(cudaMemcpyAsync(io.params, p->params.data(), sizeof(float) * MLP_NP, cudaMemcpyHostToDevice,
                            ctx.stream));
  const unsigned grid = (unsigned)std::max(1, (io.n_in + 255) / 256);
  sched_predict_kernel<<<grid, 256, 0, ctx.stream>>>(a);
  sched_parts_kernel<<<grid, 256, 0, ctx.stream>>>(a);
  sched_scan_kernel<<<1, 1024, 0, ctx.stream>>>(a);
  sched_scatter_kernel<<<grid, 256, 0, ctx.stream>>>(a);
  ctx.launches += 4;
  DM_CUDA(cudaGetLastError());
  // the task count and the error flag, through a page-locked pair (asynchronous copies)
  int* hdr = io.h_hdr;
  DM_CUDA(cudaMemcpyAsync(&hdr[0], a.n_out, sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
  DM_CUDA(cudaMemcpyAsync(&hdr[1], a.err, sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
  DM_CUDA(cudaStreamSynchronize(ctx.stream));
  if (hdr[1]) return fail(DM_EINTERNAL, "learned schedule exceeded its output capacity");
  *n_out = hdr[0];
  return DM_OK;
}

int predictor_num_params() { return MLP_NP; }

size_t learned_schedule_scratch_bytes(int n_in) {
  const size_t n = (size_t)std::max(n_in, 1);
  return 4 * 256 + (sizeof(unsigned) * SCHED_BINS + 255) / 256 * 256 + 3 * ((n * 4 + 255) / 256 * 256);
}

// Host version of the same schedule, for planning (dm_plan_roots): same costs, parts and
// flags, with ties inside a bucket in input order.
int predictor_schedule(const void* pv, dm_graph* g, int k, bool clique, int total_warps, std::vector<int32_t>& roots,
                       std::vector<int32_t>& parts) {
  const dm_predictor* p = reinterpret_cast<const dm_predictor*>(pv);
  if (g->feat[clique ? 1 : 0].empty()) return fail(DM_EINVAL, "predictor features were not prepared");
  int rc = DM_OK;
  // features are per original vertex; clique roots arrive in rank space
  std::vector<int32_t> orig(roots.size());
  if (clique) {
    std::vector<int32_t> inv(g->n);
    for (int32_t v = 0; v < g->n; ++v) inv[g->rank[v]] = v;
    for (size_t i = 0; i < roots.size(); ++i) orig[i] = inv[roots[i]];
  } else {
    orig = roots;
  }
  std::vector<float> Xr(roots.size() * MLP_F);
  for (size_t i = 0; i < roots.size(); ++i) feature_row(g, clique, k, orig[i], Xr.data() + i * MLP_F);
  std::vector<float> pred(roots.size());
  if ((rc = predict_rows(p, Xr.data(), (int64_t)roots.size(), pred.data()))) return rc;
  std::vector<double> cost(roots.size());
  std::vector<int> bin(roots.size());
  double total = 0;
  for (size_t i = 0; i < roots.size(); ++i) {
    const float y = std::min(std::max(pred[i], 0.f), 40.f);
    cost[i] = (double)std::expm1(y);
    bin[i] = SCHED_BINS - 1 - std::min(SCHED_BINS - 1, (int)(y * 64.f));
    total += cost[i];
  }
  std::vector<size_t> order(roots.size());
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return bin[a] < bin[b]; });
  const double share = total / std::max(1, total_warps);
  std::vector<int32_t> out_roots, out_parts;
  out_roots.reserve(roots.size());
  out_parts.reserve(roots.size());
  for (size_t i : order) {
    int P = 1;
    if (share > 0 && cost[i] > share) P = (int)std::min<double>(64.0, std::ceil(4.0 * cost[i] / share));
    const int eager = share > 0 && cost[i] > EAGER_SHARE * share ? PART_EAGER : 0;
    for (int q = 0; q < P; ++q) {
      out_roots.push_back(roots[i]);
      out_parts.push_back((P > 1 ? (q | (P << 16)) : 0) | eager);
    }
  }
  roots.swap(out_roots);
  parts.swap(out_parts);
  return DM_OK;
}

}  // namespace dmb

using namespace dmb;

extern "C" {

int dm_predictor_create(uint64_t seed, dm_predictor** out) {
  if (!out) return fail(DM_EINVAL, "dm_predictor_create: null argument");
  auto* p = new dm_predictor();
  p->uid = g_pred_uid++;
  p->seed = seed;
  p->params.assign(MLP_NP, 0.f);
  // He-uniform initialisation from a splitmix stream
  uint64_t s = seed;
  auto uni = [&]() {
    s = g_pred_seed_mix(s);
    return (float)((s >> 11) * (1.0 / 9007199254740992.0)) * 2.f - 1.f;
  };
  const float a1 = std::sqrt(6.f / MLP_F), a2 = std::sqrt(6.f / MLP_H);
  for (int i = 0; i < MLP_H * MLP_F; ++i) p->params[OFF_W1 + i] = a1 * uni();
  for (int i = 0; i < MLP_H * MLP_H; ++i) p->params[OFF_W2 + i] = a2 * uni();
  for (int i = 0; i < MLP_H; ++i) p->params[OFF_W3 + i] = a2 * uni() * 0.5f;
  for (int i = 0; i < MLP_H; ++i) p->params[OFF_B1 + i] = 0.01f;
  for (int i = 0; i < MLP_H; ++i) p->params[OFF_B2 + i] = 0.01f;
  p->adam_m.assign(MLP_NP, 0.f);
  p->adam_v.assign(MLP_NP, 0.f);
  *out = p;
  return DM_OK;
}

void dm_predictor_free(dm_predictor* p) { delete p; }

int dm_predictor_num_params(void) { return MLP_NP; }

int dm_predictor_get_params(const dm_predictor* p, float* params) {
  if (!p || !params) return fail(DM_EINVAL, "dm_predictor_get_params: null argument");
  std::memcpy(params, p->params.data(), sizeof(float) * MLP_NP);
  return DM_OK;
}

int dm_predictor_set_params(dm_predictor* p, const float* params) {
  if (!p || !params) return fail(DM_EINVAL, "dm_predictor_set_params: null argument");
  std::memcpy(p->params.data(), params, sizeof(float) * MLP_NP);
  ++p->version;
  return DM_OK;
}

int dm_predictor_features(dm_graph* g, int32_t k, int32_t clique, float* features) {
  if (!g || !features) return fail(DM_EINVAL, "dm_predictor_features: null argument");
  if (k < 2 || k > 12) return fail(DM_EINVAL, "dm_predictor_features: k out of range");
  int rc = ensure_features(g, clique != 0);
  if (rc) return rc;
  for (int32_t v = 0; v < g->n; ++v) feature_row(g, clique != 0, k, v, features + (size_t)v * MLP_F);
  return DM_OK;
}

int dm_predictor_predict(const dm_predictor* p, const float* X, int64_t n, float* y) {
  if (!p || (n && (!X || !y)) || n < 0) return fail(DM_EINVAL, "dm_predictor_predict: bad arguments");
  int dev = 0;
  int rc = pred_device(&dev);
  if (rc) return rc;
  return predict_rows(p, X, n, y);
}

// One full-batch gradient of the mean squared error (for checking against a CPU model).
int dm_predictor_gradients(const dm_predictor* p, const float* X, const float* T, int64_t n, float* grad,
                           float* loss) {
  if (!p || !X || !T || !grad || n <= 0) return fail(DM_EINVAL, "dm_predictor_gradients: bad arguments");
  int dev = 0;
  int rc = pred_device(&dev);
  if (rc) return rc;
  float *dP, *dX, *dT, *dG, *dL;
  DM_CUDA(cudaMalloc(&dP, sizeof(float) * MLP_NP));
  DM_CUDA(cudaMalloc(&dX, sizeof(float) * n * MLP_F));
  DM_CUDA(cudaMalloc(&dT, sizeof(float) * n));
  DM_CUDA(cudaMalloc(&dG, sizeof(float) * MLP_NP));
  DM_CUDA(cudaMalloc(&dL, sizeof(float)));
  cudaMemcpy(dP, p->params.data(), sizeof(float) * MLP_NP, cudaMemcpyHostToDevice);
  cudaMemcpy(dX, X, sizeof(float) * n * MLP_F, cudaMemcpyHostToDevice);
  cudaMemcpy(dT, T, sizeof(float) * n, cudaMemcpyHostToDevice);
  cudaMemset(dG, 0, sizeof(float) * MLP_NP);
  cudaMemset(dL, 0, sizeof(float));
  cudaFuncSetAttribute(mlp_backward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)BACKWARD_SMEM);
  mlp_backward_kernel<<<(unsigned)((n + TB - 1) / TB), TB, BACKWARD_SMEM>>>(dP, dX, dT, nullptr, (int)n,
                                                                          1.f / (float)n, dG, dL);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(grad, dG, sizeof(float) * MLP_NP, cudaMemcpyDeviceToHost);
  float ls = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&ls, dL, sizeof(float), cudaMemcpyDeviceToHost);
  cudaFree(dP);
  cudaFree(dX);
  cudaFree(dT);
  cudaFree(dG);
  cudaFree(dL);
  if (e != cudaSuccess) return fail(DM_ECUDA, std::string("predictor gradients failed: ") + cudaGetErrorString(e));
  if (loss) *loss = ls / (float)n;
  return DM_OK;
}

// Adam on minibatches for `epochs` passes over (X, T); writes the final epoch's mean loss.
int dm_predictor_train(dm_predictor* p, const float* X, const float* T, int64_t n, int32_t epochs, int32_t batch,
                       float lr, float* final_loss) {
  if (!p || !X || !T || n <= 0 || epochs <= 0 || batch <= 0 || !(lr > 0))
    return fail(DM_EINVAL, "dm_predictor_train: bad arguments");
  int dev = 0;
  int rc = pred_device(&dev);
  if (rc) return rc;
  float *dP, *dX, *dT, *dG, *dL, *dM, *dV;
  int* dIdx;
  DM_CUDA(cudaMalloc(&dP, sizeof(float) * MLP_NP));
  DM_CUDA(cudaMalloc(&dX, sizeof(float) * n * MLP_F));
  DM_CUDA(cudaMalloc(&dT, sizeof(float) * n));
  DM_CUDA(cudaMalloc(&dG, sizeof(float) * MLP_NP));
  DM_CUDA(cudaMalloc(&dL, sizeof(float)));
  DM_CUDA(cudaMalloc(&dM, sizeof(float) * MLP_NP));
  DM_CUDA(cudaMalloc(&dV, sizeof(float) * MLP_NP));
  DM_CUDA(cudaMalloc(&dIdx, sizeof(int) * n));
  cudaMemcpy(dP, p->params.data(), sizeof(float) * MLP_NP, cudaMemcpyHostToDevice);
  cudaMemcpy(dM, p->adam_m.data(), sizeof(float) * MLP_NP, cudaMemcpyHostToDevice);
  cudaMemcpy(dV, p->adam_v.data(), sizeof(float) * MLP_NP, cudaMemcpyHostToDevice);
  cudaMemcpy(dX, X, sizeof(float) * n * MLP_F, cudaMemcpyHostToDevice);
  cudaMemcpy(dT, T, sizeof(float) * n, cudaMemcpyHostToDevice);
  cudaFuncSetAttribute(mlp_backward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)BACKWARD_SMEM);
  std::vector<int> idx(n);
  std::iota(idx.begin(), idx.end(), 0);
  uint64_t s = p->seed ^ 0x5DEECE66Dull;
  double last = 0;
  const float b1 = 0.9f, b2 = 0.999f;
  for (int ep = 0; ep < epochs; ++ep) {
    for (int64_t i = n - 1; i > 0; --i) {
      s = g_pred_seed_mix(s);
      std::swap(idx[i], idx[s % (uint64_t)(i + 1)]);
    }
    cudaMemcpy(dIdx, idx.data(), sizeof(int) * n, cudaMemcpyHostToDevice);
    cudaMemset(dL, 0, sizeof(float));
    for (int64_t off = 0; off < n; off += batch) {
      const int bn = (int)std::min<int64_t>(batch, n - off);
      cudaMemsetAsync(dG, 0, sizeof(float) * MLP_NP);
      mlp_backward_kernel<<<(bn + TB - 1) / TB, TB, BACKWARD_SMEM>>>(dP, dX, dT, dIdx + off, bn, 1.f / (float)bn,
                                                                     dG, dL);
      ++p->steps;
      const float c1 = 1.f - std::pow(b1, (float)p->steps), c2 = 1.f - std::pow(b2, (float)p->steps);
      adam_kernel<<<(MLP_NP + 255) / 256, 256>>>(dP, dG, dM, dV, lr, b1, b2, 1e-8f, c1, c2);
    }
    float ls = 0;
    cudaMemcpy(&ls, dL, sizeof(float), cudaMemcpyDeviceToHost);
    last = ls / (double)n;
  }
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(p->params.data(), dP, sizeof(float) * MLP_NP, cudaMemcpyDeviceToHost);
  ++p->version;
  if (e == cudaSuccess) e = cudaMemcpy(p->adam_m.data(), dM, sizeof(float) * MLP_NP, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(p->adam_v.data(), dV, sizeof(float) * MLP_NP, cudaMemcpyDeviceToHost);
  cudaFree(dP);
  cudaFree(dX);
  cudaFree(dT);
  cudaFree(dG);
  cudaFree(dL);
  cudaFree(dM);
  cudaFree(dV);
  cudaFree(dIdx);
  if (e != cudaSuccess) return fail(DM_ECUDA, std::string("predictor training failed: ") + cudaGetErrorString(e));
  if (final_loss) *final_loss = (float)last;
  return DM_OK;
}

}  // extern "C"
