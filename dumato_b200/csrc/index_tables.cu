// Per-root tables of the clique index, built on the device: the block offsets (an exclusive
// scan of each root's block size in 16-byte units) and the plain task list (RootDesc entries
// in descending out-degree order, roots of 20..64 out-neighbours as index_split_parts
// entries). Uploading them instead would copy 20 bytes per vertex, and 16 more per extra
// part, on every re-upload of a graph.
#include <cuda_runtime.h>

#include <cub/device/device_scan.cuh>

#include "engine.hpp"

namespace dmb {

namespace {

__global__ void index_units_kernel(const int32_t* __restrict__ odeg, int n, uint32_t* __restrict__ units) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < n) {
    const int d = odeg[r];
    units[r] = (d >= 2 && d <= INDEX_MAX_DEGREE) ? index_block_units_host(d) : 0u;
  }
}

__global__ void index_boff_kernel(const uint32_t* __restrict__ units, const uint32_t* __restrict__ scan, int n,
                                  uint32_t* __restrict__ boff) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < n) boff[r] = units[r] ? scan[r] : INDEX_NONE;
}

__global__ void index_parts_kernel(const int32_t* __restrict__ deg_order, const int32_t* __restrict__ odeg, int n,
                                   uint32_t* __restrict__ parts) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) parts[i] = (uint32_t)index_split_parts(odeg[deg_order[i]]);
}

__global__ void index_desc_kernel(const int32_t* __restrict__ deg_order, const int32_t* __restrict__ odeg,
                                  const uint32_t* __restrict__ boff, const uint32_t* __restrict__ parts,
                                  const uint32_t* __restrict__ first, int n, RootDesc* __restrict__ desc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int r = deg_order[i];
  const int P = (int)parts[i];
  const uint32_t at = first[i];
  for (int q = 0; q < P; ++q) desc[at + q] = RootDesc{r, odeg[r], boff[r], P > 1 ? (q | (P << 16)) : 0};
}

// scratch: units | scan | parts | first (n words each, 256-byte aligned) | cub temporary
size_t words_bytes(int n) { return ((size_t)(n > 0 ? n : 1) * sizeof(uint32_t) + 255) / 256 * 256; }

size_t cub_bytes(int n) {
  size_t b = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, b, (const uint32_t*)nullptr, (uint32_t*)nullptr, n > 0 ? n : 1);
  return (b + 255) / 256 * 256;
}

}  // namespace

size_t index_tables_tmp_bytes(int n) { return 4 * words_bytes(n) + cub_bytes(n); }

int index_tables_build(const int32_t* odeg, const int32_t* deg_order, int n, uint32_t* boff, RootDesc* desc,
                       void* tmp, size_t tmp_bytes, LaunchCtx& ctx) {
  if (n <= 0) return DM_OK;
  if (tmp_bytes < index_tables_tmp_bytes(n)) return fail(DM_EINTERNAL, "index tables: scratch too small");
  char* w = static_cast<char*>(tmp);
  uint32_t* units = reinterpret_cast<uint32_t*>(w);
  uint32_t* scan = reinterpret_cast<uint32_t*>(w + words_bytes(n));
  uint32_t* parts = reinterpret_cast<uint32_t*>(w + 2 * words_bytes(n));
  uint32_t* first = reinterpret_cast<uint32_t*>(w + 3 * words_bytes(n));
  void* cub_tmp = w + 4 * words_bytes(n);
  size_t cb = cub_bytes(n);
  const int grid = (n + 255) / 256;
  index_units_kernel<<<grid, 256, 0, ctx.stream>>>(odeg, n, units);
  DM_CUDA(cub::DeviceScan::ExclusiveSum(cub_tmp, cb, units, scan, n, ctx.stream));
  index_boff_kernel<<<grid, 256, 0, ctx.stream>>>(units, scan, n, boff);
  index_parts_kernel<<<grid, 256, 0, ctx.stream>>>(deg_order, odeg, n, parts);
  cb = cub_bytes(n);
  DM_CUDA(cub::DeviceScan::ExclusiveSum(cub_tmp, cb, parts, first, n, ctx.stream));
  index_desc_kernel<<<grid, 256, 0, ctx.stream>>>(deg_order, odeg, boff, parts, first, n, desc);
  ctx.launches += 4;  // and two library scans
  DM_CUDA(cudaGetLastError());
  return DM_OK;
}

}  // namespace dmb
