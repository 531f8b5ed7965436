// Internal warp-level helpers of the enumeration kernels. The public step library (extend,
// filter, compact, aggregate; include/dumato_b200_gpm.cuh) is included here; the helpers
// below add explicit-mask forms used where a group mask is already at hand.
//
//   compact  - stable warp stream compaction by ballot + popc: the valid lanes of a 32-wide
//              chunk land in lane order at the list tail (DuMatoGPU.cu:317-343 write /
//              write_twice; the invalid lanes are not written here, the list tail is the
//              only thing that matters to the callers).
//   contains - membership of a value in a sorted list (binary search; the reference's
//              findMany / findOne, DuMatoGPU.cu:263-278, scan linearly).
//   pop_lowest - remove and return the lowest set bit of a warp-distributed bitset.
//
// Virtual warps (src/DM_WCV/DuMatoGPU.cu:12-37) are expressed with an explicit group
// width G and lane mask; every collective below takes the group mask.
#pragma once

#include <cstdint>

#include "dumato_b200_gpm.cuh"

namespace dmb {

constexpr unsigned FULL_MASK = 0xffffffffu;

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }
__device__ __forceinline__ int warp_in_block() { return threadIdx.x >> 5; }

// Appends the valid lanes' values at list[base ...] in lane order; returns how many.
__device__ __forceinline__ int compact(int32_t* list, int base, int32_t value, bool valid,
                                       unsigned mask = FULL_MASK) {
  unsigned b = __ballot_sync(mask, valid);
  if (valid) list[base + __popc(b & ((1u << lane_id()) - 1u))] = value;
  return __popc(b);
}

// Same, writing a second parallel array (value + its source tag / adjacency mask).
template <typename T2>
__device__ __forceinline__ int compact2(int32_t* list, T2* list2, int base, int32_t v1, T2 v2, bool valid,
                                        unsigned mask = FULL_MASK) {
  unsigned b = __ballot_sync(mask, valid);
  if (valid) {
    int p = base + __popc(b & ((1u << lane_id()) - 1u));
    list[p] = v1;
    list2[p] = v2;
  }
  return __popc(b);
}

// Lower bound of x in sorted a[lo, hi).
__device__ __forceinline__ int lower_bound(const int32_t* a, int lo, int hi, int32_t x) {
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (a[mid] < x) lo = mid + 1; else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ bool contains(const int32_t* a, int n, int32_t x) {
  int p = lower_bound(a, 0, n, x);
  return p < n && a[p] == x;
}

// Read-only 128-bit load through the non-coherent path.
__device__ __forceinline__ int4 ldg4(const int32_t* p) { return __ldg(reinterpret_cast<const int4*>(p)); }

// Warp-distributed bitset: lane l holds word l (32 bits). Removes and returns the lowest
// set bit, or -1 when empty. Warp-uniform.
__device__ __forceinline__ int pop_lowest(uint32_t& word) {
  unsigned nz = __ballot_sync(FULL_MASK, word != 0);
  if (!nz) return -1;
  int owner = __ffs(nz) - 1;
  int bit = 0;
  if (lane_id() == owner) {
    bit = __ffs(word) - 1;
    word &= word - 1;
  }
  bit = __shfl_sync(FULL_MASK, bit, owner);
  return owner * 32 + bit;
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(FULL_MASK, v, o);
  return v;
}

}  // namespace dmb
