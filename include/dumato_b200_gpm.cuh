/*
 * dumato_b200_gpm.cuh - the device-level GPM step library of dumato_b200 (sm_100a).
 *
 * The warp-level building blocks the library's enumeration kernels are written in, for
 * users who write their own pattern kernels on the same primitives. They replace the
 * reference's DuMatoGPU device API (src/main/DuMatoGPU.cu), one step per function:
 *
 *   compact / compact2      write, write_twice (DuMatoGPU.cu:317-343): stable stream
 *                           compaction of a chunk of W lanes by ballot + popc
 *   contains                findMany / findOne (DuMatoGPU.cu:263-278) as a binary search
 *                           over a sorted list (the reference scans linearly)
 *   filter                  filterClique (DuMatoGPU.cu:1747-1767): keep the members of a list
 *                           that satisfy a predicate, in order
 *   extend_intersect        extend_clique (DuMatoGPU.cu:1194-1220): the sorted intersection of
 *                           a candidate list with an adjacency list, by merge or by probe
 *   intersect_count         the last level of extend_clique + aggregate_counter: the size of
 *                           the intersection, nothing written
 *   aggregate_counter       aggregate_counter (DuMatoGPU.cu:1769-1771): one atomic per group
 *   aggregate_pattern       aggregate_pattern (DuMatoGPU.cu:930-967): a histogram add that
 *                           merges equal keys of a chunk with __match_any_sync first
 *
 * Every function is executed by all W lanes of a virtual warp (W = 8, 16 or 32 lanes of one
 * hardware warp, src/DM_WCV/DuMatoGPU.cu:12-37); Group<W> gives the lane index and mask.
 * Lists are int32 vertex ids sorted ascending; outputs are written in input order.
 */
#ifndef DUMATO_B200_GPM_CUH
#define DUMATO_B200_GPM_CUH

#include <cstdint>

namespace dm_gpm {

// A virtual warp of W lanes inside a 32-lane warp.
template <int W>
struct Group {
  static_assert(W == 8 || W == 16 || W == 32, "virtual warps are 8, 16 or 32 lanes wide");
  __device__ static __forceinline__ int lane() { return threadIdx.x & (W - 1); }
  __device__ static __forceinline__ int index() { return (threadIdx.x & 31) / W; }
  __device__ static __forceinline__ unsigned mask() {
    return W == 32 ? 0xffffffffu : (((1u << W) - 1u) << (((threadIdx.x & 31) / W) * W));
  }
  // lanes of this group below the calling lane
  __device__ static __forceinline__ unsigned below() {
    return mask() & ((1u << (threadIdx.x & 31)) - 1u);
  }
};

// Appends the valid lanes' values at list[base ...] in lane order; returns how many.
template <int W>
__device__ __forceinline__ int compact(int32_t* list, int base, int32_t value, bool valid) {
  const unsigned b = __ballot_sync(Group<W>::mask(), valid);
  if (valid) list[base + __popc(b & Group<W>::below())] = value;
  return __popc(b);
}

// Same, writing a second parallel array.
template <int W, typename T2>
__device__ __forceinline__ int compact2(int32_t* list, T2* list2, int base, int32_t v1, T2 v2, bool valid) {
  const unsigned b = __ballot_sync(Group<W>::mask(), valid);
  if (valid) {
    const int p = base + __popc(b & Group<W>::below());
    list[p] = v1;
    list2[p] = v2;
  }
  return __popc(b);
}

// First position in a[lo, hi) holding a value >= x.
__device__ __forceinline__ int lower_bound(const int32_t* a, int lo, int hi, int32_t x) {
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (a[mid] < x) lo = mid + 1; else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ bool contains(const int32_t* a, int n, int32_t x) {
  const int p = lower_bound(a, 0, n, x);
  return p < n && a[p] == x;
}

// out = the members of in[0, n) for which pred(x) holds, in order; returns how many.
template <int W, typename Pred>
__device__ __forceinline__ int filter(const int32_t* in, int n, int32_t* out, Pred pred) {
  int m = 0;
  for (int i0 = 0; i0 < n; i0 += W) {
    const int i = i0 + Group<W>::lane();
    const int32_t x = i < n ? in[i] : 0;
    m += compact<W>(out, m, x, i < n && pred(x));
  }
  return m;
}

// Slice of A owned by group lane l in a merge: [l*s, min((l+1)*s, na)), s = ceil(na / W).
template <int W>
__device__ __forceinline__ void merge_slice(int na, int& i0, int& i1) {
  const int s = (na + W - 1) / W;
  i0 = min(na, Group<W>::lane() * s);
  i1 = min(na, i0 + s);
}

// Matches of A[i0, i1) in B, merged sequentially from the first member of B >= A[i0].
// With out, writes them at out[pos ...]; returns how many.
__device__ __forceinline__ int merge_run(const int32_t* A, int i0, int i1, const int32_t* B, int nb,
                                         int32_t* out, int pos) {
  if (i0 >= i1) return 0;
  int j = lower_bound(B, 0, nb, A[i0]);
  int i = i0, m = 0;
  while (i < i1 && j < nb) {
    const int32_t a = A[i], b = B[j];
    if (a == b) {
      if (out) out[pos + m] = a;
      ++m;
      ++i;
      ++j;
    } else if (a < b) {
      ++i;
    } else {
      ++j;
    }
  }
  return m;
}

// Merge when the lists are of comparable size, probe (a binary search of every member of A
// in B) when B is much longer.
__device__ __forceinline__ bool use_merge(int na, int nb) { return nb <= 8 * na; }

// out = A cap B (both sorted ascending), in order; returns |out| (all lanes).
template <int W>
__device__ __forceinline__ int extend_intersect(const int32_t* A, int na, const int32_t* B, int nb, int32_t* out) {
  if (!use_merge(na, nb)) return filter<W>(A, na, out, [&](int32_t x) { return contains(B, nb, x); });
  int i0, i1;
  merge_slice<W>(na, i0, i1);
  const int mine = merge_run(A, i0, i1, B, nb, nullptr, 0);
  // exclusive prefix of the per-lane counts within the group
  int incl = mine;
#pragma unroll
  for (int o = 1; o < W; o <<= 1) {
    const int y = __shfl_up_sync(Group<W>::mask(), incl, o, W);
    if (Group<W>::lane() >= o) incl += y;
  }
  merge_run(A, i0, i1, B, nb, out, incl - mine);
  return __shfl_sync(Group<W>::mask(), incl, W - 1, W);
}

// |A cap B| (all lanes), nothing written.
template <int W>
__device__ __forceinline__ int intersect_count(const int32_t* A, int na, const int32_t* B, int nb) {
  int mine = 0;
  if (!use_merge(na, nb)) {
    for (int i = Group<W>::lane(); i < na; i += W) mine += contains(B, nb, A[i]) ? 1 : 0;
  } else {
    int i0, i1;
    merge_slice<W>(na, i0, i1);
    mine = merge_run(A, i0, i1, B, nb, nullptr, 0);
  }
#pragma unroll
  for (int o = W / 2; o > 0; o >>= 1) mine += __shfl_xor_sync(Group<W>::mask(), mine, o, W);
  return mine;
}

// Adds the group's per-lane counts to *total with one atomic.
template <int W>
__device__ __forceinline__ void aggregate_counter(unsigned long long* total, unsigned long long v) {
#pragma unroll
  for (int o = W / 2; o > 0; o >>= 1) v += __shfl_xor_sync(Group<W>::mask(), v, o, W);
  if (Group<W>::lane() == 0 && v) atomicAdd(total, v);
}

// hist[key] += 1 for every valid lane, with one atomic per distinct key of the chunk.
template <int W>
__device__ __forceinline__ void aggregate_pattern(unsigned* hist, int key, bool valid) {
  const unsigned gm = Group<W>::mask();
  const unsigned act = __ballot_sync(gm, valid);
  const unsigned same = __match_any_sync(gm, valid ? key : -1);
  if (valid && (same & act & Group<W>::below()) == 0) atomicAdd(hist + key, (unsigned)__popc(same & act));
}

}  // namespace dm_gpm

#endif  // DUMATO_B200_GPM_CUH
