// Warp-cooperative sorted-set primitives on int32 lists (all 32 lanes must call them
// converged; results are warp-uniform).
//
// Semantics follow the reference templates:
//   intersect / intersect_num with an optional strict upper bound and excluded ids
//     (include/set_intersect.cuh:107-115, 190-195, 352-360, 430-472, 474-507);
//   difference_set / difference_num: A \ B with lookup list A (A is not swapped), an
//     optional upper bound and one excluded id (include/set_difference.cuh:41-48, 96-102,
//     163-170, 239-245; VertexSet::difference_buf excludes other.vid, common/VertexSet.cc:21).
// Materialised outputs are in ascending order, compacted with __ballot_sync/__popc.
//
// Two intersection strategies, chosen by the length ratio of the operands (bounded
// prefixes):
//   * search: each lane takes keys of the shorter list and binary-searches the longer one
//     (the reference's only active path, include/search.cuh:31-48);
//   * merge-path: the merged sequence A' ++ B' is cut into 32 equal diagonals, each lane
//     finds its cut by a binary search along its diagonal and merges its segment
//     sequentially (Green, McColl, Bader, "GPU merge path", ICS 2012).  The reference kept
//     a merge variant only as disabled code (include/set_intersect.cuh:110-111).
#pragma once
#include <stdint.h>

namespace jgpm {

constexpr unsigned kFull = 0xffffffffu;

// Programmatic dependent launch between kernels of one count that share nothing but atomic
// result adds: pdl_open lets the next kernel (launched with programmatic stream serialization)
// start once every CTA of this one has started, so its CTAs fill the SMs this kernel's last CTAs
// leave idle; pdl_close, at the end of every CTA, waits for the previous kernel to complete, so
// a kernel completes only after all earlier ones.  Without the launch attribute both are no-ops
// in effect.  A kernel launches only after all CTAs of its predecessor have started, so the CTAs
// a wait depends on are resident and the wait always ends.
__device__ __forceinline__ void pdl_open() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
__device__ __forceinline__ void pdl_close() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

__device__ __forceinline__ int lower_bound_g(const int32_t* a, int n, int32_t key) {
  int lo = 0, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (__ldg(a + mid) < key) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ int upper_bound_g(const int32_t* a, int n, int32_t key) {
  int lo = 0, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (__ldg(a + mid) <= key) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ bool contains_g(const int32_t* a, int n, int32_t key) {
  int p = lower_bound_g(a, n, key);
  return p < n && __ldg(a + p) == key;
}

__device__ __forceinline__ int warp_sum_int(int v) {
  return __reduce_add_sync(kFull, (unsigned)v);
}

// Prefix of a sorted list below `upper` (warp-uniform; computed by lane 0 and broadcast).
__device__ __forceinline__ int warp_prefix_below(const int32_t* a, int n, int32_t upper) {
  if (upper == INT32_MAX || n == 0) return n;
  int p = 0;
  if ((threadIdx.x & 31) == 0) p = lower_bound_g(a, n, upper);
  return __shfl_sync(kFull, p, 0);
}

// Merge-path split: number of elements taken from A among the first `diag` of the merge of
// A (length na) and B (length nb), ties taken from A first.
__device__ __forceinline__ int merge_path_split(const int32_t* a, int na, const int32_t* b,
                                                int nb, int diag) {
  int lo = diag > nb ? diag - nb : 0;
  int hi = diag < na ? diag : na;
  while (lo < hi) {
    int i = (lo + hi) >> 1;  // i from A, diag-1-i from B
    if (__ldg(a + i) <= __ldg(b + diag - 1 - i)) lo = i + 1;
    else hi = i;
  }
  return lo;
}

// Counts matches in the lane's merge-path segment [d0, d1) of the merge of A and B.  A match
// is counted at the position where its A copy is consumed.  `excl*` ids are skipped.
__device__ __forceinline__ int merge_segment_count(const int32_t* a, int na, const int32_t* b,
                                                   int nb, int d0, int d1, int32_t ex0,
                                                   int32_t ex1) {
  int i = merge_path_split(a, na, b, nb, d0);
  int j = d0 - i;
  int c = 0;
  for (int d = d0; d < d1; ++d) {
    int32_t x = i < na ? __ldg(a + i) : INT32_MAX;
    int32_t y = j < nb ? __ldg(b + j) : INT32_MAX;
    if (i < na && (j >= nb || x <= y)) {
      // consuming A[i]; it matches iff B has it at j (ties take A first)
      if (j < nb && x == y && x != ex0 && x != ex1) ++c;
      ++i;
    } else {
      ++j;
    }
  }
  return c;
}

// |{x in A & B : x < upper, x not in {ex0, ex1}}| -- warp-uniform result.
__device__ __forceinline__ int warp_intersect_count(const int32_t* a, int na, const int32_t* b,
                                                    int nb, int32_t upper = INT32_MAX,
                                                    int32_t ex0 = -1, int32_t ex1 = -1) {
  const int lane = threadIdx.x & 31;
  na = warp_prefix_below(a, na, upper);
  nb = warp_prefix_below(b, nb, upper);
  if (na == 0 || nb == 0) return 0;
  if (na > nb) {
    const int32_t* t = a; a = b; b = t;
    int tn = na; na = nb; nb = tn;
  }
  int c = 0;
  // ratio rule: merge when the longer list is within ~log2 of the shorter
  int lg = 32 - __clz(nb);
  if (nb <= na * lg && na + nb >= 64) {
    const int total = na + nb;
    const int d0 = (int)((int64_t)total * lane / 32);
    const int d1 = (int)((int64_t)total * (lane + 1) / 32);
    c = merge_segment_count(a, na, b, nb, d0, d1, ex0, ex1);
  } else {
    for (int i = lane; i < na; i += 32) {
      int32_t key = __ldg(a + i);
      if (key != ex0 && key != ex1 && contains_g(b, nb, key)) ++c;
    }
  }
  return warp_sum_int(c);
}

// Materialises {x in A & B : x < upper} in ascending order into out; returns the size.
__device__ __forceinline__ int warp_intersect(const int32_t* a, int na, const int32_t* b,
                                              int nb, int32_t upper, int32_t* out) {
  const int lane = threadIdx.x & 31;
  na = warp_prefix_below(a, na, upper);
  nb = warp_prefix_below(b, nb, upper);
  if (na == 0 || nb == 0) return 0;
  if (na > nb) {
    const int32_t* t = a; a = b; b = t;
    int tn = na; na = nb; nb = tn;
  }
  int written = 0;
  for (int base = 0; base < na; base += 32) {
    int i = base + lane;
    int32_t key = i < na ? __ldg(a + i) : 0;
    bool f = i < na && contains_g(b, nb, key);
    unsigned mask = __ballot_sync(kFull, f);
    if (f) out[written + __popc(mask & ((1u << lane) - 1))] = key;
    written += __popc(mask);
  }
  __syncwarp();
  return written;
}

// {x in A : x < upper, x not in B, x != excl}; returns the size; out may be null (count).
__device__ __forceinline__ int warp_difference(const int32_t* a, int na, const int32_t* b,
                                               int nb, int32_t upper, int32_t excl,
                                               int32_t* out) {
  const int lane = threadIdx.x & 31;
  na = warp_prefix_below(a, na, upper);
  nb = warp_prefix_below(b, nb, upper);
  int written = 0;
  for (int base = 0; base < na; base += 32) {
    int i = base + lane;
    int32_t key = i < na ? __ldg(a + i) : 0;
    bool f = i < na && key != excl && !(nb > 0 && contains_g(b, nb, key));
    unsigned mask = __ballot_sync(kFull, f);
    if (out && f) out[written + __popc(mask & ((1u << lane) - 1))] = key;
    written += __popc(mask);
  }
  __syncwarp();
  return written;
}

// Splits A by B in one pass over A's keys: keys below `upper` that B lacks go to `dif`, every
// other key of A (members of B, and keys at or above upper) to `rest` (may be null), both in
// ascending order.  Returns |dif| (warp-uniform).  upper == INT32_MAX: no bound.  A key is
// looked up in the part of B below upper only, where every key that can reach `dif` lies.
// This is the one pass of both fused splits: dif_int_set (include/set_difference.cuh:346-413,
// 415-475) is one call; fuse_set (:248-343) is one call for A \ B and A & B and one with the
// operands swapped for B \ A.  The reference marks the hits of the second list in a zeroed
// per-warp map to emit B \ A; a second pass of lookups needs no scratch.
__device__ __forceinline__ int warp_split_by(const int32_t* a, int na, const int32_t* b, int nb,
                                             int32_t upper, int32_t* dif, int32_t* rest) {
  const int lane = threadIdx.x & 31;
  const unsigned below = (1u << lane) - 1u;
  nb = warp_prefix_below(b, nb, upper);
  int nd = 0, nr = 0;
  for (int base = 0; base < na; base += 32) {
    const int i = base + lane;
    const bool v = i < na;
    const int32_t key = v ? __ldg(a + i) : 0;
    const bool f = v && (upper == INT32_MAX || key < upper) && !(nb > 0 && contains_g(b, nb, key));
    const unsigned md = __ballot_sync(kFull, f);
    const unsigned mr = __ballot_sync(kFull, v && !f);
    if (f) dif[nd + __popc(md & below)] = key;
    else if (v && rest) rest[nr + __popc(mr & below)] = key;
    nd += __popc(md);
    nr += __popc(mr);
  }
  __syncwarp();
  return nd;
}

// Lists in shared or global memory that the warp reads with plain loads (no __ldg), for
// operands the warp itself just wrote.
__device__ __forceinline__ bool contains_s(const int32_t* a, int n, int32_t key) {
  int lo = 0, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (a[mid] < key) lo = mid + 1;
    else hi = mid;
  }
  return lo < n && a[lo] == key;
}

// Intersection where A was written by this warp (plain loads) and B is read-only global.
__device__ __forceinline__ int warp_intersect_w(const int32_t* a, int na, const int32_t* b,
                                                int nb, int32_t upper, int32_t* out) {
  const int lane = threadIdx.x & 31;
  int written = 0;
  if (nb == 0) return 0;
  if (upper != INT32_MAX) nb = warp_prefix_below(b, nb, upper);
  for (int base = 0; base < na; base += 32) {
    int i = base + lane;
    int32_t key = i < na ? a[i] : INT32_MAX;
    bool f = i < na && key < upper && contains_g(b, nb, key);
    unsigned mask = __ballot_sync(kFull, f);
    if (out && f) out[written + __popc(mask & ((1u << lane) - 1))] = key;
    written += __popc(mask);
  }
  __syncwarp();
  return written;
}

}  // namespace jgpm

namespace jgpm {

// Loads that are safe for lists this kernel wrote earlier (plain ld) or graph arrays
// (read-only path).
template <bool RO>
__device__ __forceinline__ int32_t ld32(const int32_t* p) {
  if (RO) return __ldg(p);
  return *p;
}

template <bool RO>
__device__ __forceinline__ int lower_bound_t(const int32_t* a, int n, int32_t key) {
  int lo = 0, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (ld32<RO>(a + mid) < key) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// Prefix below upper for a list of either kind (warp-uniform).
template <bool RO>
__device__ __forceinline__ int warp_prefix_below_t(const int32_t* a, int n, int32_t upper) {
  if (upper == INT32_MAX || n == 0) return n;
  int p = 0;
  if ((threadIdx.x & 31) == 0) p = lower_bound_t<RO>(a, n, upper);
  return __shfl_sync(kFull, p, 0);
}

// {x in A & B : x < upper, x not in {ex0, ex1}}: keys from A (either kind), lookups in B
// (graph).  out may be null.  Returns the size (warp-uniform).
template <bool ARO>
__device__ __forceinline__ int warp_isect_a(const int32_t* a, int na, const int32_t* b, int nb,
                                            int32_t upper, int32_t ex0, int32_t ex1,
                                            int32_t* out) {
  const int lane = threadIdx.x & 31;
  na = warp_prefix_below_t<ARO>(a, na, upper);
  nb = warp_prefix_below_t<true>(b, nb, upper);
  if (na == 0 || nb == 0) return 0;
  int written = 0;
  for (int base = 0; base < na; base += 32) {
    const int i = base + lane;
    const int32_t key = i < na ? ld32<ARO>(a + i) : 0;
    const bool f = i < na && key != ex0 && key != ex1 && contains_g(b, nb, key);
    const unsigned mask = __ballot_sync(kFull, f);
    if (out && f) out[written + __popc(mask & ((1u << lane) - 1))] = key;
    written += __popc(mask);
  }
  __syncwarp();
  return written;
}

// {x in A : x < upper, x not in B, x != excl}: keys from A (either kind), lookups in B (graph).
template <bool ARO>
__device__ __forceinline__ int warp_diff_a(const int32_t* a, int na, const int32_t* b, int nb,
                                           int32_t upper, int32_t excl, int32_t* out) {
  const int lane = threadIdx.x & 31;
  na = warp_prefix_below_t<ARO>(a, na, upper);
  nb = warp_prefix_below_t<true>(b, nb, upper);
  int written = 0;
  for (int base = 0; base < na; base += 32) {
    const int i = base + lane;
    const int32_t key = i < na ? ld32<ARO>(a + i) : 0;
    const bool f = i < na && key != excl && !(nb > 0 && contains_g(b, nb, key));
    const unsigned mask = __ballot_sync(kFull, f);
    if (out && f) out[written + __popc(mask & ((1u << lane) - 1))] = key;
    written += __popc(mask);
  }
  __syncwarp();
  return written;
}

}  // namespace jgpm
