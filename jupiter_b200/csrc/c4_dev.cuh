// Device building blocks of the 4-cycle wedge count, shared by the plain kernels (c4.cu) and
// the batched persistent kernel (batch.cu).
//
// On the rank-relabelled CSR (vertex id = rank by (degree, id)) every 4-cycle is counted once,
// at its top-ranked vertex v0 (the apex): with c(v0, v3) the number of common neighbours of v0
// and v3 ranked below v0,
//     C4 = sum over apexes v0, opposite vertices v3 < v0 of C(c(v0, v3), 2)
// (Chiba and Nishizeki, SIAM J. Comput. 1985).  The wedges (v0, x, v3) of an apex are
//     x in prefix(N(v0), v0),  v3 in prefix(N(x), v0)
// and c(v0, v3) is the number of wedges that end at v3.  The count equals the reference's P1
// plan (src/message_passing_gpu_kernels.cuh:104-186), which fixes each cycle at its largest
// vertex id instead.
#pragma once
#include "jgpm_internal.h"
#include "setops.cuh"

namespace jgpm {

// Apex classes by their wedge upper bound (sum of deg(x) over the prefix):
//   small  <= kC4SmallBound  one warp, shared-memory hash of kC4HashSlots (load <= 1/2);
//   mid    <= kC4MidBound    one CTA, shared-memory hash of kC4MidSlots (load <= 1/2);
//   large                    one CTA, dense counter array in global memory.
constexpr int kC4SmallBound = 256;
constexpr int kC4HashSlots = 512;
constexpr int kC4MidBound = 2048;
constexpr int kC4MidSlots = 4096;

// Per-warp shared memory of the small-apex path.
struct C4WarpHash {
  int keys[kC4HashSlots];  // -1 = empty
  int cnt[kC4HashSlots];
  int used[kC4SmallBound];  // slots taken by the current apex
  int nused;
  int pad[3];
};

// Shared memory of the mid-apex path (one per CTA).
struct C4CtaHash {
  int keys[kC4MidSlots];  // -1 = empty
  int cnt[kC4MidSlots];
  int used[kC4MidBound];
  int nused;
  int cut;
  int pad[2];
};

__device__ __forceinline__ int top_pow2_c4(int n) { return n > 0 ? 1 << (31 - __clz(n)) : 0; }

__device__ __forceinline__ int c4_lower_bound(const vid_t* a, int n, vid_t key) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(a + mid) < key) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// Visits the wedges (v, x, v3) for x = prefix[c0 .. c0+32) of N(v) below v, flattened over
// the warp's lanes; visit(v3) is called by the lane that owns the wedge.
template <typename Visit>
__device__ __forceinline__ void c4_wedge_chunk(const eid_t* rp, const vid_t* col, vid_t v,
                                               eid_t b, int cut, int c0, Visit visit) {
  const int lane = threadIdx.x & 31;
  const int i = c0 + lane;
  eid_t bx = 0;
  int lenx = 0;
  if (i < cut) {
    const vid_t x = __ldg(col + b + i);
    bx = rp[x];
    const int dx = (int)(rp[x + 1] - bx);
    lenx = c4_lower_bound(col + bx, dx, v);
  }
  int off = lenx;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(kFull, off, o);
    if (lane >= o) off += t;
  }
  const int T = __shfl_sync(kFull, off, 31);
  const int start = off - lenx;
  for (int t0 = 0; t0 < T; t0 += 32) {
    const int t = t0 + lane;
    int r = 0;
#pragma unroll
    for (int step = 16; step > 0; step >>= 1) {
      const int ov = __shfl_sync(kFull, off, r + step - 1);
      if (ov <= t) r += step;
    }
    const eid_t sb = __shfl_sync(kFull, bx, r);
    const int st = __shfl_sync(kFull, start, r);
    if (t < T) visit(__ldg(col + sb + (t - st)));
  }
}

// Adds one wedge ending at v3 to an open-addressing table (keys -1 = empty) whose load stays
// at most 1/2; slots taken for the first time are appended to used[].
template <int SLOTS, int SHIFT>
__device__ __forceinline__ void c4_hash_add(int* keys, int* cnt, int* used, int* nused,
                                            vid_t v3) {
  volatile int* vkeys = keys;
  int s = (int)(((uint32_t)v3 * 0x9E3779B1u) >> SHIFT);
  for (;;) {
    const int k = vkeys[s];
    if (k == v3) {
      atomicAdd(&cnt[s], 1);
      return;
    }
    if (k == -1) {
      const int old = atomicCAS(&keys[s], -1, v3);
      if (old == -1) {
        atomicAdd(&cnt[s], 1);
        used[atomicAdd(nused, 1)] = s;
        return;
      }
      if (old == v3) {
        atomicAdd(&cnt[s], 1);
        return;
      }
    }
    s = (s + 1) & (SLOTS - 1);
  }
}

// Empties a warp's hash table (once, before its first apex).
__device__ __forceinline__ void c4_hash_init(C4WarpHash& h) {
  const int lane = threadIdx.x & 31;
  for (int q = lane; q < kC4HashSlots; q += 32) {
    h.keys[q] = -1;
    h.cnt[q] = 0;
  }
  if (lane == 0) h.nused = 0;
  __syncwarp();
}

// One small apex v (wedge bound <= kC4SmallBound) on one warp; leaves the table empty again.
// Returns this lane's share of sum C(c, 2).
__device__ __forceinline__ acc_t c4_small_apex(const eid_t* rp, const vid_t* col, vid_t v,
                                               C4WarpHash& h) {
  const int lane = threadIdx.x & 31;
  const eid_t b = rp[v];
  const int d = (int)(rp[v + 1] - b);
  int cut = 0;
  if (lane == 0) cut = c4_lower_bound(col + b, d, v);
  cut = __shfl_sync(kFull, cut, 0);
  for (int c0 = 0; c0 < cut; c0 += 32) {
    c4_wedge_chunk(rp, col, v, b, cut, c0, [&](vid_t v3) {
      c4_hash_add<kC4HashSlots, 23>(h.keys, h.cnt, h.used, &h.nused, v3);  // 9-bit hash
    });
  }
  __syncwarp();
  acc_t sum = 0;
  const int nu = h.nused;
  for (int u = lane; u < nu; u += 32) {
    const int s = h.used[u];
    const acc_t c = (acc_t)h.cnt[s];
    sum += c * (c - 1) / 2;
    h.keys[s] = -1;
    h.cnt[s] = 0;
  }
  __syncwarp();
  if (lane == 0) h.nused = 0;
  __syncwarp();
  return sum;
}

// Empties a CTA's mid-apex table (every thread calls it; ends with a barrier).
__device__ __forceinline__ void c4_cta_hash_init(C4CtaHash& h) {
  for (int q = threadIdx.x; q < kC4MidSlots; q += blockDim.x) {
    h.keys[q] = -1;
    h.cnt[q] = 0;
  }
  if (threadIdx.x == 0) h.nused = 0;
  __syncthreads();
}

// One mid apex v (wedge bound <= kC4MidBound) on the whole CTA with the shared table (empty on
// entry, empty again on return).  Every thread calls it.  Returns this thread's share.
__device__ __forceinline__ acc_t c4_mid_apex(const eid_t* rp, const vid_t* col, vid_t v,
                                             C4CtaHash& h) {
  const int tid = threadIdx.x, warp = tid >> 5, nw = blockDim.x >> 5;
  const eid_t b = rp[v];
  const int d = (int)(rp[v + 1] - b);
  if (tid == 0) h.cut = c4_lower_bound(col + b, d, v);
  __syncthreads();
  const int cut = h.cut;
  for (int c0 = warp * 32; c0 < cut; c0 += nw * 32)
    c4_wedge_chunk(rp, col, v, b, cut, c0, [&](vid_t v3) {
      c4_hash_add<kC4MidSlots, 20>(h.keys, h.cnt, h.used, &h.nused, v3);  // 12-bit hash
    });
  __syncthreads();
  acc_t sum = 0;
  const int nu = h.nused;
  for (int u = tid; u < nu; u += blockDim.x) {
    const int s = h.used[u];
    const acc_t c = (acc_t)h.cnt[s];
    sum += c * (c - 1) / 2;
    h.keys[s] = -1;
    h.cnt[s] = 0;
  }
  __syncthreads();
  if (tid == 0) h.nused = 0;
  __syncthreads();
  return sum;
}

// Shared memory of the large-apex path for CTAs of up to NT threads.
template <int NT>
struct C4LargeSmem {
  int cut, nt;
  int off[NT + 1];  // exclusive offsets of the block's x wedge counts, off[NT] = total
  int wsum[NT / 32];
  eid_t bx[NT];     // start of prefix(N(x), v) for the block's x
};

// Binary lifting over a sorted shared-memory array (fixed trip count, top = largest power of
// two <= n): two independent searches in lockstep, p = #{a[j] < x}.
__device__ __forceinline__ void c4_count_below2(const int* a, int n, int top, int x0, int x1,
                                                int& p0, int& p1) {
  p0 = 0;
  p1 = 0;
  for (int step = top; step > 0; step >>= 1) {
    if (p0 + step <= n && a[p0 + step - 1] < x0) p0 += step;
    if (p1 + step <= n && a[p1 + step - 1] < x1) p1 += step;
  }
}

// One large apex v on the whole CTA.  The lower-ranked neighbours x are taken in blocks of
// blockDim; each block's wedges (one thread computes |prefix(N(x), v)| per x, a block scan
// gives the offsets) are spread over all threads, two per thread and iteration, so one hub x
// does not hold up a single warp.  Pass 0 adds every wedge to the dense array (zero on entry)
// and appends each vertex counted for the first time to the touched list; pass 1 reads and
// clears only the touched counters.  Every thread calls it.  Returns this thread's share of
// sum C(c, 2).
template <int NT>
__device__ __forceinline__ acc_t c4_large_apex(const eid_t* rp, const vid_t* col, vid_t v,
                                               int32_t* dense, vid_t* touched,
                                               C4LargeSmem<NT>& sh) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nth = blockDim.x;
  const eid_t b = rp[v];
  const int d = (int)(rp[v + 1] - b);
  if (tid == 0) {
    sh.cut = c4_lower_bound(col + b, d, v);
    sh.nt = 0;
  }
  __syncthreads();
  const int cut = sh.cut;
  for (int base = 0; base < cut; base += nth) {
    const int i = base + tid;
    int len = 0;
    eid_t bx = 0;
    if (i < cut) {
      const vid_t x = __ldg(col + b + i);
      bx = rp[x];
      len = c4_lower_bound(col + bx, (int)(rp[x + 1] - bx), v);
    }
    // block exclusive scan of len
    int incl = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) sh.wsum[warp] = incl;
    __syncthreads();
    int wbase = 0;
    for (int w = 0; w < warp; ++w) wbase += sh.wsum[w];
    sh.off[tid] = wbase + incl - len;
    sh.bx[tid] = bx;
    if (tid == nth - 1) sh.off[nth] = wbase + incl;
    __syncthreads();
    const int T = sh.off[nth];
    const int top = top_pow2_c4(nth - 1);
    for (int t0 = tid; t0 < T; t0 += 2 * nth) {
      const bool two = t0 + nth < T;
      const int t1 = two ? t0 + nth : t0;
      int r0, r1;  // row of element t = last r with off[r] <= t
      c4_count_below2(sh.off + 1, nth - 1, top, t0 + 1, t1 + 1, r0, r1);
      const vid_t v30 = __ldg(col + sh.bx[r0] + (t0 - sh.off[r0]));
      const vid_t v31 = __ldg(col + sh.bx[r1] + (t1 - sh.off[r1]));
      if (atomicAdd(&dense[v30], 1) == 0) touched[atomicAdd(&sh.nt, 1)] = v30;
      if (two && atomicAdd(&dense[v31], 1) == 0) touched[atomicAdd(&sh.nt, 1)] = v31;
    }
    __syncthreads();
  }
  const int nt = sh.nt;
  acc_t sum = 0;
  for (int q = tid; q < nt; q += nth) {
    const acc_t c = (acc_t)atomicExch(&dense[touched[q]], 0);
    sum += c * (c - 1) / 2;
  }
  __syncthreads();
  return sum;
}

}  // namespace jgpm
