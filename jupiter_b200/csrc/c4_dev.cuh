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
//
// Every counter add returns the count before it, and C(c, 2) = 0 + 1 + ... + (c - 1), so the
// sum of the returned counts is sum C(c, 2): no pass reads the counters back.  The passes
// after the adds only put the counters back to zero.
#pragma once
#include "jgpm_internal.h"
#include "setops.cuh"

namespace jgpm {

// Apex classes by their wedge upper bound ub (sum of deg(x) over the prefix):
//   small  ub <= kC4SmallBound  one warp, shared-memory hash of kC4HashSlots (load <= 1/2);
//   mid    ub <= kC4MidBound    one CTA, shared-memory hash of kC4MidSlots (load <= 1/2);
//   large                       one CTA, either a shared-memory slab of packed counters swept
//                               over the vertex range in slices (C4SlabForm), or a dense
//                               counter array in global memory (c4_dense_apex).
constexpr int kC4SmallBound = 256;
constexpr int kC4HashSlots = 512;
constexpr int kC4MidBound = 2048;
constexpr int kC4MidSlots = 4096;
constexpr int kC4MaxSlices = 4;

// The two slab forms of the large apexes.  Wide: one CTA of 1024 threads per SM with a 192 KB
// slab.  Narrow: two CTAs of 512 threads per SM with 96 KB each, so that one CTA's adds overlap
// the other's latency-bound phases (the loads of x, rp[x] and the boundary searches between
// barriers).  The narrow slab covers half the ids per slice, so a graph takes it only up to
// kC4NarrowMaxN vertices, where an 8-bit apex still needs at most kC4MaxSlices slices.
struct C4SlabForm {
  int threads, words;
  int slice_wedges;  // c4_dense_apex: wedge bound an apex must bring per (slice, block)
};
constexpr int kC4WideThreads = 1024, kC4WideWords = 48 * 1024;
constexpr int kC4NarrowThreads = 512, kC4NarrowWords = 24 * 1024;
constexpr int64_t kC4NarrowMaxN = (int64_t)kC4MaxSlices * (kC4NarrowWords << 2);  // 393,216
__host__ __device__ __forceinline__ C4SlabForm c4_slab_form(int64_t n) {
  return n <= kC4NarrowMaxN ? C4SlabForm{kC4NarrowThreads, kC4NarrowWords, 1024}
                            : C4SlabForm{kC4WideThreads, kC4WideWords, 8192};
}

// Per-warp shared memory of the small-apex path.
struct C4WarpHash {
  int keys[kC4HashSlots];  // -1 = empty
  int cnt[kC4HashSlots];
  int used[kC4SmallBound];  // slots taken by the current apex
  int nused;
  int pad[3];
};

// Hash table of the mid-apex path (one per CTA).
struct C4CtaHash {
  int keys[kC4MidSlots];  // -1 = empty
  int cnt[kC4MidSlots];
  int used[kC4MidBound];
  int nused;
  int cut;
  int pad[2];
};

// Block-wide wedge layout of a CTA of NT threads: the non-empty lists of the block, compacted;
// list r holds the wedges [off[r], off[r+1]) of the flattened range, read from col[bx[r] ..].
template <int NT>
struct C4LargeSmem {
  int nnz, nt;      // non-empty lists; touched-list length (dense path)
  int off[NT + 1];  // exclusive offsets, off[nnz] = total
  int wsum[NT / 32];
  int wnz[NT / 32];
  eid_t bx[NT];
};

// Shared memory of the mid-apex path: the table and the wedge layout.
template <int NT>
struct C4MidSmem {
  C4CtaHash h;
  C4LargeSmem<NT> f;
};

// log2 of the counter width of a slab apex with `cut` lower-ranked neighbours: every count is
// at most cut, so 8-bit counters do for cut < 256 and 16-bit ones for cut < 65536.
__host__ __device__ __forceinline__ int c4_slab_lgbits(int cut) {
  return cut < 256 ? 3 : cut < 65536 ? 4 : 5;
}

// Slices of `words` 32-bit words needed to cover the vertex ids [0, v).
__host__ __device__ __forceinline__ int64_t c4_slab_slices(vid_t v, int cut, int words) {
  const int64_t span = (int64_t)words << (5 - c4_slab_lgbits(cut));
  return ((int64_t)v + span - 1) / span;
}

// Threads of a dense-counter CTA (the plain dense kernel, two CTAs per SM).
constexpr int kC4DenseThreads = 1024;

// Whether a large apex counts in a dense global array rather than in the slab of form f.  The
// slab costs a layout and a boundary search per x for every (slice, block of f.threads x), so
// an apex takes it when it needs at most kC4MaxSlices slices or brings at least f.slice_wedges
// of wedge bound per (slice, block).  (Dense counters of a graph of millions of vertices do
// not stay in L2: every wedge then costs an atomic in DRAM, about ten times a slab add.)  The
// thresholds are measured: 1024 for the narrow form; 8192 for the wide one, which on an R-MAT
// graph of 16.7 M vertices took the 4-cycle count from 9.7 s (1024) to 7.8 s (4096: 8.3 s,
// 65536: 9.0 s).  The classifier decides with this one function and records it with the apex.
__host__ __device__ __forceinline__ bool c4_dense_apex(vid_t v, int cut, uint64_t ub,
                                                       C4SlabForm f) {
  const int64_t sl = c4_slab_slices(v, cut, f.words);
  const int64_t nblk = ((int64_t)cut + f.threads - 1) / f.threads;
  return sl > kC4MaxSlices && ub < (uint64_t)(sl * nblk) * (uint64_t)f.slice_wedges;
}

// Sort key of a large apex: its wedge bound, with kC4SlabKey set for slab apexes, so that a
// descending sort puts the slab apexes first and the dense ones after, each by bound.
constexpr uint64_t kC4SlabKey = 1ull << 63;

// The cut of a large apex as stored after the apex list: bit 31 set for a dense apex.
constexpr uint32_t kC4DenseFlag = 0x80000000u;

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

// First index p in [lo, n) with a[p] >= key (n if none), for a cursor lo below which every
// entry is < key: probes lo, lo+1, lo+3, lo+7, ... and then searches the last gap.  One load
// when the answer is lo, as it is for most slices of an apex that needs many of them.
__device__ __forceinline__ int c4_gallop(const vid_t* a, int lo, int n, vid_t key) {
  int p = lo, q = lo, step = 1;
  while (q < n && __ldg(a + q) < key) {
    p = q + 1;
    q += step;
    step <<= 1;
  }
  const int e = q < n ? q : n;
  return p + c4_lower_bound(a + p, e - p, key);
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
// at most 1/2; slots taken for the first time are appended to used[].  Returns the count of v3
// before this wedge.
template <int SLOTS, int SHIFT>
__device__ __forceinline__ int c4_hash_add(int* keys, int* cnt, int* used, int* nused,
                                           vid_t v3) {
  volatile int* vkeys = keys;
  int s = (int)(((uint32_t)v3 * 0x9E3779B1u) >> SHIFT);
  for (;;) {
    const int k = vkeys[s];
    if (k == v3) return atomicAdd(&cnt[s], 1);
    if (k == -1) {
      const int old = atomicCAS(&keys[s], -1, v3);
      if (old == -1) {
        used[atomicAdd(nused, 1)] = s;
        return atomicAdd(&cnt[s], 1);
      }
      if (old == v3) return atomicAdd(&cnt[s], 1);
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
  acc_t sum = 0;
  for (int c0 = 0; c0 < cut; c0 += 32) {
    c4_wedge_chunk(rp, col, v, b, cut, c0, [&](vid_t v3) {
      sum += (acc_t)c4_hash_add<kC4HashSlots, 23>(h.keys, h.cnt, h.used, &h.nused, v3);
    });
  }
  __syncwarp();
  const int nu = h.nused;
  for (int u = lane; u < nu; u += 32) {
    const int s = h.used[u];
    h.keys[s] = -1;
    h.cnt[s] = 0;
  }
  __syncwarp();
  if (lane == 0) h.nused = 0;
  __syncwarp();
  return sum;
}


// Lays out the wedges of one block of lower-ranked neighbours, one per thread: `len` wedges read
// from col[start ..].  The non-empty lists are compacted in thread order and their offsets
// scanned into sh.off; returns the total.  Every thread of the CTA (blockDim.x == NT) calls it;
// it ends with a barrier.  A caller that reads sh after it puts a barrier before the next call.
template <int NT>
__device__ __forceinline__ int c4_block_layout(int len, eid_t start, C4LargeSmem<NT>& sh) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  int incl = len;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += t;
  }
  const unsigned nz = __ballot_sync(kFull, len > 0);
  if (lane == 31) {
    sh.wsum[warp] = incl;
    sh.wnz[warp] = __popc(nz);
  }
  __syncthreads();
  int wbase = 0, zbase = 0;
  for (int w = 0; w < warp; ++w) {
    wbase += sh.wsum[w];
    zbase += sh.wnz[w];
  }
  if (len > 0) {
    const int k = zbase + __popc(nz & ((1u << lane) - 1u));
    sh.off[k] = wbase + incl - len;
    sh.bx[k] = start;
  }
  if (tid == NT - 1) {
    const int k = zbase + __popc(nz);
    sh.off[k] = wbase + incl;
    sh.nnz = k;
  }
  __syncthreads();
  return sh.off[sh.nnz];
}

// Calls visit(v3) once for each of the T wedges of the layout.  Each warp takes a contiguous
// run of 32-wedge chunks.  The list starts inside a chunk mark its bits in one OR-reduction, so
// a lane finds the list of its wedge with a popcount instead of a search; the list of the next
// chunk's first wedge follows from the same mask.  Coalesced: a warp reads 32 consecutive
// wedges.
template <int NT, typename Visit>
__device__ __forceinline__ void c4_warp_wedges(const vid_t* col, const C4LargeSmem<NT>& sh,
                                               int T, Visit visit) {
  constexpr int kWarps = NT / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nnz = sh.nnz;
  const int chunks = (T + 31) >> 5;
  const int per = (chunks + kWarps - 1) / kWarps;
  int c = warp * per;
  const int cend = min(chunks, c + per);
  if (c >= cend) return;
  int t0 = c << 5;
  int r0 = 0;  // last list with off[r0] <= t0 (off[0] = 0; offsets strictly increase)
  for (int step = top_pow2_c4(nnz); step > 0; step >>= 1)
    if (r0 + step < nnz && sh.off[r0 + step] <= t0) r0 += step;
  for (; c < cend; ++c, t0 += 32) {
    const int j = r0 + 1 + lane;  // lists after r0 start at positions >= 1 of the chunk
    const int p = j <= nnz ? sh.off[j] - t0 : 64;
    const unsigned m = __reduce_or_sync(kFull, (p > 0 && p < 32) ? (1u << p) : 0u);
    const bool next_at_32 = __any_sync(kFull, p == 32);
    const int r = r0 + __popc(m & (0xffffffffu >> (31 - lane)));
    const int t = t0 + lane;
    if (t < T) visit(__ldg(col + sh.bx[r] + (t - sh.off[r])));
    r0 += __popc(m) + (next_at_32 ? 1 : 0);
  }
}

// Lower bounds of K keys in one sorted list in lockstep (K independent loads per step):
// p[i] = #{a[j] < key[i]}.
template <int K>
__device__ __forceinline__ void c4_lower_bounds(const vid_t* a, int n, const vid_t (&key)[K],
                                                int (&p)[K]) {
#pragma unroll
  for (int i = 0; i < K; ++i) p[i] = 0;
  for (int step = top_pow2_c4(n); step > 0; step >>= 1) {
#pragma unroll
    for (int i = 0; i < K; ++i)
      if (p[i] + step <= n && __ldg(a + p[i] + step - 1) < key[i]) p[i] += step;
  }
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

// One mid apex v (wedge bound <= kC4MidBound) on the whole CTA (NT threads) with the shared
// table (empty on entry, empty again on return).  The wedges are flattened over all threads.
// Every thread calls it.  Returns this thread's share of sum C(c, 2).
template <int NT>
__device__ __forceinline__ acc_t c4_mid_apex(const eid_t* rp, const vid_t* col, vid_t v,
                                             C4MidSmem<NT>& m) {
  const int tid = threadIdx.x;
  const eid_t b = rp[v];
  const int cut = c4_lower_bound(col + b, (int)(rp[v + 1] - b), v);
  acc_t sum = 0;
  for (int base = 0; base < cut; base += NT) {
    const int i = base + tid;
    int len = 0;
    eid_t bx = 0;
    if (i < cut) {
      const vid_t x = __ldg(col + b + i);
      bx = rp[x];
      len = c4_lower_bound(col + bx, (int)(rp[x + 1] - bx), v);
    }
    const int T = c4_block_layout<NT>(len, bx, m.f);
    c4_warp_wedges<NT>(col, m.f, T, [&](vid_t v3) {
      sum += (acc_t)c4_hash_add<kC4MidSlots, 20>(m.h.keys, m.h.cnt, m.h.used, &m.h.nused, v3);
    });
    __syncthreads();
  }
  const int nu = m.h.nused;
  for (int u = tid; u < nu; u += NT) {
    const int s = m.h.used[u];
    m.h.keys[s] = -1;
    m.h.cnt[s] = 0;
  }
  __syncthreads();
  if (tid == 0) m.h.nused = 0;
  __syncthreads();
  return sum;
}

// One large apex v with `cut` lower-ranked neighbours on the whole CTA (NT threads), counted in
// a dense array of the CTA in global memory (zero on entry, zero again on return); the vertices
// counted for the first time go to the touched list, which the last pass clears.  Every thread
// calls it.  Returns this thread's share of sum C(c, 2).
template <int NT>
__device__ __forceinline__ acc_t c4_large_apex(const eid_t* rp, const vid_t* col, vid_t v,
                                               int cut, int32_t* dense, vid_t* touched,
                                               C4LargeSmem<NT>& sh) {
  const int tid = threadIdx.x;
  const eid_t b = rp[v];
  if (tid == 0) sh.nt = 0;  // ordered before the adds by the layout's barriers
  acc_t sum = 0;
  for (int base = 0; base < cut; base += NT) {
    const int i = base + tid;
    int len = 0;
    eid_t bx = 0;
    if (i < cut) {
      const vid_t x = __ldg(col + b + i);
      bx = rp[x];
      len = c4_lower_bound(col + bx, (int)(rp[x + 1] - bx), v);
    }
    const int T = c4_block_layout<NT>(len, bx, sh);
    c4_warp_wedges<NT>(col, sh, T, [&](vid_t v3) {
      const int old = atomicAdd(&dense[v3], 1);
      if (old == 0) touched[atomicAdd(&sh.nt, 1)] = v3;
      sum += (acc_t)old;
    });
    __syncthreads();
  }
  const int nt = sh.nt;
  for (int q = tid; q < nt; q += NT) atomicExch(&dense[touched[q]], 0);
  __syncthreads();
  return sum;
}

// Zeroes the first `words` words of a shared-memory slab (16-byte aligned; words % 4 == 0).
template <int NT>
__device__ __forceinline__ void c4_slab_zero(uint32_t* slab, int words) {
  uint4* p = reinterpret_cast<uint4*>(slab);
  for (int q = threadIdx.x; q < (words >> 2); q += NT) p[q] = make_uint4(0u, 0u, 0u, 0u);
}

// One large apex v with `cut` lower-ranked neighbours on the whole CTA (NT threads), counted in
// a shared-memory slab of `words` words (zero on entry, zero again on return).  The counters are
// packed 32 / 2^lgb to a word (c4_slab_lgbits: no count overflows its field), and the endpoint
// range [0, v) is swept in slices of words * 32 / 2^lgb ids.  Each prefix(N(x), v) is sorted, so
// binary searches for the slice boundaries give the wedges of each slice and no wedge is read
// twice; with one block of x and at most kC4MaxSlices slices a thread finds all of its
// boundaries in one lockstep search.  Every thread calls it.  It may return before the last
// clearing stores of other threads are done: the caller's next access to the slab or to sh
// must follow a c4_block_layout (or a barrier).  Returns this thread's share of sum C(c, 2).
template <int NT>
__device__ __forceinline__ acc_t c4_slab_apex(const eid_t* rp, const vid_t* col, vid_t v,
                                              int cut, uint32_t* slab, int words,
                                              C4LargeSmem<NT>& sh) {
  static_assert(kC4MaxSlices == 4, "the lockstep boundary search holds four slices");
  const int tid = threadIdx.x;
  const eid_t b = rp[v];
  const int lgb = c4_slab_lgbits(cut);
  const int lgper = 5 - lgb;                // log2 of counters per word
  const uint32_t lmask = (1u << lgper) - 1u;
  const uint32_t cmask = lgb == 5 ? 0xffffffffu : (1u << (1 << lgb)) - 1u;
  const int64_t span = (int64_t)words << lgper;
  const int nblk = (cut + NT - 1) / NT;
  const bool one = nblk == 1;
  const bool held = one && c4_slab_slices(v, cut, words) <= kC4MaxSlices;
  // one block: this thread's x list stays in registers; held: with the ends e[s] of its
  // wedges in slices 0..3, else with a cursor that each slice's search starts from
  eid_t xb = 0;
  int xd = 0, cur = 0;
  int e[4] = {0, 0, 0, 0};
  if (one && tid < cut) {
    const vid_t x = __ldg(col + b + tid);
    xb = rp[x];
    xd = (int)(rp[x + 1] - xb);
    if (held) {
      vid_t key[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) key[i] = (vid_t)min((int64_t)v, (int64_t)(i + 1) * span);
      c4_lower_bounds<4>(col + xb, xd, key, e);
    }
  }
  acc_t sum = 0;
  int s = 0;
  for (int64_t lo = 0; lo < (int64_t)v; lo += span, ++s) {
    const vid_t lo32 = (vid_t)lo;
    const vid_t hi = (vid_t)(lo + span < (int64_t)v ? lo + span : (int64_t)v);
    int added = 0;
    for (int blk = 0; blk < nblk; ++blk) {
      const int i = blk * NT + tid;
      int len = 0;
      eid_t start = 0;
      if (i < cut) {
        if (held) {
          const int s0 = s == 0 ? 0 : s == 1 ? e[0] : s == 2 ? e[1] : e[2];
          const int s1 = s == 0 ? e[0] : s == 1 ? e[1] : s == 2 ? e[2] : e[3];
          start = xb + s0;
          len = s1 - s0;
        } else if (one) {
          const int s1 = c4_gallop(col + xb, cur, xd, hi);
          start = xb + cur;
          len = s1 - cur;
          cur = s1;
        } else {
          const vid_t x = __ldg(col + b + i);
          const eid_t bx = rp[x];
          const vid_t key[2] = {lo32, hi};
          int p[2];
          c4_lower_bounds<2>(col + bx, (int)(rp[x + 1] - bx), key, p);
          start = bx + p[0];
          len = p[1] - p[0];
        }
      }
      const int T = c4_block_layout<NT>(len, start, sh);
      if (T > 0) {
        c4_warp_wedges<NT>(col, sh, T, [&](vid_t v3) {
          const uint32_t l = (uint32_t)(v3 - lo32);
          const int sft = (int)(l & lmask) << lgb;
          const uint32_t old = atomicAdd(slab + (l >> lgper), 1u << sft);
          sum += (acc_t)((old >> sft) & cmask);
        });
        __syncthreads();
      }
      added += T;
    }
    if (added > 0) {
      if (nblk == 1 && added <= (words >> 4)) {
        // few wedges: zero the words they touched (the layout of the one block is still in sh)
        c4_warp_wedges<NT>(col, sh, added, [&](vid_t v3) {
          slab[(uint32_t)(v3 - lo32) >> lgper] = 0u;
        });
      } else {
        c4_slab_zero<NT>(slab, ((int)(((uint32_t)(hi - lo32) + lmask) >> lgper) + 3) & ~3);
      }
      // no barrier here: whatever touches the slab or sh next (the next slice, or the next
      // apex) starts with a layout, whose barriers order it after these stores
    }
  }
  return sum;
}

}  // namespace jgpm
