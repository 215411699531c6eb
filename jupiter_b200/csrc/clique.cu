// k-clique (and triangle) counting on the degree-oriented DAG.
//
// Reference plans: P0 (triangles, src/message_passing_gpu_kernels.cuh:64-102), P13..P16
// (k = 4..7, :1208-1537) and the generic level engine (src/config.h:39-58,
// src/gpu_kernels_codegen.cuh:6-95, 261-410).  Those plans are edge-rooted: for every DAG
// arc (v0, v1) they materialise W = N+(v0) & N+(v1) and then intersect W with N+(v) for each
// candidate v, level after level.  Every k-clique is counted once, rooted at its
// DAG-minimal arc.
//
// B200 design (same counts, fewer bytes): the kernels are VERTEX-rooted.  For a root u with
// out-degree d the level-1 intersections N+(u) & N+(v_i), one per arc (u, v_i), are computed
// once and kept as a local adjacency bitmap over the positions of N+(u):
//     R_i bit j  <=>  L[j] in N+(L[i])          where L = N+(u) (sorted).
// R_i is exactly the reference's level-1 set W of the arc (u, L[i]); every deeper reference
// level "W & N+(v)" becomes a word-wise AND of bitmap rows, and the last level a popcount:
//     K_k(u) = sum_i C_{k-3}(R_i),  C_0(m) = popc(m),  C_t(m) = sum_{j in m} C_{t-1}(m & R_j).
// Each clique is enumerated once, in its (unique) topological order inside the DAG.
//
// Root tiers by out-degree d (roots with d < k-1 cannot root a k-clique and are skipped):
//   small  d <= 32     one warp per root; rows are single words; L and the row offsets
//                      live in registers and are searched with __shfl_sync;
//   mid    d <= 1024   one CTA per root; rows of ceil(d/32) words in shared memory; the
//                      count phase keeps each mask distributed one word per lane;
//   large  d > 1024    edge-rooted fallback: one warp per arc (u, v_i) with W
//                      materialised in per-warp global scratch (the reference's scheme).
// Work is handed out by a global atomic cursor (work stealing); roots are sorted by
// descending out-degree so the heaviest start first.
//
// The level-1 scan for row i reads N+(L[i]) restricted to [L[0], L[d-1]] (a binary search on
// each end when the list is long) and looks every element up in L.
#include <cuda_runtime.h>

#include "jgpm_internal.h"
#include "setops.cuh"

namespace jgpm {

struct CliqueArgs {
  const eid_t* rowptr;  // DAG row pointers
  const vid_t* col;     // DAG neighbour lists
  const vid_t* roots;
  int64_t begin, end;   // root range of this launch
  DevControl* ctl;
  int32_t* scratch;     // large tier: per-warp lists
  int64_t scratch_per_warp;
  int cursor;           // which ctl->counter this launch steals from
  uint32_t* tri;        // edge-triangle mode: triangles per DAG arc (K == 3 only)
};

namespace {

constexpr int kRangeCut = 32;  // restrict a row to [L0, Ld-1] when longer than this

// ------------------------------------------------------------------ small tier (d <= 32)
template <int D, bool STATS>
struct SmallCount {
  // m: candidate set (bits over L), R: rows, deg: out-degrees of L (stats only)
  __device__ __forceinline__ static acc_t run(uint32_t m, const uint32_t* R, const int* deg,
                                              acc_t& elems) {
    acc_t s = 0;
    const int pm = __popc(m);
    uint32_t it = m;
    while (it) {
      const int j = __ffs(it) - 1;
      it &= it - 1;
      if (STATS) elems += (acc_t)pm + (acc_t)deg[j];
      s += SmallCount<D - 1, STATS>::run(m & R[j], R, deg, elems);
    }
    return s;
  }
};

template <bool STATS>
struct SmallCount<0, STATS> {
  __device__ __forceinline__ static acc_t run(uint32_t m, const uint32_t*, const int*, acc_t&) {
    return (acc_t)__popc(m);
  }
};

template <int K, bool STATS, bool ETRI = false>
__global__ void __launch_bounds__(256) k_clique_small(CliqueArgs a) {
  __shared__ uint32_t rows_s[8][32];
  __shared__ int deg_s[8][32];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  uint32_t* R = rows_s[wib];
  int* DG = deg_s[wib];
  acc_t cnt = 0, elems = 0;
  for (;;) {
    unsigned long long idx = 0;
    if (lane == 0) idx = atomicAdd(&a.ctl->counter[a.cursor], 1ull);
    idx = __shfl_sync(kFull, idx, 0) + (unsigned long long)a.begin;
    if ((int64_t)idx >= a.end) break;
    const vid_t u = a.roots[idx];
    const eid_t base = a.rowptr[u];
    const int d = (int)(a.rowptr[u + 1] - base);
    const vid_t Lj = lane < d ? __ldg(a.col + base + lane) : INT32_MAX;
    const vid_t lo_key = __shfl_sync(kFull, Lj, 0);
    const vid_t hi_key = __shfl_sync(kFull, Lj, d - 1);
    eid_t s = 0;
    int len = 0;
    if (lane < d) {
      s = a.rowptr[Lj];
      len = (int)(a.rowptr[Lj + 1] - s);
      if (STATS) DG[lane] = len;
      if (len > kRangeCut) {
        const int lb = lower_bound_g(a.col + s, len, lo_key);
        const int ub = upper_bound_g(a.col + s, len, hi_key);
        s += lb;
        len = ub > lb ? ub - lb : 0;
      }
    }
    R[lane] = 0u;
    int off = len;  // inclusive scan of the row lengths
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(kFull, off, o);
      if (lane >= o) off += t;
    }
    const int T = __shfl_sync(kFull, off, 31);
    const int row_start = off - len;
    __syncwarp();
    for (int t0 = 0; t0 < T; t0 += 32) {
      const int t = t0 + lane;
      // row i = number of rows ending at or before t
      int i = 0;
#pragma unroll
      for (int step = 16; step > 0; step >>= 1) {
        const int ov = __shfl_sync(kFull, off, i + step - 1);
        if (ov <= t) i += step;
      }
      const eid_t si = __shfl_sync(kFull, s, i);
      const int sti = __shfl_sync(kFull, row_start, i);
      const vid_t x = t < T ? __ldg(a.col + si + (t - sti)) : INT32_MIN;
      int p = 0;
#pragma unroll
      for (int step = 16; step > 0; step >>= 1) {
        const vid_t lv = __shfl_sync(kFull, Lj, p + step - 1);
        if (lv < x) p += step;
      }
      const vid_t lp = __shfl_sync(kFull, Lj, p);
      if (t < T && lp == x) {
        atomicOr(&R[i], 1u << p);
        if (ETRI) {  // triangle (u, L[i], L[p]): one count on each of its three arcs
          atomicAdd(a.tri + si + (t - sti), 1u);
          atomicAdd(a.tri + base + i, 1u);
          atomicAdd(a.tri + base + p, 1u);
        }
      }
    }
    __syncwarp();
    if (lane < d) cnt += SmallCount<K - 3, STATS>::run(R[lane], R, DG, elems);
    __syncwarp();
  }
  // reduce and publish
  for (int o = 16; o > 0; o >>= 1) {
    cnt += __shfl_xor_sync(kFull, cnt, o);
    if (STATS) elems += __shfl_xor_sync(kFull, elems, o);
  }
  if (lane == 0) {
    if (cnt) atomicAdd(&a.ctl->count[0], cnt);
    if (STATS && elems) atomicAdd(&a.ctl->elements[0], elems);
  }
}

// ------------------------------------------------------------------ mid tier (d <= 1024)
// Shared layout for one root (dynamic shared memory):
//   L[dmax] ids | off[dmax+1] exclusive row offsets | rs[dmax] row starts (int64) |
//   deg[dmax] | R[dmax * W] rows
struct MidLayout {
  int dmax, W;
  __host__ __device__ size_t bytes() const {
    return (size_t)dmax * 4 + (size_t)(dmax + 1) * 4 + (size_t)dmax * 8 + (size_t)dmax * 4 +
           (size_t)dmax * W * 4 + 64;
  }
};

template <int D, bool STATS>
struct DistCount {
  // Mask distributed one word per lane (lane w holds word w, w < W).
  __device__ __forceinline__ static acc_t run(uint32_t mw, const uint32_t* R, int W,
                                              const int* deg, acc_t& elems) {
    const int lane = threadIdx.x & 31;
    acc_t s = 0;
    int pm = 0;
    if (STATS) pm = __reduce_add_sync(kFull, (unsigned)__popc(mw));
    unsigned nz = __ballot_sync(kFull, mw != 0u);
    while (nz) {
      const int lw = __ffs(nz) - 1;
      nz &= nz - 1;
      uint32_t word = __shfl_sync(kFull, mw, lw);
      while (word) {
        const int b = __ffs(word) - 1;
        word &= word - 1;
        const int j = lw * 32 + b;
        if (STATS && lane == 0) elems += (acc_t)pm + (acc_t)deg[j];
        const uint32_t nxt = lane < W ? (mw & R[(size_t)j * W + lane]) : 0u;
        s += DistCount<D - 1, STATS>::run(nxt, R, W, deg, elems);
      }
    }
    return s;
  }
};

template <bool STATS>
struct DistCount<0, STATS> {
  __device__ __forceinline__ static acc_t run(uint32_t mw, const uint32_t*, int, const int*,
                                              acc_t&) {
    return (acc_t)__popc(mw);  // per-lane partial; summed at the end
  }
};

template <int K, bool STATS, bool ETRI = false>
__global__ void __launch_bounds__(256) k_clique_mid(CliqueArgs a, int dmax, int W) {
  extern __shared__ __align__(16) unsigned char smem[];
  MidLayout lay{dmax, W};
  vid_t* L = reinterpret_cast<vid_t*>(smem);
  int* off = reinterpret_cast<int*>(L + dmax);
  eid_t* rs = reinterpret_cast<eid_t*>(
      (reinterpret_cast<uintptr_t>(off + dmax + 1) + 7) & ~uintptr_t(7));
  int* deg = reinterpret_cast<int*>(rs + dmax);
  uint32_t* R = reinterpret_cast<uint32_t*>(deg + dmax);
  __shared__ unsigned long long s_idx;
  __shared__ int s_wsum[8];
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int nthreads = blockDim.x;
  const int nwarps = nthreads >> 5;
  acc_t cnt = 0, elems = 0;
  (void)lay;
  for (;;) {
    if (tid == 0) s_idx = atomicAdd(&a.ctl->counter[a.cursor], 1ull);
    __syncthreads();
    const int64_t idx = (int64_t)s_idx + a.begin;
    __syncthreads();
    if (idx >= a.end) break;
    const vid_t u = a.roots[idx];
    const eid_t base = a.rowptr[u];
    const int d = (int)(a.rowptr[u + 1] - base);
    const int w_d = (d + 31) >> 5;
    for (int j = tid; j < d; j += nthreads) L[j] = __ldg(a.col + base + j);
    for (int q = tid; q < d * w_d; q += nthreads) R[q] = 0u;
    __syncthreads();
    const vid_t lo_key = L[0], hi_key = L[d - 1];
    // row extents (restricted) and lengths
    for (int i = tid; i < d; i += nthreads) {
      const vid_t v = L[i];
      eid_t s = a.rowptr[v];
      int len = (int)(a.rowptr[v + 1] - s);
      deg[i] = len;
      if (len > kRangeCut) {
        const int lb = lower_bound_g(a.col + s, len, lo_key);
        const int ub = upper_bound_g(a.col + s, len, hi_key);
        s += lb;
        len = ub > lb ? ub - lb : 0;
      }
      rs[i] = s;
      off[i] = len;
    }
    __syncthreads();
    // exclusive scan of off[0..d) (blocked per thread, then across warps)
    {
      const int per = (d + nthreads - 1) / nthreads;
      const int b0 = min(d, tid * per), b1 = min(d, b0 + per);
      int local = 0;
      for (int i = b0; i < b1; ++i) local += off[i];
      int incl = local;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += t;
      }
      if (lane == 31) s_wsum[warp] = incl;
      __syncthreads();
      int wbase = 0;
      for (int w = 0; w < warp; ++w) wbase += s_wsum[w];
      int run = wbase + incl - local;
      __syncthreads();
      for (int i = b0; i < b1; ++i) {
        const int l = off[i];
        off[i] = run;
        run += l;
      }
      if (tid == nthreads - 1) off[d] = run;
      __syncthreads();
    }
    const int T = off[d];
    for (int t = tid; t < T; t += nthreads) {
      // row i: last i with off[i] <= t
      int lo = 0, hi = d - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= t) lo = mid;
        else hi = mid - 1;
      }
      const int i = lo;
      const vid_t x = __ldg(a.col + rs[i] + (t - off[i]));
      int p0 = 0, p1 = d;
      while (p0 < p1) {
        const int mid = (p0 + p1) >> 1;
        if (L[mid] < x) p0 = mid + 1;
        else p1 = mid;
      }
      if (p0 < d && L[p0] == x) {
        atomicOr(&R[(size_t)i * w_d + (p0 >> 5)], 1u << (p0 & 31));
        if (ETRI) {
          atomicAdd(a.tri + rs[i] + (t - off[i]), 1u);
          atomicAdd(a.tri + base + i, 1u);
          atomicAdd(a.tri + base + p0, 1u);
        }
      }
    }
    __syncthreads();
    // count phase: each warp takes rows; the mask is distributed one word per lane
    for (int i = warp; i < d; i += nwarps) {
      const uint32_t mw = lane < w_d ? R[(size_t)i * w_d + lane] : 0u;
      cnt += DistCount<K - 3, STATS>::run(mw, R, w_d, deg, elems);
    }
    __syncthreads();
  }
  for (int o = 16; o > 0; o >>= 1) {
    cnt += __shfl_xor_sync(kFull, cnt, o);
    if (STATS) elems += __shfl_xor_sync(kFull, elems, o);
  }
  if (lane == 0) {
    if (cnt) atomicAdd(&a.ctl->count[0], cnt);
    if (STATS && elems) atomicAdd(&a.ctl->elements[0], elems);
  }
}

// ------------------------------------------------------------------ large tier (d > 1024)
// Edge-rooted, list based: one warp per arc (u, v_i) of a large root.  Candidate lists of
// each level live in the warp's global scratch (kMaxLevels lists of max_out entries).
constexpr int kMaxLevels = 6;

// REM = levels still to choose (compile-time, so no device-side recursion at run time).
template <int REM, bool STATS>
struct ListClique {
  __device__ static acc_t run(const CliqueArgs& a, const vid_t* cand, int nc, int32_t* buf,
                              int64_t cap, acc_t& elems) {
    const int lane = threadIdx.x & 31;
    acc_t s = 0;
    for (int i = 0; i < nc; ++i) {
      const vid_t v = cand[i];
      const eid_t b = a.rowptr[v];
      const int dv = (int)(a.rowptr[v + 1] - b);
      if (STATS && lane == 0) elems += (acc_t)nc + (acc_t)dv;
      if (REM == 1) {
        // count |cand & N+(v)| with the lookups on cand (written by this warp)
        int c = 0;
        for (int q = lane; q < nc; q += 32)
          if (contains_g(a.col + b, dv, cand[q])) ++c;
        s += (acc_t)warp_sum_int(c);
      } else {
        const int t = warp_intersect_w(cand, nc, a.col + b, dv, INT32_MAX, buf);
        if (t > 0) s += ListClique<(REM > 1 ? REM - 1 : 1), STATS>::run(a, buf, t, buf + cap, cap, elems);
      }
    }
    return s;
  }
};

template <int K, bool STATS, bool ETRI = false>
__global__ void __launch_bounds__(256) k_clique_large(CliqueArgs a) {
  const int lane = threadIdx.x & 31;
  const int64_t gwarp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int32_t* buf = a.scratch + gwarp * a.scratch_per_warp;
  const int64_t cap = a.scratch_per_warp / kMaxLevels;
  acc_t cnt = 0, elems = 0;
  // task = (root index, arc index) flattened as root-major chunks of one arc each
  for (;;) {
    unsigned long long t = 0;
    if (lane == 0) t = atomicAdd(&a.ctl->counter[a.cursor], 1ull);
    t = __shfl_sync(kFull, t, 0);
    // decode: tasks enumerate (root r in [begin,end), arc i) with i < d(r)
    // walk roots (few large roots, so a linear walk is cheap)
    int64_t r = a.begin;
    unsigned long long rem = t;
    bool found = false;
    vid_t u = 0;
    int i = 0;
    for (; r < a.end; ++r) {
      const vid_t ur = a.roots[r];
      const unsigned long long dr = (unsigned long long)(a.rowptr[ur + 1] - a.rowptr[ur]);
      if (rem < dr) {
        u = ur;
        i = (int)rem;
        found = true;
        break;
      }
      rem -= dr;
    }
    if (!found) break;
    const eid_t bu = a.rowptr[u];
    const int du = (int)(a.rowptr[u + 1] - bu);
    const vid_t v = __ldg(a.col + bu + i);
    const eid_t bv = a.rowptr[v];
    const int dv = (int)(a.rowptr[v + 1] - bv);
    int32_t* W = buf;
    const int tw = warp_intersect(a.col + bu, du, a.col + bv, dv, INT32_MAX, W);
    if (K == 3) {
      cnt += (acc_t)tw;
      if (ETRI && tw > 0) {
        if (lane == 0) atomicAdd(a.tri + bu + i, (unsigned)tw);
        for (int q = lane; q < tw; q += 32) {
          const vid_t w = W[q];
          atomicAdd(a.tri + bu + lower_bound_g(a.col + bu, du, w), 1u);
          atomicAdd(a.tri + bv + lower_bound_g(a.col + bv, dv, w), 1u);
        }
        __syncwarp();
      }
    } else if (tw > 0) {
      cnt += ListClique<(K > 3 ? K - 3 : 1), STATS>::run(a, W, tw, buf + cap, cap, elems);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    cnt += __shfl_xor_sync(kFull, cnt, o);
    if (STATS) elems += __shfl_xor_sync(kFull, elems, o);
  }
  if (lane == 0) {
    if (cnt) atomicAdd(&a.ctl->count[0], cnt);
    if (STATS && elems) atomicAdd(&a.ctl->elements[0], elems);
  }
}

// Level-1 set-op elements of the edge-rooted plan: sum over DAG arcs (u, v) of
// d+(u) + d+(v) (every arc issues the W = N+(u) & N+(v) intersection).
__global__ void k_level1_elements(const eid_t* rowptr, const vid_t* col, vid_t n,
                                  DevControl* ctl) {
  acc_t e = 0;
  const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int lane = threadIdx.x & 31;
  for (int64_t u = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < n; u += warps) {
    const eid_t b = rowptr[u];
    const int d = (int)(rowptr[u + 1] - b);
    for (int i = lane; i < d; i += 32) {
      const vid_t v = __ldg(col + b + i);
      e += (acc_t)d + (acc_t)(rowptr[v + 1] - rowptr[v]);
    }
  }
  for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(kFull, e, o);
  if (lane == 0 && e) atomicAdd(&ctl->elements[1], e);
}

struct TierRange {
  int64_t b, e;
  bool empty() const { return e <= b; }
};

template <int K, bool STATS, bool ETRI = false>
void launch_tiers(const CliqueArgs& base, TierRange large, TierRange mid, TierRange small,
                  int sms, cudaStream_t s, int mid_dmax) {
  CliqueArgs a = base;
  if (!large.empty()) {
    a.begin = large.b;
    a.end = large.e;
    a.cursor = 2;
    k_clique_large<K, STATS, ETRI><<<sms * 2, 256, 0, s>>>(a);
  }
  if (!mid.empty()) {
    a.begin = mid.b;
    a.end = mid.e;
    a.cursor = 1;
    const int W = (mid_dmax + 31) / 32;
    MidLayout lay{mid_dmax, W};
    const size_t sm = lay.bytes();
    cudaFuncSetAttribute(k_clique_mid<K, STATS, ETRI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sm);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_clique_mid<K, STATS, ETRI>, 256,
                                                  sm);
    if (per_sm < 1) per_sm = 1;
    k_clique_mid<K, STATS, ETRI><<<sms * per_sm, 256, sm, s>>>(a, mid_dmax, W);
  }
  if (!small.empty()) {
    a.begin = small.b;
    a.end = small.e;
    a.cursor = 0;
    k_clique_small<K, STATS, ETRI><<<sms * 8, 256, 0, s>>>(a);
  }
}

}  // namespace

// Launches the k-clique kernels over roots [root_begin, root_end) of g->tiers (which must
// be built for this k).  Results accumulate into g->d_ctl->count[0] (elements of levels >= 2
// into elements[0] when stats).  The caller zeroes the work cursors before each call.
int launch_clique(jgpm_graph* g, int k, bool stats, int64_t root_begin, int64_t root_end,
                  cudaStream_t s) {
  if (k < 3 || k > 8) {
    jgpm_set_error_("k-clique: k must be in [3, 8]");
    return JGPM_EPATTERN;
  }
  const int sms = device_sm_count(g->device);
  const RootTiers& t = g->tiers;
  auto cut = [&](int64_t b, int64_t e) {
    TierRange r{std::max(b, root_begin), std::min(e, root_end)};
    return r;
  };
  const TierRange large = cut(0, t.large_end);
  const TierRange mid = cut(t.large_end, t.mid_end);
  const TierRange small = cut(t.mid_end, t.small_end);
  CliqueArgs a{};
  a.rowptr = g->d_dag_rowptr;
  a.col = g->d_dag_col;
  a.roots = t.d_roots;
  a.ctl = g->d_ctl;
  if (!large.empty()) {
    const int64_t per_warp = (int64_t)kMaxLevels * (g->max_out_degree + 32);
    const int64_t warps = (int64_t)sms * 2 * 8;
    int rc = ensure_scratch(g, (size_t)(per_warp * warps) * sizeof(int32_t));
    if (rc) return rc;
    a.scratch = (int32_t*)g->d_scratch;
    a.scratch_per_warp = per_warp;
  }
  const int mid_dmax = std::max(33, std::min(g->max_out_degree, kMidMaxDeg));
  g->launches += (int)!large.empty() + (int)!mid.empty() + (int)!small.empty();
  switch (k) {
#define JGPM_K(KK)                                                              \
  case KK:                                                                      \
    if (stats) launch_tiers<KK, true>(a, large, mid, small, sms, s, mid_dmax);  \
    else launch_tiers<KK, false>(a, large, mid, small, sms, s, mid_dmax);       \
    break;
    JGPM_K(3) JGPM_K(4) JGPM_K(5) JGPM_K(6) JGPM_K(7) JGPM_K(8)
#undef JGPM_K
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    jgpm_set_error_(std::string("clique launch: ") + cudaGetErrorString(e));
    return JGPM_ECUDA;
  }
  return JGPM_OK;
}

// Triangles per DAG arc into d_tri (zeroed by the caller); the triangle total also
// accumulates into ctl->count[0].  Uses the k = 3 tiers.
int launch_edge_triangles(jgpm_graph* g, uint32_t* d_tri, cudaStream_t s) {
  int rc;
  if ((rc = ensure_tiers(g, 2))) return rc;
  if ((rc = ensure_control(g))) return rc;
  const int sms = device_sm_count(g->device);
  const RootTiers& t = g->tiers;
  CliqueArgs a{};
  a.rowptr = g->d_dag_rowptr;
  a.col = g->d_dag_col;
  a.roots = t.d_roots;
  a.ctl = g->d_ctl;
  a.tri = d_tri;
  if (t.large_end > 0) {
    const int64_t per_warp = (int64_t)kMaxLevels * (g->max_out_degree + 32);
    const int64_t warps = (int64_t)sms * 2 * 8;
    if ((rc = ensure_scratch(g, (size_t)(per_warp * warps) * sizeof(int32_t)))) return rc;
    a.scratch = (int32_t*)g->d_scratch;
    a.scratch_per_warp = per_warp;
  }
  JGPM_CUDA_TRY(cudaMemsetAsync(g->d_ctl, 0, sizeof(DevControl), s));
  const int mid_dmax = std::max(33, std::min(g->max_out_degree, kMidMaxDeg));
  g->launches += (int)(t.large_end > 0) + (int)(t.mid_end > t.large_end) +
                 (int)(t.small_end > t.mid_end);
  launch_tiers<3, false, true>(a, TierRange{0, t.large_end}, TierRange{t.large_end, t.mid_end},
                               TierRange{t.mid_end, t.small_end}, sms, s, mid_dmax);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    jgpm_set_error_(std::string("edge triangles: ") + cudaGetErrorString(e));
    return JGPM_ECUDA;
  }
  return JGPM_OK;
}

// Level-1 set-op elements of the edge-rooted plan into g->d_ctl->elements[1].
int launch_level1_elements(jgpm_graph* g, cudaStream_t s) {
  const int sms = device_sm_count(g->device);
  k_level1_elements<<<sms * 8, 256, 0, s>>>(g->d_dag_rowptr, g->d_dag_col, g->n, g->d_ctl);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    jgpm_set_error_(std::string("level-1 elements: ") + cudaGetErrorString(e));
    return JGPM_ECUDA;
  }
  return JGPM_OK;
}

}  // namespace jgpm
