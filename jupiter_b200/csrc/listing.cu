// Listing: the embeddings themselves, k vertex ids each, not only their number.
//
// The reference builds with counting or listing chosen at compile time (the COUNT switch
// that sets DO_COUNT, common.mk:60-63) and its kernels only ever count.  Here one warp per
// root arc runs the same nested loops as the literal plans (P13..P16 for the cliques,
// src/message_passing_gpu_kernels.cuh:1208-1537; P1 :104-186; P2 :188-252; the vertex-induced
// enumeration plans of plans.cu) with every level materialised, and the last level appends
// one tuple per element to the output through one atomic per warp and list.
//
// Tuple order: k-cliques in DAG order (each clique once); the 4-cycle (P1) in cycle order
// from its largest vertex, v0 - v1 - v3 - v2 with v1 > v2; the diamond (P2) as its shared
// edge (v0 > v1) and then the two other vertices (w1 < w2); the vertex-induced patterns as
// the root arc's two vertices and then the two others (their vertex set is the embedding).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <string>

#include "jgpm_internal.h"
#include "setops.cuh"

namespace jgpm {
namespace {

enum ListKind {
  kLClique = 0, kLC4 = 1, kLDiamond = 2, kLIC4 = 3, kLIDiamond = 4, kLITailed = 5,
  kLIPath4 = 6, kLIStar3 = 7,
};

constexpr int kListLevels = 6;  // per-warp scratch lists (a 8-clique needs W + 5 levels)

struct ListArgs {
  const eid_t* rowptr;
  const vid_t* col;
  vid_t n;
  int64_t nslots;
  DevControl* ctl;     // counter[0]: root-arc cursor; count[0]: embeddings found
  int32_t* scratch;
  int64_t cap;         // entries per scratch list
  int32_t* out;        // capacity tuples of k ids
  int64_t capacity;
  int k;
};

__device__ __forceinline__ const int32_t* lnbr(const ListArgs& a, vid_t v) {
  return a.col + a.rowptr[v];
}
__device__ __forceinline__ int ldg_deg(const ListArgs& a, vid_t v) {
  return (int)(a.rowptr[v + 1] - a.rowptr[v]);
}

// Reserves n tuple slots (warp-uniform n); returns the first slot index on every lane.
__device__ __forceinline__ unsigned long long reserve(const ListArgs& a, int n) {
  unsigned long long base = 0;
  if ((threadIdx.x & 31) == 0 && n > 0) base = atomicAdd(&a.ctl->count[0], (unsigned long long)n);
  return __shfl_sync(kFull, base, 0);
}

// Tuples (pre[0..np), x) for every x of X[0..nx).
__device__ __forceinline__ void emit_tail(const ListArgs& a, const int32_t* pre, int np,
                                          const int32_t* X, int nx) {
  const unsigned long long base = reserve(a, nx);
  for (int i = threadIdx.x & 31; i < nx; i += 32) {
    const unsigned long long slot = base + (unsigned long long)i;
    if (slot < (unsigned long long)a.capacity) {
      int32_t* o = a.out + slot * (unsigned long long)a.k;
      for (int q = 0; q < np; ++q) o[q] = pre[q];
      o[np] = X[i];
    }
  }
  __syncwarp();
}

// Tuples (a0, a1, f(x), g(x)) for x of X[0..nx): the 4-vertex plans' last level, with the
// two last positions given by `x_pos` (2: (a0, a1, x, b), 3: (a0, a1, b, x)) and b fixed.
__device__ __forceinline__ void emit4(const ListArgs& a, int32_t a0, int32_t a1, int32_t b,
                                      const int32_t* X, int nx, int x_pos) {
  const unsigned long long base = reserve(a, nx);
  for (int i = threadIdx.x & 31; i < nx; i += 32) {
    const unsigned long long slot = base + (unsigned long long)i;
    if (slot < (unsigned long long)a.capacity) {
      int32_t* o = a.out + slot * 4ull;
      o[0] = a0;
      o[1] = a1;
      o[2] = x_pos == 2 ? X[i] : b;
      o[3] = x_pos == 2 ? b : X[i];
    }
  }
  __syncwarp();
}

// Clique levels on materialised lists: pre holds the np chosen vertices; REM = levels
// still to choose (compile-time, no run-time recursion).
template <int REM>
struct ListClique {
  __device__ static void run(const ListArgs& a, int32_t* pre, int np, const int32_t* cand,
                             int nc, int32_t* buf) {
    if (REM == 1) {
      emit_tail(a, pre, np, cand, nc);
      return;
    }
    for (int i = 0; i < nc; ++i) {
      const vid_t v = cand[i];
      const int t = warp_isect_a<false>(cand, nc, lnbr(a, v), ldg_deg(a, v), INT32_MAX, -1, -1,
                                        buf);
      if (t > 0) {
        pre[np] = v;
        ListClique<(REM > 1 ? REM - 1 : 1)>::run(a, pre, np + 1, buf, t, buf + a.cap);
      }
    }
  }
};

template <int KIND, int K>
__device__ __forceinline__ void list_arc(const ListArgs& a, vid_t v0, vid_t v1, int32_t* W) {
  const int32_t* N0 = lnbr(a, v0);
  const int d0 = ldg_deg(a, v0);
  const int32_t* N1 = lnbr(a, v1);
  const int d1 = ldg_deg(a, v1);
  int32_t* X = W + a.cap;
  int32_t* Y = X + a.cap;
  if (KIND == kLClique) {
    const int t = warp_intersect(N0, d0, N1, d1, INT32_MAX, W);
    if (t == 0) return;
    int32_t pre[8];
    pre[0] = v0;
    pre[1] = v1;
    ListClique<(K > 2 ? K - 2 : 1)>::run(a, pre, 2, W, t, X);
  } else if (KIND == kLC4) {
    if (v1 >= v0) return;
    for (int i = 0; i < d0; ++i) {
      const vid_t v2 = __ldg(N0 + i);
      if (v2 >= v1) break;
      const int t = warp_intersect(N1, d1, lnbr(a, v2), ldg_deg(a, v2), v0, W);
      emit4(a, v0, v1, v2, W, t, 2);  // v0 - v1 - x - v2
    }
  } else if (KIND == kLDiamond) {
    if (v1 >= v0) return;
    const int t = warp_intersect(N0, d0, N1, d1, INT32_MAX, W);
    for (int i = 0; i + 1 < t; ++i) emit4(a, v0, v1, W[i], W + i + 1, t - i - 1, 3);
  } else if (KIND == kLIC4) {
    if (v1 >= v0) return;
    for (int i = 0; i < d0; ++i) {
      const vid_t v2 = __ldg(N0 + i);
      if (v2 >= v1) break;
      if (contains_g(N1, d1, v2)) continue;  // v1 ~ v2: not induced
      const int tw = warp_intersect(N1, d1, lnbr(a, v2), ldg_deg(a, v2), v0, W);
      const int ty = warp_diff_a<false>(W, tw, N0, d0, INT32_MAX, v0, X);
      emit4(a, v0, v1, v2, X, ty, 2);
    }
  } else if (KIND == kLIDiamond) {
    if (v1 >= v0) return;
    const int t = warp_intersect(N0, d0, N1, d1, INT32_MAX, W);
    for (int i = 0; i < t; ++i) {
      const vid_t x = W[i];
      const int ty = warp_diff_a<false>(W + i + 1, t - i - 1, lnbr(a, x), ldg_deg(a, x),
                                        INT32_MAX, x, X);
      emit4(a, v0, v1, x, X, ty, 3);
    }
  } else if (KIND == kLITailed) {
    const int t = warp_intersect(N0, d0, N1, d1, INT32_MAX, W);
    int start = 0;
    if ((threadIdx.x & 31) == 0) {
      int lo = 0, hi = t;
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (W[mid] <= v1) lo = mid + 1;
        else hi = mid;
      }
      start = lo;
    }
    start = __shfl_sync(kFull, start, 0);
    if (start >= t) return;
    const int nd1 = warp_diff_a<true>(N0, d0, N1, d1, INT32_MAX, v1, X);
    for (int i = start; i < t; ++i) {
      const vid_t v2 = W[i];
      const int ty = warp_diff_a<false>(X, nd1, lnbr(a, v2), ldg_deg(a, v2), INT32_MAX, v2, Y);
      emit4(a, v0, v1, v2, Y, ty, 3);
    }
  } else if (KIND == kLIPath4) {
    if (v1 >= v0) return;
    const int na = warp_diff_a<true>(N0, d0, N1, d1, INT32_MAX, v1, W);
    if (na == 0) return;
    const int nd = warp_diff_a<true>(N1, d1, N0, d0, INT32_MAX, v0, X);
    for (int i = 0; i < na; ++i) {
      const vid_t x = W[i];
      const int ty = warp_diff_a<false>(X, nd, lnbr(a, x), ldg_deg(a, x), INT32_MAX, x, Y);
      emit4(a, v0, v1, x, Y, ty, 3);  // path x - v0 - v1 - y
    }
  } else if (KIND == kLIStar3) {
    int lo = 0;
    if ((threadIdx.x & 31) == 0) lo = upper_bound_g(N0, d0, v1);
    lo = __shfl_sync(kFull, lo, 0);
    const int nd1 = warp_diff_a<true>(N0 + lo, d0 - lo, N1, d1, INT32_MAX, v1, W);
    for (int i = 0; i < nd1; ++i) {
      const vid_t y = W[i];
      const int tz = warp_diff_a<false>(W + i + 1, nd1 - i - 1, lnbr(a, y), ldg_deg(a, y),
                                        INT32_MAX, y, X);
      emit4(a, v0, v1, y, X, tz, 3);  // centre v0
    }
  }
}

template <int KIND, int K>
__global__ void __launch_bounds__(256) k_list(ListArgs a) {
  const int lane = threadIdx.x & 31;
  const int64_t gwarp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int32_t* W = a.scratch + gwarp * kListLevels * a.cap;
  constexpr int kChunk = 4;
  for (;;) {
    unsigned long long c0 = 0;
    if (lane == 0) c0 = atomicAdd(&a.ctl->counter[0], (unsigned long long)kChunk);
    c0 = __shfl_sync(kFull, c0, 0);
    if ((int64_t)c0 >= a.nslots) break;
    const int64_t s1 = min((int64_t)c0 + kChunk, a.nslots);
    int64_t lo = 0, hi = a.n;  // owner of slot c0: the last v with rowptr[v] <= c0
    while (lo < hi) {
      const int64_t mid = (lo + hi + 1) >> 1;
      if (a.rowptr[mid] <= (int64_t)c0) lo = mid;
      else hi = mid - 1;
    }
    vid_t v0 = (vid_t)lo;
    for (int64_t sl = (int64_t)c0; sl < s1; ++sl) {
      while (a.rowptr[v0 + 1] <= sl) ++v0;
      list_arc<KIND, K>(a, v0, __ldg(a.col + sl), W);
    }
  }
}

int launch_list(int kind, int k, const ListArgs& a, int grid, cudaStream_t s) {
  switch (kind) {
    case kLClique:
      switch (k) {
        case 3: k_list<kLClique, 3><<<grid, 256, 0, s>>>(a); break;
        case 4: k_list<kLClique, 4><<<grid, 256, 0, s>>>(a); break;
        case 5: k_list<kLClique, 5><<<grid, 256, 0, s>>>(a); break;
        case 6: k_list<kLClique, 6><<<grid, 256, 0, s>>>(a); break;
        case 7: k_list<kLClique, 7><<<grid, 256, 0, s>>>(a); break;
        default: k_list<kLClique, 8><<<grid, 256, 0, s>>>(a); break;
      }
      break;
    case kLC4: k_list<kLC4, 4><<<grid, 256, 0, s>>>(a); break;
    case kLDiamond: k_list<kLDiamond, 4><<<grid, 256, 0, s>>>(a); break;
    case kLIC4: k_list<kLIC4, 4><<<grid, 256, 0, s>>>(a); break;
    case kLIDiamond: k_list<kLIDiamond, 4><<<grid, 256, 0, s>>>(a); break;
    case kLITailed: k_list<kLITailed, 4><<<grid, 256, 0, s>>>(a); break;
    case kLIPath4: k_list<kLIPath4, 4><<<grid, 256, 0, s>>>(a); break;
    default: k_list<kLIStar3, 4><<<grid, 256, 0, s>>>(a); break;
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    jgpm_set_error_(std::string("listing launch: ") + cudaGetErrorString(e));
    return JGPM_ECUDA;
  }
  return JGPM_OK;
}

// Listing kind and embedding size of a pattern name, or -1.
int list_kind_of(const std::string& p, int induced, int* k) {
  if (induced) {
    *k = 4;
    if (p == "4-cycle" || p == "P1") return kLIC4;
    if (p == "diamond" || p == "P2") return kLIDiamond;
    if (p == "tailed-triangle") return kLITailed;
    if (p == "4-path") return kLIPath4;
    if (p == "3-star") return kLIStar3;
    return -1;
  }
  int kk = 0;
  if (p == "triangle" || p == "P0" || p == "3-clique") kk = 3;
  else if (p == "4-clique" || p == "P13") kk = 4;
  else if (p == "5-clique" || p == "P14") kk = 5;
  else if (p == "6-clique" || p == "P15") kk = 6;
  else if (p == "7-clique" || p == "P16") kk = 7;
  else if (p.rfind("k-clique:", 0) == 0) kk = std::atoi(p.c_str() + 9);
  if (kk != 0) {
    if (kk < 3 || kk > 8) return -1;
    *k = kk;
    return kLClique;
  }
  *k = 4;
  if (p == "4-cycle" || p == "P1") return kLC4;
  if (p == "diamond" || p == "P2") return kLDiamond;
  return -1;
}

}  // namespace
}  // namespace jgpm

using namespace jgpm;

extern "C" int jgpm_list(jgpm_graph* g, const char* pattern, int induced, int32_t* out,
                         int64_t capacity, int64_t* total, jgpm_stats* st) {
  if (!g || !pattern || !total || capacity < 0 || (capacity > 0 && !out)) {
    jgpm_set_error_("jgpm_list: bad arguments");
    return JGPM_EINVAL;
  }
  int k = 0;
  const int kind = list_kind_of(pattern, induced, &k);
  if (kind < 0) {
    jgpm_set_error_(std::string("jgpm_list: no listing plan for '") + pattern + "'" +
                    (induced ? " (vertex-induced)" : ""));
    return JGPM_EPATTERN;
  }
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != g->device) cudaSetDevice(g->device);
  struct Restore {
    int prev, dev;
    ~Restore() {
      if (prev >= 0 && prev != dev) cudaSetDevice(prev);
    }
  } restore{prev, g->device};
  int rc;
  const bool dag = kind == kLClique;
  if (dag && (rc = ensure_dag(g))) return rc;
  if ((rc = ensure_control(g))) return rc;
  const int32_t maxd = dag ? g->max_out_degree : g->max_degree;
  const int64_t cap = (int64_t)maxd + 32;
  const int64_t per_warp = (int64_t)kListLevels * cap;
  const int sms = device_sm_count(g->device);
  int64_t warps = std::min<int64_t>((int64_t)sms * 64, ((int64_t)2 << 30) / (per_warp * 4));
  warps = std::max<int64_t>(8, warps - warps % 8);
  if ((rc = ensure_scratch(g, (size_t)(warps * per_warp) * sizeof(int32_t)))) return rc;
  // the output: the caller's device buffer, or a device staging buffer copied back
  cudaPointerAttributes attr;
  const bool dev_out = capacity > 0 && cudaPointerGetAttributes(&attr, out) == cudaSuccess &&
                       attr.type == cudaMemoryTypeDevice;
  cudaGetLastError();
  int32_t* d_out = dev_out ? out : nullptr;
  const size_t out_bytes = (size_t)capacity * k * sizeof(int32_t);
  if (!dev_out && capacity > 0 && (rc = gmalloc((void**)&d_out, out_bytes, g->stream)))
    return rc;
  struct Staging {
    int32_t* p;
    bool owned;
    cudaStream_t s;
    ~Staging() {
      if (owned) gfree(p, s);
    }
  } staging{d_out, !dev_out && capacity > 0, g->stream};
  ListArgs a{};
  a.rowptr = dag ? g->d_dag_rowptr : g->d_rowptr;
  a.col = dag ? g->d_dag_col : g->d_col;
  a.n = g->n;
  a.nslots = dag ? g->m_dag : g->m;
  a.ctl = g->d_ctl;
  a.scratch = (int32_t*)g->d_scratch;
  a.cap = cap;
  a.out = d_out;
  a.capacity = capacity;
  a.k = k;
  cudaEvent_t e0, e1;
  JGPM_CUDA_TRY(cudaEventCreate(&e0));
  JGPM_CUDA_TRY(cudaEventCreate(&e1));
  JGPM_CUDA_TRY(cudaMemsetAsync(g->d_ctl, 0, sizeof(DevControl), g->stream));
  JGPM_CUDA_TRY(cudaEventRecord(e0, g->stream));
  g->launches = 0;
  if (a.nslots > 0) {
    if ((rc = launch_list(kind, k, a, (int)(warps / 8), g->stream))) return rc;
    g->launches = 1;
  }
  JGPM_CUDA_TRY(cudaEventRecord(e1, g->stream));
  JGPM_CUDA_TRY(cudaMemcpyAsync(g->h_ctl, g->d_ctl, sizeof(DevControl), cudaMemcpyDeviceToHost,
                                g->stream));
  JGPM_CUDA_TRY(cudaStreamSynchronize(g->stream));
  const uint64_t n_found = g->h_ctl->count[0];
  const uint64_t n_written = std::min<uint64_t>(n_found, (uint64_t)capacity);
  if (!dev_out && n_written > 0) {
    JGPM_CUDA_TRY(cudaMemcpyAsync(out, d_out, n_written * k * sizeof(int32_t),
                                  cudaMemcpyDeviceToHost, g->stream));
    JGPM_CUDA_TRY(cudaStreamSynchronize(g->stream));
  }
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *total = (int64_t)n_found;
  if (st) {
    memset(st, 0, sizeof(*st));
    st->count = n_found;
    st->kernel_ms = ms;
    st->rounds = 1;
    st->method = JGPM_METHOD_PLAN;
    st->launches = g->launches;
  }
  return JGPM_OK;
}
