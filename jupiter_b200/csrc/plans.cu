// Non-clique patterns: the reference's nested-loop plans as warp kernels, the
// wedge-aggregation 4-cycle count, per-edge triangle counts (diamond), and the vertex-induced
// 4-vertex census.
//
// Literal plan kernel (k_plan).  One warp per root arc, exactly the loop nests of the
// message-passing kernels in src/message_passing_gpu_kernels.cuh (P1 :104-186, P2 :188-252,
// P3 :254-334, P4 :336-420, P5 :422-502, P6 :504-576, P7 :578-659, P8 :661-745, P9 :747-825,
// P10 :827-918, P11 :920-1021, P12 :1023-1109, vsgm :1111-1206, P13..P16 :1208-1537), with
// warp set operations from setops.cuh.  The innermost "count every element of a list
// except a few ancestors" loops are evaluated as |list| minus the number of distinct
// ancestors present in the list, which is the same number.  Candidate lists live in four
// per-warp global scratch lists (the reference uses per-warp max_deg buffers,
// src/jupiter_gpm.cu:333-336).
//
// Fast methods (same counts):
//   4-cycle (P1)  wedge aggregation in degree order (Chiba and Nishizeki, SIAM J. Comput.
//                 1985): every 4-cycle is counted once at its highest-ranked vertex v0 and
//                 the opposite vertex v3, as C(c, 2) where c = common lower-ranked
//                 neighbours; rank = (degree, id), the DAG's order.
//   diamond (P2)  sum over edges of C(t_e, 2), with t_e the triangles on edge e, listed once
//                 on the DAG by the bitmap kernel.
//   vertex-induced 4-vertex patterns: from the edge-induced counts N(.) and the standard
//                 induced/non-induced identities of 4-vertex graphlets.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>

#include "jgpm_internal.h"
#include "setops.cuh"

namespace jgpm {

int launch_clique(jgpm_graph* g, int k, bool stats, int64_t root_begin, int64_t root_end,
                  cudaStream_t s);
int launch_edge_triangles(jgpm_graph* g, uint32_t* d_tri, cudaStream_t s);
int launch_diamond_pairs(jgpm_graph* g, uint32_t* d_tri, cudaStream_t s);
int launch_induced_tt(jgpm_graph* g, uint32_t* d_tri, cudaStream_t s);

enum PlanId {
  kP0 = 0, kP1 = 1, kP2 = 2, kP3 = 3, kP4 = 4, kP5 = 5, kP6 = 6, kP7 = 7, kP8 = 8, kP9 = 9,
  kP10 = 10, kP11 = 11, kP12 = 12, kVsgm = 13,
  kK4 = 14, kK5 = 15, kK6 = 16, kK7 = 17,
  kIC4 = 20, kIDiamond = 21, kITailed = 22, kIPath4 = 23, kIStar3 = 24,
  kNTailed = 30, kNPath4 = 31, kNStar3 = 32,
};

int plan_id_of(const std::string& p, int induced) {
  if (induced) {
    if (p == "4-cycle" || p == "P1") return kIC4;
    if (p == "diamond" || p == "P2") return kIDiamond;
    if (p == "tailed-triangle") return kITailed;
    if (p == "4-path") return kIPath4;
    if (p == "3-star") return kIStar3;
    return -1;
  }
  if (p == "P0") return kP0;
  if (p == "P1" || p == "4-cycle") return kP1;
  if (p == "P2" || p == "diamond") return kP2;
  if (p == "P3") return kP3;
  if (p == "P4") return kP4;
  if (p == "P5") return kP5;
  if (p == "P6") return kP6;
  if (p == "P7") return kP7;
  if (p == "P8") return kP8;
  if (p == "P9") return kP9;
  if (p == "P10") return kP10;
  if (p == "P11") return kP11;
  if (p == "P12") return kP12;
  if (p == "vsgm_last_pattern") return kVsgm;
  if (p == "P13" || p == "4-clique") return kK4;
  if (p == "P14" || p == "5-clique") return kK5;
  if (p == "P15" || p == "6-clique") return kK6;
  if (p == "P16" || p == "7-clique") return kK7;
  if (p == "tailed-triangle") return kNTailed;
  if (p == "4-path") return kNPath4;
  if (p == "3-star") return kNStar3;
  return -1;
}

bool plan_uses_dag(int id) { return id == kP0 || (id >= kK4 && id <= kK7); }

namespace {

struct PlanArgs {
  const eid_t* rowptr;
  const vid_t* col;
  vid_t n;
  // root arcs: the CSR slots slot_begin + i * slot_stride, 0 <= i < nsamp (< slot_end)
  int64_t slot_begin, slot_end;
  int64_t slot_stride, nsamp;
  DevControl* ctl;
  int32_t* scratch;
  int64_t cap;  // entries per scratch list (4 lists per warp)
};

struct Lists {
  int32_t* W;
  int32_t* X;
  int32_t* Y;
  int32_t* Z;
};

__device__ __forceinline__ const int32_t* nbr(const PlanArgs& a, vid_t v) {
  return a.col + a.rowptr[v];
}
__device__ __forceinline__ int dg(const PlanArgs& a, vid_t v) {
  return (int)(a.rowptr[v + 1] - a.rowptr[v]);
}

// Number of distinct values of ex[0..ne) present in the sorted list (plain loads).
template <bool RO>
__device__ __forceinline__ int present_distinct(const int32_t* list, int n, const int32_t* ex,
                                                int ne) {
  int c = 0;
  for (int i = 0; i < ne; ++i) {
    bool dup = false;
    for (int j = 0; j < i; ++j) dup = dup || (ex[j] == ex[i]);
    if (dup) continue;
    const int p = lower_bound_t<RO>(list, n, ex[i]);
    if (p < n && ld32<RO>(list + p) == ex[i]) ++c;
  }
  return c;
}

template <bool RO>
__device__ __forceinline__ int prefix_len(const int32_t* a, int n, int32_t upper) {
  return upper == INT32_MAX ? n : lower_bound_t<RO>(a, n, upper);
}

// Clique levels on materialised lists (P13..P16 literal); REM = levels still to choose,
// a compile-time count so the device code does not recurse at run time.
template <int REM, bool STATS>
struct PlanClique {
  __device__ static acc_t run(const PlanArgs& a, const int32_t* cand, int nc, int32_t* buf,
                              int64_t cap, acc_t& el) {
    const int lane = threadIdx.x & 31;
    acc_t s = 0;
    for (int i = 0; i < nc; ++i) {
      const vid_t v = cand[i];
      const int32_t* nv = nbr(a, v);
      const int dv = dg(a, v);
      if (STATS && lane == 0) el += (acc_t)nc + (acc_t)dv;
      if (REM == 1) {
        s += (acc_t)warp_isect_a<false>(cand, nc, nv, dv, INT32_MAX, -1, -1, nullptr);
      } else {
        const int t = warp_isect_a<false>(cand, nc, nv, dv, INT32_MAX, -1, -1, buf);
        if (t > 0)
          s += PlanClique<(REM > 1 ? REM - 1 : 1), STATS>::run(a, buf, t, buf + cap, cap, el);
      }
    }
    return s;
  }
};

// One root arc (v0, v1) of plan P.  Returns the warp-uniform contribution; `lc` collects
// per-lane partial contributions (summed at the end); `el` the set-op elements (lane 0).
template <int P, bool STATS>
__device__ __forceinline__ acc_t run_plan(const PlanArgs& a, vid_t v0, vid_t v1, Lists& L,
                                          acc_t& lc, acc_t& el) {
  const int lane = threadIdx.x & 31;
  const int32_t* N0 = nbr(a, v0);
  const int d0 = dg(a, v0);
  const int32_t* N1 = nbr(a, v1);
  const int d1 = dg(a, v1);
  acc_t u = 0;  // warp-uniform part
  if (P == kP0) {
    if (STATS && lane == 0) el += (acc_t)d0 + d1;
    u += (acc_t)warp_intersect_count(N0, d0, N1, d1);
  } else if (P == kP1) {
    if (v1 >= v0) return 0;
    for (int i = 0; i < d0; ++i) {
      const vid_t v2 = __ldg(N0 + i);
      if (v2 >= v1) break;
      const int32_t* N2 = nbr(a, v2);
      const int d2 = dg(a, v2);
      if (STATS && lane == 0)
        el += (acc_t)prefix_len<true>(N1, d1, v0) + prefix_len<true>(N2, d2, v0);
      u += (acc_t)warp_intersect_count(N1, d1, N2, d2, v0);
    }
  } else if (P == kP2) {
    if (v1 >= v0) return 0;
    if (STATS && lane == 0) el += (acc_t)d0 + d1;
    const acc_t t = (acc_t)warp_intersect_count(N0, d0, N1, d1);
    u += t * (t - (t > 0 ? 1 : 0)) / 2;
  } else if (P == kK4 || P == kK5 || P == kK6 || P == kK7) {
    constexpr int K = P == kK4 ? 4 : P == kK5 ? 5 : P == kK6 ? 6 : 7;
    if (STATS && lane == 0) el += (acc_t)d0 + d1;
    const int t = warp_intersect(N0, d0, N1, d1, INT32_MAX, L.W);
    if (t > 0) u += PlanClique<K - 3, STATS>::run(a, L.W, t, L.X, a.cap, el);
  } else {
    // plans that start with W = N(v0) & N(v1)
    if ((P == kP4 || P == kP5 || P == kP6 || P == kIC4 || P == kIDiamond || P == kIPath4) &&
        v1 >= v0)
      return 0;
    if ((P == kP9 || P == kP11 || P == kP12 || P == kVsgm) && v1 <= v0) return 0;
    int t = 0;
    if (P != kIC4 && P != kIPath4 && P != kIStar3) {
      if (STATS && lane == 0) el += (acc_t)d0 + d1;
      t = warp_intersect(N0, d0, N1, d1, INT32_MAX, L.W);
    }
    if (P == kP3) {
      for (int i3 = 0; i3 < d0; ++i3) {
        const vid_t v3 = __ldg(N0 + i3);
        if (v3 == v1) continue;
        const int32_t* N3 = nbr(a, v3);
        const int d3 = dg(a, v3);
        for (int j = lane; j < t; j += 32) {
          const vid_t v2 = L.W[j];
          if (v2 <= v1 || v2 == v3 || v2 == v0) continue;
          const int32_t ex[4] = {v0, v1, v3, v2};
          lc += (acc_t)(d3 - present_distinct<true>(N3, d3, ex, 4));
        }
      }
    } else if (P == kP4) {
      for (int i3 = 0; i3 < d1; ++i3) {
        const vid_t v3 = __ldg(N1 + i3);
        if (v3 == v0) continue;
        const int32_t* N3 = nbr(a, v3);
        const int d3 = dg(a, v3);
        if (STATS && lane == 0) el += (acc_t)d0 + d3;
        const int tx = warp_intersect(N0, d0, N3, d3, INT32_MAX, L.X);
        for (int j = lane; j < t; j += 32) {
          const vid_t v2 = L.W[j];
          if (v3 == v2) continue;
          const int32_t ex[2] = {v1, v2};
          lc += (acc_t)(tx - present_distinct<false>(L.X, tx, ex, 2));
        }
        __syncwarp();
      }
    } else if (P == kP5) {
      for (int i = 0; i < t; ++i) {
        const vid_t v2 = L.W[i];
        const int32_t* N2 = nbr(a, v2);
        const int d2 = dg(a, v2);
        if (STATS && lane == 0)
          el += (acc_t)prefix_len<false>(L.W, t, v2) + prefix_len<true>(N2, d2, v2);
        const int tx = warp_isect_a<false>(L.W, t, N2, d2, v2, -1, -1, L.X);
        for (int j = lane; j < t; j += 32) {
          const vid_t v4 = L.W[j];
          if (v2 == v4) continue;
          const int32_t ex[1] = {v4};
          lc += (acc_t)(tx - present_distinct<false>(L.X, tx, ex, 1));
        }
        __syncwarp();
      }
    } else if (P == kP6) {
      for (int i2 = 0; i2 < t; ++i2) {
        const vid_t v2 = L.W[i2];
        const int32_t* N2 = nbr(a, v2);
        const int d2 = dg(a, v2);
        for (int i3 = 0; i3 < i2; ++i3) {
          const vid_t v3 = L.W[i3];
          const int32_t* N3 = nbr(a, v3);
          const int d3 = dg(a, v3);
          if (STATS && lane == 0) el += (acc_t)d2 + d3;
          u += (acc_t)warp_intersect_count(N2, d2, N3, d3, INT32_MAX, v0, v1);
        }
      }
    } else if (P == kP7) {
      for (int i2 = 0; i2 < t; ++i2) {
        const vid_t v2 = L.W[i2];
        if (v2 <= v1) continue;
        const int32_t* N2 = nbr(a, v2);
        const int d2 = dg(a, v2);
        if (STATS && lane == 0) el += (acc_t)d0 + d2;
        const int tx = warp_intersect(N0, d0, N2, d2, INT32_MAX, L.X);
        for (int j = lane; j < tx; j += 32) {
          const vid_t v4 = L.X[j];
          if (v1 == v4) continue;
          const int32_t ex[2] = {v4, v2};
          lc += (acc_t)(t - present_distinct<false>(L.W, t, ex, 2));
        }
        __syncwarp();
      }
    } else if (P == kP8) {
      for (int i2 = 0; i2 < t; ++i2) {
        const vid_t v2 = L.W[i2];
        if (v2 >= v1) continue;
        const int32_t* N2 = nbr(a, v2);
        const int d2 = dg(a, v2);
        if (STATS && lane == 0) el += (acc_t)d0 + d2;
        const int tx = warp_intersect(N0, d0, N2, d2, INT32_MAX, L.X);
        for (int k = 0; k < tx; ++k) {
          const vid_t v3 = L.X[k];
          if (v3 >= v1) continue;
          const int32_t* N3 = nbr(a, v3);
          const int d3 = dg(a, v3);
          if (STATS && lane == 0)
            el += (acc_t)prefix_len<false>(L.W, t, v2) + prefix_len<true>(N3, d3, v2);
          u += (acc_t)warp_isect_a<false>(L.W, t, N3, d3, v2, -1, -1, nullptr);
        }
        __syncwarp();
      }
    } else if (P == kP9) {
      for (int i2 = 0; i2 < t; ++i2) {
        const vid_t v2 = L.W[i2];
        if (v2 <= v1) continue;
        const int32_t* N2 = nbr(a, v2);
        const int d2 = dg(a, v2);
        if (STATS && lane == 0) el += (acc_t)t + d2;
        const acc_t tx = (acc_t)warp_isect_a<false>(L.W, t, N2, d2, INT32_MAX, -1, -1, nullptr);
        u += tx * (tx - (tx > 0 ? 1 : 0)) / 2;
      }
    } else if (P == kP10) {
      for (int i2 = 0; i2 < t; ++i2) {
        const vid_t v2 = L.W[i2];
        const int32_t* N2 = nbr(a, v2);
        const int d2 = dg(a, v2);
        if (STATS && lane == 0) el += (acc_t)d0 + d2;
        const int tx = warp_intersect(N0, d0, N2, d2, INT32_MAX, L.X);
        for (int k = 0; k < tx; ++k) {
          const vid_t v3 = L.X[k];
          if (v3 <= v1) continue;
          const int32_t* N3 = nbr(a, v3);
          const int d3 = dg(a, v3);
          if (STATS && lane == 0) el += (acc_t)d0 + d3;
          const int ty = warp_intersect(N0, d0, N3, d3, INT32_MAX, L.Y);
          for (int j = lane; j < t; j += 32) {
            const vid_t v4 = L.W[j];
            if (v4 == v2 || v4 == v1 || v4 == v3) continue;
            const int32_t ex[4] = {v4, v1, v2, v3};
            lc += (acc_t)(ty - present_distinct<false>(L.Y, ty, ex, 4));
          }
          __syncwarp();
        }
      }
    } else if (P == kP11) {
      for (int i2 = 0; i2 < t; ++i2) {
        const vid_t v2 = L.W[i2];
        if (v2 <= v1) continue;
        const int32_t* N2 = nbr(a, v2);
        const int d2 = dg(a, v2);
        if (STATS && lane == 0) el += (acc_t)d0 + d2 + d1 + d2;
        const int tx = warp_intersect(N0, d0, N2, d2, INT32_MAX, L.X);
        const int tz = warp_intersect(N1, d1, N2, d2, INT32_MAX, L.Z);
        for (int i3 = 0; i3 < t; ++i3) {
          const vid_t v3 = L.W[i3];
          if (v3 == v2 || v3 == v1 || v3 == v0) continue;
          for (int j = lane; j < tx; j += 32) {
            const vid_t v4 = L.X[j];
            if (v4 == v3 || v4 == v2 || v4 == v1) continue;
            const int32_t ex[5] = {v4, v1, v2, v3, v0};
            lc += (acc_t)(tz - present_distinct<false>(L.Z, tz, ex, 5));
          }
        }
        __syncwarp();
      }
    } else if (P == kP12) {
      for (int i2 = 0; i2 < t; ++i2) {
        const vid_t v2 = L.W[i2];
        const int32_t* N2 = nbr(a, v2);
        const int d2 = dg(a, v2);
        if (STATS && lane == 0) el += (acc_t)t + d2;
        const int tx = warp_isect_a<false>(L.W, t, N2, d2, INT32_MAX, -1, -1, L.X);
        for (int i3 = 0; i3 < tx; ++i3) {
          const vid_t v3 = L.X[i3];
          for (int i4 = i3 + 1 + lane; i4 < tx; i4 += 32) {
            const vid_t v4 = L.X[i4];
            const int32_t ex[5] = {v4, v1, v2, v3, v0};
            lc += (acc_t)(t - present_distinct<false>(L.W, t, ex, 5));
          }
        }
        __syncwarp();
      }
    } else if (P == kVsgm) {
      for (int i2 = 0; i2 < d0; ++i2) {
        const vid_t v2 = __ldg(N0 + i2);
        if (v2 == v1) continue;
        const int32_t* N2 = nbr(a, v2);
        const int d2 = dg(a, v2);
        if (STATS && lane == 0) el += (acc_t)d1 + d2;
        const int tz = warp_intersect(N1, d1, N2, d2, INT32_MAX, L.Z);
        for (int i5 = 0; i5 < tz; ++i5) {
          const vid_t v5 = L.Z[i5];
          if (v5 == v0) continue;
          for (int j3 = lane; j3 < t; j3 += 32) {
            const vid_t v3 = L.W[j3];
            if (v3 == v2 || v3 == v1 || v3 == v0 || v3 == v5) continue;
            // w in W, w > v3, w not in {v0, v1, v2, v5}
            const int32_t* tail = L.W + j3 + 1;
            const int nt = t - j3 - 1;
            const int32_t ex[4] = {v0, v1, v2, v5};
            lc += (acc_t)(nt - present_distinct<false>(tail, nt, ex, 4));
          }
        }
        __syncwarp();
      }
    } else if (P == kIC4) {
      for (int i = 0; i < d0; ++i) {
        const vid_t v2 = __ldg(N0 + i);
        if (v2 >= v1) break;
        if (contains_g(N1, d1, v2)) continue;  // v1 ~ v2: not induced
        const int32_t* N2 = nbr(a, v2);
        const int d2 = dg(a, v2);
        if (STATS && lane == 0)
          el += (acc_t)prefix_len<true>(N1, d1, v0) + prefix_len<true>(N2, d2, v0);
        const int tw = warp_intersect(N1, d1, N2, d2, v0, L.W);
        if (STATS && lane == 0) el += (acc_t)tw + d0;
        u += (acc_t)warp_diff_a<false>(L.W, tw, N0, d0, INT32_MAX, v0, nullptr);
      }
    } else if (P == kIDiamond) {
      for (int i = 0; i < t; ++i) {
        const vid_t x = L.W[i];
        const int32_t* Nx = nbr(a, x);
        const int dx = dg(a, x);
        if (STATS && lane == 0) el += (acc_t)(t - i - 1) + dx;
        u += (acc_t)warp_diff_a<false>(L.W + i + 1, t - i - 1, Nx, dx, INT32_MAX, x, nullptr);
      }
    } else if (P == kITailed) {
      int start = 0;
      if (lane == 0) {
        int lo = 0, hi = t;
        while (lo < hi) {
          const int mid = (lo + hi) >> 1;
          if (L.W[mid] <= v1) lo = mid + 1;
          else hi = mid;
        }
        start = lo;
      }
      start = __shfl_sync(kFull, start, 0);
      if (start < t) {
        if (STATS && lane == 0) el += (acc_t)d0 + d1;
        const int nd1 = warp_diff_a<true>(N0, d0, N1, d1, INT32_MAX, v1, L.X);
        for (int i = start; i < t; ++i) {
          const vid_t v2 = L.W[i];
          const int32_t* N2 = nbr(a, v2);
          const int d2 = dg(a, v2);
          if (STATS && lane == 0) el += (acc_t)nd1 + d2;
          u += (acc_t)warp_diff_a<false>(L.X, nd1, N2, d2, INT32_MAX, v2, nullptr);
        }
      }
    } else if (P == kIPath4) {
      if (STATS && lane == 0) el += (acc_t)d0 + d1;
      const int na = warp_diff_a<true>(N0, d0, N1, d1, INT32_MAX, v1, L.W);
      if (na > 0) {
        if (STATS && lane == 0) el += (acc_t)d1 + d0;
        const int nd = warp_diff_a<true>(N1, d1, N0, d0, INT32_MAX, v0, L.X);
        for (int i = 0; i < na; ++i) {
          const vid_t x = L.W[i];
          const int32_t* Nx = nbr(a, x);
          const int dx = dg(a, x);
          if (STATS && lane == 0) el += (acc_t)nd + dx;
          u += (acc_t)warp_diff_a<false>(L.X, nd, Nx, dx, INT32_MAX, x, nullptr);
        }
      }
    } else if (P == kIStar3) {
      int lo = 0;
      if (lane == 0) lo = upper_bound_g(N0, d0, v1);
      lo = __shfl_sync(kFull, lo, 0);
      if (STATS && lane == 0) el += (acc_t)(d0 - lo) + d1;
      const int nd1 = warp_diff_a<true>(N0 + lo, d0 - lo, N1, d1, INT32_MAX, v1, L.W);
      for (int i = 0; i < nd1; ++i) {
        const vid_t y = L.W[i];
        const int32_t* Ny = nbr(a, y);
        const int dy = dg(a, y);
        if (STATS && lane == 0) el += (acc_t)(nd1 - i - 1) + dy;
        u += (acc_t)warp_diff_a<false>(L.W + i + 1, nd1 - i - 1, Ny, dy, INT32_MAX, y, nullptr);
      }
    }
  }
  __syncwarp();
  return u;
}

template <int P, bool STATS>
__global__ void __launch_bounds__(256) k_plan(PlanArgs a) {
  const int lane = threadIdx.x & 31;
  const int64_t gwarp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  Lists L;
  L.W = a.scratch + gwarp * 4 * a.cap;
  L.X = L.W + a.cap;
  L.Y = L.X + a.cap;
  L.Z = L.Y + a.cap;
  acc_t lc = 0, uc = 0, el = 0;
  constexpr int kChunk = 4;
  // owner of slot s among the vertices [lo, n): the last v with rowptr[v] <= s
  auto owner = [&](int64_t lo, int64_t s) {
    int64_t hi = a.n;
    while (lo < hi) {
      const int64_t mid = (lo + hi + 1) >> 1;
      if (a.rowptr[mid] <= s) lo = mid;
      else hi = mid - 1;
    }
    return (vid_t)lo;
  };
  for (;;) {
    unsigned long long c0 = 0;
    if (lane == 0) c0 = atomicAdd(&a.ctl->counter[0], (unsigned long long)kChunk);
    c0 = __shfl_sync(kFull, c0, 0);
    if ((int64_t)c0 >= a.nsamp) break;
    const int64_t i1 = min((int64_t)c0 + kChunk, a.nsamp);
    vid_t v0 = owner(0, a.slot_begin + (int64_t)c0 * a.slot_stride);
    for (int64_t i = (int64_t)c0; i < i1; ++i) {
      const int64_t s = a.slot_begin + i * a.slot_stride;
      if (a.slot_stride == 1) {
        while (a.rowptr[v0 + 1] <= s) ++v0;
      } else {
        v0 = owner(v0, s);
      }
      const vid_t v1 = __ldg(a.col + s);
      uc += run_plan<P, STATS>(a, v0, v1, L, lc, el);
    }
  }
  for (int o = 16; o > 0; o >>= 1) lc += __shfl_xor_sync(kFull, lc, o);
  if (lane == 0) {
    const acc_t tot = lc + uc;
    if (tot) atomicAdd(&a.ctl->count[0], tot);
    if (STATS && el) atomicAdd(&a.ctl->elements[0], el);
  }
}

// ------------------------------------------------------------------ census reductions
struct U128 {
  unsigned long long lo, hi;
};

__device__ __forceinline__ void atomic_add_u128(unsigned long long* lo, unsigned long long* hi,
                                                unsigned __int128 v) {
  const unsigned long long vlo = (unsigned long long)v;
  const unsigned long long vhi = (unsigned long long)(v >> 64);
  if (vlo) {
    const unsigned long long old = atomicAdd(lo, vlo);
    if (old + vlo < old) atomicAdd(hi, 1ull);
  }
  if (vhi) atomicAdd(hi, vhi);
}

__device__ __forceinline__ unsigned __int128 warp_sum_u128(unsigned __int128 v) {
  unsigned long long lo = (unsigned long long)v, hi = (unsigned long long)(v >> 64);
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long olo = __shfl_xor_sync(kFull, lo, o);
    const unsigned long long ohi = __shfl_xor_sync(kFull, hi, o);
    const unsigned long long nlo = lo + olo;
    hi = hi + ohi + (nlo < lo ? 1ull : 0ull);
    lo = nlo;
  }
  return ((unsigned __int128)hi << 64) | lo;
}

// acc layout (pairs lo,hi): [0] sum t_e, [1] sum C(t_e,2), [2] sum t_v (d_v - 2) * 2,
// [3] sum over edges (d_u-1)(d_v-1), [4] sum C(d_v,3)
__global__ void k_census_edges(const eid_t* dag_rowptr, const vid_t* dag_col,
                               const eid_t* rowptr, vid_t n, const uint32_t* tri,
                               unsigned long long* tv2, unsigned long long* acc) {
  unsigned __int128 s_te = 0, s_c2 = 0, s_path = 0;
  const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int lane = threadIdx.x & 31;
  for (int64_t u = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < n; u += warps) {
    const eid_t b = dag_rowptr[u];
    const int64_t d = dag_rowptr[u + 1] - b;
    const int64_t du = rowptr[u + 1] - rowptr[u];
    unsigned long long tu = 0;
    for (int64_t i = lane; i < d; i += 32) {
      const vid_t v = __ldg(dag_col + b + i);
      const unsigned long long te = tri[b + i];
      const int64_t dv = rowptr[v + 1] - rowptr[v];
      s_te += te;
      s_c2 += (unsigned __int128)te * (te > 0 ? te - 1 : 0) / 2;
      s_path += (unsigned __int128)(du - 1) * (unsigned __int128)(dv - 1);
      tu += te;
      if (te) atomicAdd(&tv2[v], te);
    }
    for (int o = 16; o > 0; o >>= 1) tu += __shfl_xor_sync(kFull, tu, o);
    if (lane == 0 && tu) atomicAdd(&tv2[u], tu);
  }
  s_te = warp_sum_u128(s_te);
  s_c2 = warp_sum_u128(s_c2);
  s_path = warp_sum_u128(s_path);
  if (lane == 0) {
    atomic_add_u128(&acc[0], &acc[1], s_te);
    atomic_add_u128(&acc[2], &acc[3], s_c2);
    atomic_add_u128(&acc[6], &acc[7], s_path);
  }
}

__global__ void k_census_vertices(const eid_t* rowptr, vid_t n, const unsigned long long* tv2,
                                  unsigned long long* acc) {
  unsigned __int128 s_tt = 0, s_star = 0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
    const unsigned __int128 d = (unsigned __int128)(rowptr[v + 1] - rowptr[v]);
    const unsigned __int128 t2 = tv2[v];  // twice the triangles at v
    if (d >= 2) s_tt += t2 * (d - 2);
    if (d >= 3) s_star += d * (d - 1) * (d - 2) / 6;
  }
  s_tt = warp_sum_u128(s_tt);
  s_star = warp_sum_u128(s_star);
  if ((threadIdx.x & 31) == 0) {
    atomic_add_u128(&acc[4], &acc[5], s_tt);
    atomic_add_u128(&acc[8], &acc[9], s_star);
  }
}

int grid_for(int64_t work, int threads = 256) {
  int64_t b = (work + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > 148 * 32) b = 148 * 32;
  return (int)b;
}

template <int P>
int launch_plan_t(const PlanArgs& a, bool stats, int grid, cudaStream_t s) {
  if (stats) k_plan<P, true><<<grid, 256, 0, s>>>(a);
  else k_plan<P, false><<<grid, 256, 0, s>>>(a);
  return JGPM_OK;
}

int launch_plan(int id, const PlanArgs& a, bool stats, int grid, cudaStream_t s) {
  switch (id) {
#define JGPM_P(ID) \
  case ID:         \
    return launch_plan_t<ID>(a, stats, grid, s);
    JGPM_P(kP0) JGPM_P(kP1) JGPM_P(kP2) JGPM_P(kP3) JGPM_P(kP4) JGPM_P(kP5) JGPM_P(kP6)
    JGPM_P(kP7) JGPM_P(kP8) JGPM_P(kP9) JGPM_P(kP10) JGPM_P(kP11) JGPM_P(kP12) JGPM_P(kVsgm)
    JGPM_P(kK4) JGPM_P(kK5) JGPM_P(kK6) JGPM_P(kK7) JGPM_P(kIC4) JGPM_P(kIDiamond)
    JGPM_P(kITailed) JGPM_P(kIPath4) JGPM_P(kIStar3)
#undef JGPM_P
  }
  jgpm_set_error_("internal: no literal plan kernel for this pattern");
  return JGPM_EPATTERN;
}

struct Timer {
  cudaEvent_t a = nullptr, b = nullptr;
  Timer() {
    cudaEventCreate(&a);
    cudaEventCreate(&b);
  }
  ~Timer() {
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  }
  double ms() {
    float f = 0.f;
    cudaEventElapsedTime(&f, a, b);
    return f;
  }
};

int read_ctl(jgpm_graph* g) {
  JGPM_CUDA_TRY(cudaMemcpyAsync(g->h_ctl, g->d_ctl, sizeof(DevControl), cudaMemcpyDeviceToHost,
                                g->stream));
  JGPM_CUDA_TRY(cudaStreamSynchronize(g->stream));
  return JGPM_OK;
}

// Warps of a literal plan launch: as many as fit a 2 GiB scratch budget of four lists of
// maxd + 32 entries each, at most 8 CTAs of 8 warps per SM.
int64_t literal_warps(int sms, int32_t maxd) {
  const int64_t per_warp = 4 * ((int64_t)maxd + 32);
  int64_t warps = std::min<int64_t>((int64_t)sms * 64, ((int64_t)2 << 30) / (per_warp * 4));
  return std::max<int64_t>(8, warps - warps % 8);
}

// Runs the literal plan kernel over the root arcs begin, begin + stride, ... < end of the
// plan's CSR (end < 0: all of them), split into chunk_size rounds of consecutive samples.
int run_literal(jgpm_graph* g, int id, int chunk_size, bool stats, uint64_t* out,
                uint64_t* elements, double* ms, int64_t begin = 0, int64_t end = -1,
                int64_t stride = 1) {
  int rc;
  const bool dag = plan_uses_dag(id);
  if (dag && (rc = ensure_dag(g))) return rc;
  if ((rc = ensure_control(g))) return rc;
  const int32_t maxd = dag ? g->max_out_degree : g->max_degree;
  const int64_t cap = (int64_t)maxd + 32;
  const int64_t per_warp = 4 * cap;
  const int64_t warps = literal_warps(device_sm_count(g->device), maxd);
  if ((rc = ensure_scratch(g, (size_t)(warps * per_warp) * sizeof(int32_t)))) return rc;
  PlanArgs a{};
  a.rowptr = dag ? g->d_dag_rowptr : g->d_rowptr;
  a.col = dag ? g->d_dag_col : g->d_col;
  a.n = g->n;
  a.ctl = g->d_ctl;
  a.scratch = (int32_t*)g->d_scratch;
  a.cap = cap;
  const int64_t m = dag ? g->m_dag : g->m;
  if (end < 0 || end > m) end = m;
  if (begin < 0) begin = 0;
  if (stride < 1) stride = 1;
  const int64_t nsamp = end > begin ? (end - begin + stride - 1) / stride : 0;
  const int grid = (int)(warps / 8);
  const int rounds = chunk_size > 1 ? chunk_size : 1;
  const int64_t per = (nsamp + rounds - 1) / rounds;
  a.slot_stride = stride;
  a.slot_end = end;
  Timer t;
  JGPM_CUDA_TRY(cudaMemsetAsync(g->d_ctl, 0, sizeof(DevControl), g->stream));
  cudaEventRecord(t.a, g->stream);
  for (int r = 0; r < rounds; ++r) {
    const int64_t i0 = std::min(nsamp, (int64_t)r * per);
    const int64_t i1 = std::min(nsamp, i0 + per);
    a.slot_begin = begin + i0 * stride;
    a.nsamp = i1 - i0;
    if (r > 0)
      JGPM_CUDA_TRY(cudaMemsetAsync(g->d_ctl->counter, 0, sizeof(g->d_ctl->counter), g->stream));
    if (a.nsamp > 0) {
      if ((rc = launch_plan(id, a, stats, grid, g->stream))) return rc;
      ++g->launches;
    }
  }
  cudaEventRecord(t.b, g->stream);
  JGPM_CUDA_TRY(cudaGetLastError());
  if ((rc = read_ctl(g))) return rc;
  *out = g->h_ctl->count[0];
  if (elements) *elements = g->h_ctl->elements[0];
  if (ms) *ms = t.ms();
  return JGPM_OK;
}

// The 4-cycle count runs on the rank-relabelled CSR (c4.cu); rounds do not change it.
int run_wedge_c4(jgpm_graph* g, int chunk_size, uint64_t* out, double* ms) {
  (void)chunk_size;
  return count_c4_wedge(g, out, ms);
}

// Diamond count (reference P2 semantics) in one pass over the DAG's triangles: every
// increment of an edge's triangle counter from o to o + k adds k*o + C(k, 2) to the total, so
// the total is sum_e C(t_e, 2).  Per-arc counters live in g->d_aux.
int run_diamond_pairs(jgpm_graph* g, uint64_t* out, double* ms) {
  int rc;
  if ((rc = ensure_dag(g))) return rc;
  const size_t bytes = (size_t)std::max<int64_t>(1, g->m_dag) * sizeof(uint32_t);
  if ((rc = ensure_aux(g, bytes))) return rc;
  Timer t;
  cudaEventRecord(t.a, g->stream);
  JGPM_CUDA_TRY(cudaMemsetAsync(g->d_aux, 0, bytes, g->stream));
  if ((rc = launch_diamond_pairs(g, (uint32_t*)g->d_aux, g->stream))) return rc;
  cudaEventRecord(t.b, g->stream);
  if ((rc = read_ctl(g))) return rc;
  *out = g->h_ctl->count[0];
  if (ms) *ms = t.ms();
  return JGPM_OK;
}

// Vertex-induced tailed-triangle count in one pass of the k = 4 bitmap tiers:
// I(TT) = N(TT) - 4 N(diamond) + 12 K4 (from N(TT) = I(TT) + 4 I(D) + 12 I(K4) and
// N(D) = I(D) + 6 I(K4)), with N(D) from the pair gains and N(TT) from the degrees of every
// triangle's vertices.  Per-arc counters live in g->d_aux.
int run_induced_tt(jgpm_graph* g, uint64_t* out, double* ms) {
  int rc;
  if ((rc = ensure_dag(g))) return rc;
  const size_t bytes = (size_t)std::max<int64_t>(1, g->m_dag) * sizeof(uint32_t);
  if ((rc = ensure_aux(g, bytes))) return rc;
  Timer t;
  cudaEventRecord(t.a, g->stream);
  JGPM_CUDA_TRY(cudaMemsetAsync(g->d_aux, 0, bytes, g->stream));
  if ((rc = launch_induced_tt(g, (uint32_t*)g->d_aux, g->stream))) return rc;
  cudaEventRecord(t.b, g->stream);
  if ((rc = read_ctl(g))) return rc;
  *out = g->h_ctl->count[0];
  if (ms) *ms = t.ms();
  return JGPM_OK;
}

// Edge-induced pieces of the 4-vertex census.
struct Census {
  unsigned __int128 sum_te, sum_c2, sum_tt, sum_path, sum_star;
  uint64_t k4, c4;
  double ms;
};

unsigned __int128 u128(const unsigned long long* p) {
  return ((unsigned __int128)p[1] << 64) | p[0];
}

int census_pieces(jgpm_graph* g, bool need_k4, bool need_c4, Census* c) {
  int rc;
  if ((rc = ensure_dag(g))) return rc;
  if ((rc = ensure_control(g))) return rc;
  cudaStream_t s = g->stream;
  memset(c, 0, sizeof(*c));
  // per-arc triangles | twice the triangles per vertex | 16 accumulator words, in g->d_aux
  const size_t tri_bytes = ((size_t)std::max<int64_t>(1, g->m_dag) * 4 + 255) & ~(size_t)255;
  const size_t tv2_bytes = (size_t)std::max<int32_t>(1, g->n) * 8;
  if ((rc = ensure_aux(g, tri_bytes + tv2_bytes + 16 * 8))) return rc;
  uint32_t* d_tri = (uint32_t*)g->d_aux;
  unsigned long long* d_tv2 = (unsigned long long*)((char*)g->d_aux + tri_bytes);
  unsigned long long* d_acc = d_tv2 + std::max<int32_t>(1, g->n);
  Timer t;
  cudaEventRecord(t.a, s);
  JGPM_CUDA_TRY(cudaMemsetAsync(g->d_aux, 0, tri_bytes + tv2_bytes + 16 * 8, s));
  if ((rc = launch_edge_triangles(g, d_tri, s))) return rc;
  k_census_edges<<<grid_for((int64_t)g->n * 32), 256, 0, s>>>(
      g->d_dag_rowptr, g->d_dag_col, g->d_rowptr, g->n, d_tri, d_tv2, d_acc);
  k_census_vertices<<<grid_for(g->n), 256, 0, s>>>(g->d_rowptr, g->n, d_tv2, d_acc);
  g->launches += 2;
  unsigned long long h[16];
  cudaEventRecord(t.b, s);
  if (cudaMemcpyAsync(h, d_acc, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    jgpm_set_error_(std::string("census: ") + cudaGetErrorString(cudaGetLastError()));
    return JGPM_ECUDA;
  }
  double ms = t.ms();
  c->sum_te = u128(&h[0]);
  c->sum_c2 = u128(&h[2]);
  c->sum_tt = u128(&h[4]) / 2;  // tv2 holds twice the triangles at each vertex
  c->sum_path = u128(&h[6]);
  c->sum_star = u128(&h[8]);
  if (need_k4) {
    double m2 = 0;
    uint64_t k4 = 0;
    if ((rc = count_clique_public(g, 4, &k4, &m2))) return rc;
    c->k4 = k4;
    ms += m2;
  }
  if (need_c4) {
    double m3 = 0;
    if ((rc = run_wedge_c4(g, 1, &c->c4, &m3))) return rc;
    ms += m3;
  }
  c->ms = ms;
  return JGPM_OK;
}

bool fits64(unsigned __int128 v) { return (v >> 64) == 0; }

}  // namespace

// Vertex-induced census from the edge-induced counts:
//   N(K4) = I(K4); N(diamond) = I(D) + 6 I(K4); N(C4) = I(C4) + I(D) + 3 I(K4);
//   N(TT) = I(TT) + 4 I(D) + 12 I(K4); N(star) = I(S) + I(TT) + 2 I(D) + 4 I(K4);
//   N(P4) = I(P4) + 2 I(TT) + 4 I(C4) + 6 I(D) + 12 I(K4).
// With T = sum t_e / 3: N(diamond) = sum_e C(t_e,2); N(TT) = sum_v t_v (d_v - 2);
// N(star) = sum_v C(d_v,3); N(P4) = sum_e (d_u-1)(d_v-1) - 3T.
// need_c4 = false skips the 4-cycle wedge pass; out[1] (4-path) and out[3] (4-cycle) are then
// not computed (set to 0) -- the other four counts do not depend on N(C4).
static int census_impl(jgpm_graph* g, uint64_t out[6], double* ms, bool need_c4) {
  Census c;
  int rc = census_pieces(g, true, need_c4, &c);
  if (rc) return rc;
  typedef __int128 i128;
  const i128 T = (i128)(c.sum_te / 3);
  const i128 nK4 = c.k4, nD = (i128)c.sum_c2, nC4 = c.c4, nTT = (i128)c.sum_tt;
  const i128 nS = (i128)c.sum_star, nP4 = (i128)c.sum_path - 3 * T;
  const i128 iK4 = nK4;
  const i128 iD = nD - 6 * iK4;
  const i128 iC4 = nC4 - iD - 3 * iK4;
  const i128 iTT = nTT - 4 * iD - 12 * iK4;
  const i128 iS = nS - iTT - 2 * iD - 4 * iK4;
  const i128 iP4 = nP4 - 2 * iTT - 4 * iC4 - 6 * iD - 12 * iK4;
  const i128 v[6] = {iS, need_c4 ? iP4 : 0, iTT, need_c4 ? iC4 : 0, iD, iK4};
  for (int i = 0; i < 6; ++i) {
    if (v[i] < 0) {
      jgpm_set_error_("census: negative induced count (internal inconsistency)");
      return JGPM_ECUDA;
    }
    if (!fits64((unsigned __int128)v[i])) {
      jgpm_set_error_("census: count exceeds uint64");
      return JGPM_EOVERFLOW;
    }
    out[i] = (uint64_t)v[i];
  }
  if (ms) *ms = c.ms;
  return JGPM_OK;
}

int count_census4(jgpm_graph* g, uint64_t out[6], double* ms) {
  return census_impl(g, out, ms, true);
}

// Returns JGPM_OK, a negative status, or never a method code; *method is set separately.
int count_plan_impl(jgpm_graph* g, int id, int chunk_size, unsigned flags, bool stats,
                    uint64_t* out, uint64_t* elements, double* ms, int* method) {
  int rc;
  const bool force_plan = (flags & JGPM_COUNT_FORCE_PLAN) != 0;
  const bool force_enum = (flags & (JGPM_COUNT_FORCE_ENUM | JGPM_COUNT_FORCE_PLAN)) != 0;
  uint64_t cnt = 0;
  double t = 0.0;
  if (id == kP1 && !force_plan) {
    if ((rc = run_wedge_c4(g, chunk_size, &cnt, &t))) return rc;
    *method = JGPM_METHOD_WEDGE;
  } else if (id == kP2 && !force_plan) {
    if ((rc = run_diamond_pairs(g, &cnt, &t))) return rc;
    *method = JGPM_METHOD_EDGE_TRIANGLE;
  } else if (id == kITailed && !force_enum) {
    if ((rc = run_induced_tt(g, &cnt, &t))) return rc;
    *method = JGPM_METHOD_EDGE_TRIANGLE;
  } else if (id >= kIC4 && id <= kIStar3 && !force_enum) {
    uint64_t v[6];
    if ((rc = census_impl(g, v, &t, id == kIC4 || id == kIPath4))) return rc;
    const int idx = id == kIStar3 ? 0 : id == kIPath4 ? 1 : id == kITailed ? 2
                  : id == kIC4 ? 3 : 4;
    cnt = v[idx];
    *method = JGPM_METHOD_CENSUS;
  } else if (id >= kNTailed && id <= kNStar3) {
    Census c;
    if ((rc = census_pieces(g, false, false, &c))) return rc;
    unsigned __int128 r = 0;
    if (id == kNTailed) r = c.sum_tt;
    else if (id == kNStar3) r = c.sum_star;
    else r = c.sum_path - 3 * (c.sum_te / 3);
    if (!fits64(r)) {
      jgpm_set_error_("count exceeds uint64");
      return JGPM_EOVERFLOW;
    }
    cnt = (uint64_t)r;
    t = c.ms;
    *method = JGPM_METHOD_EDGE_TRIANGLE;
    if (stats) {
      jgpm_set_error_("set-op statistics are not defined for closed-form counts");
      return JGPM_EINVAL;
    }
  } else {
    if ((rc = run_literal(g, id, chunk_size, false, &cnt, nullptr, &t))) return rc;
    *method = JGPM_METHOD_PLAN;
  }
  *out = cnt;
  if (ms) *ms = t;
  if (stats && elements) {
    // The canonical plan's elements come from the literal kernel (untimed); its count must
    // agree with the fast method's.
    uint64_t c2 = 0, e2 = 0;
    const int timed_launches = g->launches;
    if ((rc = run_literal(g, id, 1, true, &c2, &e2, nullptr))) return rc;
    g->launches = timed_launches;
    if (c2 != cnt) {
      jgpm_set_error_("plan accounting pass disagrees with the fast count");
      return JGPM_ECUDA;
    }
    *elements = e2;
  }
  return JGPM_OK;
}

// Plan id of a pattern name for the literal plan kernel, or -1: the plan_id_of names plus the
// clique aliases "triangle"/"3-clique" (P0 on the DAG), "4-clique".."7-clique" and
// "k-clique:<k>" for 3 <= k <= 7.  Closed-form edge-induced counts have no plan (-1).
int literal_plan_id(const std::string& p, int induced) {
  int k = 0;
  if (!induced) {
    if (p == "triangle" || p == "3-clique") k = 3;
    else if (p == "6-clique") k = 6;
    else if (p == "7-clique") k = 7;
    else if (p.rfind("k-clique:", 0) == 0) k = std::atoi(p.c_str() + 9);
    if (k != 0) return k == 3 ? (int)kP0 : (k >= 4 && k <= 7) ? (int)kK4 + (k - 4) : -1;
  }
  const int id = plan_id_of(p, induced);
  return id >= kNTailed ? -1 : id;
}

// The literal plan over a strided sample of root arcs (the reference's per-round root slice
// estart/enumber, src/jupiter_gpm.cu:373-377, generalised with a stride).
int count_roots_impl(jgpm_graph* g, int id, int64_t begin, int64_t end, int64_t stride,
                     uint64_t* out, double* ms) {
  return run_literal(g, id, 1, false, out, nullptr, ms, begin, end, stride);
}

// Device scratch that a jgpm_count of `pattern` allocates on g beyond the graph itself (0 for
// the methods that need none): the literal plan kernel's per-warp lists, or the clique
// tiers' heavy-root lists and global bitmap rows.  Needs the DAG's maximum out-degree for
// the DAG plans (0 until the DAG is built).
uint64_t count_scratch_bytes(const jgpm_graph* g, const std::string& pattern, int induced) {
  const int sms = device_sm_count(g->device);
  const int id = plan_id_of(pattern, induced);
  const bool literal = id == kP3 || id == kP4 || id == kP5 || id == kP6 || id == kP7 ||
                       id == kP8 || id == kP9 || id == kP10 || id == kP11 || id == kP12 ||
                       id == kVsgm;
  if (literal) {
    const int32_t maxd = g->max_degree;
    return (uint64_t)literal_warps(sms, maxd) * 4 * ((uint64_t)maxd + 32) * 4;
  }
  const int k = literal_plan_id(pattern, induced) == kP0 ? 3
              : (id >= kK4 && id <= kK7) ? 4 + (id - kK4) : 0;
  if (k == 0 && pattern.rfind("k-clique:", 0) != 0) return 0;
  uint64_t b = 0;
  const int32_t mo = g->max_out_degree;
  if (mo > kWideMaxDeg) b += (uint64_t)6 * ((uint64_t)mo + 32) * sms * 2 * 8 * 4;  // list tier
  if (mo > kMidMaxDeg) b += (uint64_t)96 << 20;  // wide tier rows (kept within L2 size)
  return b;
}

int64_t plan_root_arcs(jgpm_graph* g, int id) {
  if (plan_uses_dag(id)) {
    if (ensure_dag(g)) return -1;
    return g->m_dag;
  }
  return g->m;
}

}  // namespace jgpm

// ============================================================================
// Allocation-free counting: the literal plan kernel with its per-warp candidate lists in a
// fixed, file-scope device array instead of memory obtained from cudaMalloc.
//
// Some callers cannot allocate device memory at the point where they count: a host
// application whose own memory manager took the whole device at start-up and hands nothing
// back, or a latency-critical path that may not call cudaMalloc/cudaFree because those calls
// can synchronise the device and stall every other stream.  jgpm_count_noalloc serves them:
// it calls no cudaMalloc, cudaFree or allocating library routine and works in
// kNoAllocScratchInts int32 of scratch plus one control block, both static __device__
// arrays.  Every GPU that loads libjgpm holds those 32 MiB until the process exits.
namespace jgpm {
namespace {

constexpr int64_t kNoAllocScratchInts = (int64_t)8 << 20;  // 32 MiB of int32
static __device__ __align__(256) int32_t g_noalloc_scratch[kNoAllocScratchInts];
static __device__ __align__(256) DevControl g_noalloc_ctl;

struct NoAllocDevice {
  bool ready = false;
  int32_t* scratch = nullptr;
  DevControl* ctl = nullptr;
};
constexpr int kNoAllocMaxDevices = 64;
NoAllocDevice g_noalloc_dev[kNoAllocMaxDevices];
std::mutex g_noalloc_mu;

// Device addresses of the two arrays on the current device, looked up once per device by
// the first call there.  In host code the array names are host-side stand-ins, not device
// addresses, so they are never handed to a kernel directly.  The look-up can initialise the
// module on that device, so a caller that captures streams makes its first call on each
// device before any capture begins.  The addresses are kept for the life of the process: a
// cudaDeviceReset between calls would leave them stale, and is not supported.
int noalloc_setup(int device, NoAllocDevice* out) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  NoAllocDevice& d = g_noalloc_dev[device];
  if (!d.ready) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      jgpm_set_error_(std::string("jgpm_count_noalloc: cudaGetSymbolAddress(scratch): ") +
                      cudaGetErrorString(e));
      return JGPM_ECUDA;
    }
    d.scratch = static_cast<int32_t*>(p);
    e = cudaGetSymbolAddress(&p, g_noalloc_ctl);
    if (e != cudaSuccess) {
      jgpm_set_error_(std::string("jgpm_count_noalloc: cudaGetSymbolAddress(control): ") +
                      cudaGetErrorString(e));
      return JGPM_ECUDA;
    }
    d.ctl = static_cast<DevControl*>(p);
    d.ready = true;
  }
  *out = d;
  return JGPM_OK;
}

}  // namespace
}  // namespace jgpm

extern "C" int jgpm_count_noalloc(jgpm_graph* g, const char* pattern, int induced,
                                  uint64_t* out) {
  using namespace jgpm;
  if (!g || !pattern || !out) {
    jgpm_set_error_("jgpm_count_noalloc: null argument");
    return JGPM_EINVAL;
  }
  const std::string p(pattern);
  const int id = p == "triangle" ? (int)kP0 : plan_id_of(p, induced);
  if (id < 0 || id >= kNTailed) {
    jgpm_set_error_("jgpm_count_noalloc: pattern '" + p +
                    "' has no allocation-free plan kernel");
    return JGPM_EPATTERN;
  }
  const bool dag = plan_uses_dag(id);
  if (dag && !g->d_dag_rowptr) {
    jgpm_set_error_("jgpm_count_noalloc: this pattern runs on the degree-oriented DAG; build it "
                    "first (orient_dag = 1 when the graph is created, or any earlier clique "
                    "count)");
    return JGPM_EINVAL;
  }
  if (g->device < 0 || g->device >= kNoAllocMaxDevices) {
    jgpm_set_error_("jgpm_count_noalloc: device index out of range");
    return JGPM_EINVAL;
  }
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != g->device) cudaSetDevice(g->device);
  auto restore = [&]() {
    if (prev >= 0 && prev != g->device) cudaSetDevice(prev);
  };
  NoAllocDevice d;
  int rc = noalloc_setup(g->device, &d);
  if (rc) {
    restore();
    return rc;
  }
  const int32_t maxd = dag ? g->max_out_degree : g->max_degree;
  const int64_t cap = (int64_t)maxd + 32;
  const int64_t per_warp = 4 * cap;
  const int sms = device_sm_count(g->device);
  int64_t warps = std::min<int64_t>((int64_t)sms * 64, kNoAllocScratchInts / per_warp);
  warps -= warps % 8;
  if (warps < 8) {
    restore();
    jgpm_set_error_("jgpm_count_noalloc: maximum degree " + std::to_string(maxd) +
                    " needs more than the fixed 32 MiB scratch (largest supported maximum "
                    "degree: " + std::to_string(kNoAllocScratchInts / 32 - 32) + ")");
    return JGPM_ECAPACITY;
  }
  PlanArgs a{};
  a.rowptr = dag ? g->d_dag_rowptr : g->d_rowptr;
  a.col = dag ? g->d_dag_col : g->d_col;
  a.n = g->n;
  a.ctl = d.ctl;
  a.scratch = d.scratch;
  a.cap = cap;
  a.slot_begin = 0;
  a.slot_end = dag ? g->m_dag : g->m;
  a.slot_stride = 1;
  a.nsamp = a.slot_end;
  // The arrays keep the previous call's contents: the work cursors and the result must start
  // at zero.  Calls that overlap on the GPU share these arrays and race.
  cudaError_t e = cudaMemsetAsync(d.ctl, 0, sizeof(DevControl), g->stream);
  if (e == cudaSuccess && a.slot_end > 0) {
    rc = launch_plan(id, a, false, (int)(warps / 8), g->stream);
    e = cudaGetLastError();
    if (rc == JGPM_OK && e == cudaSuccess) g->launches = 1;
  }
  unsigned long long cnt = 0;
  if (e == cudaSuccess && rc == JGPM_OK)
    e = cudaMemcpyAsync(&cnt, &d.ctl->count[0], sizeof(cnt), cudaMemcpyDeviceToHost, g->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  restore();
  if (rc) return rc;
  if (e != cudaSuccess) {
    jgpm_set_error_(std::string("jgpm_count_noalloc: ") + cudaGetErrorString(e));
    return JGPM_ECUDA;
  }
  *out = cnt;
  return JGPM_OK;
}
