// k-clique (and triangle) counting on the degree-oriented DAG: the plain per-query kernels.
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
// once and kept as a local adjacency bitmap over the positions of N+(u) (clique_dev.cuh);
// every deeper reference level "W & N+(v)" becomes a word-wise AND of bitmap rows and the
// last level a popcount.  Each clique is enumerated once, in its (unique) topological order
// inside the DAG.
//
// Root tiers by out-degree d (roots with d < k-1 cannot root a k-clique and are skipped):
//   d <= 4, 8, 16, 32   groups of G = 4, 8, 16, 32 lanes, one root per group; rows are single
//                       words; L and the row offsets live in registers, searched with
//                       width-G __shfl_sync;
//   32 < d <= 128       one warp per root (up to the split degree), rows in the warp's
//                       slice of shared memory;
//   split < d <= 1024   one CTA per root; rows of ceil(d/32) words in shared memory, sized
//                       per degree band (<= 256, <= 512, <= 1024) so that the low bands keep
//                       many CTAs per SM; masks of up to 8 / 16 words are counted from
//                       registers, wider ones distributed one word per lane;
//   d > 1024            edge-rooted fallback: one warp per arc (u, v_i) with the candidate
//                       lists in per-warp global scratch (the reference's scheme).
// Work is handed out by global atomic cursors (work stealing); roots are sorted by
// descending out-degree so the heaviest start first.
#include <cuda_runtime.h>

#include "clique_dev.cuh"
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
  uint32_t* rows;       // CTA tiers with rows in global memory: dmax * W words per CTA
  int large_chunks;     // list tier: tasks per root (chunks of 32 arcs of the widest root)
  int cursor;           // which ctl->counter this launch steals from
  uint32_t* tri;        // edge-triangle mode: triangles per DAG arc (K == 3 only)
};

// Kernel variants: PAIRS (with ETRI, K == 3) returns sum_e C(t_e, 2) as the count.

namespace {

// ------------------------------------------------------------------ small tiers (d <= 32)
template <int G, int K, bool STATS, bool ETRI = false, bool PAIRS = false>
__global__ void __launch_bounds__(256) k_clique_group(CliqueArgs a) {
  __shared__ uint32_t rows_s[256];
  __shared__ int deg_s[256];
  constexpr int kGroups = 32 / G;
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int gi = lane / G;
  uint32_t* R = rows_s + wib * 32 + gi * G;
  int* DG = deg_s + wib * 32 + gi * G;
  acc_t cnt = 0, elems = 0;
  for (;;) {
    unsigned long long c0 = 0;
    if (lane == 0) c0 = atomicAdd(&a.ctl->counter[a.cursor], (unsigned long long)kGroups);
    c0 = __shfl_sync(kFull, c0, 0);
    const int64_t first = a.begin + (int64_t)c0;
    if (first >= a.end) break;
    const int64_t idx = first + gi;
    const vid_t u = idx < a.end ? a.roots[idx] : -1;
    cnt += group_root<G, K, STATS, ETRI, PAIRS>(a.rowptr, a.col, u, R, DG, a.tri, elems);
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

// ------------------------------------------------------------------ warp tier (d <= 128)
template <int K, bool STATS, bool ETRI = false, bool PAIRS = false>
__global__ void __launch_bounds__(256) k_clique_warp(CliqueArgs a) {
  extern __shared__ __align__(16) unsigned char wsmem[];
  WarpSmem& ws = reinterpret_cast<WarpSmem*>(wsmem)[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  acc_t cnt = 0, elems = 0;
  for (;;) {
    unsigned long long c0 = 0;
    if (lane == 0) c0 = atomicAdd(&a.ctl->counter[a.cursor], 1ull);
    c0 = __shfl_sync(kFull, c0, 0);
    const int64_t idx = a.begin + (int64_t)c0;
    if (idx >= a.end) break;
    cnt += warp_root<K, STATS, ETRI, PAIRS>(a.rowptr, a.col, a.roots[idx], ws, a.tri, elems);
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

// --------------------------------------------------- CTA tiers (32 < d <= kWideMaxDeg)
// GR: the bitmap rows live in global scratch (a.rows, dmax * W words per CTA, L2-resident)
// and the shared memory holds only the root's list and row offsets.
template <int K, bool STATS, bool ETRI = false, bool PAIRS = false, int ROWW = kCtaRowWords,
          int WPL = 1, bool GR = false>
__global__ void __launch_bounds__(256) k_clique_mid(CliqueArgs a, int dmax, int W) {
  extern __shared__ __align__(16) unsigned char smem[];
  const MidSmem sm = MidSmem::carve(smem, dmax, W,
                                    GR ? a.rows + (size_t)blockIdx.x * dmax * W : nullptr);
  __shared__ unsigned long long s_idx;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  acc_t cnt = 0, elems = 0;
  for (;;) {
    if (tid == 0) s_idx = atomicAdd(&a.ctl->counter[a.cursor], 1ull);
    __syncthreads();
    const int64_t idx = (int64_t)s_idx + a.begin;
    __syncthreads();
    if (idx >= a.end) break;
    cnt += cta_root<K, STATS, ETRI, PAIRS, ROWW, WPL, GR>(a.rowptr, a.col, a.roots[idx], sm,
                                                          a.tri, elems);
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
        int c = 0;  // |cand & N+(v)|, lookups of cand (written by this warp) in N+(v)
        for (int q = lane; q < nc; q += 32)
          if (contains_g(a.col + b, dv, cand[q])) ++c;
        s += (acc_t)warp_sum_int(c);
      } else {
        const int t = warp_intersect_w(cand, nc, a.col + b, dv, INT32_MAX, buf);
        if (t > 0)
          s += ListClique<(REM > 1 ? REM - 1 : 1), STATS>::run(a, buf, t, buf + cap, cap, elems);
      }
    }
    return s;
  }
};

template <int K, bool STATS, bool ETRI = false, bool PAIRS = false>
__global__ void __launch_bounds__(256) k_clique_large(CliqueArgs a) {
  const int lane = threadIdx.x & 31;
  const int64_t gwarp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int32_t* buf = a.scratch + gwarp * a.scratch_per_warp;
  const int64_t cap = a.scratch_per_warp / kMaxLevels;
  acc_t cnt = 0, elems = 0;
  for (;;) {
    // task t = chunk (t mod large_chunks) of 32 arcs of root begin + t / large_chunks
    unsigned long long t = 0;
    if (lane == 0) t = atomicAdd(&a.ctl->counter[a.cursor], 1ull);
    t = __shfl_sync(kFull, t, 0);
    const int64_t r = a.begin + (int64_t)(t / (unsigned long long)a.large_chunks);
    if (r >= a.end) break;
    const vid_t u = a.roots[r];
    const eid_t bu = a.rowptr[u];
    const int du = (int)(a.rowptr[u + 1] - bu);
    const int i0 = (int)(t % (unsigned long long)a.large_chunks) * 32;
    for (int i = i0; i < min(du, i0 + 32); ++i) {
      const vid_t v = __ldg(a.col + bu + i);
      const eid_t bv = a.rowptr[v];
      const int dv = (int)(a.rowptr[v + 1] - bv);
      int32_t* W = buf;
      const int tw = warp_intersect(a.col + bu, du, a.col + bv, dv, INT32_MAX, W);
      // tw and the ListClique sums are the same in every lane: lane 0 keeps them
      if (K == 3) {
        if (!PAIRS && lane == 0) cnt += (acc_t)tw;
        if (ETRI && tw > 0) {
          if (lane == 0) {
            const unsigned o = atomicAdd(a.tri + bu + i, (unsigned)tw);
            if (PAIRS) cnt += pair_gain(o, (unsigned)tw);
          }
          for (int q = lane; q < tw; q += 32) {
            const vid_t w = W[q];
            const unsigned o1 = atomicAdd(a.tri + bu + lower_bound_g(a.col + bu, du, w), 1u);
            const unsigned o2 = atomicAdd(a.tri + bv + lower_bound_g(a.col + bv, dv, w), 1u);
            if (PAIRS) cnt += (acc_t)o1 + (acc_t)o2;
          }
          __syncwarp();
        }
      } else if (tw > 0) {
        const acc_t c =
            ListClique<(K > 3 ? K - 3 : 1), STATS>::run(a, W, tw, buf + cap, cap, elems);
        if (lane == 0) cnt += c;
      }
      __syncwarp();  // W is rewritten by the next arc
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

// Launch plan of one count: the root ranges of each tier.  wide holds the CTA roots of
// out-degree (1024, 4096] (rows in global scratch); mid[0..2] are the CTA-root bands of
// out-degree (512, 1024], (256, 512] and (split, 256].
struct TierPlan {
  TierRange large, wide, mid[3], warp, g32, g16, g8, g4;
};

// CTAs and global row words of a wide/global-row band of out-degree <= dmax: at most
// kRowsBudget bytes of rows so that they stay in L2.
constexpr size_t kRowsBudget = (size_t)96 << 20;
inline int rows_band_grid(int dmax, int sms, int64_t roots) {
  const size_t per = (size_t)dmax * ((dmax + 31) / 32) * 4;
  const int64_t by_budget = (int64_t)std::max<size_t>(1, kRowsBudget / per);
  return (int)std::max<int64_t>(
      1, std::min<int64_t>(std::min<int64_t>((int64_t)sms * 4, by_budget), roots));
}

// One CTA-root band: bitmap layout for out-degree <= dmax, masks of up to ROWW words counted
// from registers, wider ones with WPL words per lane; GR puts the rows in global scratch.
template <int K, bool STATS, bool ETRI, bool PAIRS, int ROWW, int WPL = 1, bool GR = false>
void launch_mid_band(CliqueArgs a, const TierRange& r, int cursor, int dmax, int sms,
                     cudaStream_t s) {
  a.begin = r.b;
  a.end = r.e;
  a.cursor = cursor;
  const int W = (dmax + 31) / 32;
  const size_t sm = GR ? MidLayout{dmax, W}.bytes_no_rows() : MidLayout{dmax, W}.bytes();
  auto kern = k_clique_mid<K, STATS, ETRI, PAIRS, ROWW, WPL, GR>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, sm);
  if (per_sm < 1) per_sm = 1;
  const int64_t roots = r.e - r.b;
  int grid = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)sms * per_sm, roots));
  if (GR) grid = std::min(grid, rows_band_grid(dmax, sms, roots));
  kern<<<grid, 256, sm, s>>>(a, dmax, W);
}

template <int K, bool STATS, bool ETRI, bool PAIRS = false>
int launch_plan_k(const CliqueArgs& base, const TierPlan& p, int sms, cudaStream_t s,
                  int max_out) {
  CliqueArgs a = base;
  int n = 0;
  if (!p.large.empty()) {
    a.begin = p.large.b;
    a.end = p.large.e;
    a.cursor = 2;
    k_clique_large<K, STATS, ETRI, PAIRS><<<sms * 2, 256, 0, s>>>(a);
    ++n;
  }
  if (!p.wide.empty()) {
    launch_mid_band<K, STATS, ETRI, PAIRS, 0, 4, true>(a, p.wide, 9,
                                                       std::min(max_out, kWideMaxDeg), sms, s);
    ++n;
  }
  if (!p.mid[0].empty()) {
    launch_mid_band<K, STATS, ETRI, PAIRS, 0>(a, p.mid[0], 1, std::min(max_out, kMidMaxDeg),
                                              sms, s);
    ++n;
  }
  if (!p.mid[1].empty()) {
    launch_mid_band<K, STATS, ETRI, PAIRS, 16>(a, p.mid[1], 0, std::min(max_out, 512), sms, s);
    ++n;
  }
  if (!p.mid[2].empty()) {
    launch_mid_band<K, STATS, ETRI, PAIRS, 8>(a, p.mid[2], 8, std::min(max_out, 256), sms, s);
    ++n;
  }
  if (!p.warp.empty()) {
    a.begin = p.warp.b;
    a.end = p.warp.e;
    a.cursor = 7;
    const size_t sm = 8 * sizeof(WarpSmem);
    cudaFuncSetAttribute(k_clique_warp<K, STATS, ETRI, PAIRS>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_clique_warp<K, STATS, ETRI, PAIRS>, 256,
                                                  sm);
    if (per_sm < 1) per_sm = 1;
    k_clique_warp<K, STATS, ETRI, PAIRS><<<sms * per_sm, 256, sm, s>>>(a);
    ++n;
  }
  const TierRange* gr[4] = {&p.g32, &p.g16, &p.g8, &p.g4};
  for (int q = 0; q < 4; ++q) {
    if (gr[q]->empty()) continue;
    a.begin = gr[q]->b;
    a.end = gr[q]->e;
    a.cursor = 3 + q;
    switch (q) {
      case 0: k_clique_group<32, K, STATS, ETRI, PAIRS><<<sms * 8, 256, 0, s>>>(a); break;
      case 1: k_clique_group<16, K, STATS, ETRI, PAIRS><<<sms * 8, 256, 0, s>>>(a); break;
      case 2: k_clique_group<8, K, STATS, ETRI, PAIRS><<<sms * 8, 256, 0, s>>>(a); break;
      default: k_clique_group<4, K, STATS, ETRI, PAIRS><<<sms * 8, 256, 0, s>>>(a); break;
    }
    ++n;
  }
  return n;
}

}  // namespace

// Root ranges of a k-clique count over tier indices [root_begin, root_end): roots with
// d >= k-1 only, split by out-degree into the group widths allowed by min_group.
static TierPlan make_plan(const RootTiers& t, int k, int64_t root_begin, int64_t root_end,
                          int min_group, int split) {
  const int64_t stop = std::min(root_end, t.deg_begin[k - 2 >= 0 ? k - 2 : 0]);
  auto cut = [&](int64_t b, int64_t e) {
    TierRange r{std::max(b, root_begin), std::min(e, stop)};
    return r;
  };
  TierPlan p;
  p.large = cut(0, t.wide_begin);
  p.wide = cut(t.wide_begin, t.large_end);
  // 32 < d <= split (split in {32, 64, 128}): warp per root; above: CTA per root
  const int64_t wb = std::max(t.large_end, split >= 128 ? t.le_begin[2]
                                           : split >= 64 ? t.le_begin[1] : t.le_begin[0]);
  // CTA bands (tiers are sorted by descending out-degree, and wb >= b256 >= b512)
  const int64_t b512 = std::max(t.large_end, t.le_begin[4]);
  const int64_t b256 = std::max(b512, t.le_begin[3]);
  p.mid[0] = cut(t.large_end, b512);
  p.mid[1] = cut(b512, b256);
  p.mid[2] = cut(b256, wb);
  p.warp = cut(wb, t.mid_end);
  // small tier [mid_end, small_end): d in (16,32] -> G32, (8,16] -> G16, (4,8] -> G8, <=4 -> G4
  const int64_t b16 = min_group <= 16 ? t.deg_begin[16] : t.small_end;
  const int64_t b8 = min_group <= 8 ? t.deg_begin[8] : t.small_end;
  const int64_t b4 = min_group <= 4 ? t.deg_begin[4] : t.small_end;
  p.g32 = cut(t.mid_end, std::max(t.mid_end, b16));
  p.g16 = cut(std::max(t.mid_end, b16), std::max(b16, b8));
  p.g8 = cut(std::max(b16, b8), std::max(b8, b4));
  p.g4 = cut(std::max(b8, b4), t.small_end);
  return p;
}

// Launches the k-clique kernels over tier indices [root_begin, root_end) of g->tiers
// (built with ensure_tiers).  Results accumulate into g->d_ctl->count[0] (elements of levels
// >= 2 into elements[0] when stats); tri != null selects the edge-triangle mode (k = 3).
// The caller zeroes the work cursors before each call.
int launch_clique_ex(jgpm_graph* g, int k, bool stats, int64_t root_begin, int64_t root_end,
                     cudaStream_t s, uint32_t* tri, int min_group, bool pairs = false) {
  if (k < 3 || k > 8) {
    jgpm_set_error_("k-clique: k must be in [3, 8]");
    return JGPM_EPATTERN;
  }
  const int sms = device_sm_count(g->device);
  const RootTiers& t = g->tiers;
  const TierPlan p = make_plan(t, stats ? 3 : k, root_begin, root_end, min_group,
                               g->tune_split);
  CliqueArgs a{};
  a.rowptr = g->d_dag_rowptr;
  a.col = g->d_dag_col;
  a.roots = t.d_roots;
  a.ctl = g->d_ctl;
  a.tri = tri;
  // scratch: [per-warp lists of the list tier][bitmap rows of the wide band]
  size_t list_bytes = 0, row_bytes = 0;
  int64_t per_warp = 0;
  if (!p.large.empty()) {
    a.large_chunks = (g->max_out_degree + 31) / 32;
    per_warp = (int64_t)kMaxLevels * (g->max_out_degree + 32);
    list_bytes = (size_t)(per_warp * (int64_t)sms * 2 * 8) * sizeof(int32_t);
  }
  if (!p.wide.empty()) {
    const int dw = std::min(g->max_out_degree, kWideMaxDeg);
    row_bytes = (size_t)rows_band_grid(dw, sms, p.wide.e - p.wide.b) * dw * ((dw + 31) / 32) * 4;
  }
  if (list_bytes + row_bytes > 0) {
    int rc = ensure_scratch(g, list_bytes + row_bytes);
    if (rc) return rc;
    a.scratch = (int32_t*)g->d_scratch;
    a.scratch_per_warp = per_warp;
    a.rows = (uint32_t*)((char*)g->d_scratch + list_bytes);
  }
  const int mid_dmax = std::max(33, g->max_out_degree);
  int n = 0;
  if (tri) {
    n = pairs ? launch_plan_k<3, false, true, true>(a, p, sms, s, mid_dmax)
              : launch_plan_k<3, false, true>(a, p, sms, s, mid_dmax);
  } else {
    switch (k) {
#define JGPM_K(KK)                                                              \
  case KK:                                                                      \
    n = stats ? launch_plan_k<KK, true, false>(a, p, sms, s, mid_dmax)          \
              : launch_plan_k<KK, false, false>(a, p, sms, s, mid_dmax);        \
    break;
      JGPM_K(3) JGPM_K(4) JGPM_K(5) JGPM_K(6) JGPM_K(7) JGPM_K(8)
#undef JGPM_K
    }
  }
  g->launches += n;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    jgpm_set_error_(std::string("clique launch: ") + cudaGetErrorString(e));
    return JGPM_ECUDA;
  }
  return JGPM_OK;
}

int launch_clique(jgpm_graph* g, int k, bool stats, int64_t root_begin, int64_t root_end,
                  cudaStream_t s) {
  return launch_clique_ex(g, k, stats, root_begin, root_end, s, nullptr, g->tune_min_group);
}

// Triangles per DAG arc into d_tri (zeroed by the caller); the triangle total also
// accumulates into ctl->count[0].
int launch_edge_triangles(jgpm_graph* g, uint32_t* d_tri, cudaStream_t s) {
  int rc;
  if ((rc = ensure_tiers(g, 2))) return rc;
  if ((rc = ensure_control(g))) return rc;
  JGPM_CUDA_TRY(cudaMemsetAsync(g->d_ctl, 0, sizeof(DevControl), s));
  return launch_clique_ex(g, 3, false, 0, g->tiers.small_end, s, d_tri, g->tune_min_group);
}

// Diamond count sum_e C(t_e, 2) into ctl->count[0] in one pass; d_tri (m_dag counters) must
// be zero on entry.
int launch_diamond_pairs(jgpm_graph* g, uint32_t* d_tri, cudaStream_t s) {
  int rc;
  if ((rc = ensure_tiers(g, 2))) return rc;
  if ((rc = ensure_control(g))) return rc;
  JGPM_CUDA_TRY(cudaMemsetAsync(g->d_ctl, 0, sizeof(DevControl), s));
  return launch_clique_ex(g, 3, false, 0, g->tiers.small_end, s, d_tri, g->tune_min_group,
                          true);
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
