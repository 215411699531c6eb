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

#include "clique_tiers.cuh"

namespace jgpm {
namespace {

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

}  // namespace

// Root ranges of a k-clique count over tier indices [root_begin, root_end): roots with
// d >= k-1 only, split by out-degree into the group widths allowed by min_group.
static TierPlan make_plan(const RootTiers& t, int k, int64_t root_begin, int64_t root_end,
                          int min_group, int split, int shard, int nshards) {
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
  if (nshards > 1) {
    // shard s of n takes tier indices b + s, b + s + n, ... of every range, so each shard gets
    // an equal share of every out-degree band
    TierRange* all[] = {&p.large, &p.wide, &p.mid[0], &p.mid[1], &p.mid[2], &p.warp,
                        &p.g32, &p.g16, &p.g8, &p.g4};
    for (TierRange* r : all) {
      const int64_t b = r->b + shard;
      const int64_t cnt = b < r->e ? (r->e - b + nshards - 1) / nshards : 0;
      *r = TierRange{b, b + cnt, nshards};
    }
  }
  return p;
}

// Launches the k-clique kernels over tier indices [root_begin, root_end) of g->tiers
// (built with ensure_tiers).  Results accumulate into g->d_ctl->count[0] (elements of levels
// >= 2 into elements[0] when stats); tri != null selects the edge-triangle mode (k = 3).
// The caller zeroes the work cursors before each call.
int launch_clique_ex(jgpm_graph* g, int k, bool stats, int64_t root_begin, int64_t root_end,
                     cudaStream_t s, uint32_t* tri, int min_group, bool pairs = false,
                     bool tt = false, int shard = 0, int nshards = 1) {
  if (k < 3 || k > 8) {
    jgpm_set_error_("k-clique: k must be in [3, 8]");
    return JGPM_EPATTERN;
  }
  const int sms = device_sm_count(g->device);
  const RootTiers& t = g->tiers;
  // every triangle needs its root (out-degree >= 2) in the edge-triangle modes
  const TierPlan p = make_plan(t, (stats || tri) ? 3 : k, root_begin, root_end, min_group,
                               g->tune_split, shard, nshards);
  CliqueArgs a{};
  a.step = 1;
  a.rowptr = g->d_dag_rowptr;
  a.col = g->d_dag_col;
  a.roots = t.d_roots;
  a.ctl = g->d_ctl;
  a.tri = tri;
  a.srow = g->d_rowptr;
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
  const int mode = tt ? 4 : tri ? (pairs ? 3 : 2) : (stats ? 1 : 0);
  switch (tt ? 4 : tri ? 3 : k) {
    case 3: n = launch_tiers_k3(mode, a, p, sms, s, mid_dmax); break;
    case 4: n = launch_tiers_k4(mode, a, p, sms, s, mid_dmax); break;
    case 5: n = launch_tiers_k5(mode, a, p, sms, s, mid_dmax); break;
    case 6: n = launch_tiers_k6(mode, a, p, sms, s, mid_dmax); break;
    default: n = launch_tiers_k78(k, mode, a, p, sms, s, mid_dmax); break;
  }
  if (n < 0) return JGPM_ECUDA;  // a tier launch failed (message set)
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

// One shard of a k-clique count: the roots of every tier with index = shard (mod nshards).
int launch_clique_shard(jgpm_graph* g, int k, int shard, int nshards, cudaStream_t s) {
  return launch_clique_ex(g, k, false, 0, g->tiers.deg_begin[k - 2], s, nullptr,
                          g->tune_min_group, false, false, shard, nshards);
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

// Vertex-induced tailed-triangle count into ctl->count[0] in one pass of the k = 4 tiers
// (12 K4 - 4 sum_e C(t_e, 2) + N(tailed triangle)); d_tri (m_dag counters) must be zero.
int launch_induced_tt(jgpm_graph* g, uint32_t* d_tri, cudaStream_t s) {
  int rc;
  if ((rc = ensure_tiers(g, 2))) return rc;
  if ((rc = ensure_control(g))) return rc;
  JGPM_CUDA_TRY(cudaMemsetAsync(g->d_ctl, 0, sizeof(DevControl), s));
  return launch_clique_ex(g, 4, false, 0, g->tiers.small_end, s, d_tri, g->tune_min_group,
                          true, true);
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
