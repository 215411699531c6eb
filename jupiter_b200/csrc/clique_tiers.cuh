// The per-tier k-clique kernels and their launch templates, shared by the translation units
// that instantiate them (clique_k*.cu, one or two clique sizes each, so the build compiles
// them in parallel).  See clique.cu for the design.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>

#include "clique_dev.cuh"
#include "jgpm_internal.h"
#include "setops.cuh"

namespace jgpm {

struct CliqueArgs {
  const eid_t* rowptr;  // DAG row pointers
  const vid_t* col;     // DAG neighbour lists
  const vid_t* roots;
  int64_t begin, end;   // root range of this launch: roots[begin + (i - begin) * step],
  int64_t step;         // begin <= i < end (step > 1: one shard's roots of a tier)
  DevControl* ctl;
  int32_t* scratch;     // large tier: per-warp lists
  int64_t scratch_per_warp;
  uint32_t* rows;       // CTA tiers with rows in global memory: dmax * W words per CTA
  int large_chunks;     // list tier: tasks per root (chunks of 32 arcs of the widest root)
  int cursor;           // which ctl->counter this launch steals from
  uint32_t* tri;        // edge-triangle modes: triangles per DAG arc
  const eid_t* srow;    // TT mode: symmetric row pointers (degrees)
};

// Kernel variants: PAIRS (with ETRI, K == 3) returns sum_e C(t_e, 2) as the count; TT (with
// ETRI and PAIRS, K == 4) the vertex-induced tailed-triangle count (clique_dev.cuh).

constexpr int kMaxLevels = 6;  // list tier: candidate lists per warp

// Tier indices b, b + step, ..., (e - b) of them.
struct TierRange {
  int64_t b, e;
  int64_t step = 1;
  bool empty() const { return e <= b; }
};

// Root of launch index i (a.begin <= i < a.end).
__device__ __forceinline__ vid_t root_at(const CliqueArgs& a, int64_t i) {
  return a.roots[a.begin + (i - a.begin) * a.step];
}

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

// Launches the tiers of one count for clique size k (3..8).  mode: 0 count, 1 count with the
// set-op accounting, 2 edge triangles (k = 3), 3 diamond pairs (k = 3), 4 vertex-induced
// tailed triangles (k = 4).  Returns the number of kernels launched.
int launch_tiers_k3(int mode, const CliqueArgs& a, const TierPlan& p, int sms, cudaStream_t s,
                    int max_out);
int launch_tiers_k4(int mode, const CliqueArgs& a, const TierPlan& p, int sms, cudaStream_t s,
                    int max_out);
int launch_tiers_k5(int mode, const CliqueArgs& a, const TierPlan& p, int sms, cudaStream_t s,
                    int max_out);
int launch_tiers_k6(int mode, const CliqueArgs& a, const TierPlan& p, int sms, cudaStream_t s,
                    int max_out);
int launch_tiers_k78(int k, int mode, const CliqueArgs& a, const TierPlan& p, int sms,
                     cudaStream_t s, int max_out);

namespace {

// The tier kernels of one count share nothing but their atomic result adds (each has its own
// cursor and its own scratch), so every tier after the first is launched with programmatic
// stream serialization and overlaps the previous tier's last CTAs (pdl_open / pdl_close).

// ------------------------------------------------------------------ small tiers (d <= 32)
template <int G, int K, bool STATS, bool ETRI = false, bool PAIRS = false, bool TT = false>
__global__ void __launch_bounds__(256) k_clique_group(CliqueArgs a) {
  __shared__ uint32_t rows_s[256];
  __shared__ int deg_s[256];
  constexpr int kGroups = 32 / G;
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int gi = lane / G;
  uint32_t* R = rows_s + wib * 32 + gi * G;
  int* DG = deg_s + wib * 32 + gi * G;
  pdl_open();
  acc_t cnt = 0, elems = 0;
  for (;;) {
    unsigned long long c0 = 0;
    if (lane == 0) c0 = atomicAdd(&a.ctl->counter[a.cursor], (unsigned long long)kGroups);
    c0 = __shfl_sync(kFull, c0, 0);
    const int64_t first = a.begin + (int64_t)c0;
    if (first >= a.end) break;
    const int64_t idx = first + gi;
    const vid_t u = idx < a.end ? root_at(a, idx) : -1;
    cnt += group_root<G, K, STATS, ETRI, PAIRS, TT>(a.rowptr, a.col, u, R, DG, a.tri, elems,
                                                     a.srow);
  }
  for (int o = 16; o > 0; o >>= 1) {
    cnt += __shfl_xor_sync(kFull, cnt, o);
    if (STATS) elems += __shfl_xor_sync(kFull, elems, o);
  }
  if (lane == 0) {
    if (cnt) atomicAdd(&a.ctl->count[0], cnt);
    if (STATS && elems) atomicAdd(&a.ctl->elements[0], elems);
  }
  pdl_close();
}

// ------------------------------------------------------------------ warp tier (d <= 128)
// The warp tier's shared memory (8 x WarpSmem, 49 KB) allows four CTAs per SM, so its
// register budget is that of four CTAs.
template <int K, bool STATS, bool ETRI = false, bool PAIRS = false, bool TT = false>
__global__ void __launch_bounds__(256, 4) k_clique_warp(CliqueArgs a) {
  extern __shared__ __align__(16) unsigned char wsmem[];
  WarpSmem& ws = reinterpret_cast<WarpSmem*>(wsmem)[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  pdl_open();
  acc_t cnt = 0, elems = 0;
  for (;;) {
    unsigned long long c0 = 0;
    if (lane == 0) c0 = atomicAdd(&a.ctl->counter[a.cursor], 1ull);
    c0 = __shfl_sync(kFull, c0, 0);
    const int64_t idx = a.begin + (int64_t)c0;
    if (idx >= a.end) break;
    cnt += warp_root<K, STATS, ETRI, PAIRS, TT, (K <= 4)>(a.rowptr, a.col, root_at(a, idx), ws,
                                                           a.tri, elems, a.srow);
  }
  for (int o = 16; o > 0; o >>= 1) {
    cnt += __shfl_xor_sync(kFull, cnt, o);
    if (STATS) elems += __shfl_xor_sync(kFull, elems, o);
  }
  if (lane == 0) {
    if (cnt) atomicAdd(&a.ctl->count[0], cnt);
    if (STATS && elems) atomicAdd(&a.ctl->elements[0], elems);
  }
  pdl_close();
}

// --------------------------------------------------- CTA tiers (32 < d <= kWideMaxDeg)
// GR: the bitmap rows live in global scratch (a.rows, dmax * W words per CTA, L2-resident)
// and the shared memory holds only the root's list and row offsets.
// Register budget of the CTA bands (minimum resident CTAs per SM): the bitmap build and the
// row-parallel counts run faster with room for their masks (4-clique band of out-degree
// <= 256: 2.21 ms at the 32 registers the compiler picks by default, with a spill; 1.69 ms
// at 56), the level-2 5-clique count at 64 registers, with four CTAs per SM (the item form
// of the widest band needs more).
template <bool BAL, int ROWW>
constexpr int kMidMinBlocks() { return BAL && ROWW <= 16 ? 4 : 1; }

template <int K, bool STATS, bool ETRI = false, bool PAIRS = false, int ROWW = kCtaRowWords,
          int WPL = 1, bool GR = false, bool TT = false, bool BAL = false>
__global__ void __launch_bounds__(256, kMidMinBlocks<BAL, ROWW>()) k_clique_mid(CliqueArgs a, int dmax,
                                                                        int W) {
  extern __shared__ __align__(16) unsigned char smem[];
  const MidSmem sm = MidSmem::carve(smem, dmax, W,
                                    GR ? a.rows + (size_t)blockIdx.x * dmax * W : nullptr,
                                    BAL ? ROWW : 0);
  __shared__ unsigned long long s_idx;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  pdl_open();
  acc_t cnt = 0, elems = 0;
  for (;;) {
    if (tid == 0) s_idx = atomicAdd(&a.ctl->counter[a.cursor], 1ull);
    __syncthreads();
    const int64_t idx = (int64_t)s_idx + a.begin;
    __syncthreads();
    if (idx >= a.end) break;
    cnt += cta_root<K, STATS, ETRI, PAIRS, ROWW, WPL, GR, TT, BAL>(a.rowptr, a.col,
                                                                   root_at(a, idx), sm, a.tri,
                                                                   elems, a.srow);
  }
  for (int o = 16; o > 0; o >>= 1) {
    cnt += __shfl_xor_sync(kFull, cnt, o);
    if (STATS) elems += __shfl_xor_sync(kFull, elems, o);
  }
  if (lane == 0) {
    if (cnt) atomicAdd(&a.ctl->count[0], cnt);
    if (STATS && elems) atomicAdd(&a.ctl->elements[0], elems);
  }
  pdl_close();
}

// ------------------------------------------------------------------ large tier (d > 1024)
// Edge-rooted, list based: one warp per arc (u, v_i) of a large root.  Candidate lists of
// each level live in the warp's global scratch (kMaxLevels lists of max_out entries).
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

template <int K, bool STATS, bool ETRI = false, bool PAIRS = false, bool TT = false>
__global__ void __launch_bounds__(256) k_clique_large(CliqueArgs a) {
  const int lane = threadIdx.x & 31;
  const int64_t gwarp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int32_t* buf = a.scratch + gwarp * a.scratch_per_warp;
  const int64_t cap = a.scratch_per_warp / kMaxLevels;
  pdl_open();
  acc_t cnt = 0, elems = 0;
  for (;;) {
    // task t = chunk (t mod large_chunks) of 32 arcs of root begin + t / large_chunks
    unsigned long long t = 0;
    if (lane == 0) t = atomicAdd(&a.ctl->counter[a.cursor], 1ull);
    t = __shfl_sync(kFull, t, 0);
    const int64_t r = a.begin + (int64_t)(t / (unsigned long long)a.large_chunks);
    if (r >= a.end) break;
    const vid_t u = root_at(a, r);
    const eid_t bu = a.rowptr[u];
    const int du = (int)(a.rowptr[u + 1] - bu);
    const int i0 = (int)(t % (unsigned long long)a.large_chunks) * 32;
    for (int i = i0; i < min(du, i0 + 32); ++i) {
      const vid_t v = __ldg(a.col + bu + i);
      const eid_t bv = a.rowptr[v];
      const int dv = (int)(a.rowptr[v + 1] - bv);
      int32_t* W = buf;
      const int tw = warp_intersect(a.col + bu, du, a.col + bv, dv, INT32_MAX, W);
      // tw and the ListClique sums are the same in every lane: lane 0 keeps them.  Pair
      // gains enter the TT value with weight -4, 4-cliques with weight 12.
      const acc_t pw = TT ? (acc_t)0 - 4ull : 1ull;
      if (ETRI && tw > 0) {
        if (lane == 0) {
          const unsigned o = atomicAdd(a.tri + bu + i, (unsigned)tw);
          if (PAIRS) cnt += pw * pair_gain(o, (unsigned)tw);
        }
        const acc_t tuv = TT ? tt_deg(a.srow, u) + tt_deg(a.srow, v) : 0ull;
        for (int q = lane; q < tw; q += 32) {
          const vid_t w = W[q];
          const unsigned o1 = atomicAdd(a.tri + bu + lower_bound_g(a.col + bu, du, w), 1u);
          const unsigned o2 = atomicAdd(a.tri + bv + lower_bound_g(a.col + bv, dv, w), 1u);
          if (PAIRS) cnt += pw * ((acc_t)o1 + (acc_t)o2);
          if (TT) cnt += tuv + tt_deg(a.srow, w);
        }
        __syncwarp();
      }
      if (K == 3) {
        if (!PAIRS && lane == 0) cnt += (acc_t)tw;
      } else if (tw > 0 && (!PAIRS || TT)) {
        const acc_t c =
            ListClique<(K > 3 ? K - 3 : 1), STATS>::run(a, W, tw, buf + cap, cap, elems);
        if (lane == 0) cnt += TT ? 12ull * c : c;
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
  pdl_close();
}

// True (with the error recorded) if the kernel just launched failed to launch (rc: the
// launch call's own status), so that a count never silently misses a tier.
inline bool launch_failed(cudaError_t* err, cudaError_t rc = cudaSuccess) {
  const cudaError_t last = cudaGetLastError();
  const cudaError_t e = rc != cudaSuccess ? rc : last;
  if (e == cudaSuccess) return false;
  *err = e;
  jgpm_set_error_(std::string("clique tier launch: ") + cudaGetErrorString(e));
  return true;
}

// Launches one tier kernel of 256 threads; after the first tier of a count (pdl) with
// programmatic stream serialization.
template <typename... Args>
cudaError_t tier_launch(bool pdl, void (*kern)(Args...), int grid, size_t smem, cudaStream_t s,
                        Args... args) {
  return launch_pdl(pdl, kern, grid, 256, smem, s, args...);
}

// Register-mask width of a CTA band: k >= 7 counts warp-cooperatively (0), which keeps the
// deep register-mask recursion, and its compile time, out of the large clique sizes.
template <int K>
constexpr int kBandRowWords(int w) { return K >= 7 ? 0 : w; }

// Mask words counted from registers in the band of out-degree <= 1024 (rows of up to 32
// words): k = 4 row-parallel, k = 5 over (row, bit) pairs, one 32-word mask per thread; the
// warp-cooperative form (0) otherwise.
template <int K>
constexpr int kWideBandRowWords() { return K == 4 || K == 5 ? 32 : 0; }

// One CTA-root band: bitmap layout for out-degree <= dmax, masks of up to ROWW words counted
// from registers, wider ones with WPL words per lane; GR puts the rows in global scratch.
// A plain 5-clique count with rows in shared memory counts with the balanced form.
template <int K, bool STATS, bool ETRI, int ROWW, bool GR>
constexpr bool kBandBalanced() { return K == 5 && !STATS && !ETRI && ROWW > 0 && !GR; }

template <int K, bool STATS, bool ETRI, bool PAIRS, int ROWW, int WPL = 1, bool GR = false,
          bool TT = false>
cudaError_t launch_mid_band(CliqueArgs a, const TierRange& r, int cursor, int dmax, int sms,
                            cudaStream_t s, bool pdl) {
  a.begin = r.b;
  a.end = r.e;
  a.step = r.step;
  a.cursor = cursor;
  const int W = (dmax + 31) / 32;
  constexpr bool BAL = kBandBalanced<K, STATS, ETRI, ROWW, GR>();
  const MidLayout lay{dmax, W, BAL ? ROWW : 0};
  const size_t sm = GR ? lay.bytes_no_rows() : lay.bytes();
  auto kern = k_clique_mid<K, STATS, ETRI, PAIRS, ROWW, WPL, GR, TT, BAL>;
  raise_smem_limit((const void*)kern, sm);  // a failure shows up as the launch error
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, sm);
  if (per_sm < 1) per_sm = 1;
  const int64_t roots = r.e - r.b;
  int grid = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)sms * per_sm, roots));
  if (GR) grid = std::min(grid, rows_band_grid(dmax, sms, roots));
  return tier_launch(pdl, kern, grid, sm, s, a, dmax, W);
}

template <int K, bool STATS, bool ETRI, bool PAIRS = false, bool TT = false>
int launch_plan_k(const CliqueArgs& base, const TierPlan& p, int sms, cudaStream_t s,
                  int max_out) {
  CliqueArgs a = base;
  int n = 0;
  cudaError_t err = cudaSuccess;
  // the first tier of a count is an ordinary launch (after the control block's reset in the
  // stream); the later ones overlap their predecessor's last CTAs
  auto pdl = [&]() { return n > 0; };
  if (!p.large.empty()) {
    a.begin = p.large.b;
    a.end = p.large.e;
    a.step = p.large.step;
    a.cursor = 2;
    const cudaError_t rc =
        tier_launch(pdl(), k_clique_large<K, STATS, ETRI, PAIRS, TT>, sms * 2, 0, s, a);
    ++n;
    if (launch_failed(&err, rc)) return -1;
  }
  if (!p.wide.empty()) {
    const cudaError_t rc = launch_mid_band<K, STATS, ETRI, PAIRS, 0, 4, true, TT>(
        a, p.wide, 9, std::min(max_out, kWideMaxDeg), sms, s, pdl());
    ++n;
    if (launch_failed(&err, rc)) return -1;
  }
  if (!p.mid[0].empty()) {
    const cudaError_t rc =
        launch_mid_band<K, STATS, ETRI, PAIRS, kWideBandRowWords<K>(), 1, false, TT>(
            a, p.mid[0], 1, std::min(max_out, kMidMaxDeg), sms, s, pdl());
    ++n;
    if (launch_failed(&err, rc)) return -1;
  }
  if (!p.mid[1].empty()) {
    const cudaError_t rc =
        launch_mid_band<K, STATS, ETRI, PAIRS, kBandRowWords<K>(16), 1, false, TT>(
            a, p.mid[1], 0, std::min(max_out, 512), sms, s, pdl());
    ++n;
    if (launch_failed(&err, rc)) return -1;
  }
  if (!p.mid[2].empty()) {
    const cudaError_t rc =
        launch_mid_band<K, STATS, ETRI, PAIRS, kBandRowWords<K>(8), 1, false, TT>(
            a, p.mid[2], 8, std::min(max_out, 256), sms, s, pdl());
    ++n;
    if (launch_failed(&err, rc)) return -1;
  }
  if (!p.warp.empty()) {
    a.begin = p.warp.b;
    a.end = p.warp.e;
    a.step = p.warp.step;
    a.cursor = 7;
    const size_t sm = 8 * sizeof(WarpSmem);
    raise_smem_limit((const void*)k_clique_warp<K, STATS, ETRI, PAIRS, TT>, sm);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_clique_warp<K, STATS, ETRI, PAIRS, TT>,
                                                  256, sm);
    if (per_sm < 1) per_sm = 1;
    const cudaError_t rc =
        tier_launch(pdl(), k_clique_warp<K, STATS, ETRI, PAIRS, TT>, sms * per_sm, sm, s, a);
    ++n;
    if (launch_failed(&err, rc)) return -1;
  }
  const TierRange* gr[4] = {&p.g32, &p.g16, &p.g8, &p.g4};
  for (int q = 0; q < 4; ++q) {
    if (gr[q]->empty()) continue;
    a.begin = gr[q]->b;
    a.end = gr[q]->e;
    a.step = gr[q]->step;
    a.cursor = 3 + q;
    cudaError_t rc;
    switch (q) {
      case 0: rc = tier_launch(pdl(), k_clique_group<32, K, STATS, ETRI, PAIRS, TT>, sms * 8, 0, s, a); break;
      case 1: rc = tier_launch(pdl(), k_clique_group<16, K, STATS, ETRI, PAIRS, TT>, sms * 8, 0, s, a); break;
      case 2: rc = tier_launch(pdl(), k_clique_group<8, K, STATS, ETRI, PAIRS, TT>, sms * 8, 0, s, a); break;
      default: rc = tier_launch(pdl(), k_clique_group<4, K, STATS, ETRI, PAIRS, TT>, sms * 8, 0, s, a); break;
    }
    ++n;
    if (launch_failed(&err, rc)) return -1;
  }
  return n;
}

}  // namespace
}  // namespace jgpm
