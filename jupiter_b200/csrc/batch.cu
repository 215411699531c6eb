// Batched counting: many (graph, pattern) jobs in ONE persistent, work-stealing launch.
//
// The reference splits one query's root-edge range into `chunk_size` static rounds, one
// launch each (src/jupiter_gpm.cu:356-375).  Here every job of a batch is cut into tasks and
// all tasks of all jobs go into one global queue.  Persistent CTAs pull tasks with an atomic
// cursor until the queue is empty, so uneven jobs share the GPU without host round trips;
// every task adds its partial count into its job's counter.  Tasks are ordered heaviest
// first.
//
// Per-task work (the device code of the plain kernels, clique_dev.cuh and c4_dev.cuh):
//   GROUP_G     k-clique roots with out-degree <= G, one root per G-lane group;
//   WARP_ROOTS  roots with 32 < d <= split, one root per warp (bitmap in the warp's shared
//               slice);
//   CTA_ROOT    one root with split < d <= kBatchCtaMaxDeg on the whole CTA;
//   WIDE_ROOT   one root with kBatchCtaMaxDeg < d <= kBatchWideMaxDeg on the whole CTA, bitmap
//               rows in per-CTA global scratch (read at L2);
//   LARGE_ROOT  one root with d > kBatchWideMaxDeg, edge-rooted lists in warp scratch;
//   C4_SMALL    4-cycle apexes with few wedges, one per warp (shared-memory hash);
//   C4_MID      4-cycle apexes with up to 2048 wedges, each on the whole CTA (shared hash);
//   C4_LARGE    a heavy 4-cycle apex, or a run of lighter ones, on the whole CTA of the second
//               kernel (shared-memory counter slab; dense counters in global memory past the
//               slice cap).
// Diamond jobs (reference P2, sum over edges of C(t_e, 2)) run the k = 3 root tasks in pair
// mode: every triangle increments its three arcs' counters in the job's tri[] array and the
// adds' old values give the pairs, so the count comes out of the same single pass.  Jobs for
// the vertex-induced tailed triangle ("induced:tailed-triangle") run the k = 4 tasks in TT
// mode, 12 K4 - 4 N(diamond) + N(tailed triangle), in one pass as well.
//
// Resources: one kernel holds every task kind, so its registers and shared memory are the
// largest any kind needs.  The CTA roots count warp-cooperatively (masks one word per lane)
// instead of with per-thread register masks, and the per-CTA shared memory is one union of
// the warp slices, the 4-cycle hash tables and one CTA bitmap of out-degree <= 512, so four
// CTAs of 256 threads fit on an SM.
//
// The tuning (jgpm_tuning) picks the narrowest lane group, the out-degree split between warp
// and CTA roots, and the roots per task; jgpm_autotune picks them by timing candidates on a
// sample of the batch.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "batch.h"
#include "c4_dev.cuh"
#include "clique_dev.cuh"
#include "jgpm_internal.h"
#include "setops.cuh"

namespace jgpm {

struct BatchArgs {
  const JobDesc* jobs;
  const Task* tasks;
  int64_t nmain, ntasks;       // k_batch: tasks [0, nmain); k_batch_groups: [nmain, ntasks)
  unsigned long long* counts;
  unsigned long long* cursor;  // [0] main queue, [1] large 4-cycle apexes, [2] lane groups
  int32_t* list_scratch;  // per warp: kLevels lists of list_cap ints
  int64_t list_cap;
  int dmax, W;            // CTA-root bitmap layout
  uint32_t* rows;         // wide roots: wdmax * wW words of bitmap rows per CTA
  int wdmax, wW;
  int intersect;          // last clique level of large roots: 0 search from the shorter list,
                          // 1 always from the candidate list
};

namespace {

constexpr int kLevels = 6;

// Shared memory of one CTA of the batched kernel: the largest of the per-kind layouts.
inline size_t batch_smem_bytes(int dmax, int W, int wdmax, int wW) {
  size_t b = 8 * sizeof(WarpSmem);
  b = std::max(b, 8 * sizeof(C4WarpHash));
  b = std::max(b, sizeof(C4MidSmem<256>));
  b = std::max(b, MidLayout{dmax, W}.bytes());
  if (wdmax > 0) b = std::max(b, MidLayout{wdmax, wW}.bytes_no_rows());
  return b;
}

template <int REM>
struct BatchListClique {
  __device__ static acc_t run(const eid_t* rowptr, const vid_t* col, const vid_t* cand, int nc,
                              int32_t* buf, int64_t cap, int isect) {
    const int lane = threadIdx.x & 31;
    acc_t s = 0;
    for (int i = 0; i < nc; ++i) {
      const vid_t v = cand[i];
      const eid_t b = rowptr[v];
      const int dv = (int)(rowptr[v + 1] - b);
      if (REM == 1) {
        // |cand & N+(v)|: lanes take the keys of one list and search the other
        int c = 0;
        if (isect == 0 && dv < nc) {
          for (int q = lane; q < dv; q += 32)
            if (contains_s(cand, nc, __ldg(col + b + q))) ++c;
        } else {
          for (int q = lane; q < nc; q += 32)
            if (contains_g(col + b, dv, cand[q])) ++c;
        }
        s += (acc_t)warp_sum_int(c);
      } else {
        const int t = warp_intersect_w(cand, nc, col + b, dv, INT32_MAX, buf);
        if (t > 0)
          s += BatchListClique<(REM > 1 ? REM - 1 : 1)>::run(rowptr, col, buf, t, buf + cap, cap,
                                                             isect);
      }
    }
    return s;
  }
};

template <int G, int K, bool PAIRS, bool TT = false>
__device__ __forceinline__ acc_t task_groups(const JobDesc& j, int64_t b, int64_t e,
                                             uint32_t* rows, int* degs) {
  constexpr int kGroups = 32 / G;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int gi = lane / G;
  uint32_t* R = rows + warp * 32 + gi * G;
  int* DG = degs + warp * 32 + gi * G;
  acc_t cnt = 0, el = 0;
  for (int64_t first = b + (int64_t)warp * kGroups; first < e; first += 8 * kGroups) {
    const int64_t idx = first + gi;
    const vid_t u = idx < e ? j.roots[idx] : -1;
    cnt += group_root<G, K, false, PAIRS, PAIRS, TT>(j.drow, j.dcol, u, R, DG, j.tri, el,
                                                     j.srow);
  }
  return cnt;
}

template <int G>
__device__ __forceinline__ acc_t task_groups_k(const JobDesc& j, int64_t b, int64_t e,
                                               uint32_t* rows, int* degs) {
  if (j.kind == kJobDiamond) return task_groups<G, 3, true>(j, b, e, rows, degs);
  if (j.kind == kJobIndTT) return task_groups<G, 4, true, true>(j, b, e, rows, degs);
  switch (j.k) {
    case 3: return task_groups<G, 3, false>(j, b, e, rows, degs);
    case 4: return task_groups<G, 4, false>(j, b, e, rows, degs);
    case 5: return task_groups<G, 5, false>(j, b, e, rows, degs);
    case 6: return task_groups<G, 6, false>(j, b, e, rows, degs);
    case 7: return task_groups<G, 7, false>(j, b, e, rows, degs);
    default: return task_groups<G, 8, false>(j, b, e, rows, degs);
  }
}

// The warps take the task's roots one at a time from a shared counter (zero at task start),
// so a warp that drew cheap roots does not wait at the next task fetch for one that drew dear
// ones.
template <int K, bool PAIRS, bool TT = false>
__device__ __forceinline__ acc_t warp_roots_k(const JobDesc& j, int64_t b, int64_t e,
                                              WarpSmem& ws, int* next) {
  const int lane = threadIdx.x & 31;
  acc_t cnt = 0, el = 0;
  for (;;) {
    int q = 0;
    if (lane == 0) q = atomicAdd(next, 1);
    const int64_t r = b + __shfl_sync(kFull, q, 0);
    if (r >= e) break;
    cnt += warp_root<K, false, PAIRS, PAIRS, TT>(j.drow, j.dcol, j.roots[r], ws, j.tri, el,
                                                 j.srow);
  }
  return cnt;
}

__device__ __forceinline__ acc_t task_warp_roots(const JobDesc& j, int64_t b, int64_t e,
                                                 WarpSmem& ws, int* next) {
  if (j.kind == kJobDiamond) return warp_roots_k<3, true>(j, b, e, ws, next);
  if (j.kind == kJobIndTT) return warp_roots_k<4, true, true>(j, b, e, ws, next);
  switch (j.k) {
    case 3: return warp_roots_k<3, false>(j, b, e, ws, next);
    case 4: return warp_roots_k<4, false>(j, b, e, ws, next);
    case 5: return warp_roots_k<5, false>(j, b, e, ws, next);
    case 6: return warp_roots_k<6, false>(j, b, e, ws, next);
    case 7: return warp_roots_k<7, false>(j, b, e, ws, next);
    default: return warp_roots_k<8, false>(j, b, e, ws, next);
  }
}

// Row-mask width counted from registers for a CTA root band of up to W words (the plain
// bands' widths; the register-mask recursion is left out of k >= 7 as in the plain kernels).
template <int K, int W>
constexpr int batch_row_words() { return K >= 7 || (K >= 6 && W > 8) ? 0 : W; }

// One CTA root with rows of up to W words (out-degree <= 32 W), masks in registers.
template <int W>
__device__ __forceinline__ acc_t task_cta_root(const JobDesc& j, vid_t u, const MidSmem& sm) {
  acc_t el = 0;
  if (j.kind == kJobDiamond)  // pair mode returns before the mask counting
    return cta_root<3, false, true, true, 0>(j.drow, j.dcol, u, sm, j.tri, el);
  if (j.kind == kJobIndTT)
    return cta_root<4, false, true, true, W, 1, false, true>(j.drow, j.dcol, u, sm, j.tri, el,
                                                             j.srow);
  switch (j.k) {
    case 3: return cta_root<3, false, false, false, W>(j.drow, j.dcol, u, sm, nullptr, el);
    case 4: return cta_root<4, false, false, false, W>(j.drow, j.dcol, u, sm, nullptr, el);
    case 5: return cta_root<5, false, false, false, W>(j.drow, j.dcol, u, sm, nullptr, el);
    case 6:
      return cta_root<6, false, false, false, batch_row_words<6, W>()>(j.drow, j.dcol, u, sm,
                                                                       nullptr, el);
    case 7:
      return cta_root<7, false, false, false, batch_row_words<7, W>()>(j.drow, j.dcol, u, sm,
                                                                       nullptr, el);
    default:
      return cta_root<8, false, false, false, batch_row_words<8, W>()>(j.drow, j.dcol, u, sm,
                                                                       nullptr, el);
  }
}

// One wide root (rows in global scratch, masks two words per lane).
__device__ __forceinline__ acc_t task_wide_root(const JobDesc& j, vid_t u, const MidSmem& sm) {
  acc_t el = 0;
  if (j.kind == kJobDiamond)
    return cta_root<3, false, true, true, 0, 2, true>(j.drow, j.dcol, u, sm, j.tri, el);
  if (j.kind == kJobIndTT)
    return cta_root<4, false, true, true, 0, 2, true, true>(j.drow, j.dcol, u, sm, j.tri, el,
                                                            j.srow);
  switch (j.k) {
    case 3: return cta_root<3, false, false, false, 0, 2, true>(j.drow, j.dcol, u, sm, nullptr, el);
    case 4: return cta_root<4, false, false, false, 0, 2, true>(j.drow, j.dcol, u, sm, nullptr, el);
    case 5: return cta_root<5, false, false, false, 0, 2, true>(j.drow, j.dcol, u, sm, nullptr, el);
    case 6: return cta_root<6, false, false, false, 0, 2, true>(j.drow, j.dcol, u, sm, nullptr, el);
    case 7: return cta_root<7, false, false, false, 0, 2, true>(j.drow, j.dcol, u, sm, nullptr, el);
    default:
      return cta_root<8, false, false, false, 0, 2, true>(j.drow, j.dcol, u, sm, nullptr, el);
  }
}

// Warps of the CTA take the arcs (u, v_i) of the large root u: W = N+(u) & N+(v_i) in warp
// scratch, then the deeper clique levels on lists (or, for diamond jobs, the pair counts of
// the triangles (u, v_i, w)).  Returns this lane's partial.
__device__ acc_t task_large_root(const JobDesc& j, vid_t u, const BatchArgs& a) {
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int64_t gwarp = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp;
  int32_t* buf = a.list_scratch + gwarp * kLevels * a.list_cap;
  const int64_t cap = a.list_cap;
  const eid_t bu = j.drow[u];
  const int du = (int)(j.drow[u + 1] - bu);
  acc_t cnt = 0;
  for (int i = warp; i < du; i += 8) {
    const vid_t v = __ldg(j.dcol + bu + i);
    const eid_t bv = j.drow[v];
    const int dv = (int)(j.drow[v + 1] - bv);
    const int tw = warp_intersect(j.dcol + bu, du, j.dcol + bv, dv, INT32_MAX, buf);
    if (tw == 0) continue;
    if (j.kind == kJobDiamond || j.kind == kJobIndTT) {
      // pair gains (weight 1 for diamond, -4 in the tailed-triangle value) and, for the
      // tailed triangle, the degree terms of the triangles (u, v, w) and 12 x the 4-cliques
      const bool tt = j.kind == kJobIndTT;
      const acc_t pw = tt ? (acc_t)0 - 4ull : 1ull;
      if (lane == 0)
        cnt += pw * pair_gain(atomicAdd(j.tri + bu + i, (unsigned)tw), (unsigned)tw);
      const acc_t tuv = tt ? tt_deg(j.srow, u) + tt_deg(j.srow, v) : 0ull;
      for (int q = lane; q < tw; q += 32) {
        const vid_t w = buf[q];
        acc_t o = (acc_t)atomicAdd(j.tri + bu + lower_bound_g(j.dcol + bu, du, w), 1u);
        o += (acc_t)atomicAdd(j.tri + bv + lower_bound_g(j.dcol + bv, dv, w), 1u);
        cnt += pw * o;
        if (tt) cnt += tuv + tt_deg(j.srow, w);
      }
      __syncwarp();
      if (tt) {
        const acc_t k4 = BatchListClique<1>::run(j.drow, j.dcol, buf, tw, buf + cap, cap,
                                                 a.intersect);
        if (lane == 0) cnt += 12ull * k4;
      }
      continue;
    }
    acc_t c = (acc_t)tw;
    const int is = a.intersect;
    int32_t* nx = buf + cap;
    switch (j.k) {
      case 3: break;
      case 4: c = BatchListClique<1>::run(j.drow, j.dcol, buf, tw, nx, cap, is); break;
      case 5: c = BatchListClique<2>::run(j.drow, j.dcol, buf, tw, nx, cap, is); break;
      case 6: c = BatchListClique<3>::run(j.drow, j.dcol, buf, tw, nx, cap, is); break;
      case 7: c = BatchListClique<4>::run(j.drow, j.dcol, buf, tw, nx, cap, is); break;
      default: c = BatchListClique<5>::run(j.drow, j.dcol, buf, tw, nx, cap, is); break;
    }
    if (lane == 0) cnt += c;
  }
  return cnt;
}

__device__ __forceinline__ acc_t task_c4_small(const JobDesc& j, int64_t b, int64_t e,
                                               C4WarpHash& h) {
  acc_t s = 0;
  for (int64_t q = b + (threadIdx.x >> 5); q < e; q += 8)
    s += c4_small_apex(j.rrow, j.rcol, j.roots[q], h);
  return s;
}

__global__ void __launch_bounds__(256, 4) k_batch(BatchArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const MidSmem sm = MidSmem::carve(smem, a.dmax, a.W);
  WarpSmem& ws = reinterpret_cast<WarpSmem*>(smem)[threadIdx.x >> 5];
  C4WarpHash& hash = reinterpret_cast<C4WarpHash*>(smem)[threadIdx.x >> 5];
  C4MidSmem<256>& c4m = *reinterpret_cast<C4MidSmem<256>*>(smem);
  __shared__ unsigned long long s_task;
  __shared__ int s_next;  // next root of a warp-roots task
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  int smem_kind = -1;  // which layout the dynamic shared memory holds (hash tables persist)
  for (;;) {
    if (tid == 0) s_task = atomicAdd(&a.cursor[0], 1ull);
    __syncthreads();
    const int64_t ti = (int64_t)s_task;
    // every warp has left the previous task here, so its root counter can start over
    if (tid == 0) s_next = 0;
    __syncthreads();
    if (ti >= a.nmain) break;
    const Task t = a.tasks[ti];
    const JobDesc j = a.jobs[t.job];
    acc_t c = 0;
    switch (t.kind) {
      case kTaskWarpRoots:
        smem_kind = kTaskWarpRoots;
        c = task_warp_roots(j, t.b, t.e, ws, &s_next);
        break;
      case kTaskCtaRoot:
        smem_kind = kTaskCtaRoot;
        c = task_cta_root<16>(j, j.roots[t.b], sm);
        break;
      case kTaskCtaRoot8:
        smem_kind = kTaskCtaRoot;
        c = task_cta_root<8>(j, j.roots[t.b], sm);
        break;
      case kTaskWideRoot: {
        smem_kind = kTaskWideRoot;
        const MidSmem wsm = MidSmem::carve(
            smem, a.wdmax, a.wW, a.rows + (size_t)blockIdx.x * a.wdmax * a.wW);
        c = task_wide_root(j, j.roots[t.b], wsm);
        break;
      }
      case kTaskLargeRoot: c = task_large_root(j, j.roots[t.b], a); break;
      case kTaskC4Small:
        if (smem_kind != kTaskC4Small) {
          c4_hash_init(hash);
          smem_kind = kTaskC4Small;
        }
        c = task_c4_small(j, t.b, t.e, hash);
        break;
      case kTaskC4Mid:
        if (smem_kind != kTaskC4Mid) {
          c4_cta_hash_init(c4m.h);
          smem_kind = kTaskC4Mid;
        }
        for (int64_t q = t.b; q < t.e; ++q) c += c4_mid_apex<256>(j.rrow, j.rcol, j.mid[q], c4m);
        break;
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(kFull, c, o);
    if (lane == 0 && c) atomicAdd(&a.counts[t.job], c);
  }
}

// Lane-group tasks (roots of out-degree <= 32) of every job, on a light kernel: no dynamic
// shared memory and few registers, so that enough CTAs per SM hide the latency of these short
// roots (k_batch, which holds every other task kind, runs four).  Launched after k_batch.
__global__ void __launch_bounds__(256, 5) k_batch_groups(BatchArgs a) {
  __shared__ uint32_t rows[256];
  __shared__ int degs[256];
  __shared__ unsigned long long s_task;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  for (;;) {
    if (tid == 0) s_task = atomicAdd(&a.cursor[2], 1ull);
    __syncthreads();
    const int64_t ti = a.nmain + (int64_t)s_task;
    __syncthreads();
    if (ti >= a.ntasks) break;
    const Task t = a.tasks[ti];
    const JobDesc j = a.jobs[t.job];
    acc_t c = 0;
    switch (t.kind) {
      case kTaskGroup4: c = task_groups_k<4>(j, t.b, t.e, rows, degs); break;
      case kTaskGroup8: c = task_groups_k<8>(j, t.b, t.e, rows, degs); break;
      case kTaskGroup16: c = task_groups_k<16>(j, t.b, t.e, rows, degs); break;
      default: c = task_groups_k<32>(j, t.b, t.e, rows, degs); break;
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(kFull, c, o);
    if (lane == 0 && c) atomicAdd(&a.counts[t.job], c);
  }
}

// Large 4-cycle apexes of every 4-cycle job of the batch, heaviest first, on CTAs of 1024
// threads, launched before k_batch on the same stream.  Each CTA has a shared-memory slab of
// `words` words (a slab form of NT threads); an apex flagged dense
// counts in the CTA's dense array (and touched list) of `stride` ints instead when the batch
// has them.
struct C4BatchArgs {
  const JobDesc* jobs;
  const Task* tasks;  // (job, apex index b)
  int64_t ntasks;
  unsigned long long* counts;
  unsigned long long* cursor;
  int32_t* dense;     // null: no apex of the batch needs one
  vid_t* touched;
  int64_t stride;
  int words;
};

constexpr uint64_t kC4TaskWedges = 1u << 16;  // wedge bound of a run of light large apexes
constexpr int64_t kC4MidPerTask = 16;

template <int NT>
__global__ void __launch_bounds__(NT, NT <= 512 ? 2 : 1) k_batch_c4_large(C4BatchArgs a) {
  extern __shared__ __align__(16) uint32_t slab[];
  __shared__ C4LargeSmem<NT> sh;
  __shared__ unsigned long long s_q[2];
  int32_t* dense = a.dense ? a.dense + (int64_t)blockIdx.x * a.stride : nullptr;
  vid_t* touched = a.dense ? a.touched + (int64_t)blockIdx.x * a.stride : nullptr;
  c4_slab_zero<NT>(slab, a.words);
  if (threadIdx.x == 0) s_q[0] = atomicAdd(a.cursor, 1ull);
  __syncthreads();
  // double-buffered task fetch, as in the plain large-apex kernel: every task runs at least
  // one apex, so barriers separate each slot's store from its reads
  for (int it = 0;; ++it) {
    const int64_t q = (int64_t)s_q[it & 1];
    if (q >= a.ntasks) break;
    if (threadIdx.x == 0) s_q[(it + 1) & 1] = atomicAdd(a.cursor, 1ull);
    const Task t = a.tasks[q];
    const JobDesc j = a.jobs[t.job];
    acc_t c = 0;
    for (int64_t p = t.b; p < t.e; ++p) {
      const vid_t v = j.apexes[p];
      const uint32_t cw = (uint32_t)j.apexes[j.nlarge + p];
      const int cut = (int)(cw & ~kC4DenseFlag);
      if (!dense || !(cw & kC4DenseFlag))
        c += c4_slab_apex<NT>(j.rrow, j.rcol, v, cut, slab, a.words, sh);
      else
        c += c4_large_apex<NT>(j.rrow, j.rcol, v, cut, dense, touched, sh);
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(kFull, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(&a.counts[t.job], c);
  }
}

}  // namespace
}  // namespace jgpm

// ======================================================================= host side
namespace jgpm {

namespace {

void add_range_tasks(std::vector<Task>& out, int job, int kind, int64_t b, int64_t e,
                     int64_t chunk) {
  for (int64_t x = b; x < e; x += chunk) out.push_back(make_task(job, kind, x, std::min(e, x + chunk)));
}

// First index of the root tiers whose out-degree is <= x, x in {32, 64, 128, 256, 512}
// (tiers sorted by descending out-degree).
int64_t tier_begin(const RootTiers& t, int x) {
  return x <= 32 ? t.le_begin[0] : x <= 64 ? t.le_begin[1] : x <= 128 ? t.le_begin[2]
         : x <= 256 ? t.le_begin[3] : t.le_begin[4];
}

struct BuildOut {
  int dmax = 33;          // largest CTA-root out-degree
  int wdmax = 0;          // largest wide-root out-degree (0: no wide roots)
  int64_t c4max = 0;      // largest vertex count of a job with dense-counted 4-cycle apexes
  int64_t c4nmax = 0;     // largest vertex count of a job with large 4-cycle apexes
  int max_out = 0;        // largest out-degree among the large roots
  bool any_large = false;
  size_t tri_bytes = 0;   // diamond counters of the batch
};

// Prepares every graph (DAG, root tiers, 4-cycle apex classes) and builds the job and task
// tables on the host.  Diamond jobs get their per-arc counters at offsets of c.tri.
int build_tasks(const std::vector<BatchJobIn>& in, const jgpm_tuning& tu, BatchCtx& c,
                BuildOut* o) {
  c.h_jobs.clear();
  for (std::vector<Task>& v : c.cls) v.clear();
  c.h_c4_tasks.clear();
  std::vector<Task>&heavy = c.cls[0], &cta = c.cls[1], &c4m = c.cls[2], &warp = c.cls[3],
                     &c4s = c.cls[4], &light = c.cls[5], &c4l = c.h_c4_tasks;
  std::vector<uint64_t> c4w;  // wedge bound of each large-apex task
  std::vector<size_t> tri_off(in.size(), 0);
  const int split = tu.split_degree >= 128 ? 128 : tu.split_degree >= 64 ? 64 : 32;
  const int64_t rpt = std::max(8, tu.roots_per_task);
  for (size_t ji = 0; ji < in.size(); ++ji) {
    jgpm_graph* g = in[ji].g;
    int rc;
    JobDesc jd{};
    jd.n = g->n;
    jd.kind = in[ji].kind;
    jd.k = in[ji].kind == kJobDiamond ? 3 : in[ji].kind == kJobIndTT ? 4 : in[ji].k;
    const int job = (int)ji;
    if (in[ji].kind == kJobC4) {
      if ((rc = ensure_c4_apexes(g))) return rc;
      jd.rrow = g->d_rank_rowptr;
      jd.rcol = g->d_rank_col;
      jd.roots = g->d_c4_small;
      jd.apexes = g->d_c4_large;
      jd.nlarge = (int32_t)g->c4_nlarge;
      jd.mid = g->d_c4_mid;
      // large apexes (by descending wedge bound): a heavy one alone, lighter ones in runs of
      // at most kC4TaskWedges of wedge bound
      const std::vector<uint64_t>& key = g->c4_large_keys;
      for (int64_t q = 0, e; q < g->c4_nlarge; q = e) {
        uint64_t w = key[(size_t)q];
        for (e = q + 1; e < g->c4_nlarge && w + key[(size_t)e] <= kC4TaskWedges; ++e)
          w += key[(size_t)e];
        c4l.push_back(make_task(job, kTaskC4Large, q, e));
        c4w.push_back(w);
      }
      if (g->c4_ndense > 0) o->c4max = std::max<int64_t>(o->c4max, g->n);
      if (g->c4_nlarge > 0) o->c4nmax = std::max<int64_t>(o->c4nmax, g->n);
      add_range_tasks(c4m, job, kTaskC4Mid, 0, g->c4_nmid, kC4MidPerTask);
      add_range_tasks(c4s, job, kTaskC4Small, 0, g->c4_nsmall, std::max<int64_t>(8, rpt / 8));
      c.h_jobs.push_back(jd);
      continue;
    }
    if ((rc = ensure_dag(g))) return rc;
    if ((rc = ensure_tiers(g, 2))) return rc;
    jd.drow = g->d_dag_rowptr;
    jd.dcol = g->d_dag_col;
    const RootTiers& t = g->tiers;
    jd.roots = t.d_roots;
    jd.srow = g->d_rowptr;
    const bool per_arc = in[ji].kind == kJobDiamond || in[ji].kind == kJobIndTT;
    if (per_arc) {
      tri_off[ji] = o->tri_bytes;
      o->tri_bytes += ((size_t)std::max<int64_t>(1, g->m_dag) * 4 + 255) & ~(size_t)255;
    }
    // roots with d >= k-1; every triangle's root (d >= 2) for the per-arc counter jobs
    const int64_t stop = t.deg_begin[per_arc ? 1 : jd.k - 2];
    // roots by out-degree: > 2048 large | (512, 2048] wide | (split, 512] CTA |
    // (32, split] warp | <= 32 groups
    const int64_t wide_begin = std::min(stop, t.le_begin[5]);
    const int64_t large_end = std::min(stop, tier_begin(t, kBatchCtaMaxDeg));
    const int64_t cta_end = std::min(stop, std::max(large_end, tier_begin(t, split)));
    const int64_t warp_end = std::min(stop, std::max(cta_end, t.deg_begin[32]));
    for (int64_t r = 0; r < wide_begin; ++r) heavy.push_back(make_task(job, kTaskLargeRoot, r, r + 1));
    if (wide_begin > 0) {
      o->any_large = true;
      o->max_out = std::max(o->max_out, g->max_out_degree);
    }
    for (int64_t r = wide_begin; r < large_end; ++r)
      heavy.push_back(make_task(job, kTaskWideRoot, r, r + 1));
    if (large_end > wide_begin)
      o->wdmax = std::max(o->wdmax, std::min(g->max_out_degree, kBatchWideMaxDeg));
    // CTA roots above out-degree 256 count 16-word masks, the others 8-word ones
    const int64_t cta16_end = std::min(cta_end, std::max(large_end, tier_begin(t, 256)));
    for (int64_t r = large_end; r < cta_end; ++r)
      cta.push_back(make_task(job, r < cta16_end ? kTaskCtaRoot : kTaskCtaRoot8, r, r + 1));
    if (cta_end > large_end)
      o->dmax = std::max(o->dmax, std::min(g->max_out_degree, kBatchCtaMaxDeg));
    add_range_tasks(warp, job, kTaskWarpRoots, cta_end, warp_end, std::max<int64_t>(8, rpt / 4));
    // lane groups for d <= 32
    struct Cut { int g; int64_t b, e; };
    const int64_t b16 = tu.min_group <= 16 ? t.deg_begin[16] : t.small_end;
    const int64_t b8 = tu.min_group <= 8 ? t.deg_begin[8] : t.small_end;
    const int64_t b4 = tu.min_group <= 4 ? t.deg_begin[4] : t.small_end;
    const Cut cuts[4] = {{32, t.deg_begin[32], b16}, {16, b16, b8}, {8, b8, b4},
                         {4, b4, t.small_end}};
    for (const Cut& q : cuts) {
      const int64_t b = std::max(q.b, warp_end), e = std::min(q.e, stop);
      if (e <= b) continue;
      const int kind = q.g == 32 ? kTaskGroup32 : q.g == 16 ? kTaskGroup16
                     : q.g == 8 ? kTaskGroup8 : kTaskGroup4;
      add_range_tasks(light, job, kind, b, e, rpt);
    }
    c.h_jobs.push_back(jd);
  }
  // large 4-cycle apexes go to k_batch_c4_large job by job (so that the CTAs share one or two
  // graphs in L2 at a time), jobs by descending total wedge bound, each job's apexes by
  // descending bound (their order in the graph's list); the main queue: large roots, CTA
  // roots, mid apexes, warp roots, small apexes, lane groups
  if (c4l.size() > 1) {
    std::vector<uint64_t> weight(c.h_jobs.size(), 0);
    for (size_t q = 0; q < c4l.size(); ++q) weight[(size_t)c4l[q].job] += c4w[q];
    std::stable_sort(c4l.begin(), c4l.end(), [&](const Task& x, const Task& y) {
      const uint64_t wx = weight[(size_t)x.job], wy = weight[(size_t)y.job];
      return wx != wy ? wx > wy : x.job < y.job;
    });
  }
  size_t total = 0;
  for (const std::vector<Task>& v : c.cls) total += v.size();
  c.h_tasks.wait();  // the previous batch's copy out of the pinned table has finished
  int rc2;
  if ((rc2 = c.h_tasks.reserve(total))) return rc2;
  size_t at = 0;
  for (const std::vector<Task>& v : c.cls) {  // heavy, cta, c4m, warp, c4s, light
    if (!v.empty()) memcpy(c.h_tasks.p + at, v.data(), v.size() * sizeof(Task));
    at += v.size();
  }
  c.h_tasks.n = total;
  c.nmain = (int64_t)(total - light.size());  // lane-group tasks last: k_batch_groups
  c.tri_off.swap(tri_off);
  return JGPM_OK;
}

}  // namespace

// The stream operations of one batch: table uploads, counter resets, the large 4-cycle apex
// kernel, the task kernel, the lane-group kernel and the count read-back, in that order.
cudaError_t enqueue_plan(const LaunchPlan& p, cudaStream_t s) {
  cudaError_t e = cudaSuccess;
  auto ok = [&](cudaError_t r) {
    if (e == cudaSuccess) e = r;
  };
  if (p.tri_bytes) ok(cudaMemsetAsync(p.d_tri, 0, p.tri_bytes, s));
  ok(cudaMemcpyAsync(p.d_jobs, p.h_jobs, p.jobs_bytes, cudaMemcpyHostToDevice, s));
  if (p.tasks_bytes)
    ok(cudaMemcpyAsync(p.d_tasks, p.h_tasks, p.tasks_bytes, cudaMemcpyHostToDevice, s));
  ok(cudaMemsetAsync(p.d_counts, 0, p.counts_bytes, s));
  ok(cudaMemsetAsync(p.d_cursor, 0, 3 * sizeof(unsigned long long), s));
  if (p.c4_kernel) {
    if (p.c4_zero_bytes) ok(cudaMemsetAsync(p.d_c4_zero, 0, p.c4_zero_bytes, s));
    ok(cudaMemcpyAsync(p.d_c4_tasks, p.h_c4_tasks, p.c4_tasks_bytes, cudaMemcpyHostToDevice, s));
    C4BatchArgs b;
    memcpy(&b, p.c4_args, sizeof(b));
    if (p.c4_kernel == kC4NarrowThreads)
      k_batch_c4_large<kC4NarrowThreads><<<p.c4_ctas, kC4NarrowThreads, p.c4_smem, s>>>(b);
    else
      k_batch_c4_large<kC4WideThreads><<<p.c4_ctas, kC4WideThreads, p.c4_smem, s>>>(b);
    ok(cudaGetLastError());
  }
  BatchArgs a;
  memcpy(&a, p.args, sizeof(a));
  if (p.main_grid) k_batch<<<p.main_grid, 256, p.main_smem, s>>>(a);
  if (p.groups_grid) k_batch_groups<<<p.groups_grid, 256, 0, s>>>(a);
  ok(cudaGetLastError());
  if (p.h_counts)
    ok(cudaMemcpyAsync(p.h_counts, p.d_counts, p.d2h_bytes, cudaMemcpyDeviceToHost, s));
  return e;
}

// Issues the plan on `s`: replays the context's captured graph when the plan is unchanged,
// else captures the operations into a graph (updating the executable graph in place when its
// topology allows, instantiating a new one otherwise) and launches it.
int launch_plan(BatchCtx& c, const LaunchPlan& p, cudaStream_t s, bool use_graph) {
  if (!use_graph) {
    const cudaError_t e = enqueue_plan(p, s);
    if (e != cudaSuccess) {
      jgpm_set_error_(std::string("batch launch: ") + cudaGetErrorString(e));
      return JGPM_ECUDA;
    }
    return JGPM_OK;
  }
  if (!(c.exec && c.have_plan && memcmp(&p, &c.plan, sizeof(LaunchPlan)) == 0)) {
    cudaGraph_t g = nullptr;
    JGPM_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    const cudaError_t e = enqueue_plan(p, s);
    const cudaError_t e2 = cudaStreamEndCapture(s, &g);
    if (e != cudaSuccess || e2 != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      jgpm_set_error_(std::string("batch graph capture: ") +
                      cudaGetErrorString(e != cudaSuccess ? e : e2));
      return JGPM_ECUDA;
    }
    if (c.exec) {
      cudaGraphExecUpdateResultInfo info;
      if (cudaGraphExecUpdate(c.exec, g, &info) != cudaSuccess) {
        cudaGetLastError();
        cudaGraphExecDestroy(c.exec);
        c.exec = nullptr;
      }
    }
    if (!c.exec) {
      const cudaError_t ei = cudaGraphInstantiate(&c.exec, g, 0);
      if (ei != cudaSuccess) {
        c.exec = nullptr;
        cudaGraphDestroy(g);
        jgpm_set_error_(std::string("batch graph instantiate: ") + cudaGetErrorString(ei));
        return JGPM_ECUDA;
      }
    }
    cudaGraphDestroy(g);
    c.plan = p;
    c.have_plan = true;
  }
  JGPM_CUDA_TRY(cudaGraphLaunch(c.exec, s));
  return JGPM_OK;
}

// Enqueues one batched launch on `s`; per-job counts land in c.counts (device) and are
// copied to `h_counts` (pinned host memory, or null: the context's pinned buffer) on the same
// stream.  All allocation and kernel set-up happens before the stream operations, which are
// replayed from a CUDA graph while the launch plan repeats (tu.graphs).
int batch_enqueue(BatchCtx& c, const std::vector<BatchJobIn>& in, const jgpm_tuning& tu,
                  cudaStream_t s, uint64_t* h_counts, int* ntasks_out, int* launches_out) {
  BuildOut o;
  int rc;
  if ((rc = build_tasks(in, tu, c, &o))) return rc;  // waits for this context's last batch
  const int sms = device_sm_count(c.device);
  const int W = (o.dmax + 31) / 32;
  const int wW = (o.wdmax + 31) / 32;
  const size_t smem = batch_smem_bytes(o.dmax, W, o.wdmax, wW);
  if ((rc = raise_smem_limit((const void*)k_batch, smem))) return rc;
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch, 256, smem);
  per_sm = std::max(1, std::min(per_sm, 8));
  const int grid = sms * per_sm;
  const size_t nj = c.h_jobs.size(), nt = c.h_tasks.n;
  if ((rc = c.jobs.reserve(nj * sizeof(JobDesc)))) return rc;
  if ((rc = c.tasks.reserve(std::max<size_t>(1, nt) * sizeof(Task)))) return rc;
  if ((rc = c.counts.reserve(nj * sizeof(unsigned long long)))) return rc;
  if ((rc = c.cursor.reserve(3 * sizeof(unsigned long long)))) return rc;
  if ((rc = c.h_jobs_pin.reserve(nj * sizeof(JobDesc)))) return rc;
  if (!h_counts) {
    if ((rc = c.h_counts_pin.reserve(nj * sizeof(uint64_t)))) return rc;
    h_counts = (uint64_t*)c.h_counts_pin.p;
  }
  LaunchPlan p;
  memset(&p, 0, sizeof(p));
  if (o.tri_bytes) {
    if ((rc = c.tri.reserve(o.tri_bytes))) return rc;
    for (size_t ji = 0; ji < nj; ++ji)
      if (c.h_jobs[ji].kind == kJobDiamond || c.h_jobs[ji].kind == kJobIndTT)
        c.h_jobs[ji].tri = (uint32_t*)((char*)c.tri.p + c.tri_off[ji]);
    p.d_tri = c.tri.p;
    p.tri_bytes = o.tri_bytes;
  }
  BatchArgs a;
  memset(&a, 0, sizeof(a));
  if (o.wdmax > 0) {
    if ((rc = c.rows.reserve((size_t)grid * o.wdmax * wW * sizeof(uint32_t)))) return rc;
    a.rows = (uint32_t*)c.rows.p;
    a.wdmax = o.wdmax;
    a.wW = wW;
  }
  if (o.any_large) {
    a.list_cap = o.max_out + 32;
    if ((rc = c.lists.reserve((size_t)grid * 8 * kLevels * a.list_cap * sizeof(int32_t))))
      return rc;
    a.list_scratch = (int32_t*)c.lists.p;
  }
  memcpy(c.h_jobs_pin.p, c.h_jobs.data(), nj * sizeof(JobDesc));
  p.d_jobs = c.jobs.p;
  p.h_jobs = c.h_jobs_pin.p;
  p.jobs_bytes = nj * sizeof(JobDesc);
  p.d_tasks = c.tasks.p;
  p.h_tasks = c.h_tasks.p;
  p.tasks_bytes = nt * sizeof(Task);
  p.d_counts = c.counts.p;
  p.counts_bytes = nj * sizeof(unsigned long long);
  p.d_cursor = c.cursor.p;
  // large 4-cycle apexes: k_batch_c4_large on the same stream, before k_batch.  (Run side by
  // side on two streams the two kernels took twice their sum: the persistent k_batch CTAs hold
  // the SMs whose shared memory the slab CTAs need, and the two working sets share L2.)
  const size_t n4 = c.h_c4_tasks.size();
  if (n4 > 0) {
    // the narrow slab form when every job with large apexes has at most kC4NarrowMaxN
    // vertices (the form their dense flags assume); the wide form otherwise, which is exact
    // for every apex too
    const C4SlabForm form = c4_slab_form(o.c4nmax);
    const size_t slab_bytes = (size_t)form.words * sizeof(uint32_t);
    auto kern = form.threads == kC4NarrowThreads ? k_batch_c4_large<kC4NarrowThreads>
                                                  : k_batch_c4_large<kC4WideThreads>;
    if ((rc = raise_smem_limit((const void*)kern, slab_bytes))) return rc;
    int c4_per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c4_per_sm, kern, form.threads, slab_bytes);
    int64_t ctas = std::min<int64_t>((int64_t)sms * std::max(1, c4_per_sm), (int64_t)n4);
    const size_t per_cta = (size_t)o.c4max * sizeof(int32_t);  // 0: no dense apex
    if (per_cta) ctas = std::min<int64_t>(ctas, (int64_t)(c.c4_cap_bytes / per_cta));
    ctas = std::max<int64_t>(1, ctas);
    const size_t need = (size_t)ctas * per_cta;
    if (need) {
      if ((rc = c.c4.reserve(need))) return rc;
      if (c.c4_zeroed < need) {  // counters are zero between apexes; zero fresh memory once
        p.d_c4_zero = c.c4.p;
        p.c4_zero_bytes = c.c4.bytes;
        c.c4_zeroed = c.c4.bytes;
      }
      if ((rc = c.c4t.reserve(need))) return rc;
    }
    if ((rc = c.c4_tasks.reserve(n4 * sizeof(Task)))) return rc;
    if ((rc = c.h_c4_pin.reserve(n4 * sizeof(Task)))) return rc;
    memcpy(c.h_c4_pin.p, c.h_c4_tasks.data(), n4 * sizeof(Task));
    C4BatchArgs b;
    memset(&b, 0, sizeof(b));
    b.jobs = (const JobDesc*)c.jobs.p;
    b.tasks = (const Task*)c.c4_tasks.p;
    b.ntasks = (int64_t)n4;
    b.counts = (unsigned long long*)c.counts.p;
    b.cursor = (unsigned long long*)c.cursor.p + 1;
    b.dense = need ? (int32_t*)c.c4.p : nullptr;
    b.touched = need ? (vid_t*)c.c4t.p : nullptr;
    b.stride = o.c4max;
    b.words = form.words;
    static_assert(sizeof(C4BatchArgs) <= sizeof(p.c4_args), "plan: C4BatchArgs too large");
    memcpy(p.c4_args, &b, sizeof(b));
    p.c4_kernel = form.threads;
    p.c4_ctas = (int)ctas;
    p.c4_smem = slab_bytes;
    p.d_c4_tasks = c.c4_tasks.p;
    p.h_c4_tasks = c.h_c4_pin.p;
    p.c4_tasks_bytes = n4 * sizeof(Task);
  }
  a.jobs = (const JobDesc*)c.jobs.p;
  a.tasks = (const Task*)c.tasks.p;
  a.ntasks = (int64_t)nt;
  a.counts = (unsigned long long*)c.counts.p;
  a.cursor = (unsigned long long*)c.cursor.p;
  a.dmax = o.dmax;
  a.W = W;
  a.intersect = tu.intersect;
  const int64_t nmain = c.nmain;
  a.nmain = nmain;
  static_assert(sizeof(BatchArgs) <= sizeof(p.args), "plan: BatchArgs too large");
  memcpy(p.args, &a, sizeof(a));
  p.main_grid = nmain ? grid : 0;
  p.main_smem = smem;
  if ((int64_t)nt > nmain) {
    int gper = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&gper, k_batch_groups, 256, 0);
    p.groups_grid = sms * std::max(1, gper);
  }
  p.h_counts = h_counts;
  p.d2h_bytes = nj * sizeof(uint64_t);
  if ((rc = launch_plan(c, p, s, tu.graphs != 0))) return rc;
  // the pinned tables may be rewritten once this batch has finished
  if ((rc = c.h_tasks.record(s))) return rc;
  if (ntasks_out) *ntasks_out = (int)(nt + n4);
  if (launches_out) *launches_out = (nmain ? 1 : 0) + (p.groups_grid ? 1 : 0) + (n4 ? 1 : 0);
  return JGPM_OK;
}

int parse_batch_pattern(const char* pattern, int* kind, int* k) {
  const std::string p(pattern ? pattern : "");
  *k = 0;
  if (p == "triangle" || p == "P0" || p == "3-clique") { *kind = kJobClique; *k = 3; }
  else if (p == "4-clique" || p == "P13") { *kind = kJobClique; *k = 4; }
  else if (p == "5-clique" || p == "P14") { *kind = kJobClique; *k = 5; }
  else if (p == "6-clique" || p == "P15") { *kind = kJobClique; *k = 6; }
  else if (p == "7-clique" || p == "P16") { *kind = kJobClique; *k = 7; }
  else if (p.rfind("k-clique:", 0) == 0) {
    *kind = kJobClique;
    *k = atoi(p.c_str() + 9);
    if (*k < 3 || *k > 8) return JGPM_EPATTERN;
  } else if (p == "diamond" || p == "P2") { *kind = kJobDiamond; }
  else if (p == "induced:tailed-triangle") { *kind = kJobIndTT; *k = 4; }
  else if (p == "4-cycle" || p == "P1") { *kind = kJobC4; }
  else return JGPM_EPATTERN;
  return JGPM_OK;
}

jgpm_tuning default_tuning() {
  jgpm_tuning t;
  t.min_group = 8;
  t.split_degree = 128;
  t.roots_per_task = 256;
  t.intersect = 0;
  t.graphs = 1;
  return t;
}

int collect_jobs(const jgpm_job* jobs, int32_t njobs, std::vector<BatchJobIn>& in,
                        int* device) {
  in.clear();
  for (int32_t i = 0; i < njobs; ++i) {
    if (!jobs[i].graph) {
      jgpm_set_error_("batch: job " + std::to_string(i) + " has no graph");
      return JGPM_EINVAL;
    }
    BatchJobIn b{jobs[i].graph, 0, 0};
    if (parse_batch_pattern(jobs[i].pattern, &b.kind, &b.k)) {
      jgpm_set_error_("batch: job " + std::to_string(i) + ": pattern '" +
                      std::string(jobs[i].pattern ? jobs[i].pattern : "") +
                      "' is not batchable (triangle, k-clique, diamond, 4-cycle, "
                      "induced:tailed-triangle)");
      return JGPM_EPATTERN;
    }
    if (i == 0) *device = jobs[i].graph->device;
    else if (jobs[i].graph->device != *device) {
      jgpm_set_error_("batch: all graphs of a batch must live on one device");
      return JGPM_EINVAL;
    }
    in.push_back(b);
  }
  return JGPM_OK;
}

}  // namespace jgpm

using namespace jgpm;

namespace {
std::mutex g_batch_mu;
BatchCtx* g_sync_ctx[64] = {nullptr};

double time_batch(BatchCtx& c, const std::vector<BatchJobIn>& in, const jgpm_tuning& tu,
                  cudaStream_t s, std::vector<uint64_t>& counts, int* rc_out) {
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, s);
  int rc = batch_enqueue(c, in, tu, s, nullptr, nullptr);
  cudaEventRecord(e1, s);
  if (rc == JGPM_OK && cudaStreamSynchronize(s) != cudaSuccess) rc = JGPM_ECUDA;
  if (rc == JGPM_OK) memcpy(counts.data(), c.h_counts_pin.p, counts.size() * sizeof(uint64_t));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *rc_out = rc;
  return ms;
}
}  // namespace

extern "C" {

int jgpm_batch_count(const jgpm_job* jobs, int32_t njobs, const jgpm_tuning* tuning,
                     uint64_t* counts, jgpm_batch_stats* st) {
  if (!jobs || njobs < 0 || (!counts && njobs > 0)) {
    jgpm_set_error_("jgpm_batch_count: bad arguments");
    return JGPM_EINVAL;
  }
  if (njobs == 0) return JGPM_OK;
  std::vector<BatchJobIn> in;
  int device = 0;
  int rc = collect_jobs(jobs, njobs, in, &device);
  if (rc) return rc;
  if (device < 0 || device >= 64) return JGPM_EINVAL;
  jgpm_tuning tu = tuning ? *tuning : default_tuning();
  std::lock_guard<std::mutex> lk(g_batch_mu);
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(device);
  if (!g_sync_ctx[device]) {
    g_sync_ctx[device] = new BatchCtx;
    g_sync_ctx[device]->device = device;
  }
  BatchCtx& c = *g_sync_ctx[device];
  cudaStream_t s = jobs[0].graph->stream;
  // every graph's own stream must be idle before the batch reads it
  for (int32_t i = 0; i < njobs; ++i) cudaStreamSynchronize(jobs[i].graph->stream);
  std::vector<uint64_t> h((size_t)njobs);
  int ntasks = 0, launches = 0;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, s);
  rc = batch_enqueue(c, in, tu, s, nullptr, &ntasks, &launches);
  cudaEventRecord(e1, s);
  cudaError_t ce = cudaStreamSynchronize(s);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (prev >= 0) cudaSetDevice(prev);
  if (rc) return rc;
  if (ce != cudaSuccess) {
    jgpm_set_error_(std::string("jgpm_batch_count: ") + cudaGetErrorString(ce));
    return JGPM_ECUDA;
  }
  memcpy(counts, c.h_counts_pin.p, h.size() * sizeof(uint64_t));
  if (st) {
    st->kernel_ms = ms;
    st->launches = launches;
    st->tasks = ntasks;
    st->used = tu;
  }
  return JGPM_OK;
}

int jgpm_autotune(const jgpm_job* jobs, int32_t njobs, int32_t sample_jobs, jgpm_tuning* out) {
  if (!jobs || njobs <= 0 || !out) {
    jgpm_set_error_("jgpm_autotune: bad arguments");
    return JGPM_EINVAL;
  }
  std::vector<BatchJobIn> all;
  int device = 0;
  int rc = collect_jobs(jobs, njobs, all, &device);
  if (rc) return rc;
  // evenly spaced sample of the batch
  std::vector<BatchJobIn> in;
  const int32_t ns = sample_jobs > 0 ? std::min(sample_jobs, njobs) : std::min(njobs, 256);
  for (int32_t i = 0; i < ns; ++i) in.push_back(all[(int64_t)i * njobs / ns]);
  std::lock_guard<std::mutex> lk(g_batch_mu);
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(device);
  if (!g_sync_ctx[device]) {
    g_sync_ctx[device] = new BatchCtx;
    g_sync_ctx[device]->device = device;
  }
  BatchCtx& c = *g_sync_ctx[device];
  cudaStream_t s = jobs[0].graph->stream;
  std::vector<uint64_t> counts(in.size());
  jgpm_tuning best = default_tuning();
  auto measure = [&](const jgpm_tuning& t) {
    int r1 = 0;
    time_batch(c, in, t, s, counts, &r1);  // warm (graphs prepared, buffers sized)
    double ms = 1e30;
    for (int rep = 0; rep < 2 && r1 == JGPM_OK; ++rep) ms = std::min(ms, time_batch(c, in, t, s, counts, &r1));
    if (r1) rc = r1;
    return ms;
  };
  double best_ms = measure(best);
  // coordinate descent over the four knobs
  const int groups[] = {4, 8, 16, 32};
  const int splits[] = {32, 64, 128};
  const int rpt[] = {64, 256, 1024, 4096};
  const int isect[] = {0, 1};
  for (int pass = 0; pass < 2 && rc == JGPM_OK; ++pass) {
    for (int gsz : groups) {
      jgpm_tuning t = best;
      t.min_group = gsz;
      const double ms = measure(t);
      if (ms < best_ms) { best_ms = ms; best = t; }
    }
    for (int sp : splits) {
      jgpm_tuning t = best;
      t.split_degree = sp;
      const double ms = measure(t);
      if (ms < best_ms) { best_ms = ms; best = t; }
    }
    for (int r : rpt) {
      jgpm_tuning t = best;
      t.roots_per_task = r;
      const double ms = measure(t);
      if (ms < best_ms) { best_ms = ms; best = t; }
    }
    for (int is : isect) {
      jgpm_tuning t = best;
      t.intersect = is;
      const double ms = measure(t);
      if (ms < best_ms) { best_ms = ms; best = t; }
    }
  }
  if (prev >= 0) cudaSetDevice(prev);
  if (rc) return rc;
  *out = best;
  return JGPM_OK;
}

}  // extern "C"
