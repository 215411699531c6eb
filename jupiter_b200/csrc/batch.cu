// Batched counting: many (graph, pattern) jobs in ONE persistent, work-stealing launch.
//
// The reference splits one query's root-edge range into `chunk_size` static rounds, one
// launch each (src/jupiter_gpm.cu:356-375).  Here every job of a batch is cut into tasks --
// chunks of roots of one out-degree tier, single heavy roots, chunks of edges or of 4-cycle
// apexes -- and all tasks of all jobs go into one global queue.  Persistent CTAs (a multiple
// of the SM count) pull tasks with an atomic cursor until the queue is empty, so uneven
// jobs share the GPU without host round trips; every task adds its partial count into its
// job's counter.  Tasks are ordered heaviest first.
//
// Per-task work (same device code as the plain kernels, clique_dev.cuh):
//   GROUP_G    k-clique roots with out-degree <= G, one root per G-lane group;
//   CTA_ROOT   k-clique roots handled by the whole CTA (bitmap rows in shared memory);
//   LARGE_ROOT k-clique roots of out-degree > 1024, edge-rooted lists in warp scratch;
//   DIAMOND    DAG arcs (u, v): t = |N(u) & N(v)| on the symmetric lists, += C(t, 2)
//              (the reference P2 plan, src/message_passing_gpu_kernels.cuh:188-252);
//   C4_APEX    4-cycle apexes v0 with a per-CTA dense counter array (wedge aggregation;
//              same count as the reference P1 plan, :104-186).
// The tuning (jgpm_tuning) picks the narrowest lane group, the out-degree above which a root
// runs CTA-wide, the roots per task and the edge intersection variant; jgpm_autotune picks
// them by timing candidates on a sample of the batch.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "batch.h"
#include "clique_dev.cuh"
#include "jgpm_internal.h"
#include "setops.cuh"

namespace jgpm {

struct BatchArgs {
  const JobDesc* jobs;
  const Task* tasks;     // [0, n_c4): 4-cycle apex tasks; [n_c4, ntasks): all others
  int64_t ntasks;
  int64_t n_c4;
  int c4_ctas;           // CTAs [0, c4_ctas) own a dense counter array and drain the 4-cycle queue
  unsigned long long* counts;
  unsigned long long* cursor;  // [0] main queue, [1] 4-cycle queue
  int dmax, W;
  int32_t* c4_counters;  // per CTA: c4_stride ints
  int64_t c4_stride;
  int32_t* list_scratch;  // per warp: 6 lists of list_cap ints
  int64_t list_cap;
  int intersect;  // 0 auto, 1 binary search, 2 merge path
};

namespace {

constexpr int kLevels = 6;

template <int REM>
struct BatchListClique {
  __device__ static acc_t run(const eid_t* rowptr, const vid_t* col, const vid_t* cand, int nc,
                              int32_t* buf, int64_t cap) {
    const int lane = threadIdx.x & 31;
    acc_t s = 0;
    for (int i = 0; i < nc; ++i) {
      const vid_t v = cand[i];
      const eid_t b = rowptr[v];
      const int dv = (int)(rowptr[v + 1] - b);
      if (REM == 1) {
        int c = 0;
        for (int q = lane; q < nc; q += 32)
          if (contains_g(col + b, dv, cand[q])) ++c;
        s += (acc_t)warp_sum_int(c);
      } else {
        const int t = warp_intersect_w(cand, nc, col + b, dv, INT32_MAX, buf);
        if (t > 0)
          s += BatchListClique<(REM > 1 ? REM - 1 : 1)>::run(rowptr, col, buf, t, buf + cap, cap);
      }
    }
    return s;
  }
};

template <int G, int K>
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
    cnt += group_root<G, K, false, false>(j.drow, j.dcol, u, R, DG, nullptr, el);
  }
  return cnt;
}

template <int G>
__device__ __forceinline__ acc_t task_groups_k(const JobDesc& j, int64_t b, int64_t e,
                                               uint32_t* rows, int* degs) {
  switch (j.k) {
    case 3: return task_groups<G, 3>(j, b, e, rows, degs);
    case 4: return task_groups<G, 4>(j, b, e, rows, degs);
    case 5: return task_groups<G, 5>(j, b, e, rows, degs);
    case 6: return task_groups<G, 6>(j, b, e, rows, degs);
    case 7: return task_groups<G, 7>(j, b, e, rows, degs);
    default: return task_groups<G, 8>(j, b, e, rows, degs);
  }
}

__device__ __forceinline__ acc_t task_cta_roots(const JobDesc& j, int64_t b, int64_t e,
                                                const MidSmem& sm) {
  acc_t cnt = 0, el = 0;
  for (int64_t r = b; r < e; ++r) {
    const vid_t u = j.roots[r];
    switch (j.k) {
      case 3: cnt += cta_root<3, false, false>(j.drow, j.dcol, u, sm, nullptr, el); break;
      case 4: cnt += cta_root<4, false, false>(j.drow, j.dcol, u, sm, nullptr, el); break;
      case 5: cnt += cta_root<5, false, false>(j.drow, j.dcol, u, sm, nullptr, el); break;
      case 6: cnt += cta_root<6, false, false>(j.drow, j.dcol, u, sm, nullptr, el); break;
      case 7: cnt += cta_root<7, false, false>(j.drow, j.dcol, u, sm, nullptr, el); break;
      default: cnt += cta_root<8, false, false>(j.drow, j.dcol, u, sm, nullptr, el); break;
    }
  }
  return cnt;
}

// Warps of the CTA take the arcs of the large roots [b, e) (edge-rooted lists).
__device__ acc_t task_large_roots(const JobDesc& j, int64_t b, int64_t e, const BatchArgs& a) {
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int64_t gwarp = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp;
  int32_t* buf = a.list_scratch + gwarp * kLevels * a.list_cap;
  const int64_t cap = a.list_cap;
  acc_t cnt = 0;
  for (int64_t r = b; r < e; ++r) {
    const vid_t u = j.roots[r];
    const eid_t bu = j.drow[u];
    const int du = (int)(j.drow[u + 1] - bu);
    for (int i = warp; i < du; i += 8) {
      const vid_t v = __ldg(j.dcol + bu + i);
      const eid_t bv = j.drow[v];
      const int dv = (int)(j.drow[v + 1] - bv);
      const int tw = warp_intersect(j.dcol + bu, du, j.dcol + bv, dv, INT32_MAX, buf);
      if (lane == 0 && j.k == 3) cnt += (acc_t)tw;
      if (j.k > 3 && tw > 0) {
        acc_t c = 0;
        switch (j.k) {
          case 4: c = BatchListClique<1>::run(j.drow, j.dcol, buf, tw, buf + cap, cap); break;
          case 5: c = BatchListClique<2>::run(j.drow, j.dcol, buf, tw, buf + cap, cap); break;
          case 6: c = BatchListClique<3>::run(j.drow, j.dcol, buf, tw, buf + cap, cap); break;
          case 7: c = BatchListClique<4>::run(j.drow, j.dcol, buf, tw, buf + cap, cap); break;
          default: c = BatchListClique<5>::run(j.drow, j.dcol, buf, tw, buf + cap, cap); break;
        }
        if (lane == 0) cnt += c;
      }
    }
  }
  return cnt;
}

// DAG arcs [b, e): sum of C(|N(u) & N(v)|, 2) over the symmetric lists.
__device__ acc_t task_diamond(const JobDesc& j, int64_t b, int64_t e, int intersect) {
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  acc_t cnt = 0;
  for (int64_t arc = b + warp; arc < e; arc += 8) {
    // owner u of the DAG arc
    int64_t lo = 0, hi = j.n;
    while (lo < hi) {
      const int64_t mid = (lo + hi + 1) >> 1;
      if (j.drow[mid] <= arc) lo = mid;
      else hi = mid - 1;
    }
    const vid_t u = (vid_t)lo;
    const vid_t v = __ldg(j.dcol + arc);
    const int32_t* Nu = j.scol + j.srow[u];
    const int du = (int)(j.srow[u + 1] - j.srow[u]);
    const int32_t* Nv = j.scol + j.srow[v];
    const int dv = (int)(j.srow[v + 1] - j.srow[v]);
    acc_t t;
    if (intersect == 1) {
      // binary search of the shorter list's keys in the longer list
      const int32_t* A = du <= dv ? Nu : Nv;
      const int32_t* B = du <= dv ? Nv : Nu;
      const int na = min(du, dv), nb = max(du, dv);
      int c = 0;
      for (int q = lane; q < na; q += 32)
        if (contains_g(B, nb, __ldg(A + q))) ++c;
      t = (acc_t)warp_sum_int(c);
    } else {
      t = (acc_t)warp_intersect_count(Nu, du, Nv, dv);
    }
    if (lane == 0) cnt += t * (t - (t > 0 ? 1 : 0)) / 2;
  }
  return cnt;
}

// Apexes [b, e) of the wedge 4-cycle count; cnt_arr is this CTA's zeroed counter array.
__device__ acc_t task_c4(const JobDesc& j, int64_t b, int64_t e, int32_t* cnt_arr) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  acc_t sum = 0;
  for (int64_t vi = b; vi < e; ++vi) {
    const vid_t v0 = (vid_t)vi;
    const eid_t b0 = j.srow[v0];
    const int64_t d0 = j.srow[v0 + 1] - b0;
    if (d0 < 2) continue;
    for (int pass = 0; pass < 2; ++pass) {
      for (int64_t i = warp; i < d0; i += nw) {
        const vid_t x = __ldg(j.scol + b0 + i);
        const eid_t bx = j.srow[x];
        const int64_t dx = j.srow[x + 1] - bx;
        if (!(dx < d0 || (dx == d0 && x < v0))) continue;
        for (int64_t q = lane; q < dx; q += 32) {
          const vid_t v3 = __ldg(j.scol + bx + q);
          const int64_t d3 = j.srow[v3 + 1] - j.srow[v3];
          if (!(d3 < d0 || (d3 == d0 && v3 < v0))) continue;
          if (pass == 0) {
            atomicAdd(&cnt_arr[v3], 1);
          } else {
            const int c = atomicExch(&cnt_arr[v3], 0);
            sum += (acc_t)c * (acc_t)(c - 1) / 2;
          }
        }
      }
      __syncthreads();
    }
  }
  return sum;
}

__global__ void __launch_bounds__(256) k_batch(BatchArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const MidSmem sm = MidSmem::carve(smem, a.dmax, a.W);
  __shared__ uint32_t rows[256];
  __shared__ int degs[256];
  __shared__ unsigned long long s_task;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const bool c4_owner = a.c4_counters && (int)blockIdx.x < a.c4_ctas;
  int32_t* c4 = c4_owner ? a.c4_counters + (int64_t)blockIdx.x * a.c4_stride : nullptr;
  bool c4_done = !c4_owner;
  for (;;) {
    if (tid == 0) {
      unsigned long long t = ~0ull;
      if (!c4_done) {
        t = atomicAdd(&a.cursor[1], 1ull);
        if ((int64_t)t >= a.n_c4) t = ~0ull;
      }
      if (t == ~0ull) t = (unsigned long long)a.n_c4 + atomicAdd(&a.cursor[0], 1ull);
      s_task = t;
    }
    __syncthreads();
    const int64_t ti = (int64_t)s_task;
    __syncthreads();
    if (ti >= a.n_c4) c4_done = true;
    if (ti >= a.ntasks) break;
    const Task t = a.tasks[ti];
    const JobDesc j = a.jobs[t.job];
    acc_t c = 0;
    switch (t.kind) {
      case kTaskGroup4: c = task_groups_k<4>(j, t.b, t.e, rows, degs); break;
      case kTaskGroup8: c = task_groups_k<8>(j, t.b, t.e, rows, degs); break;
      case kTaskGroup16: c = task_groups_k<16>(j, t.b, t.e, rows, degs); break;
      case kTaskGroup32: c = task_groups_k<32>(j, t.b, t.e, rows, degs); break;
      case kTaskCtaRoot: c = task_cta_roots(j, t.b, t.e, sm); break;
      case kTaskLargeRoot: c = task_large_roots(j, t.b, t.e, a); break;
      case kTaskDiamond: c = task_diamond(j, t.b, t.e, a.intersect); break;
      case kTaskC4: c = task_c4(j, t.b, t.e, c4); break;
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(kFull, c, o);
    if (lane == 0 && c) atomicAdd(&a.counts[t.job], c);
  }
}

}  // namespace
}  // namespace jgpm

// ======================================================================= host side
namespace jgpm {

namespace {

void add_range_tasks(std::vector<Task>& out, int job, int kind, int64_t b, int64_t e,
                            int64_t chunk) {
  for (int64_t x = b; x < e; x += chunk) out.push_back(Task{job, kind, x, std::min(e, x + chunk)});
}

// Prepares every graph (DAG, root tiers) and builds the job and task tables on the host.
int build_tasks(const std::vector<BatchJobIn>& in, const jgpm_tuning& tu, BatchCtx& c,
                       int* dmax_out, int64_t* c4_n, int* max_out_deg) {
  c.h_jobs.clear();
  c.h_tasks.clear();
  int dmax = 33;
  int64_t c4max = 0;
  int maxo = 0;
  std::vector<Task> heavy, mid, light, c4t;
  const int split = std::min(32, std::max(tu.split_degree, 4));
  for (size_t ji = 0; ji < in.size(); ++ji) {
    jgpm_graph* g = in[ji].g;
    int rc;
    if ((rc = ensure_dag(g))) return rc;
    JobDesc jd{};
    jd.drow = g->d_dag_rowptr;
    jd.dcol = g->d_dag_col;
    jd.srow = g->d_rowptr;
    jd.scol = g->d_col;
    jd.n = g->n;
    jd.kind = in[ji].kind;
    jd.k = in[ji].k;
    const int job = (int)ji;
    if (in[ji].kind == kJobClique) {
      if ((rc = ensure_tiers(g, 2))) return rc;
      const RootTiers& t = g->tiers;
      jd.roots = t.d_roots;
      const int64_t stop = t.deg_begin[in[ji].k - 2];
      maxo = std::max(maxo, g->max_out_degree);
      dmax = std::max(dmax, std::min(g->max_out_degree, kMidMaxDeg));
      for (int64_t r = 0; r < std::min(stop, t.large_end); ++r)
        heavy.push_back(Task{job, kTaskLargeRoot, r, r + 1});
      // CTA roots: [large_end, deg_begin[split]) (out-degree above the split)
      const int64_t cta_end = std::min(stop, std::max(t.large_end, t.deg_begin[split]));
      for (int64_t r = t.large_end; r < cta_end; ++r) mid.push_back(Task{job, kTaskCtaRoot, r, r + 1});
      // lane groups for d <= split
      struct Cut { int g; int64_t b, e; };
      const int64_t b16 = tu.min_group <= 16 ? t.deg_begin[16] : t.small_end;
      const int64_t b8 = tu.min_group <= 8 ? t.deg_begin[8] : t.small_end;
      const int64_t b4 = tu.min_group <= 4 ? t.deg_begin[4] : t.small_end;
      const Cut cuts[4] = {{32, t.deg_begin[32], b16}, {16, b16, b8}, {8, b8, b4},
                           {4, b4, t.small_end}};
      for (const Cut& q : cuts) {
        const int64_t b = std::max(q.b, cta_end), e = std::min(q.e, stop);
        if (e <= b) continue;
        const int kind = q.g == 32 ? kTaskGroup32 : q.g == 16 ? kTaskGroup16
                       : q.g == 8 ? kTaskGroup8 : kTaskGroup4;
        add_range_tasks(light, job, kind, b, e, std::max(8, tu.roots_per_task));
      }
    } else if (in[ji].kind == kJobDiamond) {
      add_range_tasks(mid, job, kTaskDiamond, 0, g->m_dag,
                      std::max<int64_t>(64, (int64_t)tu.roots_per_task * 8));
    } else {
      c4max = std::max<int64_t>(c4max, g->n);
      add_range_tasks(c4t, job, kTaskC4, 0, g->n, std::max(16, tu.roots_per_task / 4));
    }
    c.h_jobs.push_back(jd);
  }
  // heaviest first: large roots, then CTA roots / edge / apex chunks, then lane groups
  c.h_tasks.reserve(c4t.size() + heavy.size() + mid.size() + light.size());
  c.n_c4 = (int64_t)c4t.size();
  c.h_tasks.insert(c.h_tasks.end(), c4t.begin(), c4t.end());
  c.h_tasks.insert(c.h_tasks.end(), heavy.begin(), heavy.end());
  c.h_tasks.insert(c.h_tasks.end(), mid.begin(), mid.end());
  c.h_tasks.insert(c.h_tasks.end(), light.begin(), light.end());
  *dmax_out = dmax;
  *c4_n = c4max;
  *max_out_deg = maxo;
  return JGPM_OK;
}

}  // namespace

// Enqueues one batched launch on `s`; per-job counts land in c.counts (device) and are
// copied to `h_counts` (pinned or pageable host memory) on the same stream.
int batch_enqueue(BatchCtx& c, const std::vector<BatchJobIn>& in, const jgpm_tuning& tu,
                  cudaStream_t s, uint64_t* h_counts, int* ntasks_out) {
  int dmax = 33, maxo = 0;
  int64_t c4n = 0;
  int rc;
  if ((rc = build_tasks(in, tu, c, &dmax, &c4n, &maxo))) return rc;
  const int sms = device_sm_count(c.device);
  const int W = (dmax + 31) / 32;
  const size_t smem = MidLayout{dmax, W}.bytes();
  cudaFuncSetAttribute(k_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch, 256, smem);
  per_sm = std::max(1, std::min(per_sm, 8));
  const int grid = sms * per_sm;
  const size_t nj = c.h_jobs.size(), nt = c.h_tasks.size();
  if ((rc = c.jobs.reserve(nj * sizeof(JobDesc)))) return rc;
  if ((rc = c.tasks.reserve(std::max<size_t>(1, nt) * sizeof(Task)))) return rc;
  if ((rc = c.counts.reserve(nj * sizeof(unsigned long long)))) return rc;
  if ((rc = c.cursor.reserve(2 * sizeof(unsigned long long)))) return rc;
  BatchArgs a{};
  if (c4n > 0) {
    const size_t per_cta = (size_t)c4n * sizeof(int32_t);
    a.c4_ctas = (int)std::max<size_t>(1, std::min<size_t>((size_t)grid, c.c4_cap_bytes / per_cta));
    const size_t need = (size_t)a.c4_ctas * per_cta;
    if ((rc = c.c4.reserve(need))) return rc;
    if (c.c4_zeroed < need) {  // counters are zero between apexes; zero fresh memory once
      JGPM_CUDA_TRY(cudaMemsetAsync(c.c4.p, 0, c.c4.bytes, s));
      c.c4_zeroed = c.c4.bytes;
    }
    a.c4_counters = (int32_t*)c.c4.p;
    a.c4_stride = c4n;
  }
  bool any_large = false;
  for (const Task& t : c.h_tasks) any_large = any_large || t.kind == kTaskLargeRoot;
  if (any_large) {
    a.list_cap = maxo + 32;
    if ((rc = c.lists.reserve((size_t)grid * 8 * kLevels * a.list_cap * sizeof(int32_t))))
      return rc;
    a.list_scratch = (int32_t*)c.lists.p;
  }
  JGPM_CUDA_TRY(cudaMemcpyAsync(c.jobs.p, c.h_jobs.data(), nj * sizeof(JobDesc),
                                cudaMemcpyHostToDevice, s));
  if (nt)
    JGPM_CUDA_TRY(cudaMemcpyAsync(c.tasks.p, c.h_tasks.data(), nt * sizeof(Task),
                                  cudaMemcpyHostToDevice, s));
  JGPM_CUDA_TRY(cudaMemsetAsync(c.counts.p, 0, nj * sizeof(unsigned long long), s));
  JGPM_CUDA_TRY(cudaMemsetAsync(c.cursor.p, 0, 2 * sizeof(unsigned long long), s));
  a.jobs = (const JobDesc*)c.jobs.p;
  a.tasks = (const Task*)c.tasks.p;
  a.ntasks = (int64_t)nt;
  a.n_c4 = c.n_c4;
  a.counts = (unsigned long long*)c.counts.p;
  a.cursor = (unsigned long long*)c.cursor.p;
  a.dmax = dmax;
  a.W = W;
  a.intersect = tu.intersect;
  if (nt) k_batch<<<grid, 256, smem, s>>>(a);
  JGPM_CUDA_TRY(cudaGetLastError());
  if (h_counts)
    JGPM_CUDA_TRY(cudaMemcpyAsync(h_counts, c.counts.p, nj * sizeof(uint64_t),
                                  cudaMemcpyDeviceToHost, s));
  if (ntasks_out) *ntasks_out = (int)nt;
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
  else if (p == "4-cycle" || p == "P1") { *kind = kJobC4; }
  else return JGPM_EPATTERN;
  return JGPM_OK;
}

jgpm_tuning default_tuning() {
  jgpm_tuning t;
  t.min_group = 8;
  t.split_degree = 32;
  t.roots_per_task = 256;
  t.intersect = 0;
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
                      "' is not batchable (triangle, k-clique, diamond, 4-cycle)");
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
  int rc = batch_enqueue(c, in, tu, s, counts.data(), nullptr);
  cudaEventRecord(e1, s);
  if (rc == JGPM_OK && cudaStreamSynchronize(s) != cudaSuccess) rc = JGPM_ECUDA;
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
  int ntasks = 0;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, s);
  rc = batch_enqueue(c, in, tu, s, h.data(), &ntasks);
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
  memcpy(counts, h.data(), h.size() * sizeof(uint64_t));
  if (st) {
    st->kernel_ms = ms;
    st->launches = ntasks > 0 ? 1 : 0;
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
  const int splits[] = {8, 16, 32};
  const int rpt[] = {32, 128, 512, 2048};
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
