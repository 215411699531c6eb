// 4-cycle count by wedge aggregation on the rank-relabelled CSR: the plain kernels.
//
// The reference's P1 plan (src/message_passing_gpu_kernels.cuh:104-186) counts every
// 4-cycle once, at its largest vertex v0, by intersecting N(v1) and N(v2) below v0 for every
// pair of neighbours v2 < v1 < v0 -- hub-sized intersections for every pair.  Here the same
// number is the sum over apexes of C(c(v0, v3), 2) (c4_dev.cuh), with the cycle attributed to
// its top-ranked vertex.  The apexes are classified once per graph by an upper bound on their
// wedge count (sum of deg(x) over the prefix), and the classes are kept with the graph:
//   small  (<= kC4SmallBound)  one warp per apex, counts in a shared-memory hash table;
//   mid    (<= kC4MidBound)    one CTA per apex, counts in a CTA-wide shared-memory table;
//   large                      one CTA of 1024 threads per apex, heaviest apexes first, the
//                              counts in a shared-memory slab of packed counters swept over
//                              the vertex range in slices; a light apex that would need many
//                              slices (graphs of millions of vertices; c4_dense_apex) counts
//                              in a dense per-CTA array in global memory with a touched list.
#include <cub/cub.cuh>

#include <algorithm>
#include <mutex>

#include "c4_dev.cuh"
#include "jgpm_internal.h"

namespace jgpm {
namespace {

__global__ void k_c4_classify(const eid_t* rp, const vid_t* col, vid_t n, vid_t* small_list,
                              vid_t* mid_list, vid_t* large_list, uint64_t* large_key,
                              unsigned long long* counters) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t v = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += warps) {
    const eid_t b = rp[v];
    const int d = (int)(rp[v + 1] - b);
    int cut = 0;
    if (lane == 0) cut = c4_lower_bound(col + b, d, (vid_t)v);
    cut = __shfl_sync(kFull, cut, 0);
    if (cut < 2) continue;  // a 4-cycle needs two lower-ranked neighbours of its apex
    unsigned long long ub = 0;
    for (int i = lane; i < cut; i += 32) {
      const vid_t x = __ldg(col + b + i);
      ub += (unsigned long long)(rp[x + 1] - rp[x]);
    }
    for (int o = 16; o > 0; o >>= 1) ub += __shfl_xor_sync(kFull, ub, o);
    if (lane == 0) {
      if (ub <= (unsigned long long)kC4SmallBound) {
        small_list[atomicAdd(&counters[0], 1ull)] = (vid_t)v;
      } else if (ub <= (unsigned long long)kC4MidBound) {
        mid_list[atomicAdd(&counters[2], 1ull)] = (vid_t)v;
      } else {
        const unsigned long long p = atomicAdd(&counters[1], 1ull);
        large_list[p] = (vid_t)v;
        const bool dense = c4_dense_apex((vid_t)v, cut, ub, c4_slab_form(n));
        large_key[p] = ub | (dense ? 0ull : kC4SlabKey);
        if (dense) atomicAdd(&counters[3], 1ull);
      }
    }
  }
}

__global__ void __launch_bounds__(256) k_c4_small(const eid_t* rp, const vid_t* col,
                                                  const vid_t* list, int64_t nlist,
                                                  unsigned long long* cursor, DevControl* ctl) {
  extern __shared__ __align__(16) unsigned char smem[];
  C4WarpHash& h = reinterpret_cast<C4WarpHash*>(smem)[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  c4_hash_init(h);
  acc_t sum = 0;
  for (;;) {
    unsigned long long q = 0;
    if (lane == 0) q = atomicAdd(cursor, 1ull);
    q = __shfl_sync(kFull, q, 0);
    if ((int64_t)q >= nlist) break;
    sum += c4_small_apex(rp, col, list[q], h);
  }
  for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(kFull, sum, o);
  if (lane == 0 && sum) atomicAdd(&ctl->count[0], sum);
}

// Lower-ranked neighbour count (the cut) of each large apex, stored after the apex list with
// kC4DenseFlag set for the apexes that count densely; strips kC4SlabKey from the sorted keys.
__global__ void k_c4_cuts(const eid_t* rp, const vid_t* col, const vid_t* list, uint64_t* key,
                          int64_t nlist, uint32_t* cuts) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < nlist; q += stride) {
    const vid_t v = list[q];
    const eid_t b = rp[v];
    const int cut = c4_lower_bound(col + b, (int)(rp[v + 1] - b), v);
    cuts[q] = (uint32_t)cut | ((key[q] & kC4SlabKey) ? 0u : kC4DenseFlag);
    key[q] &= ~kC4SlabKey;
  }
}

constexpr int kC4MidThreads = 256;

__global__ void __launch_bounds__(kC4MidThreads) k_c4_mid(const eid_t* rp, const vid_t* col,
                                                          const vid_t* list, int64_t nlist,
                                                          unsigned long long* cursor,
                                                          DevControl* ctl) {
  extern __shared__ __align__(16) unsigned char smem[];
  C4MidSmem<kC4MidThreads>& m = *reinterpret_cast<C4MidSmem<kC4MidThreads>*>(smem);
  __shared__ unsigned long long s_q;
  const int tid = threadIdx.x, lane = tid & 31;
  c4_cta_hash_init(m.h);
  acc_t sum = 0;
  for (;;) {
    if (tid == 0) s_q = atomicAdd(cursor, 1ull);
    __syncthreads();
    const int64_t q = (int64_t)s_q;
    __syncthreads();
    if (q >= nlist) break;
    sum += c4_mid_apex<kC4MidThreads>(rp, col, list[q], m);
  }
  for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(kFull, sum, o);
  if (lane == 0 && sum) atomicAdd(&ctl->count[0], sum);
}

// Large apexes on CTAs of NT threads.  SLAB: every apex of the list counts in the CTA's
// shared-memory slab of `words` words (a slab form: 1024 threads and one CTA per SM, or 512
// threads and two).  Otherwise every apex counts in the CTA's dense array (counters: 2n ints
// per CTA, n counters then n touched ids), a lighter kernel with two 1024-thread CTAs per SM.
// cuts: the stored cut of each apex of the list.
template <int NT, bool SLAB>
__global__ void __launch_bounds__(NT, (NT <= 512 || !SLAB) ? 2 : 1)
    k_c4_large(const eid_t* rp, const vid_t* col, vid_t n, const vid_t* list,
               const uint32_t* cuts, int64_t nlist, unsigned long long* cursor,
               int32_t* counters, int words, DevControl* ctl) {
  extern __shared__ __align__(16) uint32_t slab[];
  __shared__ unsigned long long s_q[2];
  __shared__ C4LargeSmem<NT> sh;
  int32_t* dense = SLAB ? nullptr : counters + (int64_t)blockIdx.x * 2 * n;
  vid_t* touched = SLAB ? nullptr : dense + n;
  const int tid = threadIdx.x, lane = tid & 31;
  if (SLAB) c4_slab_zero<NT>(slab, words);
  if (tid == 0) s_q[0] = atomicAdd(cursor, 1ull);
  __syncthreads();
  acc_t sum = 0;
  // Double-buffered task fetch: thread 0 takes the next apex while this one runs; every apex
  // passes barriers (its layouts) between the store and the reads of the next slot, and
  // between the reads of this slot and its next store.
  for (int it = 0;; ++it) {
    const int64_t q = (int64_t)s_q[it & 1];
    if (q >= nlist) break;
    if (tid == 0) s_q[(it + 1) & 1] = atomicAdd(cursor, 1ull);
    const vid_t v = list[q];
    const int cut = (int)(cuts[q] & ~kC4DenseFlag);
    if (SLAB)
      sum += c4_slab_apex<NT>(rp, col, v, cut, slab, words, sh);
    else
      sum += c4_large_apex<NT>(rp, col, v, cut, dense, touched, sh);
  }
  for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(kFull, sum, o);
  if (lane == 0 && sum) atomicAdd(&ctl->count[0], sum);
}

int grid_for_c4(int64_t work) {
  int64_t b = (work + 255) / 256;
  return (int)std::max<int64_t>(1, std::min<int64_t>(b, 148 * 32));
}

struct TmpBuf {
  void* p = nullptr;
  ~TmpBuf() {
    if (p) cudaFree(p);
  }
  int alloc(size_t bytes) {
    if (cudaMalloc(&p, std::max<size_t>(bytes, 16)) != cudaSuccess) {
      p = nullptr;
      cudaGetLastError();
      jgpm_set_error_("4-cycle: device allocation failed");
      return JGPM_ENOMEM;
    }
    return JGPM_OK;
  }
};

// Counter arrays of the large apexes, cached per device when they are small (a count on a
// small graph should not pay a cudaMalloc/cudaFree); larger ones are allocated per count so
// that a pool of large graphs does not keep them.  The lock is held for the whole count.
constexpr size_t kDenseCacheMax = (size_t)1 << 30;
struct DenseCache {
  std::mutex mu;
  void* p = nullptr;
  size_t bytes = 0;
};
DenseCache g_dense_cache[64];

}  // namespace

// Classifies the apexes of g's rank CSR once: g->d_c4_small (any order), g->d_c4_mid and
// g->d_c4_large (descending wedge bound, followed by the cut of each), with their lengths.
int ensure_c4_apexes(jgpm_graph* g) {
  if (g->c4_nsmall >= 0) return JGPM_OK;
  int rc;
  if ((rc = ensure_rank_csr(g))) return rc;
  cudaStream_t s = g->stream;
  const int32_t n = g->n;
  TmpBuf small, mid, large, lkey, lkey2, ctr, tmp;
  if ((rc = small.alloc((size_t)n * 4)) || (rc = mid.alloc((size_t)n * 4)) ||
      (rc = large.alloc((size_t)n * 4)) || (rc = lkey.alloc((size_t)n * 8)) ||
      (rc = ctr.alloc(4 * sizeof(unsigned long long))))
    return rc;
  unsigned long long* dctr = (unsigned long long*)ctr.p;
  JGPM_CUDA_TRY(cudaMemsetAsync(dctr, 0, 4 * sizeof(unsigned long long), s));
  k_c4_classify<<<grid_for_c4((int64_t)n * 32), 256, 0, s>>>(
      g->d_rank_rowptr, g->d_rank_col, n, (vid_t*)small.p, (vid_t*)mid.p, (vid_t*)large.p,
      (uint64_t*)lkey.p, dctr);
  JGPM_CUDA_TRY(cudaGetLastError());
  unsigned long long h[4] = {0, 0, 0, 0};
  JGPM_CUDA_TRY(cudaMemcpyAsync(h, dctr, sizeof(h), cudaMemcpyDeviceToHost, s));
  JGPM_CUDA_TRY(cudaStreamSynchronize(s));
  const int64_t nsmall = (int64_t)h[0], nlarge = (int64_t)h[1], nmid = (int64_t)h[2];
  int32_t *ds = nullptr, *dm = nullptr, *dl = nullptr;
  int arc = gmalloc((void**)&ds, std::max<int64_t>(1, nsmall) * 4, s);
  if (!arc) arc = gmalloc((void**)&dm, std::max<int64_t>(1, nmid) * 4, s);
  if (!arc) arc = gmalloc((void**)&dl, std::max<int64_t>(1, 2 * nlarge) * 4, s);
  if (arc) {
    gfree(ds, s);
    gfree(dm, s);
    return arc;
  }
  g->d_c4_small = ds;
  g->d_c4_mid = dm;
  g->d_c4_large = dl;
  if (nsmall)
    JGPM_CUDA_TRY(cudaMemcpyAsync(ds, small.p, nsmall * 4, cudaMemcpyDeviceToDevice, s));
  if (nmid)
    JGPM_CUDA_TRY(cudaMemcpyAsync(dm, mid.p, nmid * 4, cudaMemcpyDeviceToDevice, s));
  if (nlarge) {
    if ((rc = lkey2.alloc((size_t)nlarge * 8))) return rc;
    size_t tb = 0;
    JGPM_CUDA_TRY(cub::DeviceRadixSort::SortPairsDescending(
        nullptr, tb, (const uint64_t*)lkey.p, (uint64_t*)lkey2.p, (const vid_t*)large.p, dl,
        (int)nlarge, 0, 64, s));
    if ((rc = tmp.alloc(tb))) return rc;
    JGPM_CUDA_TRY(cub::DeviceRadixSort::SortPairsDescending(
        tmp.p, tb, (const uint64_t*)lkey.p, (uint64_t*)lkey2.p, (const vid_t*)large.p, dl,
        (int)nlarge, 0, 64, s));
    k_c4_cuts<<<grid_for_c4(nlarge), 256, 0, s>>>(g->d_rank_rowptr, g->d_rank_col, dl,
                                                 (uint64_t*)lkey2.p, nlarge,
                                                 (uint32_t*)(dl + nlarge));
    JGPM_CUDA_TRY(cudaGetLastError());
  }
  g->c4_large_keys.resize((size_t)nlarge);
  if (nlarge)
    JGPM_CUDA_TRY(cudaMemcpyAsync(g->c4_large_keys.data(), lkey2.p, (size_t)nlarge * 8,
                                  cudaMemcpyDeviceToHost, s));
  JGPM_CUDA_TRY(cudaStreamSynchronize(s));
  g->c4_nsmall = nsmall;
  g->c4_nmid = nmid;
  g->c4_nlarge = nlarge;
  g->c4_ndense = (int64_t)h[3];
  return JGPM_OK;
}

// Exact 4-cycle count of g (the reference P1 semantics: each cycle once).  Adds the launches
// to g->launches and the device time to *ms.
int count_c4_wedge(jgpm_graph* g, uint64_t* out, double* ms) {
  int rc;
  if ((rc = ensure_c4_apexes(g))) return rc;
  if ((rc = ensure_control(g))) return rc;
  cudaStream_t s = g->stream;
  const int32_t n = g->n;
  const int sms = device_sm_count(g->device);
  const int64_t nsmall = g->c4_nsmall, nmid = g->c4_nmid, nlarge = g->c4_nlarge;
  // Large apexes: the slab ones (first in the list) on CTAs with a shared-memory slab of the
  // graph's slab form, then the dense ones on two CTAs per SM with dense counters and touched
  // lists (2n ints per CTA, within a 12 GiB cap).  The dense arrays are allocated for this count only (a graph
  // pool would otherwise keep one such array set per graph), or taken from a small per-device
  // cache.
  const int64_t ndense = g->c4_ndense, nslab = nlarge - ndense;
  const uint32_t* cuts = (const uint32_t*)(g->d_c4_large + nlarge);
  const C4SlabForm form = c4_slab_form(n);
  const size_t slab_bytes = (size_t)form.words * sizeof(uint32_t);
  auto slab_kern = form.threads == kC4NarrowThreads ? k_c4_large<kC4NarrowThreads, true>
                                                     : k_c4_large<kC4WideThreads, true>;
  int64_t slab_ctas = 0;
  if (nslab > 0) {
    if ((rc = raise_smem_limit((const void*)slab_kern, slab_bytes))) return rc;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, slab_kern, form.threads, slab_bytes);
    slab_ctas = std::min<int64_t>((int64_t)sms * std::max(1, per_sm), nslab);
  }
  const int64_t per_cta = (int64_t)n * 8;
  int64_t ctas = std::min<int64_t>((int64_t)sms * 2,
                                   ((int64_t)12 << 30) / std::max<int64_t>(1, per_cta));
  ctas = std::max<int64_t>(1, std::min<int64_t>(ctas, ndense));
  const size_t dense_bytes = ndense > 0 ? (size_t)(ctas * per_cta) : 0;
  TmpBuf dense_tmp;
  std::unique_lock<std::mutex> cache_lk;
  void* dense = nullptr;
  if (dense_bytes > 0 && dense_bytes <= kDenseCacheMax && g->device >= 0 && g->device < 64) {
    DenseCache& dc = g_dense_cache[g->device];
    cache_lk = std::unique_lock<std::mutex>(dc.mu);
    if (dc.bytes < dense_bytes) {
      if (dc.p) cudaFree(dc.p);
      dc.p = nullptr;
      dc.bytes = 0;
      if (cudaMalloc(&dc.p, dense_bytes) != cudaSuccess) {
        cudaGetLastError();
        jgpm_set_error_("4-cycle: device allocation failed");
        return JGPM_ENOMEM;
      }
      dc.bytes = dense_bytes;
    }
    dense = dc.p;
  } else if (dense_bytes > 0) {
    if ((rc = dense_tmp.alloc(dense_bytes))) return rc;
    dense = dense_tmp.p;
  }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, s);
  JGPM_CUDA_TRY(cudaMemsetAsync(g->d_ctl, 0, sizeof(DevControl), s));
  if (nsmall > 0) {
    const size_t smem = 8 * sizeof(C4WarpHash);
    if ((rc = raise_smem_limit((const void*)k_c4_small, smem))) return rc;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_c4_small, 256, smem);
    per_sm = std::max(1, per_sm);
    const int64_t grid = std::min<int64_t>((int64_t)sms * per_sm, (nsmall + 7) / 8);
    k_c4_small<<<(int)grid, 256, smem, s>>>(g->d_rank_rowptr, g->d_rank_col, g->d_c4_small,
                                            nsmall, &g->d_ctl->counter[0], g->d_ctl);
    g->launches += 1;
  }
  if (nmid > 0) {
    const size_t smem = sizeof(C4MidSmem<kC4MidThreads>);
    if ((rc = raise_smem_limit((const void*)k_c4_mid, smem))) return rc;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_c4_mid, kC4MidThreads, smem);
    per_sm = std::max(1, per_sm);
    const int64_t grid = std::min<int64_t>((int64_t)sms * per_sm, nmid);
    k_c4_mid<<<(int)grid, kC4MidThreads, smem, s>>>(g->d_rank_rowptr, g->d_rank_col, g->d_c4_mid, nmid,
                                          &g->d_ctl->counter[2], g->d_ctl);
    g->launches += 1;
  }
  if (nslab > 0) {
    slab_kern<<<(int)slab_ctas, form.threads, slab_bytes, s>>>(
        g->d_rank_rowptr, g->d_rank_col, n, g->d_c4_large, cuts, nslab, &g->d_ctl->counter[1],
        nullptr, form.words, g->d_ctl);
    g->launches += 1;
  }
  if (ndense > 0) {
    JGPM_CUDA_TRY(cudaMemsetAsync(dense, 0, dense_bytes, s));
    k_c4_large<kC4DenseThreads, false><<<(int)ctas, kC4DenseThreads, 0, s>>>(
        g->d_rank_rowptr, g->d_rank_col, n, g->d_c4_large + nslab, cuts + nslab, ndense,
        &g->d_ctl->counter[3], (int32_t*)dense, 0, g->d_ctl);
    g->launches += 1;
  }
  cudaEventRecord(e1, s);
  JGPM_CUDA_TRY(cudaGetLastError());
  JGPM_CUDA_TRY(cudaMemcpyAsync(g->h_ctl, g->d_ctl, sizeof(DevControl), cudaMemcpyDeviceToHost,
                                s));
  JGPM_CUDA_TRY(cudaStreamSynchronize(s));
  float f = 0.f;
  cudaEventElapsedTime(&f, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *out = g->h_ctl->count[0];
  if (ms) *ms = f;
  return JGPM_OK;
}

}  // namespace jgpm
