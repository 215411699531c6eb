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
//   large                      one CTA per apex, counts in a dense per-CTA array in global
//                              memory with a list of the touched vertices, heaviest apexes
//                              first.
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
        large_key[p] = ub;
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

__global__ void __launch_bounds__(256) k_c4_mid(const eid_t* rp, const vid_t* col,
                                                const vid_t* list, int64_t nlist,
                                                unsigned long long* cursor, DevControl* ctl) {
  extern __shared__ __align__(16) unsigned char smem[];
  C4CtaHash& h = *reinterpret_cast<C4CtaHash*>(smem);
  __shared__ unsigned long long s_q;
  const int tid = threadIdx.x, lane = tid & 31;
  c4_cta_hash_init(h);
  acc_t sum = 0;
  for (;;) {
    if (tid == 0) s_q = atomicAdd(cursor, 1ull);
    __syncthreads();
    const int64_t q = (int64_t)s_q;
    __syncthreads();
    if (q >= nlist) break;
    sum += c4_mid_apex(rp, col, list[q], h);
  }
  for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(kFull, sum, o);
  if (lane == 0 && sum) atomicAdd(&ctl->count[0], sum);
}

// 1024 threads per CTA: the dense arrays are large (n ints each), so each one is shared by as
// many warps as a CTA holds, to keep enough atomics in flight.
constexpr int kC4LargeThreads = 1024;

__global__ void __launch_bounds__(kC4LargeThreads)
    k_c4_large(const eid_t* rp, const vid_t* col, vid_t n, const vid_t* list, int64_t nlist,
               unsigned long long* cursor, int32_t* counters, DevControl* ctl) {
  int32_t* dense = counters + (int64_t)blockIdx.x * 2 * n;  // n counters, then n touched ids
  vid_t* touched = dense + n;
  __shared__ unsigned long long s_q;
  __shared__ C4LargeSmem<kC4LargeThreads> sh;
  const int tid = threadIdx.x, lane = tid & 31;
  acc_t sum = 0;
  for (;;) {
    if (tid == 0) s_q = atomicAdd(cursor, 1ull);
    __syncthreads();
    const int64_t q = (int64_t)s_q;
    __syncthreads();
    if (q >= nlist) break;
    sum += c4_large_apex(rp, col, list[q], dense, touched, sh);
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

// Classifies the apexes of g's rank CSR once: g->d_c4_small (any order) and g->d_c4_large
// (descending wedge bound), with their lengths.
int ensure_c4_apexes(jgpm_graph* g) {
  if (g->c4_nsmall >= 0) return JGPM_OK;
  int rc;
  if ((rc = ensure_rank_csr(g))) return rc;
  cudaStream_t s = g->stream;
  const int32_t n = g->n;
  TmpBuf small, mid, large, lkey, lkey2, ctr, tmp;
  if ((rc = small.alloc((size_t)n * 4)) || (rc = mid.alloc((size_t)n * 4)) ||
      (rc = large.alloc((size_t)n * 4)) || (rc = lkey.alloc((size_t)n * 8)) ||
      (rc = ctr.alloc(3 * sizeof(unsigned long long))))
    return rc;
  unsigned long long* dctr = (unsigned long long*)ctr.p;
  JGPM_CUDA_TRY(cudaMemsetAsync(dctr, 0, 3 * sizeof(unsigned long long), s));
  k_c4_classify<<<grid_for_c4((int64_t)n * 32), 256, 0, s>>>(
      g->d_rank_rowptr, g->d_rank_col, n, (vid_t*)small.p, (vid_t*)mid.p, (vid_t*)large.p,
      (uint64_t*)lkey.p, dctr);
  JGPM_CUDA_TRY(cudaGetLastError());
  unsigned long long h[3] = {0, 0, 0};
  JGPM_CUDA_TRY(cudaMemcpyAsync(h, dctr, sizeof(h), cudaMemcpyDeviceToHost, s));
  JGPM_CUDA_TRY(cudaStreamSynchronize(s));
  const int64_t nsmall = (int64_t)h[0], nlarge = (int64_t)h[1], nmid = (int64_t)h[2];
  int32_t *ds = nullptr, *dm = nullptr, *dl = nullptr;
  if (cudaMalloc(&ds, std::max<int64_t>(1, nsmall) * 4) != cudaSuccess ||
      cudaMalloc(&dm, std::max<int64_t>(1, nmid) * 4) != cudaSuccess ||
      cudaMalloc(&dl, std::max<int64_t>(1, nlarge) * 4) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(ds);
    cudaFree(dm);
    jgpm_set_error_("4-cycle: device allocation failed");
    return JGPM_ENOMEM;
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
  }
  g->c4_large_keys.resize((size_t)nlarge);
  if (nlarge)
    JGPM_CUDA_TRY(cudaMemcpyAsync(g->c4_large_keys.data(), lkey2.p, (size_t)nlarge * 8,
                                  cudaMemcpyDeviceToHost, s));
  JGPM_CUDA_TRY(cudaStreamSynchronize(s));
  g->c4_nsmall = nsmall;
  g->c4_nmid = nmid;
  g->c4_nlarge = nlarge;
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
  // dense counters and touched lists for the large apexes: 2n ints per CTA, within a 12 GiB
  // cap.  They are allocated for this count only (a graph pool would otherwise keep one such
  // array set per graph).
  const int64_t per_cta = (int64_t)n * 8;
  int64_t ctas = std::min<int64_t>((int64_t)sms * 2,
                                   ((int64_t)12 << 30) / std::max<int64_t>(1, per_cta));
  ctas = std::max<int64_t>(1, std::min<int64_t>(ctas, nlarge));
  const size_t dense_bytes = nlarge > 0 ? (size_t)(ctas * per_cta) : 0;
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
    const size_t smem = sizeof(C4CtaHash);
    if ((rc = raise_smem_limit((const void*)k_c4_mid, smem))) return rc;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_c4_mid, 256, smem);
    per_sm = std::max(1, per_sm);
    const int64_t grid = std::min<int64_t>((int64_t)sms * per_sm, nmid);
    k_c4_mid<<<(int)grid, 256, smem, s>>>(g->d_rank_rowptr, g->d_rank_col, g->d_c4_mid, nmid,
                                          &g->d_ctl->counter[2], g->d_ctl);
    g->launches += 1;
  }
  if (nlarge > 0) {
    JGPM_CUDA_TRY(cudaMemsetAsync(dense, 0, dense_bytes, s));
    k_c4_large<<<(int)ctas, kC4LargeThreads, 0, s>>>(g->d_rank_rowptr, g->d_rank_col, n,
                                         g->d_c4_large, nlarge, &g->d_ctl->counter[1],
                                         (int32_t*)dense, g->d_ctl);
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
