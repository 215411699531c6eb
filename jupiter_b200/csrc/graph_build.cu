// Device-side graph construction: seeded R-MAT generation, CSR build (sort, dedup,
// symmetrise), validation of caller CSRs, degree orientation into a DAG, and the
// out-degree root tiers the clique kernels schedule from.
//
// Orientation keeps u->v iff deg(v) > deg(u) or (deg(v) == deg(u) and v > u), the rule of
// Graph::orientation (common/graph.cc:229-230, :383-384).  Because arcs are visited in
// CSR order, every DAG row stays sorted, as the reference's does.
#include <cub/cub.cuh>

#include <algorithm>
#include <map>
#include <mutex>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>

#include "jgpm_internal.h"
#include "rmat.h"

namespace jgpm {

namespace {

__global__ void k_rmat_keys(RmatParams p, int shift, uint64_t* keys, uint64_t invalid) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < p.num_edges;
       i += stride) {
    int32_t u, v;
    bool ok = rmat_edge(p, (uint64_t)i, &u, &v);
    if (!ok || u == v) {
      keys[2 * i] = invalid;
      keys[2 * i + 1] = invalid;
    } else {
      keys[2 * i] = ((uint64_t)u << shift) | (uint64_t)v;
      keys[2 * i + 1] = ((uint64_t)v << shift) | (uint64_t)u;
    }
  }
}

__global__ void k_edge_keys(const int32_t* src, const int32_t* dst, int64_t ne, int32_t n,
                            int shift, uint64_t* keys, uint64_t invalid, int* bad) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ne; i += stride) {
    int32_t u = src[i], v = dst[i];
    if (u < 0 || v < 0 || u >= n || v >= n) {
      atomicExch(bad, 1);
      keys[2 * i] = invalid;
      keys[2 * i + 1] = invalid;
      continue;
    }
    if (u == v) {
      keys[2 * i] = invalid;
      keys[2 * i + 1] = invalid;
    } else {
      keys[2 * i] = ((uint64_t)u << shift) | (uint64_t)v;
      keys[2 * i + 1] = ((uint64_t)v << shift) | (uint64_t)u;
    }
  }
}

__global__ void k_unique_flags(const uint64_t* keys, int64_t nk, uint64_t invalid, int* flags) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nk; i += stride) {
    uint64_t k = keys[i];
    flags[i] = (k != invalid && (i == 0 || keys[i - 1] != k)) ? 1 : 0;
  }
}

__global__ void k_compact_keys(const uint64_t* keys, const int* flags, const int64_t* pos,
                               int64_t nk, uint64_t mask, uint64_t* ukeys, int32_t* col) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nk; i += stride) {
    if (flags[i]) {
      uint64_t k = keys[i];
      ukeys[pos[i]] = k;
      col[pos[i]] = (int32_t)(k & mask);
    }
  }
}

// rowptr[v] = first unique key with source >= v.
__global__ void k_rowptr_from_keys(const uint64_t* ukeys, int64_t m, int32_t n, int shift,
                                   int64_t* rowptr) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v <= n; v += stride) {
    uint64_t target = (uint64_t)v << shift;
    int64_t lo = 0, hi = m;
    while (lo < hi) {
      int64_t mid = (lo + hi) >> 1;
      if (ukeys[mid] < target) lo = mid + 1;
      else hi = mid;
    }
    rowptr[v] = lo;
  }
}

// Expands rowptr into the source of every arc (one warp per vertex).
__global__ void k_arc_src(const int64_t* rowptr, int32_t n, int32_t* src) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t v = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += warps) {
    int64_t b = rowptr[v], e = rowptr[v + 1];
    for (int64_t k = b + lane; k < e; k += 32) src[k] = (int32_t)v;
  }
}

__global__ void k_validate(const int64_t* rowptr, const int32_t* col, const int32_t* src,
                           int32_t n, int64_t m, int* bad) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m; k += stride) {
    int32_t u = src[k];
    int32_t v = col[k];
    bool ok = v >= 0 && v < n && v != u;
    if (ok && k > rowptr[u]) ok = col[k - 1] < v;  // strictly increasing rows
    if (ok) {  // symmetric: u must appear in N(v)
      int64_t lo = rowptr[v], hi = rowptr[v + 1];
      while (lo < hi) {
        int64_t mid = (lo + hi) >> 1;
        if (col[mid] < u) lo = mid + 1;
        else hi = mid;
      }
      ok = lo < rowptr[v + 1] && col[lo] == u;
    }
    if (!ok) atomicExch(bad, 1);
  }
}

__global__ void k_rowptr_check(const int64_t* rowptr, int32_t n, int64_t m, int* bad) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
    if (rowptr[v + 1] < rowptr[v]) atomicExch(bad, 1);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (rowptr[0] != 0 || rowptr[n] != m) atomicExch(bad, 1);
  }
}

__global__ void k_orient_flags(const int64_t* rowptr, const int32_t* col, const int32_t* src,
                               int64_t m, int* keep) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m; k += stride) {
    int32_t u = src[k], v = col[k];
    int64_t du = rowptr[u + 1] - rowptr[u];
    int64_t dv = rowptr[v + 1] - rowptr[v];
    keep[k] = (dv > du || (dv == du && v > u)) ? 1 : 0;
  }
}

__global__ void k_orient_scatter(const int32_t* col, const int* keep, const int64_t* pos,
                                 int64_t m, int32_t* dag_col) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m; k += stride)
    if (keep[k]) dag_col[pos[k]] = col[k];
}

__global__ void k_dag_rowptr(const int64_t* rowptr, const int64_t* pos, int32_t n, int64_t m,
                             int64_t total, int64_t* dag_rowptr) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v <= n; v += stride) {
    int64_t r = rowptr[v];
    dag_rowptr[v] = (r < m) ? pos[r] : total;
  }
}

__global__ void k_max_degree(const int64_t* rowptr, int32_t n, int* out) {
  int local = 0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride)
    local = max(local, (int)(rowptr[v + 1] - rowptr[v]));
  for (int o = 16; o > 0; o >>= 1) local = max(local, __shfl_xor_sync(0xffffffffu, local, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, local);
}

// Root keys for the clique tiers: key = out-degree (roots below min_deg get key 0 and are
// dropped after the descending sort).
__global__ void k_root_keys(const int64_t* dag_rowptr, int32_t n, int min_deg, uint32_t* keys,
                            int32_t* vals) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
    int d = (int)(dag_rowptr[v + 1] - dag_rowptr[v]);
    keys[v] = d >= min_deg ? (uint32_t)d : 0u;
    vals[v] = (int32_t)v;
  }
}

std::mutex g_pool_mu;
cudaMemPool_t g_pools[64] = {};

// The library's pool on `dev`: it keeps every byte freed into it (no release threshold), so
// repeated graph life cycles reuse the same memory.  Callers that need the memory elsewhere
// get it back by the trim on an allocation failure.
cudaMemPool_t device_pool(int dev) {
  if (dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lk(g_pool_mu);
  if (!g_pools[dev]) {
    cudaMemPoolProps props;
    memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    g_pools[dev] = pool;
  }
  return g_pools[dev];
}

// Pinned host mirrors of the graphs' control blocks: slots of pinned slabs, reused.
std::mutex g_ctl_mu;
std::vector<DevControl*> g_ctl_free;

DevControl* ctl_slot() {
  std::lock_guard<std::mutex> lk(g_ctl_mu);
  if (g_ctl_free.empty()) {
    constexpr int kSlots = 256;
    DevControl* slab = nullptr;
    if (cudaMallocHost((void**)&slab, kSlots * sizeof(DevControl)) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    for (int i = kSlots - 1; i >= 0; --i) g_ctl_free.push_back(slab + i);
  }
  DevControl* p = g_ctl_free.back();
  g_ctl_free.pop_back();
  return p;
}

void ctl_release(DevControl* p) {
  if (!p) return;
  std::lock_guard<std::mutex> lk(g_ctl_mu);
  g_ctl_free.push_back(p);
}

int grid_for(int64_t work, int threads = 256) {
  int64_t b = (work + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > 148 * 32) b = 148 * 32;
  return (int)b;
}

}  // namespace

int gmalloc(void** p, size_t bytes, cudaStream_t s) {
  int dev = 0;
  cudaGetDevice(&dev);
  cudaMemPool_t pool = device_pool(dev);
  cudaError_t e = pool ? cudaMallocFromPoolAsync(p, bytes, pool, s) : cudaErrorMemoryAllocation;
  if (e == cudaErrorMemoryAllocation && pool) {  // return the cached memory, then retry once
    cudaGetLastError();
    cudaDeviceSynchronize();
    cudaMemPoolTrimTo(pool, 0);
    e = cudaMallocFromPoolAsync(p, bytes, pool, s);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    jgpm_set_error_(std::string("device allocation of ") + std::to_string(bytes) +
                    " bytes: " + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? JGPM_ENOMEM : JGPM_ECUDA;
  }
  return JGPM_OK;
}

void gfree(void* p, cudaStream_t s) {
  if (p) cudaFreeAsync(p, s);
}

namespace {

template <typename T>
int dalloc(T** p, size_t count, cudaStream_t s) {
  return gmalloc((void**)p, std::max<size_t>(count, 1) * sizeof(T), s);
}

// A temporary device buffer, returned to the pool in the order of stream s.
struct DevBuf {
  cudaStream_t s;
  void* p = nullptr;
  explicit DevBuf(cudaStream_t stream) : s(stream) {}
  ~DevBuf() {
    if (p) gfree(p, s);
  }
};

// Sorts 2*ne keys, removes duplicates and the invalid key, and fills g's symmetric CSR.
int keys_to_csr(jgpm_graph* g, int32_t n, uint64_t* d_keys, int64_t nk, int shift,
                uint64_t invalid, int end_bit) {
  cudaStream_t s = g->stream;
  DevBuf alt(g->stream), tmp(g->stream), flags(g->stream), pos(g->stream);
  int rc;
  if ((rc = dalloc((uint64_t**)&alt.p, nk, g->stream))) return rc;
  size_t tbytes = 0, tb2 = 0;
  cub::DoubleBuffer<uint64_t> db(d_keys, (uint64_t*)alt.p);
  JGPM_CUDA_TRY(cub::DeviceRadixSort::SortKeys(nullptr, tbytes, db, nk, 0, end_bit, s));
  JGPM_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tb2, (int*)nullptr, (int64_t*)nullptr,
                                              nk, s));
  tbytes = std::max(tbytes, tb2);
  if ((rc = dalloc((char**)&tmp.p, tbytes, g->stream))) return rc;
  JGPM_CUDA_TRY(cub::DeviceRadixSort::SortKeys(tmp.p, tbytes, db, nk, 0, end_bit, s));
  uint64_t* sorted = db.Current();
  uint64_t* spare = db.Alternate();
  if ((rc = dalloc((int**)&flags.p, nk, g->stream))) return rc;
  if ((rc = dalloc((int64_t**)&pos.p, nk + 1, g->stream))) return rc;
  k_unique_flags<<<grid_for(nk), 256, 0, s>>>(sorted, nk, invalid, (int*)flags.p);
  JGPM_CUDA_TRY(cub::DeviceScan::ExclusiveSum(tmp.p, tbytes, (int*)flags.p, (int64_t*)pos.p,
                                              nk, s));
  int64_t last_pos = 0;
  int last_flag = 0;
  if (nk > 0) {
    JGPM_CUDA_TRY(cudaMemcpyAsync(&last_pos, (int64_t*)pos.p + nk - 1, sizeof(int64_t),
                                  cudaMemcpyDeviceToHost, s));
    JGPM_CUDA_TRY(cudaMemcpyAsync(&last_flag, (int*)flags.p + nk - 1, sizeof(int),
                                  cudaMemcpyDeviceToHost, s));
    JGPM_CUDA_TRY(cudaStreamSynchronize(s));
  }
  const int64_t m = last_pos + last_flag;
  if ((rc = dalloc(&g->d_col, m, g->stream))) return rc;
  if ((rc = dalloc(&g->d_rowptr, (size_t)n + 1, g->stream))) return rc;
  uint64_t* ukeys = spare;  // nk >= m entries, free after the sort
  k_compact_keys<<<grid_for(nk), 256, 0, s>>>(sorted, (int*)flags.p, (int64_t*)pos.p, nk,
                                              (1ull << shift) - 1, ukeys, g->d_col);
  k_rowptr_from_keys<<<grid_for((int64_t)n + 1), 256, 0, s>>>(ukeys, m, n, shift,
                                                              g->d_rowptr);
  JGPM_CUDA_TRY(cudaGetLastError());
  g->n = n;
  g->m = m;
  return JGPM_OK;
}

int finish_sym(jgpm_graph* g) {
  DevBuf md(g->stream);
  int rc;
  if ((rc = dalloc((int**)&md.p, 1, g->stream))) return rc;
  JGPM_CUDA_TRY(cudaMemsetAsync(md.p, 0, sizeof(int), g->stream));
  k_max_degree<<<grid_for(g->n), 256, 0, g->stream>>>(g->d_rowptr, g->n, (int*)md.p);
  int h = 0;
  JGPM_CUDA_TRY(cudaMemcpyAsync(&h, md.p, sizeof(int), cudaMemcpyDeviceToHost, g->stream));
  JGPM_CUDA_TRY(cudaStreamSynchronize(g->stream));
  g->max_degree = h;
  return JGPM_OK;
}

int shift_for(int32_t n) {
  int s = 1;
  while ((int64_t(1) << s) <= (int64_t)n) ++s;  // ids and the invalid source n fit
  return s;
}

}  // namespace

int raise_smem_limit(const void* func, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, size_t> limits;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  size_t& cur = limits[std::make_pair(dev, func)];
  if (bytes <= cur) return JGPM_OK;
  const cudaError_t e =
      cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e != cudaSuccess) {
    jgpm_set_error_(std::string("raise_smem_limit: ") + cudaGetErrorString(e));
    return JGPM_ECUDA;
  }
  cur = bytes;
  return JGPM_OK;
}

int device_sm_count(int device) {
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
    return 148;
  return sms;
}

int rmat_build(jgpm_graph* g, int64_t n, int64_t num_edges, double a, double b, double c,
               uint64_t seed) {
  if (n < 2 || n > INT32_MAX - 1 || num_edges < 0 || a < 0 || b < 0 || c < 0 ||
      a + b + c > 1.0 + 1e-12) {
    jgpm_set_error_("jgpm_graph_rmat: bad parameters");
    return JGPM_EINVAL;
  }
  RmatParams p = rmat_params(n, num_edges, a, b, c, seed);
  const int shift = shift_for((int32_t)n);
  const uint64_t invalid = (uint64_t)n << shift;
  const int end_bit = 2 * shift;
  const int64_t nk = 2 * num_edges;
  DevBuf keys(g->stream);
  int rc;
  if ((rc = dalloc((uint64_t**)&keys.p, nk, g->stream))) return rc;
  k_rmat_keys<<<grid_for(num_edges), 256, 0, g->stream>>>(p, shift, (uint64_t*)keys.p, invalid);
  JGPM_CUDA_TRY(cudaGetLastError());
  if ((rc = keys_to_csr(g, (int32_t)n, (uint64_t*)keys.p, nk, shift, invalid, end_bit)))
    return rc;
  return finish_sym(g);
}

int edges_build(jgpm_graph* g, const int32_t* src, const int32_t* dst, int64_t ne, int32_t n) {
  if (n < 1 || ne < 0) {
    jgpm_set_error_("jgpm_graph_from_edges: bad sizes");
    return JGPM_EINVAL;
  }
  const int shift = shift_for(n);
  const uint64_t invalid = (uint64_t)n << shift;
  DevBuf ds(g->stream), dd(g->stream), keys(g->stream), bad(g->stream);
  int rc;
  if ((rc = dalloc((int32_t**)&ds.p, ne, g->stream))) return rc;
  if ((rc = dalloc((int32_t**)&dd.p, ne, g->stream))) return rc;
  if ((rc = dalloc((uint64_t**)&keys.p, 2 * ne, g->stream))) return rc;
  if ((rc = dalloc((int**)&bad.p, 1, g->stream))) return rc;
  JGPM_CUDA_TRY(cudaMemcpyAsync(ds.p, src, ne * sizeof(int32_t), cudaMemcpyDefault, g->stream));
  JGPM_CUDA_TRY(cudaMemcpyAsync(dd.p, dst, ne * sizeof(int32_t), cudaMemcpyDefault, g->stream));
  JGPM_CUDA_TRY(cudaMemsetAsync(bad.p, 0, sizeof(int), g->stream));
  k_edge_keys<<<grid_for(ne), 256, 0, g->stream>>>((int32_t*)ds.p, (int32_t*)dd.p, ne, n, shift,
                                                   (uint64_t*)keys.p, invalid, (int*)bad.p);
  int hbad = 0;
  JGPM_CUDA_TRY(cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, g->stream));
  JGPM_CUDA_TRY(cudaStreamSynchronize(g->stream));
  if (hbad) {
    jgpm_set_error_("jgpm_graph_from_edges: vertex id out of range");
    return JGPM_EINVAL;
  }
  if ((rc = keys_to_csr(g, n, (uint64_t*)keys.p, 2 * ne, shift, invalid, 2 * shift))) return rc;
  return finish_sym(g);
}

int upload_csr(jgpm_graph* g, const int64_t* rowptr, const int32_t* col, int32_t n, int64_t m,
               int validate) {
  if (n < 1 || m < 0 || !rowptr || (m > 0 && !col)) {
    jgpm_set_error_("jgpm_graph_from_csr: bad arguments");
    return JGPM_EINVAL;
  }
  int rc;
  if ((rc = dalloc(&g->d_rowptr, (size_t)n + 1, g->stream))) return rc;
  if ((rc = dalloc(&g->d_col, m, g->stream))) return rc;
  JGPM_CUDA_TRY(cudaMemcpyAsync(g->d_rowptr, rowptr, ((size_t)n + 1) * sizeof(int64_t),
                                cudaMemcpyDefault, g->stream));
  if (m > 0)
    JGPM_CUDA_TRY(cudaMemcpyAsync(g->d_col, col, (size_t)m * sizeof(int32_t), cudaMemcpyDefault,
                                  g->stream));
  g->n = n;
  g->m = m;
  if (validate) {
    DevBuf bad(g->stream), src(g->stream);
    if ((rc = dalloc((int**)&bad.p, 1, g->stream))) return rc;
    JGPM_CUDA_TRY(cudaMemsetAsync(bad.p, 0, sizeof(int), g->stream));
    k_rowptr_check<<<grid_for(n), 256, 0, g->stream>>>(g->d_rowptr, n, m, (int*)bad.p);
    int hbad = 0;
    JGPM_CUDA_TRY(cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, g->stream));
    JGPM_CUDA_TRY(cudaStreamSynchronize(g->stream));
    if (!hbad && m > 0) {
      if ((rc = dalloc((int32_t**)&src.p, m, g->stream))) return rc;
      k_arc_src<<<grid_for((int64_t)n * 32), 256, 0, g->stream>>>(g->d_rowptr, n,
                                                                  (int32_t*)src.p);
      k_validate<<<grid_for(m), 256, 0, g->stream>>>(g->d_rowptr, g->d_col, (int32_t*)src.p, n,
                                                     m, (int*)bad.p);
      JGPM_CUDA_TRY(cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost,
                                    g->stream));
      JGPM_CUDA_TRY(cudaStreamSynchronize(g->stream));
    }
    if (hbad) {
      jgpm_set_error_(
          "jgpm_graph_from_csr: CSR must have rowptr[0]=0, rowptr[n]=m, nondecreasing row "
          "pointers, strictly increasing rows, ids in [0,n), no self-loops and both "
          "directions of every edge");
      return JGPM_EINVAL;
    }
  }
  return finish_sym(g);
}

int ensure_dag(jgpm_graph* g) {
  if (g->d_dag_rowptr) return JGPM_OK;
  cudaStream_t s = g->stream;
  const int64_t m = g->m;
  const int32_t n = g->n;
  int rc;
  if ((rc = dalloc(&g->d_dag_rowptr, (size_t)n + 1, g->stream))) return rc;
  DevBuf src(g->stream), keep(g->stream), pos(g->stream), tmp(g->stream);
  if ((rc = dalloc((int32_t**)&src.p, m, g->stream))) return rc;
  if ((rc = dalloc((int**)&keep.p, m, g->stream))) return rc;
  if ((rc = dalloc((int64_t**)&pos.p, m + 1, g->stream))) return rc;
  k_arc_src<<<grid_for((int64_t)n * 32), 256, 0, s>>>(g->d_rowptr, n, (int32_t*)src.p);
  k_orient_flags<<<grid_for(m), 256, 0, s>>>(g->d_rowptr, g->d_col, (int32_t*)src.p, m,
                                             (int*)keep.p);
  size_t tb = 0;
  JGPM_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tb, (int*)keep.p, (int64_t*)pos.p, m, s));
  if ((rc = dalloc((char**)&tmp.p, tb, g->stream))) return rc;
  JGPM_CUDA_TRY(cub::DeviceScan::ExclusiveSum(tmp.p, tb, (int*)keep.p, (int64_t*)pos.p, m, s));
  int64_t last_pos = 0;
  int last_keep = 0;
  if (m > 0) {
    JGPM_CUDA_TRY(cudaMemcpyAsync(&last_pos, (int64_t*)pos.p + m - 1, sizeof(int64_t),
                                  cudaMemcpyDeviceToHost, s));
    JGPM_CUDA_TRY(cudaMemcpyAsync(&last_keep, (int*)keep.p + m - 1, sizeof(int),
                                  cudaMemcpyDeviceToHost, s));
    JGPM_CUDA_TRY(cudaStreamSynchronize(s));
  }
  const int64_t total = last_pos + last_keep;
  if ((rc = dalloc(&g->d_dag_col, total, g->stream))) return rc;
  k_orient_scatter<<<grid_for(m), 256, 0, s>>>(g->d_col, (int*)keep.p, (int64_t*)pos.p, m,
                                               g->d_dag_col);
  k_dag_rowptr<<<grid_for((int64_t)n + 1), 256, 0, s>>>(g->d_rowptr, (int64_t*)pos.p, n, m,
                                                        total, g->d_dag_rowptr);
  JGPM_CUDA_TRY(cudaGetLastError());
  g->m_dag = total;
  DevBuf md(g->stream);
  if ((rc = dalloc((int**)&md.p, 1, g->stream))) return rc;
  JGPM_CUDA_TRY(cudaMemsetAsync(md.p, 0, sizeof(int), s));
  k_max_degree<<<grid_for(n), 256, 0, s>>>(g->d_dag_rowptr, n, (int*)md.p);
  int h = 0;
  JGPM_CUDA_TRY(cudaMemcpyAsync(&h, md.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  JGPM_CUDA_TRY(cudaStreamSynchronize(s));
  g->max_out_degree = h;
  return JGPM_OK;
}

// out[x] for x = 0..33, then thresholds 64, 128, 256, 512, 1024, 2048, 4096: the first index
// of the descending keys[0..n) whose key is <= the threshold.
__global__ void k_tier_bounds(const uint32_t* keys, int32_t n, int64_t* out) {
  const int t = threadIdx.x;
  if (t >= 41) return;
  const uint32_t big[7] = {64u, 128u, 256u, 512u, (uint32_t)kMidMaxDeg, 2048u,
                           (uint32_t)kWideMaxDeg};
  const uint32_t x = t < 34 ? (uint32_t)t : big[t - 34];
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (keys[mid] > x) lo = mid + 1;
    else hi = mid;
  }
  out[t] = lo;
}

int ensure_tiers(jgpm_graph* g, int min_deg) {
  int rc;
  if ((rc = ensure_dag(g))) return rc;
  // One root list serves every k: it keeps all roots with out-degree >= 2 and the kernels
  // take the prefix with d >= k-1 (deg_begin).
  (void)min_deg;
  min_deg = 2;
  if (g->tiers.d_roots && g->tiers.min_deg == min_deg) return JGPM_OK;
  if (g->tiers.d_roots) {
    gfree(g->tiers.d_roots, g->stream);
    g->tiers.d_roots = nullptr;
  }
  cudaStream_t s = g->stream;
  const int32_t n = g->n;
  DevBuf k0(g->stream), k1(g->stream), v1(g->stream), tmp(g->stream);
  if ((rc = dalloc((uint32_t**)&k0.p, n, g->stream))) return rc;
  if ((rc = dalloc((uint32_t**)&k1.p, n, g->stream))) return rc;
  if ((rc = dalloc((int32_t**)&v1.p, n, g->stream))) return rc;
  if ((rc = dalloc(&g->tiers.d_roots, n, g->stream))) return rc;
  k_root_keys<<<grid_for(n), 256, 0, s>>>(g->d_dag_rowptr, n, min_deg, (uint32_t*)k0.p,
                                          g->tiers.d_roots);
  // keys are out-degrees: sort only the bits the largest one needs
  const int key_bits = std::max(1, 32 - __builtin_clz((unsigned)std::max(1, g->max_out_degree)));
  size_t tb = 0;
  JGPM_CUDA_TRY(cub::DeviceRadixSort::SortPairsDescending(
      nullptr, tb, (uint32_t*)k0.p, (uint32_t*)k1.p, g->tiers.d_roots, (int32_t*)v1.p, n, 0,
      key_bits, s));
  if ((rc = dalloc((char**)&tmp.p, tb, g->stream))) return rc;
  JGPM_CUDA_TRY(cub::DeviceRadixSort::SortPairsDescending(
      tmp.p, tb, (uint32_t*)k0.p, (uint32_t*)k1.p, g->tiers.d_roots, (int32_t*)v1.p, n, 0,
      key_bits, s));
  // keys descending: [>kMidMaxDeg][33..kMidMaxDeg][min_deg..32][0...].  The tier boundaries
  // (first index with key <= x for each threshold x) are found on the device; only they come
  // back to the host.
  JGPM_CUDA_TRY(cudaMemcpyAsync(g->tiers.d_roots, v1.p, (size_t)n * sizeof(int32_t),
                                cudaMemcpyDeviceToDevice, s));
  constexpr int kNThr = 34 + 7;  // 0..33, then 64, 128, 256, 512, 1024, 2048, 4096
  DevBuf bnd(g->stream);
  if ((rc = dalloc((int64_t**)&bnd.p, kNThr, g->stream))) return rc;
  k_tier_bounds<<<1, 64, 0, s>>>((const uint32_t*)k1.p, n, (int64_t*)bnd.p);
  JGPM_CUDA_TRY(cudaGetLastError());
  int64_t hb[kNThr];
  JGPM_CUDA_TRY(cudaMemcpyAsync(hb, bnd.p, sizeof(hb), cudaMemcpyDeviceToHost, s));
  JGPM_CUDA_TRY(cudaStreamSynchronize(s));
  for (int x = 0; x < 34; ++x) g->tiers.deg_begin[x] = hb[x];
  g->tiers.small_end = hb[0];
  g->tiers.mid_end = hb[32];
  g->tiers.large_end = hb[34 + 4];   // d <= kMidMaxDeg
  g->tiers.wide_begin = hb[34 + 6];  // d <= kWideMaxDeg
  g->tiers.le_begin[0] = hb[32];
  g->tiers.le_begin[1] = hb[34 + 0];
  g->tiers.le_begin[2] = hb[34 + 1];
  g->tiers.le_begin[3] = hb[34 + 2];
  g->tiers.le_begin[4] = hb[34 + 3];
  g->tiers.le_begin[5] = hb[34 + 5];
  g->tiers.min_deg = min_deg;
  return JGPM_OK;
}

int ensure_control(jgpm_graph* g) {
  if (g->d_ctl) return JGPM_OK;
  int rc;
  if ((rc = dalloc(&g->d_ctl, 1, g->stream))) return rc;
  g->h_ctl = ctl_slot();
  if (!g->h_ctl) {
    jgpm_set_error_("pinned host allocation of a control block failed");
    return JGPM_ENOMEM;
  }
  memset(g->h_ctl, 0, sizeof(DevControl));
  return JGPM_OK;
}

int ensure_scratch(jgpm_graph* g, size_t bytes) {
  if (g->scratch_bytes >= bytes) return JGPM_OK;
  if (g->d_scratch) gfree(g->d_scratch, g->stream);
  g->d_scratch = nullptr;
  g->scratch_bytes = 0;
  int rc;
  if ((rc = dalloc((char**)&g->d_scratch, bytes, g->stream))) return rc;
  g->scratch_bytes = bytes;
  return JGPM_OK;
}

int ensure_aux(jgpm_graph* g, size_t bytes) {
  if (g->aux_bytes >= bytes) return JGPM_OK;
  if (g->d_aux) gfree(g->d_aux, g->stream);
  g->d_aux = nullptr;
  g->aux_bytes = 0;
  int rc;
  if ((rc = dalloc((char**)&g->d_aux, bytes, g->stream))) return rc;
  g->aux_bytes = bytes;
  return JGPM_OK;
}

void free_graph_device(jgpm_graph* g) {
  gfree(g->d_rowptr, g->stream);
  gfree(g->d_col, g->stream);
  gfree(g->d_dag_rowptr, g->stream);
  gfree(g->d_dag_col, g->stream);
  gfree(g->d_rank_rowptr, g->stream);
  gfree(g->d_rank_col, g->stream);
  gfree(g->d_c4_small, g->stream);
  gfree(g->d_c4_mid, g->stream);
  gfree(g->d_c4_large, g->stream);
  gfree(g->tiers.d_roots, g->stream);
  gfree(g->d_ctl, g->stream);
  gfree(g->d_scratch, g->stream);
  gfree(g->d_aux, g->stream);
  ctl_release(g->h_ctl);
  if (g->stream) cudaStreamDestroy(g->stream);
}

}  // namespace jgpm

// ------------------------------------------------------------------- rank relabelling
namespace jgpm {
namespace {

__global__ void k_rank_keys(const int64_t* rowptr, int32_t n, uint64_t* keys, int32_t* vals) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
    keys[v] = ((uint64_t)(rowptr[v + 1] - rowptr[v]) << 32) | (uint64_t)v;
    vals[v] = (int32_t)v;
  }
}

__global__ void k_invert(const int32_t* order, int32_t n, int32_t* rank) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride)
    rank[order[p]] = (int32_t)p;
}

__global__ void k_rank_arc_keys(const int32_t* src, const int32_t* col, const int32_t* rank,
                                int64_t m, int shift, uint64_t* keys) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m; k += stride)
    keys[k] = ((uint64_t)rank[src[k]] << shift) | (uint64_t)rank[col[k]];
}

__global__ void k_low_bits(const uint64_t* keys, int64_t m, uint64_t mask, int32_t* col) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m; k += stride)
    col[k] = (int32_t)(keys[k] & mask);
}

}  // namespace

// Relabels the symmetric CSR by rank -- position in (degree, id) order, the order the DAG
// orientation uses -- and sorts every row by rank, so "neighbours ranked below v" is a prefix
// of each row.  Built once per graph.
int ensure_rank_csr(jgpm_graph* g) {
  if (g->d_rank_rowptr) return JGPM_OK;
  cudaStream_t s = g->stream;
  const int32_t n = g->n;
  const int64_t m = g->m;
  const int shift = shift_for(n);
  int rc;
  DevBuf k0(g->stream), k1(g->stream), v0(g->stream), v1(g->stream), rank(g->stream), src(g->stream), tmp(g->stream);
  if ((rc = dalloc((uint64_t**)&k0.p, n, g->stream))) return rc;
  if ((rc = dalloc((uint64_t**)&k1.p, n, g->stream))) return rc;
  if ((rc = dalloc((int32_t**)&v0.p, n, g->stream))) return rc;
  if ((rc = dalloc((int32_t**)&v1.p, n, g->stream))) return rc;
  if ((rc = dalloc((int32_t**)&rank.p, n, g->stream))) return rc;
  k_rank_keys<<<grid_for(n), 256, 0, s>>>(g->d_rowptr, n, (uint64_t*)k0.p, (int32_t*)v0.p);
  size_t tb = 0;
  JGPM_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tb, (uint64_t*)k0.p, (uint64_t*)k1.p,
                                                (int32_t*)v0.p, (int32_t*)v1.p, n, 0, 64, s));
  if ((rc = dalloc((char**)&tmp.p, tb, g->stream))) return rc;
  JGPM_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp.p, tb, (uint64_t*)k0.p, (uint64_t*)k1.p,
                                                (int32_t*)v0.p, (int32_t*)v1.p, n, 0, 64, s));
  k_invert<<<grid_for(n), 256, 0, s>>>((int32_t*)v1.p, n, (int32_t*)rank.p);
  // arcs as (rank(u), rank(v)) keys, sorted
  DevBuf ak(g->stream), ak2(g->stream), tmp2(g->stream);
  if ((rc = dalloc((int32_t**)&src.p, m, g->stream))) return rc;
  if ((rc = dalloc((uint64_t**)&ak.p, m, g->stream))) return rc;
  if ((rc = dalloc((uint64_t**)&ak2.p, m, g->stream))) return rc;
  k_arc_src<<<grid_for((int64_t)n * 32), 256, 0, s>>>(g->d_rowptr, n, (int32_t*)src.p);
  k_rank_arc_keys<<<grid_for(m), 256, 0, s>>>((int32_t*)src.p, g->d_col, (int32_t*)rank.p, m,
                                              shift, (uint64_t*)ak.p);
  cub::DoubleBuffer<uint64_t> db((uint64_t*)ak.p, (uint64_t*)ak2.p);
  size_t tb2 = 0;
  JGPM_CUDA_TRY(cub::DeviceRadixSort::SortKeys(nullptr, tb2, db, m, 0, 2 * shift, s));
  if ((rc = dalloc((char**)&tmp2.p, tb2, g->stream))) return rc;
  JGPM_CUDA_TRY(cub::DeviceRadixSort::SortKeys(tmp2.p, tb2, db, m, 0, 2 * shift, s));
  if ((rc = dalloc(&g->d_rank_rowptr, (size_t)n + 1, g->stream))) return rc;
  if ((rc = dalloc(&g->d_rank_col, m, g->stream))) {
    gfree(g->d_rank_rowptr, g->stream);
    g->d_rank_rowptr = nullptr;
    return rc;
  }
  k_low_bits<<<grid_for(m), 256, 0, s>>>(db.Current(), m, (1ull << shift) - 1, g->d_rank_col);
  k_rowptr_from_keys<<<grid_for((int64_t)n + 1), 256, 0, s>>>(db.Current(), m, n, shift,
                                                              g->d_rank_rowptr);
  JGPM_CUDA_TRY(cudaGetLastError());
  JGPM_CUDA_TRY(cudaStreamSynchronize(s));
  return JGPM_OK;
}

}  // namespace jgpm

// ------------------------------------------------------------------- file I/O (host)
namespace jgpm {

// Reads the reference's on-disk CSR (common/graph.cc:26-46): prefix.meta.txt holds
// "n m vid_size eid_size vlabel_size elabel_size max_degree feat_len nvclasses neclasses".
int read_reference_files(const std::string& prefix, std::vector<int64_t>& rowptr,
                         std::vector<int32_t>& col, int32_t* n_out) {
  std::ifstream meta(prefix + ".meta.txt");
  if (!meta) {
    jgpm_set_error_("cannot open " + prefix + ".meta.txt");
    return JGPM_EIO;
  }
  int64_t n = 0, m = 0;
  int vid_size = 0, eid_size = 0;
  meta >> n >> m >> vid_size >> eid_size;
  if (!meta || n < 1 || m < 0 || vid_size != 4 || eid_size != 8 || n > INT32_MAX) {
    jgpm_set_error_(prefix + ".meta.txt: expected n, m, vid size 4, eid size 8");
    return JGPM_EIO;
  }
  rowptr.resize((size_t)n + 1);
  col.resize((size_t)m);
  std::ifstream fv(prefix + ".vertex.bin", std::ios::binary);
  std::ifstream fe(prefix + ".edge.bin", std::ios::binary);
  if (!fv || !fe) {
    jgpm_set_error_("cannot open " + prefix + ".vertex.bin / .edge.bin");
    return JGPM_EIO;
  }
  fv.read(reinterpret_cast<char*>(rowptr.data()), (std::streamsize)((n + 1) * 8));
  fe.read(reinterpret_cast<char*>(col.data()), (std::streamsize)(m * 4));
  if (!fv || (m > 0 && !fe)) {
    jgpm_set_error_(prefix + ": truncated .vertex.bin or .edge.bin");
    return JGPM_EIO;
  }
  *n_out = (int32_t)n;
  return JGPM_OK;
}

// Writes the reference's on-disk CSR as Graph::dump_binary does (common/graph.cc:727-753).
int write_reference_files(const std::string& prefix, const std::vector<int64_t>& rowptr,
                          const std::vector<int32_t>& col, int32_t n, int32_t max_degree) {
  std::ofstream fv(prefix + ".vertex.bin", std::ios::binary);
  std::ofstream fe(prefix + ".edge.bin", std::ios::binary);
  std::ofstream meta(prefix + ".meta.txt");
  if (!fv || !fe || !meta) {
    jgpm_set_error_("cannot write " + prefix + ".*");
    return JGPM_EIO;
  }
  fv.write(reinterpret_cast<const char*>(rowptr.data()), (std::streamsize)(rowptr.size() * 8));
  fe.write(reinterpret_cast<const char*>(col.data()), (std::streamsize)(col.size() * 4));
  meta << n << "\n" << col.size() << "\n4 8 1 2\n" << max_degree << "\n0\n0\n0\n";
  if (!fv || !fe || !meta) {
    jgpm_set_error_("short write to " + prefix + ".*");
    return JGPM_EIO;
  }
  return JGPM_OK;
}

}  // namespace jgpm

namespace jgpm {

// Frees the device arrays of a graph (CSR, DAG, tiers, scratch) and keeps a host copy of the
// symmetric CSR so the graph can be made resident again (served graph pool eviction).
int evict_graph(jgpm_graph* g, std::vector<int64_t>& h_rowptr, std::vector<int32_t>& h_col) {
  if (!g->d_rowptr) return JGPM_OK;
  if (h_rowptr.empty()) {
    h_rowptr.resize((size_t)g->n + 1);
    h_col.resize((size_t)g->m);
    JGPM_CUDA_TRY(cudaMemcpyAsync(h_rowptr.data(), g->d_rowptr, ((size_t)g->n + 1) * 8,
                                  cudaMemcpyDeviceToHost, g->stream));
    if (g->m)
      JGPM_CUDA_TRY(cudaMemcpyAsync(h_col.data(), g->d_col, (size_t)g->m * 4,
                                    cudaMemcpyDeviceToHost, g->stream));
  }
  JGPM_CUDA_TRY(cudaStreamSynchronize(g->stream));
  gfree(g->d_rowptr, g->stream);
  gfree(g->d_col, g->stream);
  gfree(g->d_dag_rowptr, g->stream);
  gfree(g->d_dag_col, g->stream);
  gfree(g->d_rank_rowptr, g->stream);
  gfree(g->d_rank_col, g->stream);
  gfree(g->d_c4_small, g->stream);
  gfree(g->d_c4_mid, g->stream);
  gfree(g->d_c4_large, g->stream);
  gfree(g->tiers.d_roots, g->stream);
  gfree(g->d_scratch, g->stream);
  gfree(g->d_aux, g->stream);
  g->d_aux = nullptr;
  g->aux_bytes = 0;
  g->d_rank_rowptr = nullptr;
  g->d_rank_col = nullptr;
  g->d_c4_small = nullptr;
  g->d_c4_mid = nullptr;
  g->d_c4_large = nullptr;
  g->c4_nsmall = -1;
  g->c4_nmid = 0;
  g->c4_nlarge = 0;
  g->c4_ndense = 0;
  g->c4_large_keys.clear();
  g->d_rowptr = nullptr;
  g->d_col = nullptr;
  g->d_dag_rowptr = nullptr;
  g->d_dag_col = nullptr;
  g->tiers = RootTiers();
  g->d_scratch = nullptr;
  g->scratch_bytes = 0;
  return JGPM_OK;
}

// Uploads an evicted graph again and rebuilds its DAG and root tiers.
int restore_graph(jgpm_graph* g, const std::vector<int64_t>& h_rowptr,
                  const std::vector<int32_t>& h_col) {
  if (g->d_rowptr) return JGPM_OK;
  int rc;
  if ((rc = upload_csr(g, h_rowptr.data(), h_col.data(), g->n, (int64_t)h_col.size(), 0)))
    return rc;
  if ((rc = ensure_dag(g))) return rc;
  return ensure_tiers(g, 2);
}

// Device bytes held by a resident graph's arrays.
uint64_t graph_device_bytes(const jgpm_graph* g) {
  if (!g->d_rowptr) return 0;
  uint64_t b = (uint64_t)(g->n + 1) * 8 + (uint64_t)g->m * 4;
  if (g->d_dag_rowptr) b += (uint64_t)(g->n + 1) * 8 + (uint64_t)g->m_dag * 4;
  if (g->tiers.d_roots) b += (uint64_t)g->n * 4;
  if (g->d_rank_rowptr) b += (uint64_t)(g->n + 1) * 8 + (uint64_t)g->m * 4;
  if (g->d_c4_small) b += (uint64_t)(g->c4_nsmall + g->c4_nmid + g->c4_nlarge) * 4 + 48;
  return b + g->scratch_bytes + g->aux_bytes;
}

}  // namespace jgpm
