// extern "C" entry points of libjgpm (declared in include/jgpm.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "jgpm_internal.h"
#include "rmat.h"
#include "setops.cuh"

namespace {
thread_local std::string g_last_error;
thread_local int g_device = 0;
}  // namespace

void jgpm_set_error_(const std::string& msg) { g_last_error = msg; }

namespace jgpm {
int read_reference_files(const std::string& prefix, std::vector<int64_t>& rowptr,
                         std::vector<int32_t>& col, int32_t* n_out);
int write_reference_files(const std::string& prefix, const std::vector<int64_t>& rowptr,
                          const std::vector<int32_t>& col, int32_t n, int32_t max_degree);
int edges_build(jgpm_graph* g, const int32_t* src, const int32_t* dst, int64_t ne, int32_t n);
int launch_clique(jgpm_graph* g, int k, bool stats, int64_t root_begin, int64_t root_end,
                  cudaStream_t s);
int launch_level1_elements(jgpm_graph* g, cudaStream_t s);
int launch_clique_shard(jgpm_graph* g, int k, int shard, int nshards, cudaStream_t s);
}  // namespace jgpm

using namespace jgpm;

namespace {

int new_graph(jgpm_graph** out) {
  if (!out) {
    jgpm_set_error_("null output handle");
    return JGPM_EINVAL;
  }
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    jgpm_set_error_("no CUDA device");
    return JGPM_ENODEV;
  }
  jgpm_graph* g = new jgpm_graph;
  g->device = g_device < ndev ? g_device : 0;
  cudaError_t e = cudaSetDevice(g->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    jgpm_set_error_(std::string("stream create: ") + cudaGetErrorString(e));
    delete g;
    return JGPM_ECUDA;
  }
  *out = g;
  return JGPM_OK;
}

int fail_graph(jgpm_graph* g, int rc) {
  free_graph_device(g);
  delete g;
  return rc;
}

struct ScopedDevice {
  int prev = -1;
  explicit ScopedDevice(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~ScopedDevice() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

int clique_k_of(const std::string& p) {
  if (p == "P0" || p == "triangle" || p == "3-clique") return 3;
  if (p == "P13" || p == "4-clique") return 4;
  if (p == "P14" || p == "5-clique") return 5;
  if (p == "P15" || p == "6-clique") return 6;
  if (p == "P16" || p == "7-clique") return 7;
  if (p.rfind("k-clique:", 0) == 0) {
    int k = std::atoi(p.c_str() + 9);
    if (k >= 3 && k <= 8) return k;
    return -1;
  }
  return 0;
}

int reset_control(jgpm_graph* g, cudaStream_t s) {
  JGPM_CUDA_TRY(cudaMemsetAsync(g->d_ctl, 0, sizeof(DevControl), s));
  return JGPM_OK;
}

int read_control(jgpm_graph* g, cudaStream_t s) {
  JGPM_CUDA_TRY(cudaMemcpyAsync(g->h_ctl, g->d_ctl, sizeof(DevControl), cudaMemcpyDeviceToHost,
                                s));
  JGPM_CUDA_TRY(cudaStreamSynchronize(s));
  return JGPM_OK;
}

// k-clique count (k >= 3) with the bitmap kernels; rounds split the root list.
int count_clique(jgpm_graph* g, int k, int chunk_size, bool stats, uint64_t* out,
                 uint64_t* elements, double* ms) {
  int rc;
  if ((rc = ensure_dag(g))) return rc;
  if ((rc = ensure_tiers(g, k - 1))) return rc;
  if ((rc = ensure_control(g))) return rc;
  cudaStream_t s = g->stream;
  cudaEvent_t e0, e1;
  JGPM_CUDA_TRY(cudaEventCreate(&e0));
  JGPM_CUDA_TRY(cudaEventCreate(&e1));
  if ((rc = reset_control(g, s))) return rc;
  const int64_t nroots = g->tiers.deg_begin[k - 2];
  const int rounds = chunk_size > 1 ? chunk_size : 1;
  const int64_t per = (nroots + rounds - 1) / rounds;
  JGPM_CUDA_TRY(cudaEventRecord(e0, s));
  for (int r = 0; r < rounds; ++r) {
    const int64_t b = (int64_t)r * per, e = std::min(nroots, b + per);
    if (r > 0)
      JGPM_CUDA_TRY(cudaMemsetAsync(g->d_ctl->counter, 0, sizeof(g->d_ctl->counter), s));
    if (e > b && (rc = launch_clique(g, k, false, b, e, s))) return rc;
  }
  JGPM_CUDA_TRY(cudaEventRecord(e1, s));
  if ((rc = read_control(g, s))) return rc;
  float fms = 0.f;
  cudaEventElapsedTime(&fms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *out = g->h_ctl->count[0];
  if (ms) *ms = fms;
  if (stats) {
    const int timed_launches = g->launches;
    // Untimed accounting pass: all roots with out-degree >= 2 issue deeper plan levels.
    if ((rc = ensure_tiers(g, 2))) return rc;
    if ((rc = reset_control(g, s))) return rc;
    if ((rc = launch_clique(g, k, true, 0, g->tiers.small_end, s))) return rc;
    if ((rc = launch_level1_elements(g, s))) return rc;
    if ((rc = read_control(g, s))) return rc;
    if (g->h_ctl->count[0] != *out) {
      jgpm_set_error_("k-clique: accounting pass disagrees with the timed count");
      return JGPM_ECUDA;
    }
    if (elements) *elements = g->h_ctl->elements[0] + g->h_ctl->elements[1];
    g->launches = timed_launches;
  }
  return JGPM_OK;
}

}  // namespace

namespace jgpm {
int count_clique_public(jgpm_graph* g, int k, uint64_t* out, double* ms) {
  return count_clique(g, k, 1, false, out, nullptr, ms);
}
}  // namespace jgpm

extern "C" {

const char* jgpm_version(void) { return "jgpm-b200 1.0 (sm_100a)"; }

const char* jgpm_last_error(void) { return g_last_error.c_str(); }

int jgpm_device_count(int* n) {
  if (!n) return JGPM_EINVAL;
  int c = 0;
  if (cudaGetDeviceCount(&c) != cudaSuccess) {
    cudaGetLastError();
    c = 0;
  }
  *n = c;
  return JGPM_OK;
}

int jgpm_set_device(int device) {
  int n = 0;
  jgpm_device_count(&n);
  if (device < 0 || device >= n) {
    jgpm_set_error_("jgpm_set_device: no such device");
    return n == 0 ? JGPM_ENODEV : JGPM_EINVAL;
  }
  g_device = device;
  return JGPM_OK;
}

int jgpm_graph_load(const char* prefix, int orient_dag, jgpm_graph** g) {
  if (!prefix || !g) {
    jgpm_set_error_("jgpm_graph_load: null argument");
    return JGPM_EINVAL;
  }
  std::vector<int64_t> rowptr;
  std::vector<int32_t> col;
  int32_t n = 0;
  int rc = read_reference_files(prefix, rowptr, col, &n);
  if (rc) return rc;
  rc = jgpm_graph_from_csr(rowptr.data(), col.data(), n, (int64_t)col.size(), orient_dag, g);
  if (rc == JGPM_OK) (*g)->name = prefix;
  return rc;
}

int jgpm_graph_from_csr(const int64_t* rowptr, const int32_t* col, int32_t n, int64_t m,
                        int orient_dag, jgpm_graph** out) {
  jgpm_graph* g = nullptr;
  int rc = new_graph(&g);
  if (rc) return rc;
  ScopedDevice sd(g->device);
  if ((rc = upload_csr(g, rowptr, col, n, m, 1))) return fail_graph(g, rc);
  if (orient_dag && (rc = ensure_dag(g))) return fail_graph(g, rc);
  *out = g;
  return JGPM_OK;
}

int jgpm_graph_from_edges(const int32_t* src, const int32_t* dst, int64_t num_edges, int32_t n,
                          int orient_dag, jgpm_graph** out) {
  if ((!src || !dst) && num_edges > 0) {
    jgpm_set_error_("jgpm_graph_from_edges: null edge arrays");
    return JGPM_EINVAL;
  }
  jgpm_graph* g = nullptr;
  int rc = new_graph(&g);
  if (rc) return rc;
  ScopedDevice sd(g->device);
  if ((rc = edges_build(g, src, dst, num_edges, n))) return fail_graph(g, rc);
  if (orient_dag && (rc = ensure_dag(g))) return fail_graph(g, rc);
  *out = g;
  return JGPM_OK;
}

int jgpm_graph_rmat(int64_t n, int64_t num_edges, double a, double b, double c, uint64_t seed,
                    int orient_dag, jgpm_graph** out) {
  jgpm_graph* g = nullptr;
  int rc = new_graph(&g);
  if (rc) return rc;
  ScopedDevice sd(g->device);
  if ((rc = rmat_build(g, n, num_edges, a, b, c, seed))) return fail_graph(g, rc);
  if (orient_dag && (rc = ensure_dag(g))) return fail_graph(g, rc);
  *out = g;
  return JGPM_OK;
}

int jgpm_rmat_edges(int64_t n, int64_t num_edges, double a, double b, double c, uint64_t seed,
                    int32_t* src, int32_t* dst, int64_t* out_count) {
  if (n < 2 || n > INT32_MAX - 1 || num_edges < 0 || !out_count || (num_edges > 0 && (!src || !dst)) ||
      a < 0 || b < 0 || c < 0 || a + b + c > 1.0 + 1e-12) {
    jgpm_set_error_("jgpm_rmat_edges: bad parameters");
    return JGPM_EINVAL;
  }
  RmatParams p = rmat_params(n, num_edges, a, b, c, seed);
  int64_t k = 0;
  for (int64_t i = 0; i < num_edges; ++i) {
    int32_t u, v;
    if (rmat_edge(p, (uint64_t)i, &u, &v)) {
      src[k] = u;
      dst[k] = v;
      ++k;
    }
  }
  *out_count = k;
  return JGPM_OK;
}

int jgpm_graph_get_info(const jgpm_graph* g, jgpm_graph_info* info) {
  if (!g || !info) {
    jgpm_set_error_("jgpm_graph_get_info: null argument");
    return JGPM_EINVAL;
  }
  info->num_vertices = g->n;
  info->num_arcs = g->m;
  info->max_degree = g->max_degree;
  info->num_dag_arcs = g->d_dag_rowptr ? g->m_dag : 0;
  info->max_out_degree = g->d_dag_rowptr ? g->max_out_degree : 0;
  info->device = g->device;
  uint64_t bytes = (uint64_t)(g->n + 1) * 8 + (uint64_t)g->m * 4;
  if (g->d_dag_rowptr) bytes += (uint64_t)(g->n + 1) * 8 + (uint64_t)g->m_dag * 4;
  if (g->tiers.d_roots) bytes += (uint64_t)g->n * 4;
  bytes += g->scratch_bytes;
  info->device_bytes = bytes;
  return JGPM_OK;
}

int jgpm_graph_copy_csr(jgpm_graph* g, int dag, int64_t* rowptr, int32_t* col) {
  if (!g || !rowptr || !col) {
    jgpm_set_error_("jgpm_graph_copy_csr: null argument");
    return JGPM_EINVAL;
  }
  ScopedDevice sd(g->device);
  int rc;
  if (dag && (rc = ensure_dag(g))) return rc;
  const int64_t* rp = dag ? g->d_dag_rowptr : g->d_rowptr;
  const int32_t* cp = dag ? g->d_dag_col : g->d_col;
  const int64_t m = dag ? g->m_dag : g->m;
  JGPM_CUDA_TRY(cudaMemcpyAsync(rowptr, rp, ((size_t)g->n + 1) * 8, cudaMemcpyDeviceToHost,
                                g->stream));
  if (m > 0)
    JGPM_CUDA_TRY(cudaMemcpyAsync(col, cp, (size_t)m * 4, cudaMemcpyDeviceToHost, g->stream));
  JGPM_CUDA_TRY(cudaStreamSynchronize(g->stream));
  return JGPM_OK;
}

int jgpm_graph_save(jgpm_graph* g, const char* prefix, int dag) {
  if (!g || !prefix) {
    jgpm_set_error_("jgpm_graph_save: null argument");
    return JGPM_EINVAL;
  }
  ScopedDevice sd(g->device);
  int rc;
  if (dag && (rc = ensure_dag(g))) return rc;
  std::vector<int64_t> rowptr((size_t)g->n + 1);
  std::vector<int32_t> col((size_t)(dag ? g->m_dag : g->m));
  if ((rc = jgpm_graph_copy_csr(g, dag, rowptr.data(), col.data()))) return rc;
  return write_reference_files(prefix, rowptr, col, g->n,
                               dag ? g->max_out_degree : g->max_degree);
}

void jgpm_graph_free(jgpm_graph* g) {
  if (!g) return;
  ScopedDevice sd(g->device);
  if (g->stream) cudaStreamSynchronize(g->stream);
  free_graph_device(g);
  delete g;
}

int jgpm_count_ex(jgpm_graph* g, const char* pattern, int induced, int chunk_size,
                  unsigned flags, uint64_t* out, jgpm_stats* st) {
  if (!g || !pattern || !out) {
    jgpm_set_error_("jgpm_count: null argument");
    return JGPM_EINVAL;
  }
  ScopedDevice sd(g->device);
  const std::string p(pattern);
  const bool stats = (flags & JGPM_COUNT_STATS) != 0;
  uint64_t count = 0, elems = 0;
  double ms = 0.0;
  int method = 0;
  int rc;
  g->launches = 0;
  const int k = clique_k_of(p);
  if (k < 0) {
    jgpm_set_error_("jgpm_count: k-clique needs 3 <= k <= 8");
    return JGPM_EPATTERN;
  }
  if (k > 0 && !(flags & JGPM_COUNT_FORCE_PLAN)) {
    rc = count_clique(g, k, chunk_size, stats, &count, &elems, &ms);
    method = JGPM_METHOD_BITMAP_CLIQUE;
  } else {
    const int id = plan_id_of(p, induced);
    if (id < 0) {
      jgpm_set_error_("jgpm_count: unknown pattern '" + p + "'" +
                      (induced ? " (vertex-induced)" : ""));
      return JGPM_EPATTERN;
    }
    rc = count_plan_impl(g, id, chunk_size, flags, stats, &count, &elems, &ms, &method);
  }
  if (rc) return rc;
  *out = count;
  g->last_kernel_ms = ms;
  if (st) {
    st->count = count;
    st->setop_elements = stats ? elems : 0;
    st->kernel_ms = ms;
    st->rounds = chunk_size > 1 ? chunk_size : 1;
    st->method = method;
    st->launches = g->launches;
    st->reserved = 0;
  }
  return JGPM_OK;
}

int jgpm_graph_set_tuning(jgpm_graph* g, const jgpm_tuning* t) {
  if (!g || !t) {
    jgpm_set_error_("jgpm_graph_set_tuning: null argument");
    return JGPM_EINVAL;
  }
  if (t->min_group != 4 && t->min_group != 8 && t->min_group != 16 && t->min_group != 32) {
    jgpm_set_error_("jgpm_graph_set_tuning: min_group must be 4, 8, 16 or 32");
    return JGPM_EINVAL;
  }
  if (t->split_degree != 32 && t->split_degree != 64 && t->split_degree != 128) {
    jgpm_set_error_("jgpm_graph_set_tuning: split_degree must be 32, 64 or 128");
    return JGPM_EINVAL;
  }
  g->tune_min_group = t->min_group;
  g->tune_split = t->split_degree;
  return JGPM_OK;
}

int jgpm_graph_stream(jgpm_graph* g, void** stream) {
  if (!g || !stream) {
    jgpm_set_error_("jgpm_graph_stream: null argument");
    return JGPM_EINVAL;
  }
  *stream = (void*)g->stream;
  return JGPM_OK;
}

int jgpm_count(jgpm_graph* g, const char* pattern, int induced, int chunk_size, uint64_t* out,
               jgpm_stats* st) {
  return jgpm_count_ex(g, pattern, induced, chunk_size, 0u, out, st);
}

int jgpm_count_roots(jgpm_graph* g, const char* pattern, int induced, int64_t begin,
                     int64_t end, int64_t stride, uint64_t* out, jgpm_stats* st) {
  if (!g || !pattern || !out) {
    jgpm_set_error_("jgpm_count_roots: null argument");
    return JGPM_EINVAL;
  }
  if (begin < 0 || stride < 1 || (end >= 0 && end < begin)) {
    jgpm_set_error_("jgpm_count_roots: need 0 <= begin <= end (or end < 0) and stride >= 1");
    return JGPM_EINVAL;
  }
  ScopedDevice sd(g->device);
  const int id = literal_plan_id(pattern, induced);
  if (id < 0) {
    jgpm_set_error_(std::string("jgpm_count_roots: no nested-loop plan for '") + pattern + "'" +
                    (induced ? " (vertex-induced)" : ""));
    return JGPM_EPATTERN;
  }
  const int64_t m = plan_root_arcs(g, id);
  if (m < 0) return JGPM_ECUDA;  // DAG build failed (message set)
  if (end > m) {
    jgpm_set_error_("jgpm_count_roots: end is past the last root arc (" + std::to_string(m) +
                    ")");
    return JGPM_EINVAL;
  }
  g->launches = 0;
  uint64_t count = 0;
  double ms = 0.0;
  int rc = count_roots_impl(g, id, begin, end < 0 ? m : end, stride, &count, &ms);
  if (rc) return rc;
  *out = count;
  if (st) {
    memset(st, 0, sizeof(*st));
    st->count = count;
    st->kernel_ms = ms;
    st->rounds = 1;
    st->method = JGPM_METHOD_PLAN;
    st->launches = g->launches;
  }
  return JGPM_OK;
}

int jgpm_count_shard(jgpm_graph* g, const char* pattern, int induced, int32_t shard,
                     int32_t nshards, uint64_t* out, jgpm_stats* st) {
  if (!g || !pattern || !out) {
    jgpm_set_error_("jgpm_count_shard: null argument");
    return JGPM_EINVAL;
  }
  if (nshards < 1 || shard < 0 || shard >= nshards) {
    jgpm_set_error_("jgpm_count_shard: need 0 <= shard < nshards");
    return JGPM_EINVAL;
  }
  ScopedDevice sd(g->device);
  const std::string p(pattern);
  const int k = clique_k_of(p);
  if (k < 0) {
    jgpm_set_error_("jgpm_count_shard: k-clique needs 3 <= k <= 8");
    return JGPM_EPATTERN;
  }
  g->launches = 0;
  uint64_t count = 0;
  double ms = 0.0;
  int method = 0;
  int rc;
  if (k > 0) {
    if ((rc = ensure_dag(g))) return rc;
    if ((rc = ensure_tiers(g, k - 1))) return rc;
    if ((rc = ensure_control(g))) return rc;
    cudaStream_t s = g->stream;
    cudaEvent_t e0, e1;
    JGPM_CUDA_TRY(cudaEventCreate(&e0));
    JGPM_CUDA_TRY(cudaEventCreate(&e1));
    if ((rc = reset_control(g, s))) return rc;
    JGPM_CUDA_TRY(cudaEventRecord(e0, s));
    if ((rc = launch_clique_shard(g, k, shard, nshards, s))) return rc;
    JGPM_CUDA_TRY(cudaEventRecord(e1, s));
    if ((rc = read_control(g, s))) return rc;
    float fms = 0.f;
    cudaEventElapsedTime(&fms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    count = g->h_ctl->count[0];
    ms = fms;
    method = JGPM_METHOD_BITMAP_CLIQUE;
  } else {
    const int id = literal_plan_id(p, induced);
    if (id < 0) {
      jgpm_set_error_("jgpm_count_shard: no nested-loop plan for '" + p + "'" +
                      (induced ? " (vertex-induced)" : ""));
      return JGPM_EPATTERN;
    }
    const int64_t m = plan_root_arcs(g, id);
    if (m < 0) return JGPM_ECUDA;
    if ((rc = count_roots_impl(g, id, shard, m, nshards, &count, &ms))) return rc;
    method = JGPM_METHOD_PLAN;
  }
  *out = count;
  if (st) {
    memset(st, 0, sizeof(*st));
    st->count = count;
    st->kernel_ms = ms;
    st->rounds = 1;
    st->method = method;
    st->launches = g->launches;
  }
  return JGPM_OK;
}

int jgpm_census4(jgpm_graph* g, uint64_t out[6], jgpm_stats* st) {
  if (!g || !out) {
    jgpm_set_error_("jgpm_census4: null argument");
    return JGPM_EINVAL;
  }
  ScopedDevice sd(g->device);
  double ms = 0.0;
  g->launches = 0;
  int rc = count_census4(g, out, &ms);
  if (rc) return rc;
  if (st) {
    memset(st, 0, sizeof(*st));
    st->kernel_ms = ms;
    st->method = JGPM_METHOD_CENSUS;
    st->rounds = 1;
    st->launches = g->launches;
  }
  return JGPM_OK;
}

}  // extern "C"
