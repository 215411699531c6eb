// Internal declarations shared by the CUDA translation units of libjgpm.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>

#include "../../include/jgpm.h"

namespace jgpm {

typedef int32_t vid_t;
typedef int64_t eid_t;
typedef unsigned long long acc_t;

// Device view of a CSR: row pointers (n+1, int64) and sorted neighbour lists (int32).
struct DevCsr {
  vid_t n;
  eid_t m;
  const eid_t* rowptr;
  const vid_t* col;
};

// Roots of a clique count (vertices with DAG out-degree >= min_deg), sorted by out-degree
// descending, so the array holds three tiers back to back:
//   large  [0, large_end)          d > kMidMaxDeg
//   mid    [large_end, mid_end)    32 < d <= kMidMaxDeg
//   small  [mid_end, small_end)    min_deg <= d <= 32
constexpr int kMidMaxDeg = 1024;
// Roots of out-degree kMidMaxDeg < d <= kWideMaxDeg still run on local bitmaps, with the
// bitmap rows in global scratch; larger ones run on edge-rooted lists.
constexpr int kWideMaxDeg = 4096;

//   deg_begin[x] = first index whose out-degree is <= x (0 <= x <= 33), so the roots with
//   d >= k-1 are the prefix [0, deg_begin[k-2]).
struct RootTiers {
  vid_t* d_roots = nullptr;
  int64_t large_end = 0, mid_end = 0, small_end = 0;
  int64_t deg_begin[34] = {0};
  // first index with out-degree <= 32, 64, 128, 256, 512, 2048
  int64_t le_begin[6] = {0, 0, 0, 0, 0, 0};
  int64_t wide_begin = 0;  // first index with out-degree <= kWideMaxDeg
  int min_deg = -1;  // smallest out-degree kept
};

struct jgpm_graph_impl;

// Per-launch device control block: work counters and results.  No kernel has an error to
// report: capacities are sized on the host before each launch and no kernel waits.
struct DevControl {
  unsigned long long counter[12]; // work-stealing cursors
  unsigned long long count[4];    // pattern results
  unsigned long long elements[4]; // set-op elements (stats launches)
  int pad[8];
};

std::string cuda_error_string(cudaError_t e);

}  // namespace jgpm

// The opaque graph handle of the C-ABI.
struct jgpm_graph {
  int device = 0;
  cudaStream_t stream = nullptr;
  int32_t n = 0;
  // symmetric CSR
  int64_t m = 0;
  int64_t* d_rowptr = nullptr;
  int32_t* d_col = nullptr;
  int32_t max_degree = 0;
  // degree-oriented DAG (built on demand)
  int64_t m_dag = 0;
  int64_t* d_dag_rowptr = nullptr;
  int32_t* d_dag_col = nullptr;
  // rank-relabelled symmetric CSR (vertex ids replaced by their (degree, id) rank, rows sorted
  // by rank), built on demand for the 4-cycle wedge count
  int64_t* d_rank_rowptr = nullptr;
  int32_t* d_rank_col = nullptr;
  // 4-cycle apexes of the rank CSR by wedge bound (built on demand): one-warp, one-CTA
  // hash and large (slab or dense counter) classes, the last sorted by descending bound
  int32_t* d_c4_small = nullptr;
  int32_t* d_c4_mid = nullptr;
  int32_t* d_c4_large = nullptr;  // c4_nlarge apexes, then the cut of each
  int64_t c4_nsmall = -1;  // -1 = not built
  int64_t c4_nmid = 0;
  int64_t c4_nlarge = 0;
  int64_t c4_ndense = 0;   // large apexes that count in dense arrays (c4_dense_apex)
  std::vector<uint64_t> c4_large_keys;  // host copy: wedge bound of each large apex, descending
  int32_t max_out_degree = 0;
  jgpm::RootTiers tiers;
  // per-graph reusable launch state
  jgpm::DevControl* d_ctl = nullptr;
  jgpm::DevControl* h_ctl = nullptr;  // pinned mirror
  void* d_scratch = nullptr;          // per-CTA scratch for heavy roots
  size_t scratch_bytes = 0;
  void* d_aux = nullptr;              // per-arc counters (edge triangles, diamond pairs)
  size_t aux_bytes = 0;
  // statistics of the last count
  double last_kernel_ms = 0.0;
  int launches = 0;  // kernels launched since the counting call began
  int tune_min_group = 4;  // narrowest lane group for the d <= 32 roots (4, 8, 16 or 32)
  int tune_split = 128;    // roots with 32 < d <= tune_split run one per warp, above per CTA
  std::string name;
};

#define JGPM_CUDA_TRY(expr)                                   \
  do {                                                        \
    cudaError_t _e = (expr);                                  \
    if (_e != cudaSuccess) {                                  \
      jgpm_set_error_(std::string(#expr) + ": " + cudaGetErrorString(_e)); \
      return (_e == cudaErrorMemoryAllocation) ? JGPM_ENOMEM : JGPM_ECUDA; \
    }                                                         \
  } while (0)

void jgpm_set_error_(const std::string& msg);

namespace jgpm {
// Launches `kern`; with pdl, with programmatic stream serialization, so that it may start
// while the previous kernel of the stream drains (the kernels pair pdl_open / pdl_close).
template <typename... Args>
cudaError_t launch_pdl(bool pdl, void (*kern)(Args...), int grid, int block, size_t smem,
                       cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kern, args...);
}

// graph_build.cu
// Device memory of graphs and their temporaries: a per-device stream-ordered pool that keeps
// freed memory for reuse (freed memory is reused in the order of the freeing stream), so a
// graph's life cycle does not pay cudaMalloc / cudaFree.  gfree(nullptr) does nothing.
int gmalloc(void** p, size_t bytes, cudaStream_t s);
void gfree(void* p, cudaStream_t s);
int build_from_edges_device(jgpm_graph* g, int32_t n, int64_t* d_keys, int64_t nkeys_valid_cap);
int rmat_build(jgpm_graph* g, int64_t n, int64_t num_edges, double a, double b, double c,
               uint64_t seed);
int upload_csr(jgpm_graph* g, const int64_t* rowptr, const int32_t* col, int32_t n, int64_t m,
               int validate);
int ensure_dag(jgpm_graph* g);
int ensure_rank_csr(jgpm_graph* g);
// c4.cu: apex classes of the 4-cycle count (needs the rank CSR)
int ensure_c4_apexes(jgpm_graph* g);
int count_c4_wedge(jgpm_graph* g, uint64_t* out, double* ms);
int ensure_tiers(jgpm_graph* g, int min_deg);
int ensure_control(jgpm_graph* g);
int ensure_scratch(jgpm_graph* g, size_t bytes);
int ensure_aux(jgpm_graph* g, size_t bytes);
void free_graph_device(jgpm_graph* g);
int device_sm_count(int device);
// Raises the dynamic shared-memory limit of kernel `func` on the current device to at least
// `bytes`, never lowering it.  The limit is process-wide state and several host threads launch
// the same kernels with different sizes, so it only grows (under a lock).
int raise_smem_limit(const void* func, size_t bytes);
int evict_graph(jgpm_graph* g, std::vector<int64_t>& h_rowptr, std::vector<int32_t>& h_col);
int restore_graph(jgpm_graph* g, const std::vector<int64_t>& h_rowptr,
                  const std::vector<int32_t>& h_col);
uint64_t graph_device_bytes(const jgpm_graph* g);
// k-clique count through the bitmap kernels (capi.cu)
int count_clique_public(jgpm_graph* g, int k, uint64_t* out, double* ms);
// non-clique dispatch (plans.cu); *method receives a JGPM_METHOD_* code
int count_plan_impl(jgpm_graph* g, int id, int chunk_size, unsigned flags, bool stats,
                    uint64_t* out, uint64_t* elements, double* ms, int* method);
int plan_id_of(const std::string& name, int induced);
bool plan_uses_dag(int plan_id);
// literal plan over sampled root arcs (plans.cu)
int literal_plan_id(const std::string& name, int induced);
int count_roots_impl(jgpm_graph* g, int id, int64_t begin, int64_t end, int64_t stride,
                     uint64_t* out, double* ms);
int64_t plan_root_arcs(jgpm_graph* g, int id);  // CSR slots of the plan's graph (-1: error)
uint64_t count_scratch_bytes(const jgpm_graph* g, const std::string& pattern, int induced);
int count_census4(jgpm_graph* g, uint64_t out[6], double* ms);
}  // namespace jgpm
