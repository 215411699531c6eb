// Batched-kernel types shared by batch.cu (the kernel and its synchronous C-ABI) and
// server.cu (continuous batching on several streams).
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "jgpm_internal.h"

namespace jgpm {

enum BatchKind : int32_t {
  kJobClique = 0,
  kJobDiamond = 1,
  kJobC4 = 2,
};

enum TaskKind : int32_t {
  kTaskGroup4 = 0,
  kTaskGroup8 = 1,
  kTaskGroup16 = 2,
  kTaskGroup32 = 3,
  kTaskCtaRoot = 4,
  kTaskLargeRoot = 5,
  kTaskDiamond = 6,
  kTaskC4 = 7,
};

struct JobDesc {
  const eid_t* drow;  // DAG
  const vid_t* dcol;
  const eid_t* srow;  // symmetric
  const vid_t* scol;
  const vid_t* roots;  // root tiers (descending out-degree)
  int32_t n;
  int32_t kind;
  int32_t k;
  int32_t pad;
};

struct Task {
  int32_t job;
  int32_t kind;
  int64_t b, e;
};

// Growable device buffer.
struct DevArena {
  void* p = nullptr;
  size_t bytes = 0;
  int reserve(size_t want) {
    if (want <= bytes) return JGPM_OK;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    size_t sz = std::max<size_t>(want, 4096);
    if (cudaMalloc(&p, sz) != cudaSuccess) {
      cudaGetLastError();
      jgpm_set_error_("batch: device allocation failed");
      return JGPM_ENOMEM;
    }
    bytes = sz;
    return JGPM_OK;
  }
};

// Reusable per-device launch state of the batched kernel (task/job tables, counters,
// scratch).  One per server slot or per synchronous caller.
struct BatchCtx {
  int device = 0;
  DevArena jobs, tasks, counts, cursor, c4, lists;
  std::vector<JobDesc> h_jobs;
  std::vector<Task> h_tasks;
  int64_t n_c4 = 0;
  size_t c4_zeroed = 0;
  size_t c4_cap_bytes = (size_t)4 << 30;  // memory cap of the 4-cycle counter arrays
  ~BatchCtx() {
    for (DevArena* d : {&jobs, &tasks, &counts, &cursor, &c4, &lists})
      if (d->p) cudaFree(d->p);
  }
};

struct BatchJobIn {
  jgpm_graph* g;
  int kind;
  int k;
};

int parse_batch_pattern(const char* pattern, int* kind, int* k);
jgpm_tuning default_tuning();
int batch_enqueue(BatchCtx& c, const std::vector<BatchJobIn>& in, const jgpm_tuning& tu,
                  cudaStream_t s, uint64_t* h_counts, int* ntasks_out);

}  // namespace jgpm
