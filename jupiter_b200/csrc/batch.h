// Batched-kernel types shared by batch.cu (the kernel and its synchronous C-ABI) and
// server.cu (continuous batching on several streams).
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "jgpm_internal.h"

namespace jgpm {

enum BatchKind : int32_t {
  kJobClique = 0,
  kJobDiamond = 1,
  kJobC4 = 2,
  kJobIndTT = 3,  // vertex-induced tailed triangle (k = 4 tasks in TT mode)
};

enum TaskKind : int32_t {
  kTaskGroup4 = 0,     // roots [b, e) of out-degree <= 4 .. 32, one per lane group
  kTaskGroup8 = 1,
  kTaskGroup16 = 2,
  kTaskGroup32 = 3,
  kTaskWarpRoots = 4,  // roots [b, e) of out-degree 32 < d <= split, one per warp
  kTaskCtaRoot = 5,    // root b, max(split, 256) < d <= kBatchCtaMaxDeg, the whole CTA, masks
                       // of up to 16 words in registers
  kTaskLargeRoot = 6,  // root b, d > kBatchWideMaxDeg, warps take its arcs (edge-rooted lists)
  kTaskC4Small = 7,    // small 4-cycle apexes [b, e) of the job's list, one per warp
  kTaskC4Large = 8,    // large 4-cycle apexes [b, e) of the job's list (k_batch_c4_large)
  kTaskC4Mid = 9,      // mid 4-cycle apexes [b, e) of the job's list, one after another per CTA
  kTaskWideRoot = 10,  // root b, kBatchCtaMaxDeg < d <= kBatchWideMaxDeg, the whole CTA with
                       // its bitmap rows in global scratch
  kTaskCtaRoot8 = 11,  // root b, split < d <= 256, the whole CTA, masks of up to 8 words in
                       // registers
};

// Out-degree limits of the batched root tasks: the CTA bitmap of a root of out-degree d takes
// about 20 d + d^2 / 8 bytes; up to kBatchCtaMaxDeg all of it is in shared memory, up to
// kBatchWideMaxDeg the d^2 / 8 bytes of rows go to global scratch, above that the root runs on
// edge-rooted lists.
constexpr int kBatchCtaMaxDeg = 512;
constexpr int kBatchWideMaxDeg = 2048;

struct JobDesc {
  const eid_t* drow;    // DAG (cliques, diamond)
  const vid_t* dcol;
  const eid_t* rrow;    // rank-relabelled symmetric CSR (4-cycle)
  const vid_t* rcol;
  const vid_t* roots;   // root tiers (descending out-degree), or the small 4-cycle apexes
  const vid_t* apexes;  // large 4-cycle apexes (descending wedge bound), then their cuts
  const vid_t* mid;     // mid 4-cycle apexes
  uint32_t* tri;        // diamond, tailed triangle: per-arc triangle counters (zero at launch)
  const eid_t* srow;    // tailed triangle: symmetric row pointers (degrees)
  int32_t n;
  int32_t kind;
  int32_t k;
  int32_t nlarge;       // large 4-cycle apexes
};

struct Task {
  int32_t job;
  int32_t kind;
  int32_t b, e;  // index range in the job's root or apex list
};

inline Task make_task(int job, int kind, int64_t b, int64_t e) {
  return Task{(int32_t)job, (int32_t)kind, (int32_t)b, (int32_t)e};
}

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

// Pinned host copy of a batch's task table, from which the device copy is made.  `done`
// marks the end of the last copy out of it: a new batch waits for it before writing.
struct PinnedTasks {
  Task* p = nullptr;
  size_t cap = 0, n = 0;
  cudaEvent_t done = nullptr;
  bool pending = false;
  void wait() {
    if (pending) cudaEventSynchronize(done);
    pending = false;
  }
  int reserve(size_t want) {
    if (want <= cap) return JGPM_OK;
    wait();
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    const size_t sz = std::max<size_t>(want + want / 4, (size_t)1 << 16);
    if (cudaHostAlloc((void**)&p, sz * sizeof(Task), cudaHostAllocDefault) != cudaSuccess) {
      p = nullptr;
      cudaGetLastError();
      jgpm_set_error_("batch: pinned host allocation failed");
      return JGPM_ENOMEM;
    }
    cap = sz;
    return JGPM_OK;
  }
  int record(cudaStream_t s) {
    if (!done && cudaEventCreateWithFlags(&done, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      jgpm_set_error_("batch: event creation failed");
      return JGPM_ECUDA;
    }
    if (cudaEventRecord(done, s) != cudaSuccess) {
      jgpm_set_error_("batch: event record failed");
      return JGPM_ECUDA;
    }
    pending = true;
    return JGPM_OK;
  }
  ~PinnedTasks() {
    wait();
    if (p) cudaFreeHost(p);
    if (done) cudaEventDestroy(done);
  }
};

// Reusable per-device launch state of the batched kernel (task/job tables, counters,
// scratch).  One per server slot or per synchronous caller.
// Pinned host staging reused across batches (written only after the previous batch of the
// same context has finished).
struct PinnedBytes {
  void* p = nullptr;
  size_t cap = 0;
  int reserve(size_t want) {
    if (want <= cap) return JGPM_OK;
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    const size_t sz = std::max<size_t>(want + want / 4, 4096);
    if (cudaHostAlloc(&p, sz, cudaHostAllocDefault) != cudaSuccess) {
      p = nullptr;
      cudaGetLastError();
      jgpm_set_error_("batch: pinned host allocation failed");
      return JGPM_ENOMEM;
    }
    cap = sz;
    return JGPM_OK;
  }
  ~PinnedBytes() {
    if (p) cudaFreeHost(p);
  }
};

// Everything the stream operations of one batch need, as plain data: two batches with equal
// plans (bytewise) issue identical operations, so a captured CUDA graph can be replayed.
struct LaunchPlan {
  void* d_jobs;
  const void* h_jobs;
  size_t jobs_bytes;
  void* d_tasks;
  const void* h_tasks;
  size_t tasks_bytes;
  void* d_c4_tasks;
  const void* h_c4_tasks;
  size_t c4_tasks_bytes;
  void* d_tri;
  size_t tri_bytes;
  void* d_counts;
  size_t counts_bytes;
  void* d_cursor;
  void* d_c4_zero;
  size_t c4_zero_bytes;
  int c4_kernel;  // 0 none, else the slab form's threads
  int c4_ctas;
  size_t c4_smem;
  unsigned char c4_args[128];
  int main_grid;
  size_t main_smem;
  int groups_grid;
  unsigned char args[128];
  void* h_counts;
  size_t d2h_bytes;
};

struct BatchCtx {
  int device = 0;
  PinnedBytes h_jobs_pin, h_c4_pin, h_counts_pin;
  cudaGraphExec_t exec = nullptr;  // the captured launches of `plan`
  LaunchPlan plan;
  bool have_plan = false;
  DevArena jobs, tasks, counts, cursor, c4, c4t, lists, tri, rows, c4_tasks;
  std::vector<JobDesc> h_jobs;
  PinnedTasks h_tasks;           // the main queue
  std::vector<Task> h_c4_tasks;  // large 4-cycle apexes, by job, heaviest first
  std::vector<Task> cls[6];      // per-class task lists while building (capacity kept)
  int64_t nmain = 0;             // tasks of k_batch; the lane-group tasks follow them
  std::vector<size_t> tri_off;  // diamond jobs: offset of the job's counters in `tri`
  size_t c4_zeroed = 0;
  size_t c4_cap_bytes = (size_t)4 << 30;  // memory cap of the 4-cycle counter arrays
  ~BatchCtx() {
    if (exec) cudaGraphExecDestroy(exec);
    for (DevArena* d : {&jobs, &tasks, &counts, &cursor, &c4, &c4t, &lists, &tri, &rows,
                        &c4_tasks})
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
                  cudaStream_t s, uint64_t* h_counts, int* ntasks_out,
                  int* launches_out = nullptr);

}  // namespace jgpm
