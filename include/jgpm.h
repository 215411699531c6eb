/*
 * jgpm.h -- C-ABI of libjgpm, the B200 subgraph-pattern counting library.
 *
 * Plain C types only: pointers, sizes and status codes; no CUDA or torch types cross this
 * boundary.  Every entry point returns JGPM_OK (0) or a negative JGPM_E* status and never
 * calls exit(); jgpm_last_error() gives the message of the calling thread's last failure.
 * The library owns the device memory it allocates; callers own their host arrays.  A graph
 * handle may be used by one host thread at a time.
 *
 * Reference interfaces replaced (paths inside the AnySparse/Jupiter tree) are cited per entry
 * point.  The reference exposes no plugin API or FFI of its own; its operator surface is
 * the CLI `jupiter_gpm <graph_prefix> <pattern> [rounds]` (src/main.cc:7-47), the solver
 * SubgraphSolver(Graph&, uint64_t&, argc, argv, MPI_Comm&, rank, nranks)
 * (src/jupiter_gpm.cu:27), the loader Graph(prefix, use_dag) (include/graph.h:41-42) and
 * the device set-operation templates (include/set_intersect.cuh, include/set_difference.cuh).
 */
#ifndef JGPM_H_
#define JGPM_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------------------- */
#define JGPM_OK 0
#define JGPM_EINVAL (-1)     /* bad argument or malformed graph */
#define JGPM_ENOMEM (-2)     /* device or host allocation failed */
#define JGPM_ECUDA (-3)      /* CUDA runtime error */
#define JGPM_EIO (-4)        /* graph file missing or unreadable */
#define JGPM_EPATTERN (-5)   /* unknown pattern name, or pattern/induced combination */
#define JGPM_ETIMEDOUT (-6)  /* a bounded device wait gave up */
#define JGPM_EOVERFLOW (-7)  /* a count does not fit in uint64 */
#define JGPM_ENODEV (-8)     /* no CUDA device */
#define JGPM_EBUSY (-9)      /* the server has no free slot */
#define JGPM_ECAPACITY (-10) /* a per-root list exceeded a fixed capacity */
#define JGPM_EADMISSION (-11)/* a query or graph does not fit the memory budget */
#define JGPM_ENOTFOUND (-12) /* unknown ticket or graph id */

typedef struct jgpm_graph jgpm_graph;

typedef struct {
  int32_t num_vertices;
  int64_t num_arcs;        /* symmetric CSR slots (2 x undirected edges) */
  int32_t max_degree;
  int64_t num_dag_arcs;    /* 0 until the degree-oriented DAG is built */
  int32_t max_out_degree;
  int32_t device;
  uint64_t device_bytes;   /* device memory held by the handle */
} jgpm_graph_info;

typedef struct {
  uint64_t count;          /* the pattern count (also written to *out) */
  uint64_t setop_elements; /* algorithmic set-op elements of the canonical plan; filled only
                              when JGPM_COUNT_STATS is set */
  double kernel_ms;        /* device time of the counting launches (CUDA events) */
  int32_t rounds;          /* root-range rounds launched */
  int32_t method;          /* implementation path taken (JGPM_METHOD_*) */
  int32_t launches;        /* kernels launched by the counting call (timed part) */
  int32_t reserved;
} jgpm_stats;

#define JGPM_METHOD_BITMAP_CLIQUE 1  /* vertex-rooted local-bitmap k-clique kernels */
#define JGPM_METHOD_PLAN 2           /* per-root nested-loop plan kernel */
#define JGPM_METHOD_WEDGE 3          /* wedge aggregation (4-cycle) */
#define JGPM_METHOD_EDGE_TRIANGLE 4  /* per-arc triangle counters (diamond, tailed triangle) */
#define JGPM_METHOD_CENSUS 5         /* vertex-induced counts from the 4-vertex census */

#define JGPM_COUNT_STATS 1u          /* also compute setop_elements (an extra untimed pass) */
#define JGPM_COUNT_FORCE_PLAN 2u     /* use the literal nested-loop plan kernel */
#define JGPM_COUNT_FORCE_ENUM 4u     /* vertex-induced patterns: enumerate with set difference */

/* ---- library --------------------------------------------------------------------- */
/* The library's version string, naming its sm_100a build.  No reference counterpart. */
const char* jgpm_version(void);
/* Message of the calling thread's last failed call ("" if none).  Replaces the reference's
 * print-and-exit error handling (CUDA_SAFE_CALL, include/cutil_subset.h:4-16). */
const char* jgpm_last_error(void);
/* Number of visible CUDA devices; replaces cudaGetDeviceCount in SubgraphSolver
 * (src/jupiter_gpm.cu:33). */
int jgpm_device_count(int* n);
/* Selects the device used by graphs created afterwards on this thread; replaces the per-rank
 * cudaSetDevice (src/jupiter_gpm.cu:53, 310). */
int jgpm_set_device(int device);

/* ---- graphs ---------------------------------------------------------------------- */
/* Loads prefix.meta.txt / prefix.vertex.bin (int64 row pointers) / prefix.edge.bin (int32
 * sorted neighbour lists), the reference's on-disk CSR.  Replaces Graph::Graph(prefix,
 * use_dag) (common/graph.cc:8-124, include/graph.h:41-42).  orient_dag=1 builds the
 * degree-oriented DAG eagerly (Graph::orientation, common/graph.cc:210-401); the symmetric
 * CSR is kept either way, and every pattern picks the CSR its plan needs. */
int jgpm_graph_load(const char* prefix, int orient_dag, jgpm_graph** g);

/* Builds a graph from a host symmetric CSR (sorted, duplicate-free rows, no self-loops, both
 * directions present).  Replaces the CSR half of the reference loader and
 * NvsGraphGPU::init (include/graph_gpu_nvs.h:243-304).  Malformed input gives JGPM_EINVAL. */
int jgpm_graph_from_csr(const int64_t* rowptr, const int32_t* col, int32_t n, int64_t m,
                        int orient_dag, jgpm_graph** g);

/* Builds a graph from an undirected host edge list: both directions are added, self-loops
 * dropped, rows sorted and deduplicated on the device.  No reference counterpart (the
 * reference reads prebuilt CSRs only; this is the ingest step before its loader). */
int jgpm_graph_from_edges(const int32_t* src, const int32_t* dst, int64_t num_edges,
                          int32_t n, int orient_dag, jgpm_graph** g);

/* Generates a seeded R-MAT graph on the device: edge i draws its quadrants from a
 * counter-based hash of (seed, i) with integer thresholds, so the result does not depend on
 * the thread layout; ids >= n are redrawn.  Then symmetrised, deduplicated, self-loops
 * dropped.  No reference counterpart (the reference reads external datasets). */
int jgpm_graph_rmat(int64_t n, int64_t num_edges, double a, double b, double c, uint64_t seed,
                    int orient_dag, jgpm_graph** g);

/* The same seeded R-MAT edges on the host (no GPU needed): writes up to num_edges pairs and
 * the number written (edges with no valid draw in 64 attempts are dropped).  No reference
 * counterpart. */
int jgpm_rmat_edges(int64_t n, int64_t num_edges, double a, double b, double c, uint64_t seed,
                    int32_t* src, int32_t* dst, int64_t* out_count);

/* Sizes and degrees of a graph: Graph::num_vertices / num_edges / get_max_degree
 * (include/graph.h:50-59). */
int jgpm_graph_get_info(const jgpm_graph* g, jgpm_graph_info* info);

/* Copies the symmetric CSR (dag=0) or the DAG (dag=1, built if needed) to host arrays of
 * n+1 and num_arcs / num_dag_arcs entries: Graph::out_rowptr / out_colidx
 * (include/graph.h:69-70). */
int jgpm_graph_copy_csr(jgpm_graph* g, int dag, int64_t* rowptr, int32_t* col);

/* Writes the symmetric CSR (dag=0) or the DAG (dag=1) in the reference's on-disk format.
 * Replaces Graph::dump_binary (common/graph.cc:727-753). */
int jgpm_graph_save(jgpm_graph* g, const char* prefix, int dag);

/* Releases the handle and its device memory: Graph::~Graph (include/graph.h:45) and the
 * device CSR's teardown. */
void jgpm_graph_free(jgpm_graph* g);

/* The CUDA stream (a cudaStream_t, as an opaque pointer) on which every kernel of this graph
 * runs, so callers can order their own work or record events on it.  No reference
 * counterpart. */
int jgpm_graph_stream(jgpm_graph* g, void** stream);

/* ---- counting -------------------------------------------------------------------- */
/* Counts `pattern` in g exactly.  Replaces SubgraphSolver's pattern dispatch, round loop and
 * count reduction (src/jupiter_gpm.cu:356-375, 393-428, 873-908).  Pattern names:
 *   reference IDs  "P1".."P16", "vsgm_last_pattern" (edge-induced, reference semantics);
 *   aliases        "triangle" (= P0 on the DAG), "4-clique" (= P13), "5-clique" (= P14),
 *                  "6-clique", "7-clique", "k-clique:<k>" (3 <= k <= 8), "4-cycle" (= P1),
 *                  "diamond" (= P2), "tailed-triangle", "4-path", "3-star".
 * induced=0 counts edge-induced copies (reference semantics); induced=1 counts
 * vertex-induced copies of the 4-vertex patterns (each 4-vertex subset whose induced
 * subgraph is isomorphic to the pattern, once).  chunk_size is the reference's round count
 * (the root range is split into that many launches; <= 1 means one); it does not change
 * the result.  st may be NULL. */
int jgpm_count(jgpm_graph* g, const char* pattern, int induced, int chunk_size, uint64_t* out,
               jgpm_stats* st);

/* jgpm_count with JGPM_COUNT_* flags (the same reference interface,
 * src/jupiter_gpm.cu:356-375, 393-428, 873-908). */
int jgpm_count_ex(jgpm_graph* g, const char* pattern, int induced, int chunk_size,
                  unsigned flags, uint64_t* out, jgpm_stats* st);

/* Counts the embeddings rooted at a strided sample of root arcs: the CSR slots begin,
 * begin + stride, ... below end (end < 0: all) of the CSR the pattern's nested-loop plan
 * runs on -- the DAG for "triangle" (P0) and the cliques P13..P16 ("4-clique".."7-clique",
 * "k-clique:<k>" with k <= 7), the symmetric CSR otherwise.  Every embedding is rooted at
 * exactly one arc, so counts over disjoint samples add up, and begin = 0, end < 0, stride = 1
 * gives jgpm_count's result.  Runs the literal plan kernel (JGPM_COUNT_FORCE_PLAN; with
 * induced = 1 the set-difference enumeration), so it matches a CPU run of the same plans on
 * the same sample root arc for root arc.  The slots of one vertex v, [rowptr[v],
 * rowptr[v+1]), count the embeddings rooted at v.  Replaces the reference's per-round root
 * slice estart/enumber (src/jupiter_gpm.cu:373-377), here with a stride so that a sample
 * spreads over the whole graph.  Closed-form patterns ("tailed-triangle", "4-path",
 * "3-star" with induced = 0) have no plan: JGPM_EPATTERN.  end past the last root arc:
 * JGPM_EINVAL. */
int jgpm_count_roots(jgpm_graph* g, const char* pattern, int induced, int64_t begin,
                     int64_t end, int64_t stride, uint64_t* out, jgpm_stats* st);

/* The part of jgpm_count's result that shard `shard` of `nshards` owns, for splitting one
 * count over several GPUs (each holding the whole graph): the shards' results add up to the
 * full count, so one sum over the shards -- an all-reduce of one uint64 per count -- gives
 * it.  k-cliques ("triangle", "4-clique" .. "k-clique:<k>") shard the roots of every
 * out-degree tier of the bitmap kernels: shard s takes tier indices s, s + nshards, ..., so
 * every shard gets the same mix of heavy and light roots.  Every other pattern runs its
 * nested-loop plan (as jgpm_count_roots) over the root arcs shard, shard + nshards, ....
 * Replaces the reference's split of the root edges over ranks (src/jupiter_gpm.cu:91-150)
 * and its sum of the ranks' counts (:880-904). */
int jgpm_count_shard(jgpm_graph* g, const char* pattern, int induced, int32_t shard,
                     int32_t nshards, uint64_t* out, jgpm_stats* st);

/* Allocation-free count.  No counterpart in the reference: it exists for callers that may
 * not allocate device memory while they count (a host whose own allocator holds the device,
 * or a latency-critical path that must not call cudaMalloc/cudaFree).  It calls no
 * cudaMalloc, cudaFree or allocating routine; the literal plan kernel's per-warp lists live
 * in a fixed 32 MiB static device array, which limits the largest maximum degree to 262112
 * (maximum out-degree for the DAG plans); larger graphs get JGPM_ECAPACITY.  Patterns: the
 * reference IDs "P1".."P16", "vsgm_last_pattern" and "triangle" with induced=0, and
 * "4-cycle", "diamond", "tailed-triangle", "4-path", "3-star" with induced=1.  The DAG plans
 * (triangle, P13..P16) need the DAG already built (JGPM_EINVAL otherwise).  The count equals
 * jgpm_count's.  The static arrays are shared per device: calls that overlap on one device
 * race, so callers serialise them.  The first call on each device looks up the arrays'
 * addresses and keeps them for the life of the process; make it before any stream capture
 * begins, and do not reset the device (cudaDeviceReset) between calls. */
int jgpm_count_noalloc(jgpm_graph* g, const char* pattern, int induced, uint64_t* out);

/* Listing mode: writes the embeddings themselves, k vertex ids each (k = the pattern's size),
 * to out[0 .. k * min(total, capacity)) and their number to *total (all of them, also when
 * more than capacity exist: call with capacity 0 to size the buffer).  out may be host or
 * device memory.  Patterns: "triangle" and the k-cliques up to k = 8 (vertices in DAG order),
 * "4-cycle"/"P1" (cycle order v0 - v1 - v3 - v2 from the largest vertex v0, v1 > v2) and
 * "diamond"/"P2" (the shared edge v0 > v1, then the other two, ascending) with induced = 0;
 * "4-cycle", "diamond", "tailed-triangle", "4-path", "3-star" with induced = 1 (the root arc's
 * two vertices, then the other two).  The order of the tuples is unspecified.  The
 * reference chooses counting or listing when it is built (common.mk:60-63) and only counts;
 * this is the listing counterpart of jgpm_count's plans. */
int jgpm_list(jgpm_graph* g, const char* pattern, int induced, int32_t* out, int64_t capacity,
              int64_t* total, jgpm_stats* st);

/* Vertex-induced census of the six connected 4-vertex graphlets, out[0..5] = 3-star,
 * 4-path, tailed triangle, 4-cycle, diamond, 4-clique.  No reference counterpart (the
 * reference has no vertex-induced plans). */
int jgpm_census4(jgpm_graph* g, uint64_t out[6], jgpm_stats* st);

/* ---- batched counting -------------------------------------------------------------- */
/* One (graph, pattern) job.  Batchable patterns: "triangle", "4-clique" .. "7-clique",
 * "k-clique:<k>", "diamond" (= P2) and "4-cycle" (= P1), all with reference semantics. */
typedef struct {
  jgpm_graph* graph;
  const char* pattern;
} jgpm_job;

/* Work-split knobs of the batched kernel (and of the plain clique kernels). */
typedef struct {
  int32_t min_group;      /* narrowest lane group for roots of out-degree <= 32: 4, 8, 16, 32 */
  int32_t split_degree;   /* 32, 64 or 128: roots of out-degree 32 < d <= split run one per
                             warp, larger ones one per CTA (batched: up to out-degree 512,
                             above that on edge-rooted lists) */
  int32_t roots_per_task; /* lane-group roots per queued task (warp roots 1/16x, 4-cycle
                             apexes 1/8x) */
  int32_t intersect;      /* last clique level on edge-rooted lists: 0 searches the keys of
                             the shorter list in the longer one, 1 always the candidates */
  int32_t graphs;         /* 1: a batch's launches (table copies, the one to three persistent
                             kernels, the count read-back) are captured in a CUDA graph and
                             replayed while the launch plan is unchanged; 0: launched directly */
} jgpm_tuning;

typedef struct {
  double kernel_ms;       /* time of the batch on its stream, from before the host builds the
                             task tables to the count read-back (task building and upload,
                             kernels, read-back) */
  int32_t launches;       /* kernels launched, one to three: the persistent task kernel, a
                             light persistent kernel for the lane-group tasks, and one for the
                             large 4-cycle apexes, each when it has work */
  int32_t tasks;          /* tasks in the queues */
  jgpm_tuning used;
} jgpm_batch_stats;

/* Counts every job exactly in one persistent work-stealing launch: all jobs' work is cut into
 * tasks of one global queue that persistent CTAs drain; counts[i] receives job i's count.  Two
 * kinds of task have queues and persistent kernels of their own, on the same stream: the large
 * 4-cycle apexes of all jobs, drained first by CTAs that hold a shared-memory counter slab, and
 * the lane-group roots (out-degree <= 32), drained last by a light kernel with more CTAs per
 * SM.
 * Replaces, for a whole batch, the reference's per-query round loop and static chunking
 * (src/jupiter_gpm.cu:356-375).  tuning = NULL uses the defaults.  All graphs must be on one
 * device. */
/* Counts every job of `jobs` in one batched launch (one to three persistent kernels) and
 * writes counts[i] for job i.  Replaces one SubgraphSolver run per (graph, pattern)
 * (src/jupiter_gpm.cu:356-428) with its root-edge task queue in place of chunk_size's static
 * slices (:373-377). */
int jgpm_batch_count(const jgpm_job* jobs, int32_t njobs, const jgpm_tuning* tuning,
                     uint64_t* counts, jgpm_batch_stats* st);

/* Sets the lane-group and split knobs (min_group, split_degree) the plain clique kernels of
 * this graph use; split_degree in {32, 64, 128} (roots of out-degree 32 < d <= split run one per
 * warp, larger ones one per CTA).  Counts do not depend on it.  No reference counterpart. */
int jgpm_graph_set_tuning(jgpm_graph* g, const jgpm_tuning* tuning);

/* Picks the tuning by timing candidate settings (coordinate descent over the four knobs) on
 * an evenly spaced sample of at most sample_jobs jobs (<= 0: 256).  No reference
 * counterpart. */
int jgpm_autotune(const jgpm_job* jobs, int32_t njobs, int32_t sample_jobs, jgpm_tuning* out);

/* ---- serving: continuous batching over a memory-budgeted graph pool -------------- */
/* No reference counterpart (the reference runs one query per process invocation). */
typedef struct jgpm_server jgpm_server;

typedef struct {
  uint64_t memory_budget_bytes; /* device memory for resident graphs + in-flight frontiers */
  int32_t max_inflight;         /* batches in flight on the device at once (streams) */
  int32_t max_batch;            /* queries packed into one batched launch */
  int32_t device;
  int32_t reserved;
  jgpm_tuning tuning;           /* min_group == 0: defaults */
} jgpm_server_config;

typedef struct {
  uint64_t submitted, completed, rejected;
  uint64_t batches;             /* batched launches issued */
  uint64_t evictions, restores; /* graph pool traffic */
  uint64_t resident_bytes;      /* graph bytes resident now */
  uint64_t peak_frontier_bytes; /* largest admitted in-flight frontier estimate */
  double mean_batch;            /* queries per batch */
} jgpm_server_stats;

/* Starts a server (its scheduler thread, slots and plain lanes) on cfg->device.  No reference
 * counterpart. */
int jgpm_server_create(const jgpm_server_config* cfg, jgpm_server** s);

/* Adds a graph to the pool; the server takes ownership of the handle (it frees it in
 * jgpm_server_destroy).  The graph's DAG and root tiers are built now.  Evicted graphs keep a
 * host copy and are uploaded again on demand (least recently used graphs go first).  No
 * reference counterpart. */
int jgpm_server_add_graph(jgpm_server* s, jgpm_graph* g, int32_t* graph_id);

/* Queues a counting query and returns its ticket at once.  Batchable patterns (see jgpm_job)
 * are packed into batched launches; any other jgpm_count pattern runs on the server's plain
 * lane (one jgpm_count at a time, concurrently with the batches); the prefix "induced:"
 * (e.g. "induced:tailed-triangle") asks for the vertex-induced count.
 * A query is admitted to the device when its graph is resident and its estimated frontier
 * memory fits the budget; JGPM_EADMISSION if it can never fit.  Pending queries are admitted
 * shortest estimated work first, with aging: the estimate is the running average of the
 * service times measured for the same (graph, pattern) (before the first, a prior from the
 * graph's DAG arcs and the pattern), less 0.1 s per second the query has waited, so light
 * queries do not wait behind heavy ones and no query waits for ever.  No reference
 * counterpart. */
int jgpm_server_submit(jgpm_server* s, int32_t graph_id, const char* pattern, uint64_t* ticket);

/* Waits up to timeout_ms (< 0: no limit) for a ticket; JGPM_ETIMEDOUT if it is not done.
 * No reference counterpart. */
int jgpm_server_wait(jgpm_server* s, uint64_t ticket, int32_t timeout_ms, uint64_t* count,
                     double* latency_ms);

/* Query, batch and pool counters since the server started.  No reference counterpart. */
int jgpm_server_get_stats(jgpm_server* s, jgpm_server_stats* st);

/* Replays an open-loop trace: query i (graph_ids[i], patterns[i]) is submitted at
 * arrival_s[i] seconds after the start, from a generator thread inside the library.
 * mode 0 = through the server (continuous batching); mode 1 = each query as its own plain
 * jgpm_count call, served one at a time in arrival order.  Fills counts[i] and
 * latency_ms[i] (completion - arrival) and the wall time of the whole replay.  No reference
 * counterpart. */
int jgpm_server_replay(jgpm_server* s, int32_t mode, int64_t n, const int32_t* graph_ids,
                       const char* const* patterns, const double* arrival_s, uint64_t* counts,
                       double* latency_ms, double* wall_s);

/* Stops the server: its threads exit, the batches already on the device complete, queries
 * not yet launched are dropped, and its graphs are freed.  No reference counterpart. */
int jgpm_server_destroy(jgpm_server* s);

/* ---- set operations -------------------------------------------------------------- */
#define JGPM_OP_INTERSECT 0        /* materialise {x in A & B : x < upper} */
#define JGPM_OP_INTERSECT_COUNT 1  /* |{x in A & B : x < upper, x != exclude}| */
#define JGPM_OP_DIFFERENCE 2       /* materialise {x in A \ B : x < upper, x != exclude} */
#define JGPM_OP_DIFFERENCE_COUNT 3 /* |{x in A \ B : x < upper, x != exclude}| */

/* One sorted-set operation on int32 lists (device or host pointers; host buffers are
 * staged).  upper = INT32_MAX for no bound; exclude = -1 for none.  For the materialising
 * ops `out` must hold min(na, nb) (intersect) or na (difference) entries.  Replaces the
 * warp templates intersect / intersect_num (include/set_intersect.cuh:107-115, 190-195,
 * 352-360, 430-472) and difference_set / difference_num (include/set_difference.cuh:41-48,
 * 96-102, 163-170, 239-245) and the VertexSet operators (include/VertexSet.h:53-160).
 * Note: the reference's difference_num returns 0 when B is empty
 * (include/set_difference.cuh:44-45); this entry point returns |A'| as the set algebra
 * says, and as the reference's own bool-flag overload of difference_num does (:506-520). */
int jgpm_setop(int op, const int32_t* a, int32_t na, const int32_t* b, int32_t nb,
               int32_t upper, int32_t exclude, int32_t* out, int32_t* out_n);

/* A batch of set operations in one launch (the templates jgpm_setop replaces,
 * include/set_intersect.cuh and include/set_difference.cuh, one warp per pair): pair i is
 * A = a[a_off[i] .. a_off[i+1]) and
 * B = b[b_off[i] .. b_off[i+1]), with per-pair bounds (upper/exclude arrays may be NULL).
 * Counts go to counts[i]; for the materialising ops results go to out[out_off[i] ..) where
 * out_off (nops+1 entries, host) gives each pair's capacity.  Host or device arrays. */
int jgpm_setop_batch(int op, const int32_t* a, const int64_t* a_off, const int32_t* b,
                     const int64_t* b_off, int64_t nops, const int32_t* upper,
                     const int32_t* exclude, int32_t* counts, int32_t* out,
                     const int64_t* out_off);

/* Fused splits: one call yields several of the sets above at once.
 *   JGPM_SPLIT_FUSE     c = A \ B, d = A & B, e = B \ A;  count = |A & B|
 *                       (fuse_set, include/set_difference.cuh:248-343)
 *   JGPM_SPLIT_DIF_INT  c = {x in A : x < upper, x not in B}, d = the rest of A (members of B
 *                       and keys at or above upper);  count = |c|
 *                       (dif_int_set, include/set_difference.cuh:346-413; with upper =
 *                       INT32_MAX the unbounded form, :415-475)
 * Every output is in ascending order; |c| and |d| follow from count and na (and |e| from nb).
 * Capacities: c and d na entries, e nb entries (e is unused by JGPM_SPLIT_DIF_INT and may be
 * NULL); upper is ignored by JGPM_SPLIT_FUSE.  Outputs the sizes leave unwritten keep their
 * contents.  Note: the reference's templates return 0 and write nothing when A or B is empty;
 * these entry points follow the set algebra there too (B empty: c = A below upper). */
#define JGPM_SPLIT_FUSE 0
#define JGPM_SPLIT_DIF_INT 1
int jgpm_setop_split(int kind, const int32_t* a, int32_t na, const int32_t* b, int32_t nb,
                     int32_t upper, int32_t* c, int32_t* d, int32_t* e, int32_t* count);

/* A batch of fused splits in one launch (fuse_set / dif_int_set,
 * include/set_difference.cuh:248-475, one warp per pair), pairs given by offsets as in
 * jgpm_setop_batch.  Pair i writes c[a_off[i] ..) and d[a_off[i] ..) (arrays of a_off[nops]
 * entries) and e[b_off[i] ..) (b_off[nops] entries): the outputs are laid out like the
 * inputs.  upper may be NULL (no bounds).  Host or device arrays. */
int jgpm_setop_split_batch(int kind, const int32_t* a, const int64_t* a_off, const int32_t* b,
                           const int64_t* b_off, int64_t nops, const int32_t* upper,
                           int32_t* counts, int32_t* c, int32_t* d, int32_t* e);

#ifdef __cplusplus
}
#endif
#endif /* JGPM_H_ */
