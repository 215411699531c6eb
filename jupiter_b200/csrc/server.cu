// Serving: continuous batching of counting queries over a memory-budgeted graph pool.
//
// A scheduler thread owns `max_inflight` slots (a stream, a batched-kernel context and a
// pinned count buffer each).  Whenever a slot is free and queries are pending, it packs up to
// `max_batch` admissible queries into one batched persistent launch on that slot's stream and
// moves on.  Queries are taken shortest estimated work first, with aging: a query's estimate
// is the running average of the service times measured for its (graph, pattern), or before
// the first one a prior of DAG arcs x a per-pattern factor, and its priority is that estimate
// minus kAging x its wait, so light queries do not queue behind heavy ones and a heavy one is
// not passed over for ever; completions are detected with events, so batches of queries that
// arrived while others run overlap on the device.  Admission: a query's graph must be
// resident (the pool uploads it again, evicting least-recently-used idle graphs, if needed)
// and the resident graph bytes plus the estimated frontier memory of everything in flight
// must stay within the budget.  Queries on heavy graphs (more than kHeavyArcs DAG arcs) and
// patterns the batched kernel does not cover go to kPlainWorkers plain lanes, one jgpm_count
// each: on large graphs the per-tier plain kernels use the GPU better than the one-size batch
// kernel, while batches win on the many small queries.  A graph is used by one batch or one
// plain query at a time.  A batch's frontier is the sum of its queries' own scratch
// (diamond per-arc counters) plus the largest shared scratch any of them needs (4-cycle
// counter arena, edge-rooted list scratch), since the batch shares one context.  Counts are those of the batched kernel, i.e. exact and
// identical to the plain per-query path.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "batch.h"
#include "jgpm_internal.h"

namespace jgpm {
namespace {

using Clock = std::chrono::steady_clock;

constexpr int kPlainWorkers = 2;
constexpr int64_t kHeavyArcs = (int64_t)16 << 20;  // DAG arcs (symmetric arcs / 2)
constexpr double kAging = 0.1;  // seconds of estimated work forgiven per second of waiting

double now_s() {
  return std::chrono::duration<double>(Clock::now().time_since_epoch()).count();
}

struct Query {
  uint64_t ticket = 0;
  int32_t graph_id = 0;
  int kind = 0, k = 0;
  double t_submit = 0.0, t_done = 0.0;
  uint64_t count = 0;
  uint64_t frontier = 0;       // plain lane: bytes this query may allocate while it runs
  uint64_t fr_own = 0;         // batched: scratch of this query alone (adds up in a batch)
  uint64_t fr_shared = 0;      // batched: shared scratch of the batch this query needs
  int status = 1;  // 1 pending, 0 done, < 0 error
  bool plain = false;   // not batchable: runs through jgpm_count on the plain lane
  int induced = 0;
  std::string pattern;
  std::string cost_key;  // pattern as submitted (with the "induced:" prefix)
  double est = 0.0;      // estimated service time (s)
};

struct PoolGraph {
  jgpm_graph* g = nullptr;
  std::vector<int64_t> h_rowptr;  // host copy once evicted
  std::vector<int32_t> h_col;
  uint64_t bytes = 0;             // device bytes when resident
  uint64_t last_use = 0;
  int inflight = 0;
  bool plain_busy = false;        // a plain-lane query is running on this graph
  bool resident = true;
};

struct Slot {
  BatchCtx ctx;
  cudaStream_t stream = nullptr;
  cudaEvent_t done_ev = nullptr;
  uint64_t* h_counts = nullptr;  // pinned
  std::vector<std::shared_ptr<Query>> queries;
  uint64_t frontier = 0;  // of the batch in flight
  double t_launch = 0.0;
  bool busy = false;
};

}  // namespace
}  // namespace jgpm

struct jgpm_server {
  jgpm_server_config cfg;
  std::mutex mu;
  std::condition_variable cv_work;   // wakes the scheduler
  std::condition_variable cv_done;   // wakes waiters
  std::deque<std::shared_ptr<jgpm::Query>> pending;
  std::deque<std::shared_ptr<jgpm::Query>> plain_pending;
  std::condition_variable cv_plain;
  std::vector<std::thread> plain_threads;
  std::unordered_map<uint64_t, std::shared_ptr<jgpm::Query>> tickets;
  std::vector<jgpm::PoolGraph> graphs;
  std::vector<std::unique_ptr<jgpm::Slot>> slots;
  std::thread sched;
  std::atomic<bool> stop{false};
  uint64_t next_ticket = 1;
  uint64_t use_clock = 0;
  uint64_t resident_bytes = 0;
  uint64_t inflight_frontier = 0;
  jgpm_server_stats st{};
  std::string sched_error;
  // measured service time (s) per (graph, pattern): the scheduler's work estimates
  std::unordered_map<std::string, double> cost;
};

namespace jgpm {
namespace {

std::string cost_id(int32_t graph_id, const std::string& pattern) {
  return std::to_string(graph_id) + "/" + pattern;
}

// Prior service time of a query before any has been measured: DAG arcs x a per-pattern
// factor (seconds per arc; measured ratios of the plain kernels on R-MAT graphs).
double prior_cost(const jgpm_graph* g, const std::string& pattern) {
  const double arcs = (double)(g->m_dag > 0 ? g->m_dag : g->m / 2);
  double f = 2.0;  // literal plans and census pieces
  if (pattern == "triangle" || pattern == "P0" || pattern == "3-clique") f = 0.1;
  else if (pattern == "4-clique" || pattern == "P13") f = 0.45;
  else if (pattern == "5-clique" || pattern == "P14") f = 1.0;
  else if (pattern == "diamond" || pattern == "P2") f = 0.5;
  else if (pattern == "induced:tailed-triangle") f = 0.55;
  else if (pattern == "4-cycle" || pattern == "P1") f = 3.0;
  return arcs * f * 1e-9;
}

// Folds a measured service time into the running average of its (graph, pattern) (mu held).
void learn_cost(jgpm_server* s, const Query& q, double seconds) {
  const std::string id = cost_id(q.graph_id, q.cost_key);
  auto it = s->cost.find(id);
  if (it == s->cost.end()) s->cost.emplace(id, seconds);
  else it->second = 0.5 * it->second + 0.5 * seconds;
}

// Priority of a pending query (lower first): estimated work, less credit for waiting.
double priority(const Query& q, double now) { return q.est - kAging * (now - q.t_submit); }

// Indices of `pending` in priority order.
std::vector<size_t> by_priority(const std::deque<std::shared_ptr<Query>>& pending) {
  const double now = now_s();
  std::vector<std::pair<double, size_t>> k(pending.size());
  for (size_t i = 0; i < pending.size(); ++i) k[i] = {priority(*pending[i], now), i};
  std::stable_sort(k.begin(), k.end());
  std::vector<size_t> out(k.size());
  for (size_t i = 0; i < k.size(); ++i) out[i] = k[i].second;
  return out;
}

bool over_budget(jgpm_server* s, uint64_t extra) {
  return s->resident_bytes + s->inflight_frontier + extra > s->cfg.memory_budget_bytes;
}

// Makes graph `gid` resident, evicting idle LRU graphs while over budget (mu held).
int make_resident(jgpm_server* s, int gid, uint64_t frontier) {
  PoolGraph& pg = s->graphs[gid];
  if (pg.resident) return JGPM_OK;
  while (over_budget(s, pg.bytes + frontier)) {
    int victim = -1;
    for (int i = 0; i < (int)s->graphs.size(); ++i) {
      PoolGraph& o = s->graphs[i];
      if (i == gid || !o.resident || o.inflight > 0) continue;
      if (victim < 0 || o.last_use < s->graphs[victim].last_use) victim = i;
    }
    if (victim < 0) return JGPM_EBUSY;  // try again when something completes
    PoolGraph& v = s->graphs[victim];
    int rc = evict_graph(v.g, v.h_rowptr, v.h_col);
    if (rc) return rc;
    v.resident = false;
    s->resident_bytes -= v.bytes;
    s->st.evictions++;
  }
  int rc = restore_graph(pg.g, pg.h_rowptr, pg.h_col);
  if (rc) return rc;
  pg.resident = true;
  pg.bytes = graph_device_bytes(pg.g);
  s->resident_bytes += pg.bytes;
  s->st.restores++;
  return JGPM_OK;
}

// Packs admissible pending queries into the free slot and launches them (mu held).
int launch_batch(jgpm_server* s, Slot& slot) {
  std::vector<std::shared_ptr<Query>> batch;
  std::vector<BatchJobIn> in;
  uint64_t own = 0, shared = 0;
  std::vector<bool> taken(s->pending.size(), false);
  for (size_t idx : by_priority(s->pending)) {
    if ((int)batch.size() >= s->cfg.max_batch) break;
    std::shared_ptr<Query> q = s->pending[idx];
    PoolGraph& pg = s->graphs[q->graph_id];
    if (pg.plain_busy) continue;  // the graph is in a plain-lane query: next launch
    const uint64_t with_q = own + q->fr_own + std::max(shared, q->fr_shared);
    if (!pg.resident) {
      int rc = make_resident(s, q->graph_id, with_q);
      if (rc == JGPM_EBUSY) continue;
      if (rc) return rc;
    }
    if (over_budget(s, with_q) && (!batch.empty() || s->inflight_frontier > 0))
      continue;  // wait for in-flight work to release memory
    own += q->fr_own;
    shared = std::max(shared, q->fr_shared);
    pg.inflight++;
    pg.last_use = ++s->use_clock;
    in.push_back(BatchJobIn{pg.g, q->kind, q->k});
    batch.push_back(q);
    taken[idx] = true;
  }
  if (batch.empty()) return JGPM_OK;
  {
    std::deque<std::shared_ptr<Query>> rest;
    for (size_t i = 0; i < s->pending.size(); ++i)
      if (!taken[i]) rest.push_back(s->pending[i]);
    s->pending.swap(rest);
  }
  slot.t_launch = now_s();
  int ntasks = 0;
  int rc = batch_enqueue(slot.ctx, in, s->cfg.tuning, slot.stream, slot.h_counts, &ntasks);
  if (rc) {
    for (auto& q : batch) {
      q->status = rc;
      s->graphs[q->graph_id].inflight--;
    }
    s->cv_done.notify_all();
    return rc;
  }
  cudaEventRecord(slot.done_ev, slot.stream);
  const uint64_t frontier = own + shared;
  s->inflight_frontier += frontier;
  slot.frontier = frontier;
  s->st.peak_frontier_bytes = std::max<uint64_t>(s->st.peak_frontier_bytes, s->inflight_frontier);
  s->st.batches++;
  slot.queries = std::move(batch);
  slot.busy = true;
  return JGPM_OK;
}

void complete_slot(jgpm_server* s, Slot& slot) {
  const double t = now_s();
  // the batch's service time, shared out over its queries by their estimates
  double est_sum = 0.0;
  for (auto& qp : slot.queries) est_sum += qp->est;
  for (size_t i = 0; i < slot.queries.size(); ++i) {
    Query& q = *slot.queries[i];
    q.count = slot.h_counts[i];
    q.t_done = t;
    q.status = 0;
    s->graphs[q.graph_id].inflight--;
    s->st.completed++;
    if (est_sum > 0.0) learn_cost(s, q, (t - slot.t_launch) * q.est / est_sum);
  }
  // derived structures (DAG, tiers, 4-cycle classes) may have grown the graphs
  for (auto& qp : slot.queries) {
    PoolGraph& pg = s->graphs[qp->graph_id];
    const uint64_t b = graph_device_bytes(pg.g);
    s->resident_bytes += b - pg.bytes;
    pg.bytes = b;
  }
  s->inflight_frontier -= slot.frontier;
  slot.frontier = 0;
  slot.queries.clear();
  slot.busy = false;
}

void scheduler(jgpm_server* s) {
  cudaSetDevice(s->cfg.device);
  std::unique_lock<std::mutex> lk(s->mu);
  while (!s->stop.load()) {
    bool progress = false;
    for (auto& sp : s->slots) {
      Slot& slot = *sp;
      if (slot.busy && cudaEventQuery(slot.done_ev) == cudaSuccess) {
        complete_slot(s, slot);
        progress = true;
      }
    }
    if (progress) {
      s->cv_done.notify_all();
      s->cv_plain.notify_all();  // graphs of completed batches are free for the plain lanes
    }
    for (auto& sp : s->slots) {
      if (s->pending.empty()) break;
      Slot& slot = *sp;
      if (slot.busy) continue;
      const uint64_t before = s->st.batches;
      int rc = launch_batch(s, slot);
      if (rc) s->sched_error = std::string(jgpm_last_error());
      if (s->st.batches != before) progress = true;
      else break;  // nothing admissible now
    }
    if (!progress) {
      bool any_busy = false;
      for (auto& sp : s->slots) any_busy = any_busy || sp->busy;
      // poll completions quickly while work is in flight; otherwise sleep until a submit
      s->cv_work.wait_for(lk, any_busy ? std::chrono::microseconds(20)
                                       : std::chrono::milliseconds(50));
    }
  }
}

// Plain lane: queries the batched kernel does not cover (vertex-induced patterns, the
// reference's P3..P12, ...) run one at a time through jgpm_count on their graph's stream,
// concurrently with the batches.
void plain_worker(jgpm_server* s) {
  cudaSetDevice(s->cfg.device);
  std::unique_lock<std::mutex> lk(s->mu);
  while (!s->stop.load()) {
    if (s->plain_pending.empty()) {
      s->cv_plain.wait_for(lk, std::chrono::milliseconds(50));
      continue;
    }
    // the first pending query, in priority order, whose graph no batch or other plain query
    // is using
    auto pick = s->plain_pending.end();
    for (size_t idx : by_priority(s->plain_pending)) {
      const PoolGraph& c = s->graphs[s->plain_pending[idx]->graph_id];
      if (c.inflight == 0 && !c.plain_busy) {
        pick = s->plain_pending.begin() + (std::ptrdiff_t)idx;
        break;
      }
    }
    if (pick == s->plain_pending.end()) {
      s->cv_plain.wait_for(lk, std::chrono::microseconds(200));
      continue;
    }
    std::shared_ptr<Query> q = *pick;
    PoolGraph& pg = s->graphs[q->graph_id];
    if (!pg.resident) {
      int rc = make_resident(s, q->graph_id, q->frontier);
      if (rc == JGPM_EBUSY) {
        s->cv_plain.wait_for(lk, std::chrono::microseconds(200));
        continue;
      }
      if (rc) {
        s->plain_pending.erase(pick);
        q->status = rc;
        s->cv_done.notify_all();
        continue;
      }
    }
    if (over_budget(s, q->frontier) && s->inflight_frontier > 0) {
      s->cv_plain.wait_for(lk, std::chrono::microseconds(200));
      continue;
    }
    s->plain_pending.erase(pick);
    pg.inflight++;
    pg.plain_busy = true;
    pg.last_use = ++s->use_clock;
    s->inflight_frontier += q->frontier;
    s->st.peak_frontier_bytes = std::max<uint64_t>(s->st.peak_frontier_bytes, s->inflight_frontier);
    jgpm_graph* g = pg.g;
    lk.unlock();
    uint64_t cnt = 0;
    const double t_start = now_s();
    const int rc = jgpm_count_ex(g, q->pattern.c_str(), q->induced, 1, 0u, &cnt, nullptr);
    const std::string err = rc ? std::string(jgpm_last_error()) : std::string();
    lk.lock();
    {
      PoolGraph& pg2 = s->graphs[q->graph_id];
      pg2.inflight--;
      pg2.plain_busy = false;
      const uint64_t b = graph_device_bytes(pg2.g);
      s->resident_bytes += b - pg2.bytes;
      pg2.bytes = b;
    }
    s->inflight_frontier -= q->frontier;
    q->count = cnt;
    q->t_done = now_s();
    q->status = rc;
    if (rc) s->sched_error = err;
    else {
      s->st.completed++;
      learn_cost(s, *q, q->t_done - t_start);
    }
    s->cv_done.notify_all();
    s->cv_work.notify_one();  // the graph is free for batches again
  }
}

}  // namespace
}  // namespace jgpm

using namespace jgpm;

namespace {

// Scratch a batched query needs: *own adds up over a batch (diamond per-arc counters), *shared
// is charged once per batch at its largest (4-cycle counter and touched arrays of the owner
// CTAs, within the slot's cap; edge-rooted lists of the heavy roots).  The DAG and the
// 4-cycle apex classes count as graph bytes once built.
void estimate_frontier(const jgpm_server* s, const jgpm_graph* g, int kind, uint64_t* own,
                       uint64_t* shared) {
  const uint64_t sms = (uint64_t)device_sm_count(s->cfg.device);
  const uint64_t grid = sms * 4;
  *own = 0;
  *shared = 0;
  const uint64_t m_dag = g->m_dag > 0 ? (uint64_t)g->m_dag : (uint64_t)g->m / 2;
  if (kind == kJobC4) {
    const uint64_t cap = s->slots.empty() ? ((uint64_t)4 << 30) : s->slots[0]->ctx.c4_cap_bytes;
    *shared = 2 * std::min<uint64_t>(cap, grid * (uint64_t)g->n * 4);
  } else {
    if (kind == kJobDiamond || kind == kJobIndTT) *own = m_dag * 4 + 256;
    const int maxo = g->max_out_degree > 0 ? g->max_out_degree : g->max_degree;
    if (maxo > kBatchCtaMaxDeg) {  // wide roots: bitmap rows per CTA
      const uint64_t wd = (uint64_t)std::min(maxo, kBatchWideMaxDeg);
      *shared += grid * wd * ((wd + 31) / 32) * 4;
    }
    if (maxo > kBatchWideMaxDeg) *shared += grid * 8 * 6 * ((uint64_t)maxo + 32) * 4;
  }
}

bool pattern_known(const std::string& p, int induced) {
  if (!induced) {
    int kind = 0, k = 0;
    if (parse_batch_pattern(p.c_str(), &kind, &k) == JGPM_OK) return true;
  }
  return plan_id_of(p, induced) >= 0;
}

int check_server(jgpm_server* s) {
  if (!s) {
    jgpm_set_error_("null server");
    return JGPM_EINVAL;
  }
  return JGPM_OK;
}

}  // namespace

extern "C" {

int jgpm_server_create(const jgpm_server_config* cfg, jgpm_server** out) {
  if (!cfg || !out || cfg->max_inflight < 1 || cfg->max_batch < 1 || cfg->memory_budget_bytes == 0) {
    jgpm_set_error_("jgpm_server_create: bad config");
    return JGPM_EINVAL;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    jgpm_set_error_("no CUDA device");
    return JGPM_ENODEV;
  }
  if (cfg->device < 0 || cfg->device >= ndev) {
    jgpm_set_error_("jgpm_server_create: no such device");
    return JGPM_EINVAL;
  }
  jgpm_server* s = new jgpm_server;
  s->cfg = *cfg;
  if (s->cfg.tuning.min_group == 0) s->cfg.tuning = default_tuning();
  cudaSetDevice(cfg->device);
  const uint64_t c4cap = std::max<uint64_t>((uint64_t)64 << 20,
                                            cfg->memory_budget_bytes / 8 / cfg->max_inflight);
  for (int i = 0; i < cfg->max_inflight; ++i) {
    auto sl = std::make_unique<Slot>();
    sl->ctx.device = cfg->device;
    sl->ctx.c4_cap_bytes = c4cap;
    if (cudaStreamCreateWithFlags(&sl->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&sl->done_ev, cudaEventDisableTiming) != cudaSuccess ||
        cudaMallocHost((void**)&sl->h_counts, sizeof(uint64_t) * cfg->max_batch) != cudaSuccess) {
      jgpm_set_error_("jgpm_server_create: stream/event/pinned allocation failed");
      delete s;
      return JGPM_ECUDA;
    }
    s->slots.push_back(std::move(sl));
  }
  s->sched = std::thread(scheduler, s);
  for (int i = 0; i < kPlainWorkers; ++i) s->plain_threads.emplace_back(plain_worker, s);
  *out = s;
  return JGPM_OK;
}

int jgpm_server_add_graph(jgpm_server* s, jgpm_graph* g, int32_t* graph_id) {
  int rc;
  if ((rc = check_server(s))) return rc;
  if (!g || !graph_id) {
    jgpm_set_error_("jgpm_server_add_graph: null argument");
    return JGPM_EINVAL;
  }
  if (g->device != s->cfg.device) {
    jgpm_set_error_("jgpm_server_add_graph: graph lives on another device");
    return JGPM_EINVAL;
  }
  cudaSetDevice(g->device);
  if ((rc = ensure_dag(g)) || (rc = ensure_tiers(g, 2)) || (rc = ensure_control(g))) return rc;
  std::unique_lock<std::mutex> lk(s->mu);
  PoolGraph pg;
  pg.g = g;
  pg.bytes = graph_device_bytes(g);
  pg.last_use = ++s->use_clock;
  s->graphs.push_back(std::move(pg));
  s->resident_bytes += s->graphs.back().bytes;
  *graph_id = (int32_t)s->graphs.size() - 1;
  // keep the pool within budget: evict idle LRU graphs (never the one just added)
  while (s->resident_bytes > s->cfg.memory_budget_bytes) {
    int victim = -1;
    for (int i = 0; i + 1 < (int)s->graphs.size(); ++i) {
      PoolGraph& o = s->graphs[i];
      if (!o.resident || o.inflight > 0) continue;
      if (victim < 0 || o.last_use < s->graphs[victim].last_use) victim = i;
    }
    if (victim < 0) break;
    PoolGraph& v = s->graphs[victim];
    if ((rc = evict_graph(v.g, v.h_rowptr, v.h_col))) return rc;
    v.resident = false;
    s->resident_bytes -= v.bytes;
    s->st.evictions++;
  }
  if (s->graphs.back().bytes > s->cfg.memory_budget_bytes) {
    jgpm_set_error_("jgpm_server_add_graph: graph alone exceeds the memory budget");
    return JGPM_EADMISSION;
  }
  return JGPM_OK;
}

int jgpm_server_submit(jgpm_server* s, int32_t graph_id, const char* pattern, uint64_t* ticket) {
  int rc;
  if ((rc = check_server(s))) return rc;
  if (!ticket || !pattern) {
    jgpm_set_error_("jgpm_server_submit: null argument");
    return JGPM_EINVAL;
  }
  auto q = std::make_shared<Query>();
  std::string p(pattern);
  if (parse_batch_pattern(pattern, &q->kind, &q->k) == JGPM_OK) {
    // batchable, including "induced:tailed-triangle"
  } else if (p.rfind("induced:", 0) == 0) {
    q->plain = true;
    q->induced = 1;
    q->pattern = p.substr(8);
  } else {
    q->plain = true;
    q->pattern = p;
  }
  if (q->plain && !pattern_known(q->pattern, q->induced)) {
    jgpm_set_error_(std::string("jgpm_server_submit: unknown pattern '") + pattern + "'");
    return JGPM_EPATTERN;
  }
  std::unique_lock<std::mutex> lk(s->mu);
  if (graph_id < 0 || graph_id >= (int32_t)s->graphs.size()) {
    jgpm_set_error_("jgpm_server_submit: unknown graph id");
    return JGPM_ENOTFOUND;
  }
  q->graph_id = graph_id;
  const jgpm_graph* g = s->graphs[graph_id].g;
  if (!q->plain && g->m / 2 > kHeavyArcs) {  // heavy graph: plain lane
    q->plain = true;
    q->induced = p.rfind("induced:", 0) == 0 ? 1 : 0;
    q->pattern = q->induced ? p.substr(8) : p;
  }
  if (q->plain) {
    const uint64_t m_dag = g->m_dag > 0 ? (uint64_t)g->m_dag : (uint64_t)g->m / 2;
    q->frontier = m_dag * 4 + (uint64_t)g->n * 8 + ((uint64_t)256 << 20);
    const std::string& qp = q->pattern;
    if (qp == "4-cycle" || qp == "P1" || (q->induced && qp == "4-path"))
      // the 4-cycle count's dense counters (2n ints per CTA, at most 12 GiB)
      q->frontier += std::min<uint64_t>((uint64_t)12 << 30,
                                        (uint64_t)device_sm_count(s->cfg.device) * 2 *
                                            (uint64_t)g->n * 8);
    // the literal plan kernel's per-warp lists (up to 2 GiB) or the clique tiers' scratch,
    // allocated on the graph while the query runs
    q->frontier += count_scratch_bytes(g, qp, q->induced);
  } else {
    estimate_frontier(s, g, q->kind, &q->fr_own, &q->fr_shared);
  }
  q->cost_key = p;
  {
    auto it = s->cost.find(cost_id(graph_id, p));
    q->est = it != s->cost.end() ? it->second : prior_cost(g, p);
  }
  const uint64_t need = q->plain ? q->frontier : q->fr_own + q->fr_shared;
  if (need + s->graphs[graph_id].bytes > s->cfg.memory_budget_bytes) {
    s->st.rejected++;
    jgpm_set_error_("jgpm_server_submit: query frontier + graph exceed the memory budget");
    return JGPM_EADMISSION;
  }
  q->ticket = s->next_ticket++;
  q->t_submit = now_s();
  s->tickets[q->ticket] = q;
  if (q->plain) s->plain_pending.push_back(q);
  else s->pending.push_back(q);
  s->st.submitted++;
  *ticket = q->ticket;
  lk.unlock();
  if (q->plain) s->cv_plain.notify_one();
  else s->cv_work.notify_one();
  return JGPM_OK;
}

int jgpm_server_wait(jgpm_server* s, uint64_t ticket, int32_t timeout_ms, uint64_t* count,
                     double* latency_ms) {
  int rc;
  if ((rc = check_server(s))) return rc;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) {
    jgpm_set_error_("jgpm_server_wait: unknown ticket");
    return JGPM_ENOTFOUND;
  }
  std::shared_ptr<Query> q = it->second;
  auto ready = [&] { return q->status <= 0; };
  if (timeout_ms < 0) {
    s->cv_done.wait(lk, ready);
  } else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) {
    jgpm_set_error_("jgpm_server_wait: timed out");
    return JGPM_ETIMEDOUT;
  }
  s->tickets.erase(ticket);
  if (q->status < 0) {
    jgpm_set_error_("jgpm_server_wait: the batch failed: " + s->sched_error);
    return q->status;
  }
  if (count) *count = q->count;
  if (latency_ms) *latency_ms = (q->t_done - q->t_submit) * 1e3;
  return JGPM_OK;
}

int jgpm_server_get_stats(jgpm_server* s, jgpm_server_stats* st) {
  int rc;
  if ((rc = check_server(s))) return rc;
  if (!st) return JGPM_EINVAL;
  std::unique_lock<std::mutex> lk(s->mu);
  *st = s->st;
  st->resident_bytes = s->resident_bytes;
  st->mean_batch = s->st.batches ? (double)s->st.completed / (double)s->st.batches : 0.0;
  return JGPM_OK;
}

int jgpm_server_replay(jgpm_server* s, int32_t mode, int64_t n, const int32_t* graph_ids,
                       const char* const* patterns, const double* arrival_s, uint64_t* counts,
                       double* latency_ms, double* wall_s) {
  int rc;
  if ((rc = check_server(s))) return rc;
  if (n < 0 || (n > 0 && (!graph_ids || !patterns || !arrival_s || !counts || !latency_ms))) {
    jgpm_set_error_("jgpm_server_replay: bad arguments");
    return JGPM_EINVAL;
  }
  cudaSetDevice(s->cfg.device);
  const double t0 = now_s();
  auto sleep_until = [&](double t_rel) {
    const double target = t0 + t_rel;
    for (;;) {
      const double d = target - now_s();
      if (d <= 0) return;
      if (d > 200e-6) std::this_thread::sleep_for(std::chrono::duration<double>(d - 100e-6));
    }
  };
  if (mode == 0) {
    std::vector<uint64_t> tk((size_t)n);
    for (int64_t i = 0; i < n; ++i) {
      sleep_until(arrival_s[i]);
      if ((rc = jgpm_server_submit(s, graph_ids[i], patterns[i], &tk[i]))) return rc;
    }
    for (int64_t i = 0; i < n; ++i) {
      double lat = 0;
      if ((rc = jgpm_server_wait(s, tk[i], -1, &counts[i], &lat))) return rc;
      latency_ms[i] = lat;
    }
  } else {
    // plain: one jgpm_count per query, in arrival order, one at a time
    for (int64_t i = 0; i < n; ++i) {
      sleep_until(arrival_s[i]);
      jgpm_graph* g = nullptr;
      {
        std::unique_lock<std::mutex> lk(s->mu);
        if (graph_ids[i] < 0 || graph_ids[i] >= (int32_t)s->graphs.size()) return JGPM_ENOTFOUND;
        PoolGraph& pg = s->graphs[graph_ids[i]];
        if (!pg.resident && (rc = make_resident(s, graph_ids[i], 0))) return rc;
        pg.last_use = ++s->use_clock;
        pg.inflight++;
        g = pg.g;
      }
      const std::string pat(patterns[i]);
      const bool ind = pat.rfind("induced:", 0) == 0;
      rc = jgpm_count(g, ind ? pat.c_str() + 8 : pat.c_str(), ind ? 1 : 0, 1, &counts[i],
                      nullptr);
      {
        std::unique_lock<std::mutex> lk(s->mu);
        s->graphs[graph_ids[i]].inflight--;
      }
      if (rc) return rc;
      latency_ms[i] = (now_s() - (t0 + arrival_s[i])) * 1e3;
    }
  }
  if (wall_s) *wall_s = now_s() - t0;
  return JGPM_OK;
}

int jgpm_server_destroy(jgpm_server* s) {
  if (!s) return JGPM_EINVAL;
  {
    std::unique_lock<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  s->cv_plain.notify_all();
  if (s->sched.joinable()) s->sched.join();
  for (auto& t : s->plain_threads)
    if (t.joinable()) t.join();
  for (auto& sl : s->slots) {
    if (sl->stream) cudaStreamSynchronize(sl->stream);
    if (sl->done_ev) cudaEventDestroy(sl->done_ev);
    if (sl->h_counts) cudaFreeHost(sl->h_counts);
    if (sl->stream) cudaStreamDestroy(sl->stream);
  }
  for (auto& pg : s->graphs) jgpm_graph_free(pg.g);
  delete s;
  return JGPM_OK;
}

}  // extern "C"
