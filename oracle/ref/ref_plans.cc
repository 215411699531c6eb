// Plan driver over the reference's OWN host code (test infrastructure and timed CPU baseline).
//
// The reference ships no CPU plan driver (its common/intersect.cc has no caller), so this
// file, written for this project, drives the plans with the reference's compiled host code:
//   * the graph loader and degree orientation, Graph::Graph / Graph::orientation
//     (common/graph.cc:8-124, 210-401), reading the reference's .meta.txt/.vertex.bin/.edge.bin;
//   * SetIntersection::get_num / ComputeCandidates (common/intersect.cc:6-79), AVX2 (SI == 0);
//   * VertexSet differences (common/VertexSet.cc:21-89) for the vertex-induced plans.
// The plans are those of src/message_passing_gpu_kernels.cuh (P0 :64-102, P1 :104-186,
// P2 :188-252, P13..P16 :1208-1537) and the vertex-induced definitions of oracle/oracle.cc.
// Built by oracle/build_ref.py into oracle/_ref/libjref.so.
#include <omp.h>
#include <chrono>
#include <cstdint>
#include <string>
#include <vector>

#include "graph.h"
#include "intersect.h"

namespace {

struct RefCtx {
  Graph* g;
  bool dag;
};

inline vidType bounded_len(const vidType* a, vidType n, vidType upper) {
  return bs(const_cast<vidType*>(a), n, upper);  // include/VertexSet.h:9-19
}

struct Buf {
  std::vector<vidType> w[6];
  explicit Buf(vidType md) {
    for (auto& x : w) x.resize((size_t)md + 16);
  }
};

uint64_t clique_rec(Graph& g, const vidType* cand, vidType nc, int remaining, Buf& b, int depth) {
  uint64_t c = 0;
  if (remaining == 1) {
    for (vidType i = 0; i < nc; ++i) {
      vidType v = cand[i];
      c += SetIntersection::get_num(cand, nc, g.adj_ptr(v), g.get_degree(v));
    }
    return c;
  }
  vidType* next = b.w[depth].data();
  for (vidType i = 0; i < nc; ++i) {
    vidType v = cand[i];
    vidType t = 0;
    SetIntersection::ComputeCandidates(cand, nc, g.adj_ptr(v), g.get_degree(v), next, t);
    c += clique_rec(g, next, t, remaining - 1, b, depth + 1);
  }
  return c;
}

}  // namespace

extern "C" {

void* ref_graph_load(const char* prefix, int use_dag) {
  RefCtx* ctx = new RefCtx;
  ctx->g = new Graph(std::string(prefix), use_dag != 0);
  ctx->dag = use_dag != 0;
  return ctx;
}

void ref_graph_free(void* h) {
  RefCtx* ctx = (RefCtx*)h;
  delete ctx->g;
  delete ctx;
}

int64_t ref_graph_info(void* h, int64_t* num_vertices, int64_t* num_arcs) {
  RefCtx* ctx = (RefCtx*)h;
  *num_vertices = ctx->g->V();
  *num_arcs = ctx->g->E();
  return 0;
}

// Copies the loaded (and, for a DAG, oriented) CSR out, so tests can compare the reference's
// own orientation with the product's.
int ref_graph_copy(void* h, int64_t* rowptr, int32_t* col) {
  RefCtx* ctx = (RefCtx*)h;
  Graph& g = *ctx->g;
  for (int64_t v = 0; v <= g.V(); ++v) rowptr[v] = g.out_rowptr()[v];
  for (int64_t e = 0; e < g.E(); ++e) col[e] = g.out_colidx()[e];
  return 0;
}

// Counts `pattern` over root arcs [begin, end) every `stride`-th, with `nthreads` OpenMP
// threads.  Patterns: clique3..clique7 (P0 on the DAG and P13..P16), P1, P2 and the
// vertex-induced induced-4-cycle / induced-diamond / induced-tailed-triangle /
// induced-4-path / induced-3-star.  Returns -1 for an unknown pattern.
int ref_count(void* h, const char* pattern, int64_t begin, int64_t end, int64_t stride,
              int nthreads, uint64_t* count, double* seconds) {
  RefCtx* ctx = (RefCtx*)h;
  Graph& g = *ctx->g;
  std::string p(pattern);
  int k = 0;
  if (p == "clique3" || p == "P0") k = 3;
  else if (p == "P13" || p == "clique4") k = 4;
  else if (p == "P14" || p == "clique5") k = 5;
  else if (p == "P15" || p == "clique6") k = 6;
  else if (p == "P16" || p == "clique7") k = 7;
  int kind = -1;
  if (k) kind = 0;
  else if (p == "P1") kind = 1;
  else if (p == "P2") kind = 2;
  else if (p == "induced-4-cycle") kind = 3;
  else if (p == "induced-diamond") kind = 4;
  else if (p == "induced-tailed-triangle") kind = 5;
  else if (p == "induced-4-path") kind = 6;
  else if (p == "induced-3-star") kind = 7;
  if (kind < 0) return -1;
  if (stride < 1) stride = 1;
  const eidType* rp = g.out_rowptr();
  const vidType* ci = g.out_colidx();
  const vidType n = g.V();
  vidType md = g.get_max_degree();
  for (vidType v = 0; v < n; ++v) md = std::max(md, g.get_degree(v));
  int64_t nslots = end > begin ? (end - begin + stride - 1) / stride : 0;
  uint64_t total = 0;
  auto t0 = std::chrono::steady_clock::now();
#pragma omp parallel num_threads(nthreads) reduction(+ : total)
  {
    Buf b(md);
    uint64_t c = 0;
#pragma omp for schedule(dynamic, 64)
    for (int64_t t = 0; t < nslots; ++t) {
      int64_t slot = begin + t * stride;
      vidType v0 = (vidType)(std::upper_bound(rp, rp + n + 1, slot) - rp - 1);
      vidType v1 = ci[slot];
      const vidType* n0 = g.adj_ptr(v0);
      vidType d0 = g.get_degree(v0);
      const vidType* n1 = g.adj_ptr(v1);
      vidType d1 = g.get_degree(v1);
      vidType* w = b.w[0].data();
      vidType tw = 0;
      switch (kind) {
        case 0:
          if (k == 3) {
            c += SetIntersection::get_num(n0, d0, n1, d1);
          } else {
            SetIntersection::ComputeCandidates(n0, d0, n1, d1, w, tw);
            c += clique_rec(g, w, tw, k - 3, b, 1);
          }
          break;
        case 1:  // P1
          if (v1 >= v0) break;
          for (vidType i = 0; i < d0 && n0[i] < v1; ++i) {
            vidType v2 = n0[i];
            vidType l1 = bounded_len(n1, d1, v0);
            vidType l2 = bounded_len(g.adj_ptr(v2), g.get_degree(v2), v0);
            c += SetIntersection::get_num(n1, l1, g.adj_ptr(v2), l2);
          }
          break;
        case 2:  // P2
          if (v1 >= v0) break;
          {
            uint64_t t2 = SetIntersection::get_num(n0, d0, n1, d1);
            c += t2 * (t2 - (t2 > 0 ? 1 : 0)) / 2;
          }
          break;
        case 3:  // induced 4-cycle
          if (v1 >= v0) break;
          for (vidType i = 0; i < d0 && n0[i] < v1; ++i) {
            vidType v2 = n0[i];
            if (std::binary_search(n1, n1 + d1, v2)) continue;  // v1 ~ v2
            vidType l1 = bounded_len(n1, d1, v0);
            vidType l2 = bounded_len(g.adj_ptr(v2), g.get_degree(v2), v0);
            SetIntersection::ComputeCandidates(n1, l1, g.adj_ptr(v2), l2, w, tw);
            VertexSet W(w, tw, -1);
            c += W.difference_ns(g.N(v0), INT32_MAX);
          }
          break;
        case 4:  // induced diamond
          if (v1 >= v0) break;
          SetIntersection::ComputeCandidates(n0, d0, n1, d1, w, tw);
          for (vidType i = 0; i < tw; ++i) {
            VertexSet rest(w + i + 1, tw - i - 1, -1);
            c += rest.difference_ns(g.N(w[i]), INT32_MAX);
          }
          break;
        case 5: {  // induced tailed triangle
          SetIntersection::ComputeCandidates(n0, d0, n1, d1, w, tw);
          vidType* b1 = b.w[1].data();
          VertexSet D1(b1, g.N(v0).difference_buf(b1, g.N(v1)), -1);  // N(v0) \ N(v1) \ {v1}
          for (vidType i = 0; i < tw; ++i) {
            if (w[i] <= v1) continue;
            c += D1.difference_ns(g.N(w[i]), INT32_MAX);
          }
          break;
        }
        case 6: {  // induced 4-path
          if (v1 >= v0) break;
          vidType* ba = b.w[1].data();
          vidType* bd = b.w[2].data();
          VertexSet A(ba, g.N(v0).difference_buf(ba, g.N(v1)), -1);
          VertexSet D(bd, g.N(v1).difference_buf(bd, g.N(v0)), -1);
          for (vidType i = 0; i < A.size(); ++i) c += D.difference_ns(g.N(A.data()[i]), INT32_MAX);
          break;
        }
        case 7: {  // induced 3-star
          vidType lo = (vidType)(std::upper_bound(n0, n0 + d0, v1) - n0);
          VertexSet hi(const_cast<vidType*>(n0) + lo, d0 - lo, -1);
          vidType* b1 = b.w[1].data();
          VertexSet D1(b1, hi.difference_buf(b1, g.N(v1)), -1);
          for (vidType i = 0; i < D1.size(); ++i) {
            VertexSet rest(D1.data() + i + 1, D1.size() - i - 1, -1);
            c += rest.difference_ns(g.N(D1.data()[i]), INT32_MAX);
          }
          break;
        }
      }
    }
    total += c;
  }
  auto t1 = std::chrono::steady_clock::now();
  *count = total;
  *seconds = std::chrono::duration<double>(t1 - t0).count();
  return 0;
}

}  // extern "C"
