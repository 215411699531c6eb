// Jupiter subgraph-counting ORACLE -- test infrastructure only.
//
// This file is the CPU restatement that the tests, the smoke check and the bench's
// cpu_baseline leg use to CHECK the CUDA path.  It is never linked into, loaded by or called
// from the product library (jupiter_b200/), which fails loudly without its CUDA extension.
//
// What it restates (reference paths are relative to the AnySparse/Jupiter tree):
//   * CSR construction and degree orientation: common/graph.cc:210-401 (rule at :229-230).
//   * The scalar merge set operations of VertexSet: include/VertexSet.h:53-160 and
//     common/VertexSet.cc:21-89 (difference excludes other.vid, the AutoMine convention).
//   * The fused splits fuse_set and dif_int_set, include/set_difference.cuh:248-475, and the
//     cached two-phase search they and the intersect templates use, with the other search
//     variants and the hash-bin intersection, include/search.cuh:5-203 and
//     include/operations.cuh:359-410.
//   * The per-pattern nested-loop plans of the message-passing kernels,
//     src/message_passing_gpu_kernels.cuh: P0 :64-102, P1 :104-186, P2 :188-252,
//     P3 :254-334, P4 :336-420, P5 :422-502, P6 :504-576, P7 :578-659, P8 :661-745,
//     P9 :747-825, P10 :827-918, P11 :920-1021, P12 :1023-1109, vsgm :1111-1206,
//     P13 :1208-1286, P14 :1288-1356, P15 :1358-1440, P16 :1442-1537; and the generic
//     k-clique level engine, src/config.h:39-58 with src/gpu_kernels_codegen.cuh:6-95,261-410.
//   * Vertex-induced 4-vertex plans built on set difference.  The reference has no
//     vertex-induced plan; these are defined here from the mathematics (each 4-vertex subset
//     whose induced subgraph is isomorphic to the pattern is counted once).
//
// Every set operation a plan issues adds |A'| + |B'| to `elements`, where A' and B' are the
// operand prefixes below the operation's upper bound (the whole lists when unbounded).  That
// sum is the algorithmic unit of the throughput and roofline figures.
//
// Parity pins: the reference repository ships no tests, fixtures or golden counts.  The
// plans here are pinned by brute force (orc_count_embeddings, orc_census4) on small graphs,
// by closed forms, and against the reference's own compiled set-operation code
// (oracle/ref/, built into oracle/_ref/).
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>
#include <omp.h>

#include "rmat_oracle.h"

typedef int32_t vid_t;
typedef int64_t eid_t;
typedef unsigned long long acc_t;

namespace {

struct Csr {
  vid_t n;
  const eid_t* rowptr;
  const vid_t* col;
  inline const vid_t* N(vid_t v) const { return col + rowptr[v]; }
  inline vid_t deg(vid_t v) const { return (vid_t)(rowptr[v + 1] - rowptr[v]); }
};

inline vid_t prefix_below(const vid_t* a, vid_t na, vid_t upper) {
  return (vid_t)(std::lower_bound(a, a + na, upper) - a);
}

// {x in A intersect B : x < upper}; VertexSet::intersect(other, upper), include/VertexSet.h:95-108.
inline vid_t isect(const vid_t* a, vid_t na, const vid_t* b, vid_t nb, vid_t upper, vid_t* out,
                   acc_t* elems) {
  vid_t la = prefix_below(a, na, upper), lb = prefix_below(b, nb, upper);
  *elems += (acc_t)la + (acc_t)lb;
  vid_t i = 0, j = 0, k = 0;
  while (i < la && j < lb) {
    vid_t x = a[i], y = b[j];
    if (x <= y) ++i;
    if (y <= x) ++j;
    if (x == y) {
      if (out) out[k] = x;
      ++k;
    }
  }
  return k;
}

// |A intersect B| excluding the listed ancestors; the (T* ancestor, int n) counting variant,
// include/set_intersect.cuh:474-507.
inline vid_t isect_except(const vid_t* a, vid_t na, const vid_t* b, vid_t nb, const vid_t* anc,
                          int nanc, acc_t* elems) {
  *elems += (acc_t)na + (acc_t)nb;
  vid_t i = 0, j = 0, k = 0;
  while (i < na && j < nb) {
    vid_t x = a[i], y = b[j];
    if (x <= y) ++i;
    if (y <= x) ++j;
    if (x == y) {
      bool ok = true;
      for (int t = 0; t < nanc; ++t) ok = ok && (x != anc[t]);
      if (ok) ++k;
    }
  }
  return k;
}

// {x in A : x not in B, x != excl, x < upper}; VertexSet::difference_buf with other.vid as
// the excluded id, common/VertexSet.cc:43-67.
inline vid_t diff(const vid_t* a, vid_t na, const vid_t* b, vid_t nb, vid_t excl, vid_t upper,
                  vid_t* out, acc_t* elems) {
  vid_t la = prefix_below(a, na, upper), lb = prefix_below(b, nb, upper);
  *elems += (acc_t)la + (acc_t)lb;
  vid_t i = 0, j = 0, k = 0;
  while (i < la) {
    vid_t x = a[i];
    while (j < lb && b[j] < x) ++j;
    bool in_b = (j < lb && b[j] == x);
    if (!in_b && x != excl) {
      if (out) out[k] = x;
      ++k;
    }
    ++i;
  }
  return k;
}

// Elements of a list greater than `lower` (plan-internal range restriction; not a set op).
inline vid_t first_above(const vid_t* a, vid_t na, vid_t lower) {
  return (vid_t)(std::upper_bound(a, a + na, lower) - a);
}

inline bool adjacent(const Csr& g, vid_t u, vid_t v) {
  const vid_t* a = g.N(u);
  vid_t d = g.deg(u);
  return std::binary_search(a, a + d, v);
}

struct Scratch {
  std::vector<vid_t> b[6];
  explicit Scratch(vid_t maxdeg) {
    for (auto& x : b) x.resize((size_t)maxdeg + 1);
  }
};

vid_t max_degree(const Csr& g) {
  vid_t m = 0;
  for (vid_t v = 0; v < g.n; ++v) m = std::max(m, g.deg(v));
  return m;
}

// Runs `body(v0, v1, scratch, count, elems)` over the root arcs (CSR slots) in
// [begin, end) taken every `stride`-th slot.  The reference's root edges are exactly the CSR
// slots (src/jupiter_gpm.cu:129-146, include/graph_gpu_nvs.h:362-372).
template <typename F>
void over_arcs(const Csr& g, eid_t begin, eid_t end, eid_t stride, int nthreads, acc_t* count,
               acc_t* elems, F body) {
  vid_t md = max_degree(g);
  // owner of each slot via binary search on rowptr
  acc_t c_tot = 0, e_tot = 0;
  eid_t nslots = (end - begin + stride - 1) / stride;
  if (nslots < 0) nslots = 0;
#pragma omp parallel num_threads(nthreads) reduction(+ : c_tot, e_tot)
  {
    Scratch s(md);
    acc_t c = 0, e = 0;
#pragma omp for schedule(dynamic, 64)
    for (eid_t t = 0; t < nslots; ++t) {
      eid_t slot = begin + t * stride;
      vid_t v0 = (vid_t)(std::upper_bound(g.rowptr, g.rowptr + g.n + 1, slot) - g.rowptr - 1);
      vid_t v1 = g.col[slot];
      body(v0, v1, s, c, e);
    }
    c_tot += c;
    e_tot += e;
  }
  *count = c_tot;
  *elems = e_tot;
}

const vid_t kNoBound = INT32_MAX;

// ---------------------------------------------------------------- reference plans
// P0 / triangle on the DAG: src/message_passing_gpu_kernels.cuh:64-102.
void plan_p0(const Csr& g, vid_t v0, vid_t v1, Scratch&, acc_t& c, acc_t& e) {
  c += isect(g.N(v0), g.deg(v0), g.N(v1), g.deg(v1), kNoBound, nullptr, &e);
}

// P1 (edge-induced 4-cycle): src/message_passing_gpu_kernels.cuh:104-186.
void plan_p1(const Csr& g, vid_t v0, vid_t v1, Scratch&, acc_t& c, acc_t& e) {
  if (v1 >= v0) return;
  const vid_t* n0 = g.N(v0);
  vid_t d0 = g.deg(v0);
  for (vid_t i = 0; i < d0; ++i) {
    vid_t v2 = n0[i];
    if (v2 >= v1) break;
    c += isect(g.N(v1), g.deg(v1), g.N(v2), g.deg(v2), v0, nullptr, &e);
  }
}

// P2 (edge-induced diamond): src/message_passing_gpu_kernels.cuh:188-252.  The warp loop
// sum over x in W of count_smaller(x, W) is the number of pairs in W, since W is sorted and
// duplicate free and every bound is a member of W (include/operations.cuh:80-124).
void plan_p2(const Csr& g, vid_t v0, vid_t v1, Scratch& s, acc_t& c, acc_t& e) {
  if (v1 >= v0) return;
  vid_t* w = s.b[0].data();
  vid_t t = isect(g.N(v0), g.deg(v0), g.N(v1), g.deg(v1), kNoBound, w, &e);
  for (vid_t i = 0; i < t; ++i) c += (acc_t)i;  // count_smaller(w[i], W) == i
}

// P3: src/message_passing_gpu_kernels.cuh:254-334.
void plan_p3(const Csr& g, vid_t v0, vid_t v1, Scratch& s, acc_t& c, acc_t& e) {
  vid_t* w = s.b[0].data();
  vid_t t = isect(g.N(v0), g.deg(v0), g.N(v1), g.deg(v1), kNoBound, w, &e);
  const vid_t* n0 = g.N(v0);
  vid_t d0 = g.deg(v0);
  for (vid_t i3 = 0; i3 < d0; ++i3) {
    vid_t v3 = n0[i3];
    if (v3 == v1) continue;
    const vid_t* n3 = g.N(v3);
    vid_t d3 = g.deg(v3);
    for (vid_t i = 0; i < t; ++i) {
      vid_t v2 = w[i];
      if (v2 <= v1 || v2 == v3 || v2 == v0) continue;
      for (vid_t i4 = 0; i4 < d3; ++i4) {
        vid_t v4 = n3[i4];
        if (v4 == v0 || v4 == v1 || v4 == v3 || v4 == v2) continue;
        ++c;
      }
    }
  }
}

// P4 (house): src/message_passing_gpu_kernels.cuh:336-420.
void plan_p4(const Csr& g, vid_t v0, vid_t v1, Scratch& s, acc_t& c, acc_t& e) {
  if (v1 >= v0) return;
  vid_t* w = s.b[0].data();
  vid_t* x = s.b[1].data();
  vid_t t = isect(g.N(v0), g.deg(v0), g.N(v1), g.deg(v1), kNoBound, w, &e);
  const vid_t* n1 = g.N(v1);
  vid_t d1 = g.deg(v1);
  for (vid_t i3 = 0; i3 < d1; ++i3) {
    vid_t v3 = n1[i3];
    if (v3 == v0) continue;
    vid_t tx = isect(g.N(v0), g.deg(v0), g.N(v3), g.deg(v3), kNoBound, x, &e);
    for (vid_t i = 0; i < t; ++i) {
      vid_t v2 = w[i];
      if (v3 == v2) continue;
      for (vid_t k = 0; k < tx; ++k) {
        vid_t y = x[k];
        if (y == v1 || y == v2) continue;
        ++c;
      }
    }
  }
}

// P5: src/message_passing_gpu_kernels.cuh:422-502.
void plan_p5(const Csr& g, vid_t v0, vid_t v1, Scratch& s, acc_t& c, acc_t& e) {
  if (v1 >= v0) return;
  vid_t* w = s.b[0].data();
  vid_t* x = s.b[1].data();
  vid_t t = isect(g.N(v0), g.deg(v0), g.N(v1), g.deg(v1), kNoBound, w, &e);
  for (vid_t i = 0; i < t; ++i) {
    vid_t v2 = w[i];
    vid_t tx = isect(w, t, g.N(v2), g.deg(v2), v2, x, &e);
    for (vid_t j = 0; j < t; ++j) {
      vid_t v4 = w[j];
      if (v2 == v4) continue;
      for (vid_t k = 0; k < tx; ++k)
        if (x[k] != v4) ++c;
    }
  }
}

// P6: src/message_passing_gpu_kernels.cuh:504-576.
void plan_p6(const Csr& g, vid_t v0, vid_t v1, Scratch& s, acc_t& c, acc_t& e) {
  if (v1 >= v0) return;
  vid_t* w = s.b[0].data();
  vid_t t = isect(g.N(v0), g.deg(v0), g.N(v1), g.deg(v1), kNoBound, w, &e);
  vid_t anc[2] = {v0, v1};
  for (vid_t i2 = 0; i2 < t; ++i2) {
    vid_t v2 = w[i2];
    for (vid_t i3 = 0; i3 < i2; ++i3) {
      vid_t v3 = w[i3];
      c += isect_except(g.N(v2), g.deg(v2), g.N(v3), g.deg(v3), anc, 2, &e);
    }
  }
}

// P7 (gem): src/message_passing_gpu_kernels.cuh:578-659.  Every arc is a root.
void plan_p7(const Csr& g, vid_t v0, vid_t v1, Scratch& s, acc_t& c, acc_t& e) {
  vid_t* w = s.b[0].data();
  vid_t* x = s.b[1].data();
  vid_t t = isect(g.N(v0), g.deg(v0), g.N(v1), g.deg(v1), kNoBound, w, &e);
  for (vid_t i2 = 0; i2 < t; ++i2) {
    vid_t v2 = w[i2];
    if (v2 <= v1) continue;
    vid_t tx = isect(g.N(v0), g.deg(v0), g.N(v2), g.deg(v2), kNoBound, x, &e);
    for (vid_t k = 0; k < tx; ++k) {
      vid_t v4 = x[k];
      if (v1 == v4) continue;
      for (vid_t j = 0; j < t; ++j) {
        vid_t y = w[j];
        if (y == v4 || y == v2) continue;
        ++c;
      }
    }
  }
}

// P8 (4-wheel): src/message_passing_gpu_kernels.cuh:661-745.  Every arc is a root.
void plan_p8(const Csr& g, vid_t v0, vid_t v1, Scratch& s, acc_t& c, acc_t& e) {
  vid_t* w = s.b[0].data();
  vid_t* x = s.b[1].data();
  vid_t t = isect(g.N(v0), g.deg(v0), g.N(v1), g.deg(v1), kNoBound, w, &e);
  for (vid_t i2 = 0; i2 < t; ++i2) {
    vid_t v2 = w[i2];
    if (v2 >= v1) continue;
    vid_t tx = isect(g.N(v0), g.deg(v0), g.N(v2), g.deg(v2), kNoBound, x, &e);
    for (vid_t k = 0; k < tx; ++k) {
      vid_t v3 = x[k];
      if (v3 >= v1) continue;
      c += isect(w, t, g.N(v3), g.deg(v3), v2, nullptr, &e);
    }
  }
}

// P9 (K5 minus an edge): src/message_passing_gpu_kernels.cuh:747-825.
void plan_p9(const Csr& g, vid_t v0, vid_t v1, Scratch& s, acc_t& c, acc_t& e) {
  if (v1 <= v0) return;
  vid_t* w = s.b[0].data();
  vid_t* x = s.b[1].data();
  vid_t t = isect(g.N(v0), g.deg(v0), g.N(v1), g.deg(v1), kNoBound, w, &e);
  for (vid_t i2 = 0; i2 < t; ++i2) {
    vid_t v2 = w[i2];
    if (v2 <= v1) continue;
    vid_t tx = isect(w, t, g.N(v2), g.deg(v2), kNoBound, x, &e);
    for (vid_t k = 0; k < tx; ++k) c += (acc_t)k;  // count_smaller(x[k], X) == k
  }
}

// P10: src/message_passing_gpu_kernels.cuh:827-918.  Every arc is a root.
void plan_p10(const Csr& g, vid_t v0, vid_t v1, Scratch& s, acc_t& c, acc_t& e) {
  vid_t* w = s.b[0].data();
  vid_t* x = s.b[1].data();
  vid_t* y = s.b[2].data();
  vid_t t = isect(g.N(v0), g.deg(v0), g.N(v1), g.deg(v1), kNoBound, w, &e);
  for (vid_t i2 = 0; i2 < t; ++i2) {
    vid_t v2 = w[i2];
    vid_t tx = isect(g.N(v0), g.deg(v0), g.N(v2), g.deg(v2), kNoBound, x, &e);
    for (vid_t k = 0; k < tx; ++k) {
      vid_t v3 = x[k];
      if (v3 <= v1) continue;
      vid_t ty = isect(g.N(v0), g.deg(v0), g.N(v3), g.deg(v3), kNoBound, y, &e);
      for (vid_t i4 = 0; i4 < t; ++i4) {
        vid_t v4 = w[i4];
        if (v4 == v2 || v4 == v1 || v4 == v3) continue;
        for (vid_t q = 0; q < ty; ++q) {
          vid_t z = y[q];
          if (z == v4 || z == v1 || z == v2 || z == v3) continue;
          ++c;
        }
      }
    }
  }
}

// P11: src/message_passing_gpu_kernels.cuh:920-1021.
void plan_p11(const Csr& g, vid_t v0, vid_t v1, Scratch& s, acc_t& c, acc_t& e) {
  if (v1 <= v0) return;
  vid_t* w = s.b[0].data();
  vid_t* x = s.b[1].data();
  vid_t* z = s.b[2].data();
  vid_t t = isect(g.N(v0), g.deg(v0), g.N(v1), g.deg(v1), kNoBound, w, &e);
  for (vid_t i2 = 0; i2 < t; ++i2) {
    vid_t v2 = w[i2];
    if (v2 <= v1) continue;
    vid_t tx = isect(g.N(v0), g.deg(v0), g.N(v2), g.deg(v2), kNoBound, x, &e);
    vid_t tz = isect(g.N(v1), g.deg(v1), g.N(v2), g.deg(v2), kNoBound, z, &e);
    for (vid_t i3 = 0; i3 < t; ++i3) {
      vid_t v3 = w[i3];
      if (v3 == v2 || v3 == v1 || v3 == v0) continue;
      for (vid_t i4 = 0; i4 < tx; ++i4) {
        vid_t v4 = x[i4];
        if (v4 == v3 || v4 == v2 || v4 == v1) continue;
        for (vid_t q = 0; q < tz; ++q) {
          vid_t y = z[q];
          if (y == v4 || y == v1 || y == v2 || y == v3 || y == v0) continue;
          ++c;
        }
      }
    }
  }
}

// P12: src/message_passing_gpu_kernels.cuh:1023-1109.
void plan_p12(const Csr& g, vid_t v0, vid_t v1, Scratch& s, acc_t& c, acc_t& e) {
  if (v1 <= v0) return;
  vid_t* w = s.b[0].data();
  vid_t* x = s.b[1].data();
  vid_t t = isect(g.N(v0), g.deg(v0), g.N(v1), g.deg(v1), kNoBound, w, &e);
  for (vid_t i2 = 0; i2 < t; ++i2) {
    vid_t v2 = w[i2];
    vid_t tx = isect(w, t, g.N(v2), g.deg(v2), kNoBound, x, &e);
    for (vid_t i3 = 0; i3 < tx; ++i3) {
      vid_t v3 = x[i3];
      for (vid_t i4 = i3 + 1; i4 < tx; ++i4) {
        vid_t v4 = x[i4];
        for (vid_t q = 0; q < t; ++q) {
          vid_t y = w[q];
          if (y == v4 || y == v1 || y == v2 || y == v3 || y == v0) continue;
          ++c;
        }
      }
    }
  }
}

// vsgm_last_pattern: src/message_passing_gpu_kernels.cuh:1111-1206.
void plan_vsgm(const Csr& g, vid_t v0, vid_t v1, Scratch& s, acc_t& c, acc_t& e) {
  if (v1 <= v0) return;
  vid_t* w = s.b[0].data();
  vid_t* z = s.b[1].data();
  vid_t t = isect(g.N(v0), g.deg(v0), g.N(v1), g.deg(v1), kNoBound, w, &e);
  const vid_t* n0 = g.N(v0);
  vid_t d0 = g.deg(v0);
  for (vid_t i2 = 0; i2 < d0; ++i2) {
    vid_t v2 = n0[i2];
    if (v2 == v1) continue;
    vid_t tz = isect(g.N(v1), g.deg(v1), g.N(v2), g.deg(v2), kNoBound, z, &e);
    for (vid_t i5 = 0; i5 < tz; ++i5) {
      vid_t v5 = z[i5];
      if (v5 == v0) continue;
      for (vid_t i3 = 0; i3 < t; ++i3) {
        vid_t v3 = w[i3];
        if (v3 == v2 || v3 == v1 || v3 == v0 || v3 == v5) continue;
        for (vid_t q = 0; q < t; ++q) {
          vid_t y = w[q];
          if (y == v0 || y == v1 || y == v2 || y <= v3 || y == v5) continue;
          ++c;
        }
      }
    }
  }
}

// k-clique on the DAG, P13 (k=4) :1208-1286, P14 (k=5) :1288-1356, P15 (k=6) :1358-1440,
// P16 (k=7) :1442-1537; the level engine src/config.h:39-58 is the same recursion: level 1
// W = N+(v0) & N+(v1); each deeper level intersects the current candidate set with N+(v);
// the last level only counts.
void clique_level(const Csr& g, const vid_t* cand, vid_t nc, int remaining, Scratch& s,
                  int depth, acc_t& c, acc_t& e) {
  if (remaining == 1) {
    for (vid_t i = 0; i < nc; ++i) {
      vid_t v = cand[i];
      c += isect(cand, nc, g.N(v), g.deg(v), kNoBound, nullptr, &e);
    }
    return;
  }
  vid_t* next = s.b[depth].data();
  for (vid_t i = 0; i < nc; ++i) {
    vid_t v = cand[i];
    vid_t t = isect(cand, nc, g.N(v), g.deg(v), kNoBound, next, &e);
    clique_level(g, next, t, remaining - 1, s, depth + 1, c, e);
  }
}

void plan_clique(const Csr& g, int k, vid_t v0, vid_t v1, Scratch& s, acc_t& c, acc_t& e) {
  vid_t* w = s.b[0].data();
  vid_t t = isect(g.N(v0), g.deg(v0), g.N(v1), g.deg(v1), kNoBound, w, &e);
  if (k == 3) {
    c += t;
    return;
  }
  clique_level(g, w, t, k - 3, s, 1, c, e);
}

// ---------------------------------------------------------------- vertex-induced plans
// No reference implementation exists; each induced copy is counted exactly once.
// Induced 4-cycle rooted at its largest vertex v0 with v1, v2 its cycle neighbours
// (v2 < v1 < v0, v1 and v2 non-adjacent) and the opposite vertex v3 < v0, v3 not adjacent to v0.
void plan_i_c4(const Csr& g, vid_t v0, vid_t v1, Scratch& s, acc_t& c, acc_t& e) {
  if (v1 >= v0) return;
  vid_t* w = s.b[0].data();
  const vid_t* n0 = g.N(v0);
  vid_t d0 = g.deg(v0);
  for (vid_t i = 0; i < d0; ++i) {
    vid_t v2 = n0[i];
    if (v2 >= v1) break;
    if (adjacent(g, v1, v2)) continue;
    vid_t t = isect(g.N(v1), g.deg(v1), g.N(v2), g.deg(v2), v0, w, &e);
    c += diff(w, t, n0, d0, v0, kNoBound, nullptr, &e);
  }
}

// Induced diamond: the adjacent degree-3 pair is the root edge (v1 < v0); the two
// degree-2 vertices x < y lie in W = N(v0) & N(v1) and are not adjacent.
void plan_i_diamond(const Csr& g, vid_t v0, vid_t v1, Scratch& s, acc_t& c, acc_t& e) {
  if (v1 >= v0) return;
  vid_t* w = s.b[0].data();
  vid_t t = isect(g.N(v0), g.deg(v0), g.N(v1), g.deg(v1), kNoBound, w, &e);
  for (vid_t i = 0; i < t; ++i) {
    vid_t x = w[i];
    vid_t lo = i + 1;
    c += diff(w + lo, t - lo, g.N(x), g.deg(x), x, kNoBound, nullptr, &e);
  }
}

// Induced tailed triangle: the degree-3 vertex v0 is the root, the arc (v0, v1) names one
// triangle partner; the other partner v2 > v1 is in N(v0) & N(v1); the tail t is in
// N(v0) \ N(v1) \ N(v2), t not in {v1, v2}.
void plan_i_tailed(const Csr& g, vid_t v0, vid_t v1, Scratch& s, acc_t& c, acc_t& e) {
  vid_t* w = s.b[0].data();
  vid_t* d1 = s.b[1].data();
  vid_t t = isect(g.N(v0), g.deg(v0), g.N(v1), g.deg(v1), kNoBound, w, &e);
  vid_t start = first_above(w, t, v1);
  if (start >= t) return;
  // D1 = N(v0) \ N(v1) \ {v1}
  vid_t nd1 = diff(g.N(v0), g.deg(v0), g.N(v1), g.deg(v1), v1, kNoBound, d1, &e);
  for (vid_t i = start; i < t; ++i) {
    vid_t v2 = w[i];
    c += diff(d1, nd1, g.N(v2), g.deg(v2), v2, kNoBound, nullptr, &e);
  }
}

// Induced 4-path a-b-c-d: the middle edge (b, c) with c < b is the root arc (v0 = b,
// v1 = c); A = N(b) \ N(c) \ {c}, D = N(c) \ N(b) \ {b}, and d not adjacent to a.
void plan_i_path4(const Csr& g, vid_t v0, vid_t v1, Scratch& s, acc_t& c, acc_t& e) {
  if (v1 >= v0) return;
  vid_t* a = s.b[0].data();
  vid_t* d = s.b[1].data();
  vid_t na = diff(g.N(v0), g.deg(v0), g.N(v1), g.deg(v1), v1, kNoBound, a, &e);
  if (na == 0) return;
  vid_t nd = diff(g.N(v1), g.deg(v1), g.N(v0), g.deg(v0), v0, kNoBound, d, &e);
  for (vid_t i = 0; i < na; ++i) {
    vid_t x = a[i];
    c += diff(d, nd, g.N(x), g.deg(x), x, kNoBound, nullptr, &e);
  }
}

// Induced 3-star: the centre v0 is the root, the arc (v0, v1) names the smallest leaf;
// the leaves v1 < y < z are pairwise non-adjacent.
void plan_i_star3(const Csr& g, vid_t v0, vid_t v1, Scratch& s, acc_t& c, acc_t& e) {
  vid_t* d1 = s.b[0].data();
  const vid_t* n0 = g.N(v0);
  vid_t d0 = g.deg(v0);
  vid_t lo = first_above(n0, d0, v1);
  // D1 = {y in N(v0) : y > v1} \ N(v1)
  vid_t nd1 = diff(n0 + lo, d0 - lo, g.N(v1), g.deg(v1), v1, kNoBound, d1, &e);
  for (vid_t i = 0; i < nd1; ++i) {
    vid_t y = d1[i];
    vid_t lo2 = i + 1;
    c += diff(d1 + lo2, nd1 - lo2, g.N(y), g.deg(y), y, kNoBound, nullptr, &e);
  }
}

typedef void (*PlanFn)(const Csr&, vid_t, vid_t, Scratch&, acc_t&, acc_t&);

struct PlanEntry {
  const char* name;
  PlanFn fn;
  int clique_k;  // >0: k-clique recursion on the DAG
};

const PlanEntry kPlans[] = {
    {"P0", plan_p0, 0},          {"P1", plan_p1, 0},       {"P2", plan_p2, 0},
    {"P3", plan_p3, 0},          {"P4", plan_p4, 0},       {"P5", plan_p5, 0},
    {"P6", plan_p6, 0},          {"P7", plan_p7, 0},       {"P8", plan_p8, 0},
    {"P9", plan_p9, 0},          {"P10", plan_p10, 0},     {"P11", plan_p11, 0},
    {"P12", plan_p12, 0},        {"vsgm_last_pattern", plan_vsgm, 0},
    {"P13", nullptr, 4},         {"P14", nullptr, 5},      {"P15", nullptr, 6},
    {"P16", nullptr, 7},         {"clique3", nullptr, 3},  {"clique8", nullptr, 8},
    {"induced-4-cycle", plan_i_c4, 0},     {"induced-diamond", plan_i_diamond, 0},
    {"induced-tailed-triangle", plan_i_tailed, 0}, {"induced-4-path", plan_i_path4, 0},
    {"induced-3-star", plan_i_star3, 0},
};

}  // namespace

extern "C" {

// Edges of an R-MAT graph (same generator definition as the product's; restated in
// rmat_oracle.h).  Returns the number of edges written (edges with no valid draw are
// dropped).
int64_t orc_rmat_edges(int64_t n, int64_t num_edges, double a, double b, double c,
                       uint64_t seed, int32_t* src, int32_t* dst, int nthreads) {
  orc::RmatSpec p = orc::make_spec(n, num_edges, a, b, c, seed);
  std::vector<uint8_t> ok((size_t)num_edges);
#pragma omp parallel for num_threads(nthreads) schedule(static)
  for (int64_t i = 0; i < num_edges; ++i) {
    int32_t u, v;
    ok[i] = orc::edge(p, (uint64_t)i, &u, &v) ? 1 : 0;
    src[i] = u;
    dst[i] = v;
  }
  int64_t k = 0;
  for (int64_t i = 0; i < num_edges; ++i)
    if (ok[i]) {
      src[k] = src[i];
      dst[k] = dst[i];
      ++k;
    }
  return k;
}

// Undirected CSR from an edge list: both directions, self-loops dropped, rows sorted and
// deduplicated.  rowptr has n+1 entries; col must hold 2*ne entries.  Returns the arc count.
int64_t orc_build_csr(int32_t n, int64_t ne, const int32_t* src, const int32_t* dst,
                      int64_t* rowptr, int32_t* col) {
  std::vector<int64_t> cnt((size_t)n + 1, 0);
  for (int64_t i = 0; i < ne; ++i) {
    if (src[i] == dst[i]) continue;
    cnt[src[i] + 1]++;
    cnt[dst[i] + 1]++;
  }
  for (int32_t v = 0; v < n; ++v) cnt[v + 1] += cnt[v];
  std::vector<int64_t> pos(cnt.begin(), cnt.end() - 1);
  std::vector<int32_t> tmp((size_t)cnt[n]);
  for (int64_t i = 0; i < ne; ++i) {
    if (src[i] == dst[i]) continue;
    tmp[pos[src[i]]++] = dst[i];
    tmp[pos[dst[i]]++] = src[i];
  }
  int64_t m = 0;
  rowptr[0] = 0;
  for (int32_t v = 0; v < n; ++v) {
    auto b = tmp.begin() + cnt[v], en = tmp.begin() + cnt[v + 1];
    std::sort(b, en);
    auto last = std::unique(b, en);
    for (auto it = b; it != last; ++it) col[m++] = *it;
    rowptr[v + 1] = m;
  }
  return m;
}

// Degree orientation, common/graph.cc:210-401: keep u->v iff deg(v) > deg(u), or the
// degrees tie and v > u (rule at :229-230).  dag_col must hold rowptr[n] entries.
int64_t orc_orient(int32_t n, const int64_t* rowptr, const int32_t* col, int64_t* dag_rowptr,
                   int32_t* dag_col) {
  dag_rowptr[0] = 0;
  int64_t m = 0;
  for (int32_t u = 0; u < n; ++u) {
    int64_t du = rowptr[u + 1] - rowptr[u];
    for (int64_t k = rowptr[u]; k < rowptr[u + 1]; ++k) {
      int32_t v = col[k];
      int64_t dv = rowptr[v + 1] - rowptr[v];
      if (dv > du || (dv == du && v > u)) dag_col[m++] = v;
    }
    dag_rowptr[u + 1] = m;
  }
  return m;
}

// Runs a plan over root arcs [root_begin, root_end) with stride (a full run is 0, m, 1).
// Pattern names: P0..P16, vsgm_last_pattern, clique3, clique8, induced-4-cycle,
// induced-diamond, induced-tailed-triangle, induced-4-path, induced-3-star.  The caller
// passes the DAG for P0, P13..P16 and the cliques, the symmetric graph otherwise.
// Returns 0, or -1 for an unknown pattern.
int orc_count(const char* pattern, int32_t n, const int64_t* rowptr, const int32_t* col,
              int64_t root_begin, int64_t root_end, int64_t root_stride, int nthreads,
              uint64_t* count, uint64_t* elements) {
  Csr g{n, rowptr, col};
  const PlanEntry* pe = nullptr;
  for (const auto& p : kPlans)
    if (std::string(p.name) == pattern) pe = &p;
  if (!pe) return -1;
  if (root_stride < 1) root_stride = 1;
  acc_t c = 0, e = 0;
  if (pe->clique_k > 0) {
    int k = pe->clique_k;
    over_arcs(g, root_begin, root_end, root_stride, nthreads, &c, &e,
              [&](vid_t v0, vid_t v1, Scratch& s, acc_t& cc, acc_t& ee) {
                plan_clique(g, k, v0, v1, s, cc, ee);
              });
  } else {
    PlanFn fn = pe->fn;
    over_arcs(g, root_begin, root_end, root_stride, nthreads, &c, &e,
              [&](vid_t v0, vid_t v1, Scratch& s, acc_t& cc, acc_t& ee) {
                fn(g, v0, v1, s, cc, ee);
              });
  }
  *count = c;
  *elements = e;
  return 0;
}

// General k-clique count (k >= 3) on a DAG.
int orc_count_clique(int k, int32_t n, const int64_t* rowptr, const int32_t* col, int nthreads,
                     uint64_t* count, uint64_t* elements) {
  if (k < 3 || k > 8) return -1;
  Csr g{n, rowptr, col};
  acc_t c = 0, e = 0;
  over_arcs(g, 0, rowptr[n], 1, nthreads, &c, &e,
            [&](vid_t v0, vid_t v1, Scratch& s, acc_t& cc, acc_t& ee) {
              plan_clique(g, k, v0, v1, s, cc, ee);
            });
  *count = c;
  *elements = e;
  return 0;
}

// Brute-force vertex-induced census of the six connected 4-vertex graphlets by enumerating
// every 4-subset (tiny graphs only).  out[0..5] = 3-star, 4-path, tailed triangle, 4-cycle,
// diamond, 4-clique.
// The reference's cached two-phase membership search, binary_search_2phase
// (include/search.cuh:70-105) with width 32, its CTA form binary_search_2phase_cta (:107-140)
// with width 256, and the hit index the marking form binary_search_2phase_map (:164-203)
// records.  The caller caches list[k * size / width] for k < width; phase 1 bisects the cache,
// phase 2 searches the list between the two bracketing pivots.  For each key: found[i] and
// marked[i] (the list index the map form marks, -1 when not found).  The tests run it over
// every key of many lists to pin that it is exact, so a plain lookup gives the same answers.
void orc_search_2phase(const int32_t* list, int32_t size, int32_t width, const int32_t* keys,
                       int64_t nkeys, uint8_t* found, int32_t* marked) {
  std::vector<int32_t> cache((size_t)width);
  for (int k = 0; k < width; ++k) cache[k] = list[(int64_t)k * size / width];
  for (int64_t i = 0; i < nkeys; ++i) {
    const int32_t key = keys[i];
    found[i] = 0;
    marked[i] = -1;
    int bottom = 0, top = width, mid = 0;
    bool hit = false;
    while (top > bottom + 1) {
      mid = (top + bottom) / 2;
      const int32_t y = cache[mid];
      if (key == y) {
        hit = true;
        marked[i] = (int32_t)((int64_t)mid * size / width);
        break;
      }
      if (key < y) top = mid;
      if (key > y) bottom = mid;
    }
    if (!hit) {
      int lo = (int)((int64_t)bottom * size / width);
      int hi = (int)((int64_t)top * size / width) - 1;
      while (hi >= lo) {
        mid = (hi + lo) / 2;
        const int32_t y = list[mid];
        if (key == y) {
          hit = true;
          marked[i] = mid;
          break;
        }
        if (key < y) hi = mid - 1;
        else lo = mid + 1;
      }
    }
    found[i] = hit ? 1 : 0;
  }
}

// count_smaller (include/operations.cuh:80-124), the rank of `bound` in a sorted list as P2
// and P9 use it (src/message_passing_gpu_kernels.cuh:241, 815), for one warp: lane 0 narrows
// [begin, end) while it spans more than 128 elements (returning mid on a hit, and moving end to
// mid - 1 on a miss above), then the warp counts the elements below the bound 32 at a time until
// a chunk is not all below.
uint32_t orc_count_smaller(int32_t bound, const int32_t* a, int32_t size) {
  if (size == 0) return 0;
  unsigned begin = 0, end = (unsigned)size;
  int l = 0, r = size, mid = 0;
  while (r - l > 32 * 4) {
    mid = l + (r - l) / 2;
    const int32_t value = a[mid];
    if (value == bound) return (uint32_t)mid;
    if (value < bound) begin = mid + 1;
    else end = mid - 1;
    l = (int)begin;
    r = (int)end;
  }
  unsigned count = begin;
  for (int base = l; base < r; base += 32) {
    const int lanes = std::min(32, r - base);
    unsigned below = 0;
    for (int q = 0; q < lanes; ++q) below += a[base + q] < bound ? 1u : 0u;
    count += below;
    if (below != 32u) break;  // the ballot is not the full mask
  }
  return count;
}

// binary_search_bound (include/search.cuh:142-162, unused by the reference's plans): the
// position the search ends at for each key, as the reference computes it.
void orc_search_bound(const int32_t* list, int32_t size, const int32_t* keys, int64_t nkeys,
                      int32_t* pos) {
  for (int64_t i = 0; i < nkeys; ++i) {
    const int32_t key = keys[i];
    int l = 0, r = size - 1, mid = 0;
    int32_t value = 0;
    while (r >= l) {
      mid = l + (r - l) / 2;
      value = list[mid];
      if (value == key) break;
      if (value < key) l = mid + 1;
      else r = mid - 1;
    }
    pos[i] = value >= key ? mid : mid + 1;
  }
}

// intersect_warp_hindex (include/operations.cuh:359-410, unused by the reference's plans):
// |A & B| by hashing the shorter list into 128 bins by id mod 128 (1,024 slots each) and
// probing every key of the longer list with a linear scan of its bin (linear_search,
// include/search.cuh:15-29).  Returns the count, or -1 when a bin would overflow its 1,024
// slots (the reference then writes past the bin).
int64_t orc_hindex_count(const int32_t* a, int32_t na, const int32_t* b, int32_t nb) {
  constexpr int kBuckets = 128, kBucketSize = 1024;
  const int32_t* lookup = a;
  const int32_t* search = b;
  int32_t nl = na, ns = nb;
  if (na > nb) {
    lookup = b;
    search = a;
    nl = nb;
    ns = na;
  }
  std::vector<int32_t> bins((size_t)kBuckets * kBucketSize);
  std::vector<int32_t> count(kBuckets, 0);
  for (int32_t i = 0; i < nl; ++i) {
    const int32_t key = lookup[i] % kBuckets;
    if (count[key] == kBucketSize) return -1;
    bins[(size_t)count[key]++ * kBuckets + key] = lookup[i];
  }
  int64_t c = 0;
  for (int32_t i = 0; i < ns; ++i) {
    const int32_t v = search[i], key = v % kBuckets;
    for (int32_t q = 0; q < count[key]; ++q)
      if (bins[(size_t)q * kBuckets + key] == v) {
        ++c;
        break;
      }
  }
  return c;
}

// fuse_set (include/set_difference.cuh:248-343): c = A \ B, d = A & B, e = B \ A of two sorted
// lists; returns |A & B|.  As the reference's wrapper (:338-343) does, an empty A or B returns
// 0 and writes nothing.  The reference searches the shorter list's keys in the longer one and
// marks the hits in a map to emit the longer list's remainder; one merge gives the same sets.
int32_t orc_fuse_set(const int32_t* a, int32_t na, const int32_t* b, int32_t nb, int32_t* c,
                     int32_t* d, int32_t* e) {
  if (na == 0 || nb == 0) return 0;
  int32_t i = 0, j = 0, nc = 0, nd = 0, ne = 0;
  while (i < na || j < nb) {
    if (j == nb || (i < na && a[i] < b[j])) {
      c[nc++] = a[i++];
    } else if (i == na || b[j] < a[i]) {
      e[ne++] = b[j++];
    } else {
      d[nd++] = a[i];
      ++i;
      ++j;
    }
  }
  return nd;
}

// dif_int_set (include/set_difference.cuh:346-413): keys x of A with x < upper and x not in B
// go to c, every other key of A to d (keys at or above upper included, the active branch at
// :379-382); returns |c|.  upper == INT32_MAX is the unbounded form (:415-475).  An empty A or
// B returns 0 and writes nothing (:407-413).
int32_t orc_dif_int_set(const int32_t* a, int32_t na, const int32_t* b, int32_t nb,
                        int32_t upper, int32_t* c, int32_t* d) {
  if (na == 0 || nb == 0) return 0;
  int32_t j = 0, nc = 0, nd = 0;
  for (int32_t i = 0; i < na; ++i) {
    const int32_t x = a[i];
    while (j < nb && b[j] < x) ++j;
    const bool in_b = j < nb && b[j] == x;
    const bool below = upper == INT32_MAX || x < upper;
    if (below && !in_b) c[nc++] = x;
    else d[nd++] = x;
  }
  return nc;
}

int orc_census4(int32_t n, const int64_t* rowptr, const int32_t* col, uint64_t* out) {
  if (n > 400) return -1;
  std::vector<uint8_t> adj((size_t)n * n, 0);
  for (int32_t u = 0; u < n; ++u)
    for (int64_t k = rowptr[u]; k < rowptr[u + 1]; ++k) adj[(size_t)u * n + col[k]] = 1;
  for (int i = 0; i < 6; ++i) out[i] = 0;
  for (int32_t a = 0; a < n; ++a)
    for (int32_t b = a + 1; b < n; ++b)
      for (int32_t c = b + 1; c < n; ++c)
        for (int32_t d = c + 1; d < n; ++d) {
          int32_t v[4] = {a, b, c, d};
          int deg[4] = {0, 0, 0, 0}, m = 0;
          for (int i = 0; i < 4; ++i)
            for (int j = i + 1; j < 4; ++j)
              if (adj[(size_t)v[i] * n + v[j]]) {
                ++deg[i];
                ++deg[j];
                ++m;
              }
          int dmax = 0, dmin = 4;
          for (int i = 0; i < 4; ++i) {
            dmax = std::max(dmax, deg[i]);
            dmin = std::min(dmin, deg[i]);
          }
          if (dmin == 0) continue;  // disconnected (an isolated vertex)
          if (m == 3) {
            if (dmax == 3) out[0]++;            // 3-star
            else out[1]++;                      // 4-path (a 3-edge, 4-vertex graph with
                                                // no isolated vertex and no degree 3 is P4)
          } else if (m == 4) {
            if (dmax == 3) out[2]++;            // tailed triangle
            else out[3]++;                      // 4-cycle
          } else if (m == 5) {
            out[4]++;                           // diamond
          } else if (m == 6) {
            out[5]++;                           // 4-clique
          }
        }
  return 0;
}

// Number of injective maps phi: V(H) -> V(G) with every edge of H mapped onto an edge of G
// (tiny graphs only).  H has k vertices and `ne` edges given as pairs in `hedges`.
uint64_t orc_count_embeddings(int k, int ne, const int32_t* hedges, int32_t n,
                              const int64_t* rowptr, const int32_t* col) {
  std::vector<uint8_t> adj((size_t)n * n, 0);
  for (int32_t u = 0; u < n; ++u)
    for (int64_t q = rowptr[u]; q < rowptr[u + 1]; ++q) adj[(size_t)u * n + col[q]] = 1;
  std::vector<std::vector<int>> back(k);  // edges to earlier pattern vertices
  for (int i = 0; i < ne; ++i) {
    int a = hedges[2 * i], b = hedges[2 * i + 1];
    if (a < b) back[b].push_back(a);
    else back[a].push_back(b);
  }
  std::vector<int32_t> phi(k, -1);
  uint64_t total = 0;
  std::vector<uint8_t> used(n, 0);
  // iterative DFS
  std::vector<int32_t> next(k, 0);
  int lvl = 0;
  next[0] = 0;
  while (lvl >= 0) {
    if (lvl == k) {
      ++total;
      --lvl;
      used[phi[lvl]] = 0;
      continue;
    }
    bool placed = false;
    while (next[lvl] < n) {
      int32_t x = next[lvl]++;
      if (used[x]) continue;
      bool ok = true;
      for (int p : back[lvl])
        if (!adj[(size_t)phi[p] * n + x]) {
          ok = false;
          break;
        }
      if (!ok) continue;
      phi[lvl] = x;
      used[x] = 1;
      placed = true;
      break;
    }
    if (placed) {
      ++lvl;
      if (lvl < k) next[lvl] = 0;
    } else {
      --lvl;
      if (lvl >= 0) used[phi[lvl]] = 0;
    }
  }
  return total;
}

}  // extern "C"
