// Device building blocks of the vertex-rooted local-bitmap k-clique count, shared by the
// plain per-query kernels (clique.cu) and the batched persistent kernel (batch.cu).
//
// For a root u with out-degree d, L = N+(u) (sorted) and the bitmap rows
//     R_i bit j  <=>  L[j] in N+(L[i])
// are the level-1 sets of the reference's edge-rooted plans (W of arc (u, L[i]));
// K_k(u) = sum_i C_{k-3}(R_i) with C_0(m) = popc(m), C_t(m) = sum_{j in m} C_{t-1}(m & R_j).
//
// Modes of the k = 3 root kernels:
//   ETRI   every triangle adds one to each of its three DAG arcs in tri[] (edge triangles);
//   PAIRS  ETRI whose adds return the old value; an add of k to a counter holding o creates
//          k*o + C(k, 2) new pairs of triangles on that edge, so the sum over all adds is
//          sum_e C(t_e, 2) -- the diamond count -- in one pass (tri[] starts at zero).
//   TT     (k = 4, with ETRI and PAIRS) the vertex-induced tailed-triangle count in the same
//          pass: I(TT) = N(TT) - 4 N(diamond) + 12 K4, where N(TT) = sum over triangles of
//          (d_a - 2) + (d_b - 2) + (d_c - 2) with d the symmetric degree (srow).  Each root
//          returns 12 K4 - 4 pairs + its triangles' degree terms in wrapping 64-bit
//          arithmetic; the sum over all roots is the exact (non-negative) count.
//   The root kernels return the pair count in PAIRS mode, the TT value in TT mode and the
//   clique count otherwise.

#pragma once
#include "jgpm_internal.h"
#include "setops.cuh"

namespace jgpm {

// Pairs of triangles created on one edge by adding k to a counter that held o.
__device__ __forceinline__ acc_t pair_gain(unsigned o, unsigned k) {
  return (acc_t)k * (acc_t)o + (acc_t)k * (acc_t)(k - 1) / 2;
}

// Symmetric degree minus two (the tailed-triangle degree term of a triangle vertex).
__device__ __forceinline__ acc_t tt_deg(const eid_t* srow, vid_t v) {
  return (acc_t)(srow[v + 1] - srow[v]) - 2ull;
}

constexpr int kRangeCut = 32;  // restrict a row to [L0, Ld-1] when longer than this
// Rows of at least this many elements (after the range cut) are scanned by a whole warp, one
// row at a time; shorter ones are flattened over the lanes.
constexpr int kLongRow = 32;

// Largest power of two <= n (0 for n <= 0).
__device__ __forceinline__ int top_pow2(int n) { return n > 0 ? 1 << (31 - __clz(n)) : 0; }

// Two independent searches in the same sorted shared-memory array a[0..n) in lockstep:
// p0 = #{a[j] < x0}, p1 = #{a[j] < x1}.  Binary lifting with a fixed trip count (top =
// top_pow2(n)), so the two dependent load chains overlap.
__device__ __forceinline__ void count_below2(const int* a, int n, int top, int x0, int x1,
                                             int& p0, int& p1) {
  p0 = 0;
  p1 = 0;
  for (int step = top; step > 0; step >>= 1) {
    if (p0 + step <= n && a[p0 + step - 1] < x0) p0 += step;
    if (p1 + step <= n && a[p1 + step - 1] < x1) p1 += step;
  }
}

// Row elements staged per warp when a row is searched for the root's list.
constexpr int kStage = 256;

// Row i of a root's bitmap when the row (len elements from col + rsi, sorted) is longer than
// the root's list L[0..d): the list is looked up in the row, as the reference does with the
// shorter of two lists.  Used by the warp tier, whose lists (out-degree <= 128) are mostly
// shorter than their rows; in the CTA bands the extra registers cost more than it saves.  A warp stages up to kStage row elements at a time in shared memory
// (one coalesced copy), each lane binary-searches two list entries in them, and the ballot
// of the hits of 32 entries is one word of the row (ORed into Ri, which starts at zero).
// on_hit(j, e) runs for every hit in the edge-triangle modes (j = list index, e = the slot
// of L[j] in the row).
// One staged piece of a row (cl elements in stage[], the first at slot e0 of col) searched
// for the root's list: each lane binary-searches two list entries, and the ballot of the hits
// of 32 entries is one word of the row.
template <bool ETRI, typename F>
__device__ __forceinline__ void flip_search(const vid_t* stage, int cl, eid_t e0, const vid_t* L,
                                            int d, int w_d, uint32_t* Ri, F&& on_hit) {
  const int lane = threadIdx.x & 31;
  const int top = top_pow2(cl);
  for (int q0 = 0; q0 < w_d; q0 += 2) {
    const int ja = 32 * q0 + lane, jb = ja + 32;
    const vid_t xa = ja < d ? L[ja] : INT32_MAX;
    const vid_t xb = jb < d ? L[jb] : INT32_MAX;
    int pa, pb;
    count_below2(stage, cl, top, xa, xb, pa, pb);
    const bool fa = ja < d && pa < cl && stage[pa] == xa;
    const bool fb = jb < d && pb < cl && stage[pb] == xb;
    const unsigned ma = __ballot_sync(kFull, fa), mb = __ballot_sync(kFull, fb);
    if (lane == 0) {
      if (ma) atomicOr(Ri + q0, ma);
      if (mb && q0 + 1 < w_d) atomicOr(Ri + q0 + 1, mb);
    }
    if (ETRI) {
      if (fa) on_hit(ja, e0 + pa);
      if (fb) on_hit(jb, e0 + pb);
    }
  }
}

// Row i of a root's bitmap when the row (len elements from col + rsi, sorted) is longer than
// the root's list L[0..d): the list is looked up in the row, as the reference does with the
// shorter of two lists.  Used by the warp tier, whose lists (out-degree <= 128) are mostly
// shorter than their rows; in the CTA bands the extra registers cost more than they save.  A
// warp stages up to kStage row elements at a time in shared memory (one coalesced copy) and
// searches them (flip_search); the hits are ORed into Ri, which starts at zero.  on_hit(j, e)
// runs for every hit in the edge-triangle modes (j = list index, e = the slot of L[j] in the
// row).
template <bool ETRI, typename F>
__device__ __forceinline__ void flip_row(const vid_t* __restrict__ col, eid_t rsi, int len,
                                         const vid_t* L, int d, int w_d, uint32_t* Ri,
                                         vid_t* stage, F&& on_hit) {
  const int lane = threadIdx.x & 31;
  for (int c0 = 0; c0 < len; c0 += kStage) {
    const int cl = min(kStage, len - c0);
    __syncwarp();
    for (int t = lane; t < cl; t += 32) stage[t] = __ldg(col + rsi + c0 + t);
    __syncwarp();
    flip_search<ETRI>(stage, cl, rsi + c0, L, d, w_d, Ri, on_hit);
  }
  __syncwarp();
}

// Position of the r-th set bit (r counted from 0) of the W-word row.
__device__ __forceinline__ int select_bit(const uint32_t* row, int W, int r) {
  for (int q = 0; q < W; ++q) {
    const uint32_t w = row[q];
    const int c = __popc(w);
    if (r < c) return q * 32 + (int)__fns(w, 0, r + 1);
    r -= c;
  }
  return 0;  // not reached: r < popc(row)
}

// Word w of a register array, by an unrolled select (the array stays in registers).
template <int WMAX>
__device__ __forceinline__ uint32_t pick_word(const uint32_t (&m)[WMAX], int w) {
  uint32_t r = 0u;
#pragma unroll
  for (int q = 0; q < WMAX; ++q) r = (q == w) ? m[q] : r;
  return r;
}

// ---------------------------------------------------------------- single-word rows
template <int D, bool STATS>
struct SmallCount {
  // m: candidate set (bits over L), R: rows, deg: out-degrees of L (stats only)
  __device__ __forceinline__ static acc_t run(uint32_t m, const uint32_t* R, const int* deg,
                                              acc_t& elems) {
    acc_t s = 0;
    const int pm = __popc(m);
    uint32_t it = m;
    while (it) {
      const int j = __ffs(it) - 1;
      it &= it - 1;
      if (STATS) elems += (acc_t)pm + (acc_t)deg[j];
      s += SmallCount<D - 1, STATS>::run(m & R[j], R, deg, elems);
    }
    return s;
  }
};

template <bool STATS>
struct SmallCount<0, STATS> {
  __device__ __forceinline__ static acc_t run(uint32_t m, const uint32_t*, const int*, acc_t&) {
    return (acc_t)__popc(m);
  }
};

// One root per group of G lanes (G in {4, 8, 16, 32}); every lane of the warp calls this
// with its group's root u (or u < 0 for an idle group).  R and DG point at the group's G
// shared words.  Returns this lane's partial count.  tri (edge-triangle mode) receives one
// count per triangle arc.
template <int G, int K, bool STATS, bool ETRI, bool PAIRS = false, bool TT = false>
__device__ __forceinline__ acc_t group_root(const eid_t* __restrict__ rowptr,
                                            const vid_t* __restrict__ col, vid_t u,
                                            uint32_t* R, int* DG, uint32_t* tri,
                                            acc_t& elems, const eid_t* srow = nullptr) {
  const int lane = threadIdx.x & 31;
  const int gl = lane & (G - 1);
  eid_t base = 0;
  int d = 0;
  if (u >= 0) {
    base = rowptr[u];
    d = (int)(rowptr[u + 1] - base);
  }
  const vid_t Lj = gl < d ? __ldg(col + base + gl) : INT32_MAX;
  const vid_t lo_key = __shfl_sync(kFull, Lj, 0, G);
  const vid_t hi_key = __shfl_sync(kFull, Lj, d > 0 ? d - 1 : 0, G);
  eid_t s = 0;
  int len = 0;
  if (gl < d) {
    s = rowptr[Lj];
    len = (int)(rowptr[Lj + 1] - s);
    if (STATS) DG[gl] = len;
    if (len > kRangeCut) {
      const int lb = lower_bound_g(col + s, len, lo_key);
      const int ub = upper_bound_g(col + s, len, hi_key);
      s += lb;
      len = ub > lb ? ub - lb : 0;
    }
  }
  R[gl] = 0u;
  if (ETRI) DG[gl] = 0;  // column counts (DG is free when STATS is off)
  int off = len;  // inclusive scan of the row lengths within the group
#pragma unroll
  for (int o = 1; o < G; o <<= 1) {
    const int t = __shfl_up_sync(kFull, off, o, G);
    if (gl >= o) off += t;
  }
  const int T = __shfl_sync(kFull, off, G - 1, G);
  const int Tmax = (G == 32) ? T : (int)__reduce_max_sync(kFull, (unsigned)T);
  const int row_start = off - len;
  acc_t pairs = 0;
  __syncwarp();
  for (int t0 = 0; t0 < Tmax; t0 += G) {
    const int t = t0 + gl;
    // row i = number of rows of the group ending at or before t
    int i = 0;
#pragma unroll
    for (int step = G / 2; step > 0; step >>= 1) {
      const int ov = __shfl_sync(kFull, off, i + step - 1, G);
      if (ov <= t) i += step;
    }
    const eid_t si = __shfl_sync(kFull, s, i, G);
    const int sti = __shfl_sync(kFull, row_start, i, G);
    const vid_t x = t < T ? __ldg(col + si + (t - sti)) : INT32_MIN;
    int p = 0;
#pragma unroll
    for (int step = G / 2; step > 0; step >>= 1) {
      const vid_t lv = __shfl_sync(kFull, Lj, p + step - 1, G);
      if (lv < x) p += step;
    }
    const vid_t lp = __shfl_sync(kFull, Lj, p, G);
    if (t < T && lp == x) {
      atomicOr(&R[i], 1u << p);
      if (ETRI) {  // triangle (u, L[i], L[p]): the arc L[i] -> L[p] gets its count now
        const unsigned o = atomicAdd(tri + si + (t - sti), 1u);
        if (PAIRS) pairs += (acc_t)o;
        atomicAdd(&DG[p], 1);
      }
    }
  }
  __syncwarp();
  acc_t cnt = 0, tt = 0;
  if ((!PAIRS || TT) && gl < d) cnt = SmallCount<K - 3, STATS>::run(R[gl], R, DG, elems);
  if (ETRI && gl < d) {
    // the root's own arc (u, L[gl]) lies on popc(R_gl) + (rows with bit gl) triangles
    const unsigned tu = (unsigned)__popc(R[gl]) + (unsigned)DG[gl];
    if (tu) {
      const unsigned o = atomicAdd(tri + base + gl, tu);
      if (PAIRS) pairs += pair_gain(o, tu);
    }
    // L[gl] is the middle vertex of popc(R_gl) of the root's triangles and the top of DG[gl]
    if (TT && tu) {
      const acc_t dg = tt_deg(srow, Lj);
      tt = (acc_t)__popc(R[gl]) * (tt_deg(srow, u) + dg) + (acc_t)DG[gl] * dg;
    }
  }
  __syncwarp();
  if (TT) return 12ull * cnt - 4ull * pairs + tt;
  return PAIRS ? pairs : cnt;
}

// ---------------------------------------------------------------- multi-word rows
// Row loads: rows in global memory (GR) are built with L2 atomics, so they are read at L2
// (ld.global.cg), never from a possibly stale L1 line; shared-memory rows are read directly.
template <bool GR>
__device__ __forceinline__ uint32_t ld_row(const uint32_t* p) {
  if (GR) return __ldcg(p);
  return *p;
}

// Mask distributed over the warp, WPL words per lane: lane l holds words l + 32 q (q < WPL,
// word index < W).  Rows are W words long.
template <int D, int WPL, bool STATS, bool GR = false>
struct DistCount {
  __device__ __forceinline__ static acc_t run(const uint32_t (&mw)[WPL], const uint32_t* R,
                                              int W, const int* deg, acc_t& elems, int S) {
    const int lane = threadIdx.x & 31;
    acc_t s = 0;
    int pm = 0;
    if (STATS) {
      int c = 0;
#pragma unroll
      for (int q = 0; q < WPL; ++q) c += __popc(mw[q]);
      pm = __reduce_add_sync(kFull, (unsigned)c);
    }
    // one recursive call site per level (a rolled loop over the lane's words, picked from
    // registers), so the code does not grow as WPL^depth
#pragma unroll 1
    for (int q = 0; q < WPL; ++q) {
      const uint32_t mq = pick_word<WPL>(mw, q);
      unsigned nz = __ballot_sync(kFull, mq != 0u);
      while (nz) {
        const int lw = __ffs(nz) - 1;
        nz &= nz - 1;
        uint32_t word = __shfl_sync(kFull, mq, lw);
        while (word) {
          const int b = __ffs(word) - 1;
          word &= word - 1;
          const int j = (q * 32 + lw) * 32 + b;
          if (STATS && lane == 0) elems += (acc_t)pm + (acc_t)deg[j];
          const uint32_t* Rj = R + (size_t)j * S;
          uint32_t nxt[WPL];
#pragma unroll
          for (int r = 0; r < WPL; ++r) {
            const int w = r * 32 + lane;
            nxt[r] = w < W ? (mw[r] & ld_row<GR>(Rj + w)) : 0u;
          }
          s += DistCount<D - 1, WPL, STATS, GR>::run(nxt, R, W, deg, elems, S);
        }
      }
    }
    return s;
  }
};

template <int WPL, bool STATS, bool GR>
struct DistCount<0, WPL, STATS, GR> {
  __device__ __forceinline__ static acc_t run(const uint32_t (&mw)[WPL], const uint32_t*, int,
                                              const int*, acc_t&, int) {
    acc_t s = 0;  // per-lane partial; summed at the end
#pragma unroll
    for (int q = 0; q < WPL; ++q) s += (acc_t)__popc(mw[q]);
    return s;
  }
};

// Row-parallel counting with the candidate mask in registers (WMAX words, W <= WMAX used):
// one thread owns one first-level row and walks the deeper levels itself.  Each level has a
// single recursive call site (code size stays linear in the depth); words are picked out of
// the register array with an unrolled select so the masks never go to local memory.

template <int D, int WMAX, bool STATS>
struct RowCount {
  __device__ static acc_t run(const uint32_t (&m)[WMAX], const uint32_t* R, int W,
                              const int* deg, acc_t& elems, int S) {
    acc_t s = 0;
    int pm = 0;
    if (STATS) {
#pragma unroll
      for (int w = 0; w < WMAX; ++w) pm += __popc(m[w]);
    }
    int w = 0;
    uint32_t bits = m[0];
    for (;;) {
      while (bits == 0u) {
        if (++w >= W) return s;
        bits = pick_word<WMAX>(m, w);
      }
      const int j = w * 32 + __ffs(bits) - 1;
      bits &= bits - 1;
      if (STATS) elems += (acc_t)pm + (acc_t)deg[j];
      uint32_t nxt[WMAX];
      const uint32_t* Rj = R + (size_t)j * S;
#pragma unroll
      for (int q = 0; q < WMAX; ++q) nxt[q] = q < W ? (m[q] & Rj[q]) : 0u;
      s += RowCount<D - 1, WMAX, STATS>::run(nxt, R, W, deg, elems, S);
    }
  }
};

template <int WMAX, bool STATS>
struct RowCount<0, WMAX, STATS> {
  __device__ __forceinline__ static acc_t run(const uint32_t (&m)[WMAX], const uint32_t*, int,
                                              const int*, acc_t&, int) {
    acc_t s = 0;
#pragma unroll
    for (int w = 0; w < WMAX; ++w) s += (acc_t)__popc(m[w]);
    return s;
  }
};

// ---------------------------------------------------------------- warp per root
// One root of out-degree 32 < d <= kWarpMaxDeg per warp, with the warp's own slice of shared
// memory (no CTA barriers).
constexpr int kWarpMaxDeg = 128;
constexpr int kWarpW = kWarpMaxDeg / 32;

struct WarpSmem {
  vid_t L[kWarpMaxDeg];
  int off[kWarpMaxDeg + 1];
  int deg[kWarpMaxDeg];
  eid_t rs[kWarpMaxDeg];
  uint32_t R[kWarpMaxDeg * kWarpW];
  int colcnt[kWarpMaxDeg];  // edge-triangle mode: rows with bit j set
  vid_t stage[kStage];      // a long row, staged to look the root's list up in it
};

// PIPE: the rows that are looked up in (flip rows) go through a register pipeline: while a
// warp searches one staged piece, the next piece (of this row or of the next flip row) is
// already on its way into registers, so the row loads no longer stall the searches.  It costs
// kStage / 32 registers per lane, which pays in the plain k <= 4 warp tier only.
template <int K, bool STATS, bool ETRI, bool PAIRS = false, bool TT = false, bool PIPE = false>
__device__ __forceinline__ acc_t warp_root(const eid_t* __restrict__ rowptr,
                                           const vid_t* __restrict__ col, vid_t u, WarpSmem& ws,
                                           uint32_t* tri, acc_t& elems,
                                           const eid_t* srow = nullptr) {
  const int lane = threadIdx.x & 31;
  const eid_t base = rowptr[u];
  const int d = (int)(rowptr[u + 1] - base);
  const int w_d = (d + 31) >> 5;
  for (int j = lane; j < d; j += 32) ws.L[j] = __ldg(col + base + j);
  for (int q = lane; q < d * w_d; q += 32) ws.R[q] = 0u;
  if (ETRI)
    for (int q = lane; q < d; q += 32) ws.colcnt[q] = 0;
  __syncwarp();
  const vid_t lo_key = ws.L[0], hi_key = ws.L[d - 1];
  for (int i = lane; i < d; i += 32) {
    const vid_t v = ws.L[i];
    eid_t s = rowptr[v];
    int len = (int)(rowptr[v + 1] - s);
    ws.deg[i] = len;
    if (len > kRangeCut) {
      const int lb = lower_bound_g(col + s, len, lo_key);
      const int ub = upper_bound_g(col + s, len, hi_key);
      s += lb;
      len = ub > lb ? ub - lb : 0;
    }
    ws.rs[i] = s;
    // rows of kLongRow or more elements are scanned row by row below (deg[] then holds the
    // cut length; the accounting pass needs the full one and scans every row flattened)
    const bool lng = !STATS && len >= kLongRow;
    if (!STATS) ws.deg[i] = len;
    ws.off[i] = lng ? 0 : len;
  }
  __syncwarp();
  {  // exclusive scan: lane takes rows [4 lane, 4 lane + 4)
    const int b0 = min(d, lane * kWarpW), b1 = min(d, b0 + kWarpW);
    int local = 0;
    for (int i = b0; i < b1; ++i) local += ws.off[i];
    int incl = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += t;
    }
    int run = incl - local;
    __syncwarp();
    for (int i = b0; i < b1; ++i) {
      const int l = ws.off[i];
      ws.off[i] = run;
      run += l;
    }
    if (lane == 31) ws.off[d] = incl;
    __syncwarp();
  }
  const int T = ws.off[d];
  acc_t pairs = 0, tt = 0;
  const int topL = top_pow2(d), topO = top_pow2(d - 1);
  auto hit = [&](int i, int p, vid_t x, eid_t e) {
    if (p < d && ws.L[p] == x) {
      atomicOr(&ws.R[i * w_d + (p >> 5)], 1u << (p & 31));
      if (ETRI) {
        const unsigned o = atomicAdd(tri + e, 1u);
        if (PAIRS) pairs += (acc_t)o;
        atomicAdd(&ws.colcnt[p], 1);
      }
    }
  };
  auto etri_hit = [&](int j, eid_t e) {
    const unsigned o = atomicAdd(tri + e, 1u);
    if (PAIRS) pairs += (acc_t)o;
    atomicAdd(&ws.colcnt[j], 1);
  };
  if (PIPE && !STATS) {
    constexpr int kPer = kStage / 32;
    auto next_flip = [&](int r) {
      for (++r; r < d; ++r) {
        const int l = ws.deg[r];
        if (l >= kLongRow && l > d) break;
      }
      return r;
    };
    vid_t nb[kPer];
    auto fetch = [&](int r, int c) {
      const eid_t s = ws.rs[r] + c;
      const int n = min(kStage, ws.deg[r] - c);
#pragma unroll
      for (int q = 0; q < kPer; ++q) {
        const int t = q * 32 + lane;
        nb[q] = t < n ? __ldg(col + s + t) : 0;
      }
    };
    int i = next_flip(-1), c0 = 0;
    if (i < d) fetch(i, 0);
    while (i < d) {
      const int cl = min(kStage, ws.deg[i] - c0);
      __syncwarp();
#pragma unroll
      for (int q = 0; q < kPer; ++q)
        if (q * 32 + lane < cl) ws.stage[q * 32 + lane] = nb[q];
      __syncwarp();
      int ni = i, nc = c0 + kStage;
      if (nc >= ws.deg[i]) {
        ni = next_flip(i);
        nc = 0;
      }
      if (ni < d) fetch(ni, nc);
      flip_search<ETRI>(ws.stage, cl, ws.rs[i] + c0, ws.L, d, w_d, ws.R + i * w_d, etri_hit);
      i = ni;
      c0 = nc;
    }
    __syncwarp();
  }
  // long rows: the warp scans one row at a time, two elements per lane and iteration, so no
  // element searches for its row
  if (!STATS) {
    for (int i = 0; i < d; ++i) {
      const int len = ws.deg[i];
      if (len < kLongRow) continue;
      const eid_t rsi = ws.rs[i];
      if (len > d) {  // the row is the longer list: look the root's list up in it
        if (PIPE) continue;
        flip_row<ETRI>(col, rsi, len, ws.L, d, w_d, ws.R + i * w_d, ws.stage, etri_hit);
        continue;
      }
      for (int t0 = lane; t0 < len; t0 += 64) {
        const bool two = t0 + 32 < len;
        const int t1 = two ? t0 + 32 : t0;
        const vid_t x0 = __ldg(col + rsi + t0), x1 = __ldg(col + rsi + t1);
        int p0, p1;
        count_below2(ws.L, d, topL, x0, x1, p0, p1);
        hit(i, p0, x0, rsi + t0);
        if (two) hit(i, p1, x1, rsi + t1);
      }
    }
  }
  // two scanned elements per lane and iteration; row i of element t = last i with off[i] <= t
  for (int t0 = lane; t0 < T; t0 += 64) {
    const bool two = t0 + 32 < T;
    const int t1 = two ? t0 + 32 : t0;
    int i0, i1;
    count_below2(ws.off + 1, d - 1, topO, t0 + 1, t1 + 1, i0, i1);
    const eid_t e0 = ws.rs[i0] + (t0 - ws.off[i0]), e1 = ws.rs[i1] + (t1 - ws.off[i1]);
    const vid_t x0 = __ldg(col + e0), x1 = __ldg(col + e1);
    int p0, p1;
    count_below2(ws.L, d, topL, x0, x1, p0, p1);
    hit(i0, p0, x0, e0);
    if (two) hit(i1, p1, x1, e1);
  }
  __syncwarp();
  acc_t cnt = 0;
  if (K >= 5 && !ETRI) {
    // k >= 5: the first two levels flattened over the lanes as (row i, bit j of R_i) pairs,
    // so one dense row does not hold up the warp.  off[i] = pairs before row i.
    const int b0 = min(d, lane * kWarpW), b1 = min(d, b0 + kWarpW);
    int local = 0;
    for (int i = b0; i < b1; ++i) {
      int c = 0;
      for (int q = 0; q < w_d; ++q) c += __popc(ws.R[i * w_d + q]);
      ws.off[i] = c;
      local += c;
    }
    int incl = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += t;
    }
    int run = incl - local;
    for (int i = b0; i < b1; ++i) {
      const int c = ws.off[i];
      ws.off[i] = run;
      run += c;
    }
    if (lane == 31) ws.off[d] = incl;
    __syncwarp();
    const int P = ws.off[d];
    for (int p = lane; p < P; p += 32) {
      int i, i2;
      count_below2(ws.off + 1, d - 1, topO, p + 1, p + 1, i, i2);
      const uint32_t* Ri = ws.R + i * w_d;
      const int j = select_bit(Ri, w_d, p - ws.off[i]);
      const uint32_t* Rj = ws.R + j * w_d;
      uint32_t m2[kWarpW];
#pragma unroll
      for (int q = 0; q < kWarpW; ++q) m2[q] = q < w_d ? (Ri[q] & Rj[q]) : 0u;
      if (STATS) elems += (acc_t)(ws.off[i + 1] - ws.off[i]) + (acc_t)ws.deg[j];
      cnt += RowCount<(K >= 5 ? K - 4 : 1), kWarpW, STATS>::run(m2, ws.R, w_d, ws.deg, elems,
                                                                  w_d);
    }
    __syncwarp();
    return cnt;
  }
  for (int i = lane; i < d && !(K >= 5 && !ETRI); i += 32) {
    uint32_t m[kWarpW];
#pragma unroll
    for (int q = 0; q < kWarpW; ++q) m[q] = q < w_d ? ws.R[i * w_d + q] : 0u;
    if (!PAIRS || TT)
      cnt += RowCount<K - 3, kWarpW, STATS>::run(m, ws.R, w_d, ws.deg, elems, w_d);
    if (ETRI) {
      unsigned pc = 0;
#pragma unroll
      for (int q = 0; q < kWarpW; ++q) pc += (unsigned)__popc(m[q]);
      const unsigned tu = pc + (unsigned)ws.colcnt[i];
      if (tu) {
        const unsigned o = atomicAdd(tri + base + i, tu);
        if (PAIRS) pairs += pair_gain(o, tu);
        if (TT) {
          const acc_t di = tt_deg(srow, ws.L[i]);
          tt += (acc_t)pc * (tt_deg(srow, u) + di) + (acc_t)ws.colcnt[i] * di;
        }
      }
    }
  }
  __syncwarp();
  if (TT) return 12ull * cnt - 4ull * pairs + tt;
  return PAIRS ? pairs : cnt;
}

// Row stride in words of a root with w_d-word rows: odd in shared memory, so that the rows
// that the threads of a warp read at the same word index fall into different banks; rows in
// global memory (GR) are packed.
__host__ __device__ __forceinline__ int row_stride(int w_d, bool global_rows) {
  return global_rows ? w_d : (w_d | 1);
}

// Balanced 5-clique count (BAL): per warp, the R_i & R_j masks of 32 (i, j) pairs (RW words
// each, word q of lane l at q * 32 + l) and a list of kBalCap packed items (k | lane << 10).
constexpr int kBalCap = 512;
__host__ __device__ __forceinline__ size_t bal_bytes(int rw) {
  return rw > 0 ? (size_t)8 * ((size_t)rw * 32 * 4 + (size_t)kBalCap * 2) : 0;
}

// Level-2 bitmaps of the 5-clique count (rows of up to 16 words): per warp, the positions of
// the members of one row R_i (kL2Max of them) and their induced adjacency, kL2Stride words
// per member (odd, so that 32 members' words fall into 32 banks).
constexpr int kL2Max = 128;
constexpr int kL2Words = kL2Max / 32;
constexpr int kL2Stride = kL2Words + 1;
__host__ __device__ __forceinline__ size_t l2_bytes() {
  return (size_t)8 * ((size_t)kL2Max * kL2Stride * 4 + (size_t)kL2Max * 2);
}
// Buffers of the balanced 5-clique count for masks of rw words: a row counter, then the
// level-2 buffers (rw <= 16) or the item buffers (rw = 32), over the same memory.
__host__ __device__ __forceinline__ size_t k5_bytes(int rw) {
  if (rw <= 0) return 0;
  const size_t b = rw <= 16 ? l2_bytes() : bal_bytes(rw);
  return 16 + b + 16;  // counter, buffers, alignment slack
}

// Shared layout for one mid-tier root (dynamic shared memory):
//   L[dmax] ids | off[dmax+1] exclusive row offsets | rs[dmax] row starts (int64) |
//   deg[dmax] | ln[dmax] row lengths | R[dmax * row_stride(W)] rows | 8 warp sums |
//   balanced-count buffers (bal_rw)
struct MidLayout {
  int dmax, W;
  int bal_rw = 0;  // mask words of the balanced 5-clique buffers (0: none)
  __host__ __device__ size_t bytes() const {
    return bytes_no_rows() + (size_t)dmax * row_stride(W, false) * 4;
  }
  __host__ __device__ size_t bytes_no_rows() const {
    return (size_t)dmax * 4 + (size_t)(dmax + 1) * 4 + (size_t)dmax * 8 + (size_t)dmax * 8 +
           64 + 64 + k5_bytes(bal_rw);
  }
};

struct MidSmem {
  vid_t* L;
  int* off;
  eid_t* rs;
  int* deg;
  int* ln;  // row lengths after the range cut
  uint32_t* R;
  int* wsum;
  int* k5_next;        // balanced 5-clique count: next row to take (level-2 form)
  uint32_t* bal_m;     // item form: 8 warps x RW x 32 mask words
  uint16_t* bal_list;  // item form: 8 warps x kBalCap items
  uint32_t* l2_a;      // level-2 form: 8 warps x kL2Max x kL2Stride adjacency words
  uint16_t* l2_p;      // level-2 form: 8 warps x kL2Max member positions
  // rows = nullptr: the rows follow in shared memory (MidLayout); otherwise they live at
  // rows (dmax * W words of global scratch for this CTA) and shared memory holds the rest
  // (MidLayout::bytes_no_rows).
  __device__ __forceinline__ static MidSmem carve(unsigned char* smem, int dmax, int W,
                                                  uint32_t* rows = nullptr, int bal_rw = 0) {
    MidSmem m;
    m.L = reinterpret_cast<vid_t*>(smem);
    m.off = reinterpret_cast<int*>(m.L + dmax);
    m.rs = reinterpret_cast<eid_t*>(
        (reinterpret_cast<uintptr_t>(m.off + dmax + 1) + 7) & ~uintptr_t(7));
    m.deg = reinterpret_cast<int*>(m.rs + dmax);
    m.ln = m.deg + dmax;
    uint32_t* after = reinterpret_cast<uint32_t*>(m.ln + dmax);
    if (rows) {
      m.R = rows;
      m.wsum = reinterpret_cast<int*>(after);
    } else {
      m.R = after;
      m.wsum = reinterpret_cast<int*>(m.R + (size_t)dmax * row_stride(W, false));
    }
    m.k5_next = reinterpret_cast<int*>(
        (reinterpret_cast<uintptr_t>(m.wsum + 8) + 15) & ~uintptr_t(15));
    m.bal_m = reinterpret_cast<uint32_t*>(m.k5_next + 4);
    m.bal_list = reinterpret_cast<uint16_t*>(m.bal_m + (size_t)8 * bal_rw * 32);
    m.l2_a = m.bal_m;
    m.l2_p = reinterpret_cast<uint16_t*>(m.l2_a + (size_t)8 * kL2Max * kL2Stride);
    return m;
  }
};

// Rows up to this many words (out-degree <= 512) are counted row-parallel from registers.
constexpr int kCtaRowWords = 16;

// Exclusive scan of off[0..d) in place over the CTA (blocked per thread, then across
// warps); off[d] receives the total.
__device__ __forceinline__ void cta_exclusive_scan(int* off, int d, int* wsum) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nthreads = blockDim.x;
  const int per = (d + nthreads - 1) / nthreads;
  const int b0 = min(d, tid * per), b1 = min(d, b0 + per);
  int local = 0;
  for (int i = b0; i < b1; ++i) local += off[i];
  int incl = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) wsum[warp] = incl;
  __syncthreads();
  int wbase = 0;
  for (int w = 0; w < warp; ++w) wbase += wsum[w];
  int run = wbase + incl - local;
  __syncthreads();
  for (int i = b0; i < b1; ++i) {
    const int l = off[i];
    off[i] = run;
    run += l;
  }
  if (tid == nthreads - 1) off[d] = run;
  __syncthreads();
}

// Items t = lane, lane + 32, ... < nit of a balanced round: popc(M_owner & R_k) over the
// first W words (W a compile-time multiple of 4 >= w_d; the mask words past w_d are zero).
template <int W>
__device__ __forceinline__ acc_t bal_items_w(const uint16_t* Lw, int nit, const uint32_t* Mw,
                                             const uint32_t* R, int S) {
  acc_t cnt = 0;
  for (int t2 = threadIdx.x & 31; t2 < nit; t2 += 32) {
    const uint32_t v = Lw[t2];
    const uint32_t* Rk = R + (size_t)(v & 1023u) * S;
    const uint32_t* Mo = Mw + (v >> 10);
    int s = 0;
#pragma unroll
    for (int q = 0; q < W; ++q) s += __popc(Mo[q * 32] & Rk[q]);
    cnt += (acc_t)s;
  }
  return cnt;
}

template <int RW>
__device__ __forceinline__ acc_t bal_items(const uint16_t* Lw, int nit, const uint32_t* Mw,
                                           const uint32_t* R, int S, int w_d) {
  switch ((w_d + 3) >> 2) {
    case 1: return bal_items_w<4>(Lw, nit, Mw, R, S);
    case 2: return bal_items_w<(RW >= 8 ? 8 : 4)>(Lw, nit, Mw, R, S);
    case 3: return bal_items_w<(RW >= 12 ? 12 : 4)>(Lw, nit, Mw, R, S);
    case 4: return bal_items_w<(RW >= 16 ? 16 : 4)>(Lw, nit, Mw, R, S);
    case 5: return bal_items_w<(RW >= 20 ? 20 : 4)>(Lw, nit, Mw, R, S);
    case 6: return bal_items_w<(RW >= 24 ? 24 : 4)>(Lw, nit, Mw, R, S);
    case 7: return bal_items_w<(RW >= 28 ? 28 : 4)>(Lw, nit, Mw, R, S);
    default: return bal_items_w<(RW >= 32 ? 32 : 4)>(Lw, nit, Mw, R, S);
  }
}

// 5-cliques of one root from its bitmap rows, with the work spread evenly over the lanes.
// off[0..d] holds the exclusive prefix of the row popcounts (P = off[d] pairs (i, j), j a
// bit of R_i).  A warp takes 32 pairs at a time: each lane forms m = R_i & R_j, then the
// bits k of all 32 masks are expanded into an item list (at most kBalCap per round) that
// the lanes take round-robin; an item adds popc(m & R_k).  The work per item is the same
// for every lane, whatever the masks' sizes.
template <int RW>
__device__ __forceinline__ acc_t bal_count5(const int* off, int d, int topO,
                                            const uint32_t* R, int w_d, int S,
                                            uint32_t* Mw, uint16_t* Lw) {
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  const int P = off[d];
  acc_t cnt = 0;
  for (int base = warp * 32; base < P; base += nwarps * 32) {
    const int p = base + lane;
    uint32_t m2[RW];
    int c = 0;
    if (p < P) {
      int i, i2;
      count_below2(off + 1, d - 1, topO, p + 1, p + 1, i, i2);
      const uint32_t* Ri = R + (size_t)i * S;
      const int j = select_bit(Ri, w_d, p - off[i]);
      const uint32_t* Rj = R + (size_t)j * S;
#pragma unroll
      for (int q = 0; q < RW; ++q) {
        m2[q] = q < w_d ? (Ri[q] & Rj[q]) : 0u;
        c += __popc(m2[q]);
      }
    } else {
#pragma unroll
      for (int q = 0; q < RW; ++q) m2[q] = 0u;
    }
#pragma unroll
    for (int q = 0; q < RW; ++q)
      if (q < ((w_d + 3) & ~3)) Mw[q * 32 + lane] = m2[q];  // m2[q] = 0 for q >= w_d
    int incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += t;
    }
    const int first = incl - c;
    const int C = __shfl_sync(kFull, incl, 31);
    for (int r0 = 0; r0 < C; r0 += kBalCap) {
      // this lane's items with index in [r0, r0 + kBalCap)
      const int tend = min(first + c, r0 + kBalCap);
      int t = first;
      if (t < tend) {
#pragma unroll
        for (int q = 0; q < RW; ++q) {
          uint32_t w = m2[q];
          const int pc = __popc(w);
          if (t + pc <= r0) {  // the whole word lies before this round
            t += pc;
            continue;
          }
          while (w != 0u && t < tend) {
            const int b = __ffs(w) - 1;
            w &= w - 1;
            if (t >= r0) Lw[t - r0] = (uint16_t)((q * 32 + b) | (lane << 10));
            ++t;
          }
        }
      }
      __syncwarp();
      const int nit = min(C - r0, kBalCap);
      cnt += bal_items<RW>(Lw, nit, Mw, R, S, w_d);
      __syncwarp();
    }
  }
  return cnt;
}

// 5-cliques through row i of a root: the triangles of the sub-DAG that the rows induce on the
// c members of R_i (c <= 32 P), counted by one warp.  The members' positions go to Pw; the
// induced adjacency A (member x -> member y iff position p_y is in row p_x) is built one
// member at a time with a ballot per 32 members, into Aw (kL2Stride words per member); then
// lane x sums popc(A_x & A_y) over the y in A_x.  Every mask is P words instead of the
// row's w_d, and no lane waits for another.
template <int P>
__device__ __forceinline__ int l2_row(const uint32_t* Ri, int w_d, int c, const uint32_t* R,
                                      int S, uint32_t* Aw, uint16_t* Pw) {
  const int lane = threadIdx.x & 31;
  {  // member positions: word q of R_i on lane q, inclusive prefix of the word popcounts
    const uint32_t wq = lane < w_d ? Ri[lane] : 0u;
    int incl = __popc(wq);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += t;
    }
    const int excl = incl - __popc(wq);
#pragma unroll
    for (int w = 0; w < P; ++w) {
      const int y = lane + 32 * w;
      int q = 0;  // the word holding member y: the number of words ending at or before y
#pragma unroll
      for (int step = 16; step > 0; step >>= 1) {
        const int v = __shfl_sync(kFull, incl, q + step - 1);
        if (v <= y) q += step;
      }
      const uint32_t word = __shfl_sync(kFull, wq, q & 31);
      const int ex = __shfl_sync(kFull, excl, q & 31);
      if (y < c) Pw[y] = (uint16_t)(q * 32 + (int)__fns(word, 0, y - ex + 1));
    }
  }
  __syncwarp();
  int pw[P], pb[P];  // word and bit of member y = lane + 32 w
#pragma unroll
  for (int w = 0; w < P; ++w) {
    const int y = lane + 32 * w;
    const int p = y < c ? (int)Pw[y] : 0;
    pw[w] = p >> 5;
    pb[w] = p & 31;
  }
  for (int x = 0; x < c; ++x) {
    const uint32_t* Rx = R + (size_t)Pw[x] * S;
#pragma unroll
    for (int w = 0; w < P; ++w) {
      const bool b = lane + 32 * w < c && ((Rx[pw[w]] >> pb[w]) & 1u);
      const uint32_t m = __ballot_sync(kFull, b);
      if (lane == w) Aw[x * kL2Stride + w] = m;
    }
  }
  __syncwarp();
  int s = 0;
#pragma unroll
  for (int pass = 0; pass < P; ++pass) {
    const int x = lane + 32 * pass;
    uint32_t ax[P];
#pragma unroll
    for (int w = 0; w < P; ++w) ax[w] = x < c ? Aw[x * kL2Stride + w] : 0u;
#pragma unroll
    for (int wy = 0; wy < P; ++wy) {
      const int ylim = min(32, c - 32 * wy);
      for (int yb = 0; yb < ylim; ++yb) {
        const uint32_t* Ay = Aw + (32 * wy + yb) * kL2Stride;
        int t = 0;
#pragma unroll
        for (int w = 0; w < P; ++w) t += __popc(ax[w] & Ay[w]);
        s += ((ax[wy] >> yb) & 1u) ? t : 0;
      }
    }
  }
  __syncwarp();
  return s;
}

// 5-cliques of one root through the level-2 bitmaps of each row, rows taken by the CTA's warps
// from a shared counter; rows of more than kL2Max members are counted pair by pair.
template <int RW>
__device__ __forceinline__ acc_t l2_count5(const uint32_t* R, int d, int w_d, int S,
                                           int* next, uint32_t* Aw, uint16_t* Pw,
                                           const int* deg, acc_t& elems) {
  const int lane = threadIdx.x & 31;
  acc_t cnt = 0;
  for (;;) {
    int i = 0;
    if (lane == 0) i = atomicAdd(next, 1);
    i = __shfl_sync(kFull, i, 0);
    if (i >= d) break;
    const uint32_t* Ri = R + (size_t)i * S;
    int c = 0;
#pragma unroll
    for (int q = 0; q < RW; ++q) c += q < w_d ? __popc(Ri[q]) : 0;
    if (c < 3) continue;
    if (c <= 32) cnt += (acc_t)l2_row<1>(Ri, w_d, c, R, S, Aw, Pw);
    else if (c <= 64) cnt += (acc_t)l2_row<2>(Ri, w_d, c, R, S, Aw, Pw);
    else if (c <= 96) cnt += (acc_t)l2_row<3>(Ri, w_d, c, R, S, Aw, Pw);
    else if (c <= kL2Max) cnt += (acc_t)l2_row<4>(Ri, w_d, c, R, S, Aw, Pw);
    else {  // a dense row: its pairs (i, j) one per lane
      for (int jj = lane; jj < c; jj += 32) {
        const int j = select_bit(Ri, w_d, jj);
        const uint32_t* Rj = R + (size_t)j * S;
        uint32_t m2[RW];
#pragma unroll
        for (int q = 0; q < RW; ++q) m2[q] = q < w_d ? (Ri[q] & Rj[q]) : 0u;
        cnt += RowCount<1, RW, false>::run(m2, R, w_d, deg, elems, S);
      }
    }
  }
  return cnt;
}

// One root of out-degree 32 < d <= dmax processed by the whole CTA (blockDim = 256).
// Every thread calls it; returns this thread's partial count.  Rows of up to ROWW words are
// counted row-parallel from registers, wider ones (or all, with ROWW = 0) warp-cooperatively
// with WPL mask words per lane (rows of up to 32 WPL words).  BAL (k = 5, rows of up to ROWW
// words in shared memory, no accounting) counts with bal_count5; the layout then carries the
// balanced-count buffers (MidLayout::bal_rw = ROWW).
template <int K, bool STATS, bool ETRI, bool PAIRS = false, int ROWW = kCtaRowWords,
          int WPL = 1, bool GR = false, bool TT = false, bool BAL = false>
__device__ __forceinline__ acc_t cta_root(const eid_t* __restrict__ rowptr,
                                          const vid_t* __restrict__ col, vid_t u,
                                          const MidSmem& sm, uint32_t* tri, acc_t& elems,
                                          const eid_t* srow = nullptr) {
  static_assert(!BAL || (K == 5 && !STATS && !ETRI && !GR && ROWW > 0),
                "the balanced count is for plain 5-clique counts with rows in shared memory");
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int nthreads = blockDim.x;
  const int nwarps = nthreads >> 5;
  vid_t* L = sm.L;
  int* off = sm.off;
  eid_t* rs = sm.rs;
  int* deg = sm.deg;
  uint32_t* R = sm.R;
  const eid_t base = rowptr[u];
  const int d = (int)(rowptr[u + 1] - base);
  const int w_d = (d + 31) >> 5;
  const int S = row_stride(w_d, GR);
  for (int j = tid; j < d; j += nthreads) L[j] = __ldg(col + base + j);
  // global rows are built by L2 atomics and read at L2: clear them at L2 as well
  for (int q = tid; q < d * S; q += nthreads) {
    if (GR) __stcg(R + q, 0u);
    else R[q] = 0u;
  }
  __syncthreads();
  const vid_t lo_key = L[0], hi_key = L[d - 1];
  for (int i = tid; i < d; i += nthreads) {
    const vid_t v = L[i];
    eid_t s = rowptr[v];
    int len = (int)(rowptr[v + 1] - s);
    deg[i] = ETRI ? 0 : len;  // edge-triangle mode reuses deg[] as column counts
    if (len > kRangeCut) {
      const int lb = lower_bound_g(col + s, len, lo_key);
      const int ub = upper_bound_g(col + s, len, hi_key);
      s += lb;
      len = ub > lb ? ub - lb : 0;
    }
    rs[i] = s;
    sm.ln[i] = len;
    // rows of kLongRow or more elements are scanned row by row below; the accounting pass
    // scans every row flattened
    off[i] = (!STATS && len >= kLongRow) ? 0 : len;
  }
  __syncthreads();
  cta_exclusive_scan(off, d, sm.wsum);
  const int T = off[d];
  acc_t pairs = 0, tt = 0;
  const int topL = top_pow2(d), topO = top_pow2(d - 1);
  auto hit = [&](int i, int p, vid_t x, eid_t e) {
    if (p < d && L[p] == x) {
      atomicOr(&R[(size_t)i * S + (p >> 5)], 1u << (p & 31));
      if (ETRI) {
        const unsigned o = atomicAdd(tri + e, 1u);
        if (PAIRS) pairs += (acc_t)o;
        atomicAdd(&deg[p], 1);
      }
    }
  };
  // long rows: one warp per row, two elements per lane and iteration, so no element
  // searches for its row
  if (!STATS) {
    for (int i = warp; i < d; i += nwarps) {
      const int len = sm.ln[i];
      if (len < kLongRow) continue;
      const eid_t rsi = rs[i];
      for (int t0 = lane; t0 < len; t0 += 64) {
        const bool two = t0 + 32 < len;
        const int t1 = two ? t0 + 32 : t0;
        const vid_t x0 = __ldg(col + rsi + t0), x1 = __ldg(col + rsi + t1);
        int p0, p1;
        count_below2(L, d, topL, x0, x1, p0, p1);
        hit(i, p0, x0, rsi + t0);
        if (two) hit(i, p1, x1, rsi + t1);
      }
    }
  }
  // short rows: two scanned elements per thread and iteration; row i of element t = last i
  // with off[i] <= t
  for (int t0 = tid; t0 < T; t0 += 2 * nthreads) {
    const bool two = t0 + nthreads < T;
    const int t1 = two ? t0 + nthreads : t0;
    int i0, i1;
    count_below2(off + 1, d - 1, topO, t0 + 1, t1 + 1, i0, i1);
    const eid_t e0 = rs[i0] + (t0 - off[i0]), e1 = rs[i1] + (t1 - off[i1]);
    const vid_t x0 = __ldg(col + e0), x1 = __ldg(col + e1);
    int p0, p1;
    count_below2(L, d, topL, x0, x1, p0, p1);
    hit(i0, p0, x0, e0);
    if (two) hit(i1, p1, x1, e1);
  }
  __syncthreads();
  if (ETRI) {  // the root's own arcs: popc(R_i) + (rows with bit i) triangles each
    for (int i = tid; i < d; i += nthreads) {
      unsigned pc = 0;
      for (int q = 0; q < w_d; ++q) pc += (unsigned)__popc(ld_row<GR>(R + (size_t)i * S + q));
      const unsigned tu = pc + (unsigned)deg[i];
      if (tu) {
        const unsigned o = atomicAdd(tri + base + i, tu);
        if (PAIRS) pairs += pair_gain(o, tu);
        if (TT) {
          const acc_t di = tt_deg(srow, L[i]);
          tt += (acc_t)pc * (tt_deg(srow, u) + di) + (acc_t)deg[i] * di;
        }
      }
    }
  }
  if (PAIRS && !TT) {
    __syncthreads();
    return pairs;
  }
  acc_t cnt = 0;
  static_assert(!GR || ROWW == 0, "rows in global memory are counted warp-cooperatively");
  constexpr int RW = ROWW > 0 ? ROWW : 1;
  if (BAL && RW <= 16 && w_d <= ROWW) {
    // 5-cliques through level-2 bitmaps, one row per warp (rows from a shared counter)
    if (tid == 0) *sm.k5_next = 0;
    __syncthreads();
    cnt += l2_count5<RW>(R, d, w_d, S, sm.k5_next, sm.l2_a + (size_t)warp * kL2Max * kL2Stride,
                         sm.l2_p + (size_t)warp * kL2Max, deg, elems);
  } else if (ROWW > 0 && w_d <= ROWW && K >= 5 && !ETRI) {
    // k >= 5: the first two levels flattened over the threads as (row i, bit j of R_i)
    // pairs, so one dense row does not hold up the CTA.  off[i] = pairs before row i.
    for (int i = tid; i < d; i += nthreads) {
      int c = 0;
      for (int q = 0; q < w_d; ++q) c += __popc(R[(size_t)i * S + q]);
      off[i] = c;
    }
    __syncthreads();
    cta_exclusive_scan(off, d, sm.wsum);
    if (BAL) {
      cnt += bal_count5<RW>(off, d, topO, R, w_d, S, sm.bal_m + (size_t)warp * RW * 32,
                            sm.bal_list + (size_t)warp * kBalCap);
    } else {
      const int P = off[d];
      for (int p = tid; p < P; p += nthreads) {
        int i, i2;
        count_below2(off + 1, d - 1, topO, p + 1, p + 1, i, i2);
        const uint32_t* Ri = R + (size_t)i * S;
        const int j = select_bit(Ri, w_d, p - off[i]);
        const uint32_t* Rj = R + (size_t)j * S;
        uint32_t m2[RW];
#pragma unroll
        for (int q = 0; q < RW; ++q) m2[q] = q < w_d ? (Ri[q] & Rj[q]) : 0u;
        if (STATS) elems += (acc_t)(off[i + 1] - off[i]) + (acc_t)deg[j];
        cnt += RowCount<(K >= 5 ? K - 4 : 1), RW, STATS>::run(m2, R, w_d, deg, elems, S);
      }
    }
  } else if (ROWW > 0 && w_d <= ROWW) {
    // row-parallel: each thread owns rows, masks in registers
    for (int i = tid; i < d; i += nthreads) {
      uint32_t m[RW];
#pragma unroll
      for (int q = 0; q < RW; ++q) m[q] = q < w_d ? R[(size_t)i * S + q] : 0u;
      cnt += RowCount<K - 3, RW, STATS>::run(m, R, w_d, deg, elems, S);
    }
  } else {
    // wide rows: the mask is distributed over the lanes, WPL words each
    for (int i = warp; i < d; i += nwarps) {
      uint32_t mw[WPL];
#pragma unroll
      for (int q = 0; q < WPL; ++q) {
        const int w = q * 32 + lane;
        mw[q] = w < w_d ? ld_row<GR>(R + (size_t)i * S + w) : 0u;
      }
      cnt += DistCount<K - 3, WPL, STATS, GR>::run(mw, R, w_d, deg, elems, S);
    }
  }
  __syncthreads();
  if (TT) return 12ull * cnt - 4ull * pairs + tt;
  return cnt;
}

}  // namespace jgpm
