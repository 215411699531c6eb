// Deterministic, counter-based R-MAT edge generator shared by the host and the device.
//
// Edge i of a graph with seed s is a pure function of (s, i): the quadrant choices at each
// of the `scale` recursion levels come from 32-bit draws cut out of a counter-based 64-bit
// hash, and the quadrant thresholds are integers (a, a+b, a+b+c scaled to 2^32).  So a
// CPU and a GPU that generate the same edge index get the same endpoints bit for bit,
// whatever the thread layout.
//
// The hash is the SplitMix64 output function (Steele, Lea and Flood, "Fast splittable
// pseudorandom number generators", OOPSLA 2014), used here as a stateless mixer of a
// counter.  No noise is added and no vertex permutation is applied, so R-MAT's hubs sit
// at the low vertex ids, as in the plain R-MAT model (Chakrabarti, Zhan and Faloutsos,
// SDM 2004).
//
// When the vertex count n is not a power of two, the edge is drawn on 2^ceil(log2 n)
// vertices and redrawn (a fresh counter block per attempt) while either endpoint is >= n.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define JGPM_HD __host__ __device__ __forceinline__
#else
#define JGPM_HD inline
#endif

namespace jgpm {

struct RmatParams {
  int32_t scale;      // log2 of the generated id range
  int64_t n;          // vertex count (<= 2^scale); ids >= n are redrawn
  int64_t num_edges;  // edges drawn (edge factor * n)
  uint32_t t_a;       // floor(a * 2^32)
  uint32_t t_ab;      // floor((a+b) * 2^32)
  uint32_t t_abc;     // floor((a+b+c) * 2^32)
  uint64_t seed;
  int32_t max_attempts;
};

JGPM_HD uint64_t splitmix64_mix(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

// 64-bit draw number k of edge i.
JGPM_HD uint64_t rmat_draw(uint64_t seed, uint64_t i, uint64_t k) {
  const uint64_t g = 0x9e3779b97f4a7c15ULL;
  uint64_t base = splitmix64_mix(seed + g * (i + 1));
  return splitmix64_mix(base + g * (k + 1));
}

// Generates edge i.  Returns false when every attempt fell outside [0, n).
JGPM_HD bool rmat_edge(const RmatParams& p, uint64_t i, int32_t* u_out, int32_t* v_out) {
  const int words_per_attempt = (p.scale + 1) / 2;
  for (int attempt = 0; attempt < p.max_attempts; ++attempt) {
    uint64_t u = 0, v = 0;
    uint64_t word = 0;
    for (int l = 0; l < p.scale; ++l) {
      uint32_t r;
      if ((l & 1) == 0) {
        word = rmat_draw(p.seed, i, (uint64_t)attempt * words_per_attempt + (l >> 1));
        r = (uint32_t)word;
      } else {
        r = (uint32_t)(word >> 32);
      }
      uint64_t rb, cb;
      if (r < p.t_a) { rb = 0; cb = 0; }
      else if (r < p.t_ab) { rb = 0; cb = 1; }
      else if (r < p.t_abc) { rb = 1; cb = 0; }
      else { rb = 1; cb = 1; }
      const int bit = p.scale - 1 - l;
      u |= rb << bit;
      v |= cb << bit;
    }
    if ((int64_t)u < p.n && (int64_t)v < p.n) {
      *u_out = (int32_t)u;
      *v_out = (int32_t)v;
      return true;
    }
  }
  return false;
}

// Threshold from a probability, saturating at 2^32 - 1.
inline uint32_t rmat_threshold(double p) {
  if (p <= 0.0) return 0u;
  double t = p * 4294967296.0;
  if (t >= 4294967295.0) return 4294967295u;
  return (uint32_t)t;
}

inline RmatParams rmat_params(int64_t n, int64_t num_edges, double a, double b, double c,
                              uint64_t seed) {
  RmatParams p;
  int s = 0;
  while ((int64_t(1) << s) < n) ++s;
  p.scale = s;
  p.n = n;
  p.num_edges = num_edges;
  p.t_a = rmat_threshold(a);
  p.t_ab = rmat_threshold(a + b);
  p.t_abc = rmat_threshold(a + b + c);
  p.seed = seed;
  p.max_attempts = 64;
  return p;
}

}  // namespace jgpm
