// Oracle-side restatement of the seeded R-MAT edge definition (test infrastructure only).
//
// Edge i of seed s: for each of `scale` levels take a 32-bit draw (two per 64-bit word of
// a SplitMix64-mixed counter, Steele/Lea/Flood OOPSLA 2014) and pick the quadrant by the
// integer thresholds floor(a*2^32), floor((a+b)*2^32), floor((a+b+c)*2^32): below the first
// is (0,0), then (0,1), then (1,0), else (1,1); level l sets bit scale-1-l.  An edge with an
// endpoint >= n is redrawn from the next block of words, up to 64 attempts.  Written
// independently of the product's generator so the tests can compare the two.
#pragma once
#include <cstdint>

namespace orc {

struct RmatSpec {
  int scale;
  int64_t n;
  uint32_t ta, tab, tabc;
  uint64_t seed;
};

inline uint32_t thr(double p) {
  if (p <= 0.0) return 0u;
  double t = p * 4294967296.0;
  return t >= 4294967295.0 ? 4294967295u : (uint32_t)t;
}

inline RmatSpec make_spec(int64_t n, int64_t, double a, double b, double c, uint64_t seed) {
  RmatSpec s;
  s.scale = 0;
  while ((int64_t(1) << s.scale) < n) s.scale++;
  s.n = n;
  s.ta = thr(a);
  s.tab = thr(a + b);
  s.tabc = thr(a + b + c);
  s.seed = seed;
  return s;
}

inline uint64_t mix(uint64_t z) {
  z ^= z >> 30;
  z *= 0xbf58476d1ce4e5b9ULL;
  z ^= z >> 27;
  z *= 0x94d049bb133111ebULL;
  z ^= z >> 31;
  return z;
}

inline bool edge(const RmatSpec& s, uint64_t i, int32_t* u, int32_t* v) {
  const uint64_t g = 0x9e3779b97f4a7c15ULL;
  const uint64_t base = mix(s.seed + g * (i + 1));
  const int wpa = (s.scale + 1) / 2;
  for (int att = 0; att < 64; ++att) {
    uint64_t x = 0, y = 0;
    for (int l = 0; l < s.scale; ++l) {
      uint64_t word = mix(base + g * ((uint64_t)att * wpa + (uint64_t)(l / 2) + 1));
      uint32_t r = (l % 2 == 0) ? (uint32_t)word : (uint32_t)(word >> 32);
      int q = r < s.ta ? 0 : (r < s.tab ? 1 : (r < s.tabc ? 2 : 3));
      x |= (uint64_t)(q >> 1) << (s.scale - 1 - l);
      y |= (uint64_t)(q & 1) << (s.scale - 1 - l);
    }
    if ((int64_t)x < s.n && (int64_t)y < s.n) {
      *u = (int32_t)x;
      *v = (int32_t)y;
      return true;
    }
  }
  return false;
}

}  // namespace orc
