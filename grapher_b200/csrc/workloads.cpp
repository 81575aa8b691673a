// workloads.cpp -- seeded synthetic graphs for tests and benchmarks, a
// host-only library of its own (libgvizworkloads.so, include/gvizworkloads.h)
// so that a process can build the same inputs without loading the layout
// library itself.
//
// The grid and random-connected generators reproduce the reference's own
// fixtures edge for edge (src/utils/graphs.c:285-316, 598-639) by drawing
// from the same libc rand_r stream; the Barabasi-Albert, Erdos-Renyi and
// R-MAT generators are this project's own (seeded splitmix64).
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <unordered_set>
#include <vector>

#include "gvizworkloads.h"

namespace {

struct SplitMix {
  uint64_t s;
  explicit SplitMix(uint64_t seed) : s(seed) {}
  uint64_t next() {
    uint64_t z = (s += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
  }
  // uniform in [0, n), n < 2^32 (multiply-shift)
  uint32_t below(uint64_t n) {
    return (uint32_t)(((next() >> 32) * n) >> 32);
  }
  double unit() { return (double)(next() >> 11) * 0x1.0p-53; }
};

inline uint64_t pair_key(uint32_t a, uint32_t b) {
  uint32_t lo = a < b ? a : b, hi = a < b ? b : a;
  return ((uint64_t)lo << 32) | hi;
}

inline void put(uint32_t *ea, uint32_t *eb, size_t e, uint32_t a, uint32_t b) {
  if (ea) ea[e] = a;
  if (eb) eb[e] = b;
}

}  // namespace

extern "C" {

size_t gvizGenGrid(size_t L, size_t W, uint32_t *ea, uint32_t *eb) {
  size_t e = 0;
  for (size_t i = 0; i < L; i++)
    for (size_t j = 0; j < W; j++) {
      size_t idx = i * W + j;
      if (j + 1 < W) put(ea, eb, e++, (uint32_t)idx, (uint32_t)(idx + 1));
      if (i + 1 < L) put(ea, eb, e++, (uint32_t)idx, (uint32_t)(idx + W));
    }
  return e;
}

size_t gvizGenRandomConnected(size_t n, double density, unsigned seed,
                                  uint32_t *ea, uint32_t *eb) {
  if (density < 0.0) density = 0.0;
  if (density > 1.0) density = 1.0;
  if (n < 2) return 0;
  std::unordered_set<uint64_t> have;
  size_t e = 0;
  for (size_t i = 1; i < n; i++) {
    size_t j = (size_t)(rand_r(&seed) % i);
    put(ea, eb, e++, (uint32_t)i, (uint32_t)j);
    have.insert(pair_key((uint32_t)i, (uint32_t)j));
  }
  size_t treeEdges = n - 1;
  size_t maxEdges = n * (n - 1) / 2;
  size_t maxExtra = maxEdges - treeEdges;
  size_t targetExtra = (size_t)(density * (double)maxExtra + 0.5);
  size_t added = 0, attempts = 0;
  size_t maxAttempts = targetExtra * 20 + 100;
  while (added < targetExtra && attempts < maxAttempts) {
    attempts++;
    size_t a = (size_t)(rand_r(&seed) % n);
    size_t b = (size_t)(rand_r(&seed) % n);
    if (a == b || have.count(pair_key((uint32_t)a, (uint32_t)b))) continue;
    put(ea, eb, e++, (uint32_t)a, (uint32_t)b);
    have.insert(pair_key((uint32_t)a, (uint32_t)b));
    added++;
  }
  return e;
}

size_t gvizGenBarabasiAlbert(size_t n, uint32_t m, uint64_t seed,
                                 uint32_t *ea, uint32_t *eb) {
  if (m == 0 || n == 0) return 0;
  const size_t m0 = (size_t)m + 1;
  if (n <= m0) {  // complete graph on n vertices
    size_t e = 0;
    for (size_t i = 0; i < n; i++)
      for (size_t j = i + 1; j < n; j++) put(ea, eb, e++, (uint32_t)i, (uint32_t)j);
    return e;
  }
  SplitMix rng(seed * 0x2545F4914F6CDD1DULL + 0x1234567ULL);
  std::vector<uint32_t> ends;
  ends.reserve(2 * (m0 * (m0 - 1) / 2 + (n - m0) * (size_t)m));
  size_t e = 0;
  for (size_t i = 0; i < m0; i++)
    for (size_t j = i + 1; j < m0; j++) {
      put(ea, eb, e++, (uint32_t)i, (uint32_t)j);
      ends.push_back((uint32_t)i);
      ends.push_back((uint32_t)j);
    }
  std::vector<uint32_t> pick(m);
  for (size_t v = m0; v < n; v++) {
    const size_t L = ends.size();
    for (uint32_t t = 0; t < m; t++) {
      uint32_t u;
      bool dup;
      do {
        u = ends[rng.below(L)];
        dup = false;
        for (uint32_t q = 0; q < t; q++) dup |= pick[q] == u;
      } while (dup);
      pick[t] = u;
    }
    for (uint32_t t = 0; t < m; t++) {
      put(ea, eb, e++, (uint32_t)v, pick[t]);
      ends.push_back((uint32_t)v);
      ends.push_back(pick[t]);
    }
  }
  return e;
}

size_t gvizGenErdosRenyi(size_t n, size_t m, uint64_t seed, uint32_t *ea,
                             uint32_t *eb) {
  if (n < 2) return 0;
  const size_t maxEdges = n * (n - 1) / 2;
  if (m > maxEdges) m = maxEdges;
  SplitMix rng(seed ^ 0xA5A5A5A5DEADBEEFULL);
  std::unordered_set<uint64_t> have;
  have.reserve(m * 2);
  size_t e = 0;
  while (e < m) {
    uint32_t a = rng.below(n), b = rng.below(n);
    if (a == b) continue;
    if (!have.insert(pair_key(a, b)).second) continue;
    put(ea, eb, e++, a, b);
  }
  return e;
}

size_t gvizGenRmat(uint32_t scale, size_t draws, double a, double b,
                       double c, uint64_t seed, uint32_t *ea, uint32_t *eb) {
  if (scale == 0 || scale > 31) return 0;
  SplitMix rng(seed ^ 0x5DEECE66DULL);
  std::vector<uint64_t> keys;
  keys.reserve(draws);
  const double ab = a + b, abc = a + b + c;
  for (size_t d = 0; d < draws; d++) {
    uint32_t u = 0, v = 0;
    for (uint32_t bit = 0; bit < scale; bit++) {
      double r = rng.unit();
      uint32_t du = 0, dv = 0;
      if (r < a) {
      } else if (r < ab) {
        dv = 1;
      } else if (r < abc) {
        du = 1;
      } else {
        du = 1;
        dv = 1;
      }
      u = (u << 1) | du;
      v = (v << 1) | dv;
    }
    if (u == v) continue;
    keys.push_back(pair_key(u, v));
  }
  std::sort(keys.begin(), keys.end());
  keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
  for (size_t e = 0; e < keys.size(); e++)
    put(ea, eb, e, (uint32_t)(keys[e] >> 32), (uint32_t)(keys[e] & 0xffffffffu));
  return keys.size();
}

}  // extern "C"
