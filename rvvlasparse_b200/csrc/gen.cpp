// gen.cpp — seeded synthetic sparse matrices for the workloads the library is
// measured on (host side, OpenMP).  Every row draws from its own counter-based
// stream (splitmix64 keyed by seed and row), so the output does not depend on
// the number of threads.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "rvvla.h"

namespace {

inline uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

struct Rng {
  uint64_t s;
  Rng(uint64_t seed, uint64_t stream) : s(mix64(seed * 0x9e3779b97f4a7c15ULL + stream * 0xd1b54a32d192ed03ULL + 0x632be59bd9b4e019ULL)) {}
  uint64_t next() { s += 0x9e3779b97f4a7c15ULL; return mix64(s); }
  double uni() { return (double)(next() >> 11) * 0x1.0p-53; }           // [0, 1)
  double uni_open() { return ((double)(next() >> 11) + 0.5) * 0x1.0p-53; }  // (0, 1)
  double normal() {  // Box-Muller
    double u1 = uni_open(), u2 = uni();
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  }
  int64_t below(int64_t n) { return (int64_t)(uni() * (double)n) % n; }
};

// Small set of distinct columns for one row: linear probe table.
struct ColSet {
  std::vector<int64_t> tab;
  size_t mask = 0;
  void reset(int64_t want) {
    size_t cap = 16;
    while (cap < (size_t)want * 2) cap <<= 1;
    tab.assign(cap, -1);
    mask = cap - 1;
  }
  bool insert(int64_t c) {
    size_t h = (size_t)mix64((uint64_t)c) & mask;
    while (tab[h] >= 0) {
      if (tab[h] == c) return false;
      h = (h + 1) & mask;
    }
    tab[h] = c;
    return true;
  }
};

template <class F>
void parallel_rows(int64_t m, F&& f) {
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t i = 0; i < m; ++i) f(i);
}

int64_t finish_rst(std::vector<int64_t>& len, int64_t m, int32_t* Rst) {
  int64_t acc = 0;
  for (int64_t i = 0; i < m; ++i) {
    if (Rst) Rst[i] = (int32_t)acc;
    acc += len[(size_t)i];
  }
  if (Rst) Rst[m] = (int32_t)acc;
  return acc;
}

}  // namespace

extern "C" {

int64_t rvvla_gen_laplace2d(int64_t g, int32_t* Rst, int32_t* Col, double* Val) {
  const int64_t n = g * g;
  std::vector<int64_t> len((size_t)n);
  for (int64_t i = 0; i < n; ++i) {
    int64_t r = i / g, c = i % g;
    len[(size_t)i] = 1 + (r > 0) + (r < g - 1) + (c > 0) + (c < g - 1);
  }
  int64_t nz = finish_rst(len, n, Rst);
  if (!Rst || !Col || !Val) return nz;
  parallel_rows(n, [&](int64_t i) {
    int64_t r = i / g, c = i % g, k = Rst[i];
    if (r > 0) { Col[k] = (int32_t)(i - g); Val[k++] = -1.0; }
    if (c > 0) { Col[k] = (int32_t)(i - 1); Val[k++] = -1.0; }
    Col[k] = (int32_t)i; Val[k++] = 4.0;
    if (c < g - 1) { Col[k] = (int32_t)(i + 1); Val[k++] = -1.0; }
    if (r < g - 1) { Col[k] = (int32_t)(i + g); Val[k++] = -1.0; }
  });
  return nz;
}

int64_t rvvla_gen_stencil27(int64_t g, uint64_t seed, int32_t* Rst, int32_t* Col, double* Val) {
  if (g < 3) return -1;
  const int64_t n = g * g * g;
  if (Rst) for (int64_t i = 0; i <= n; ++i) Rst[i] = (int32_t)(27 * i);
  if (!Rst || !Col || !Val) return 27 * n;
  parallel_rows(n, [&](int64_t i) {
    int64_t z = i / (g * g), y = (i / g) % g, x = i % g;
    int64_t cols[27];
    int q = 0;
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          int64_t zz = (z + dz + g) % g, yy = (y + dy + g) % g, xx = (x + dx + g) % g;
          cols[q++] = (zz * g + yy) * g + xx;
        }
    std::sort(cols, cols + 27);
    Rng rng(seed, (uint64_t)i);
    for (int k = 0; k < 27; ++k) {
      Col[27 * i + k] = (int32_t)cols[k];
      Val[27 * i + k] = 1.0 + 0.1 * rng.normal();
    }
  });
  return 27 * n;
}

int64_t rvvla_gen_powerlaw(int64_t n, double mean, double sigma, int64_t cap, int64_t band,
                           double band_frac, uint64_t seed, int32_t* Rst, int32_t* Col,
                           double* Val) {
  if (n <= 0) return 0;
  cap = std::min(cap, n);
  const double mu = std::log(mean) - 0.5 * sigma * sigma;
  std::vector<int64_t> len((size_t)n);
  parallel_rows(n, [&](int64_t i) {
    Rng rng(seed, (uint64_t)i);
    double l = std::exp(mu + sigma * rng.normal());
    int64_t L = (int64_t)std::llround(l);
    len[(size_t)i] = std::max<int64_t>(1, std::min(cap, L));
  });
  int64_t nz = finish_rst(len, n, Rst);
  if (!Rst || !Col || !Val) return nz;
  parallel_rows(n, [&](int64_t i) {
    Rng rng(seed, (uint64_t)i);
    (void)rng.normal();  // the length draw
    const int64_t L = len[(size_t)i];
    thread_local ColSet set;
    set.reset(L);
    int32_t* c = Col + Rst[i];
    for (int64_t k = 0; k < L; ++k) {
      int64_t col = -1;
      for (int attempt = 0; attempt < 64 && col < 0; ++attempt) {
        int64_t cand;
        if (rng.uni() < band_frac) {
          cand = i + rng.below(2 * band + 1) - band;
          cand = std::min(std::max<int64_t>(cand, 0), n - 1);
        } else {
          cand = rng.below(n);
        }
        if (set.insert(cand)) col = cand;
      }
      while (col < 0) {  // band exhausted: uniform draws until unique
        int64_t cand = rng.below(n);
        if (set.insert(cand)) col = cand;
      }
      c[k] = (int32_t)col;
    }
    std::sort(c, c + L);
    for (int64_t k = 0; k < L; ++k) Val[Rst[i] + k] = 2.0 * rng.uni() - 1.0;
  });
  return nz;
}

int64_t rvvla_gen_random_rows(int64_t m, int64_t n, int dist, double param, int val_dist,
                              uint64_t seed, int32_t* Rst, int32_t* Col, double* Val) {
  if (m <= 0 || n <= 0) { if (Rst && m >= 0) for (int64_t i = 0; i <= m; ++i) Rst[i] = 0; return 0; }
  std::vector<int64_t> len((size_t)m);
  parallel_rows(m, [&](int64_t i) {
    Rng rng(seed, (uint64_t)i);
    int64_t L;
    if (dist == 0) {  // geometric on {1, 2, ...} with success probability param
      double u = rng.uni_open();
      L = 1 + (int64_t)std::floor(std::log(u) / std::log1p(-param));
    } else {  // Poisson(param), Knuth
      double lim = std::exp(-param), p = 1.0;
      L = -1;
      do { L++; p *= rng.uni(); } while (p > lim);
    }
    len[(size_t)i] = std::max<int64_t>(0, std::min(L, n));
  });
  int64_t nz = finish_rst(len, m, Rst);
  if (!Rst || !Col || !Val) return nz;
  parallel_rows(m, [&](int64_t i) {
    Rng rng(seed ^ 0x5bd1e995ULL, (uint64_t)i);
    const int64_t L = len[(size_t)i];
    thread_local ColSet set;
    set.reset(L);
    int32_t* c = Col + Rst[i];
    for (int64_t k = 0; k < L; ++k) {
      int64_t col;
      do { col = rng.below(n); } while (!set.insert(col));
      c[k] = (int32_t)col;
    }
    std::sort(c, c + L);
    for (int64_t k = 0; k < L; ++k) Val[Rst[i] + k] = val_dist == 0 ? rng.normal() : 2.0 * rng.uni() - 1.0;
  });
  return nz;
}

void rvvla_gen_vector(int64_t n, uint64_t seed, int normal, double lo, double hi, double* out) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    Rng rng(seed, (uint64_t)i);
    out[i] = normal ? rng.normal() : lo + (hi - lo) * rng.uni();
  }
}

}  // extern "C"
