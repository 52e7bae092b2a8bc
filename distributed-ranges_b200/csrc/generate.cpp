// generate.cpp -- seeded synthetic CSR workloads (see include/drb_gen.h).
//
// Counter-based randomness: each row (or block of vector entries) seeds its
// own splitmix64 stream from (seed, stream id, index), so any thread count
// produces the same matrix.
#include "drb_gen.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <limits>
#include <thread>
#include <vector>

namespace {

inline uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

struct Rng {
  uint64_t s;
  Rng(uint64_t seed, uint64_t stream, uint64_t idx)
      : s(mix64(seed * 0x9E3779B97F4A7C15ull + stream) ^
          mix64(idx * 0xD1B54A32D192ED03ull + 0x632BE59BD9B4E019ull * (stream + 1))) {}
  uint64_t next() {
    s += 0x9E3779B97F4A7C15ull;
    return mix64(s);
  }
  double uniform01() { return (double)(next() >> 11) * 0x1.0p-53; }
  // uniform integer in [0, r] (Lemire's multiply-shift; bias < 2^-40 here)
  uint64_t below_incl(uint64_t r) {
    return (uint64_t)(((unsigned __int128)next() * (unsigned __int128)(r + 1)) >> 64);
  }
  double normal() {
    double u1 = uniform01(), u2 = uniform01();
    if (u1 < 1e-300)
      u1 = 1e-300;
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  }
};

int pick_threads(int nthreads) {
  if (nthreads > 0)
    return nthreads;
  unsigned h = std::thread::hardware_concurrency();
  return (int)std::max(1u, std::min(h, 64u));
}

template <class F> void parallel_chunks(int64_t total, int64_t chunk, int nth, F f) {
  std::atomic<int64_t> next{0};
  auto work = [&] {
    for (;;) {
      const int64_t lo = next.fetch_add(chunk);
      if (lo >= total)
        return;
      f(lo, std::min(total, lo + chunk));
    }
  };
  if (nth <= 1 || total <= chunk) {
    work();
    return;
  }
  std::vector<std::thread> th;
  for (int t = 0; t < nth; t++)
    th.emplace_back(work);
  for (auto &t : th)
    t.join();
}

double draw_value(Rng &g, int dist, double row_scale) {
  switch (dist) {
  case DRB_GEN_UNIFORM_PM1:
    return 2.0 * g.uniform01() - 1.0;
  case DRB_GEN_NORMAL:
    return g.normal();
  case DRB_GEN_NORMAL_ROWSCALE:
    return g.normal() * row_scale;
  default:
    return 1.0;
  }
}

} // namespace

extern "C" {

double drb_gen_zipf_mean(int64_t lo, int64_t hi, double alpha) {
  long double num = 0, den = 0;
  for (int64_t k = lo; k <= hi; k++) {
    const long double w = std::pow((long double)k, -(long double)alpha);
    num += w * k;
    den += w;
  }
  return (double)(num / den);
}

double drb_gen_zipf_alpha_for_mean(int64_t lo, int64_t hi, double mean) {
  if (!(mean > (double)lo && mean < (double)hi))
    return std::numeric_limits<double>::quiet_NaN();
  double a = -10.0, b = 10.0; // mean decreases as alpha grows
  for (int it = 0; it < 200; it++) {
    const double c = 0.5 * (a + b);
    if (drb_gen_zipf_mean(lo, hi, c) > mean)
      a = c;
    else
      b = c;
  }
  return 0.5 * (a + b);
}

int64_t drb_gen_rowptr_zipf(int64_t m, int64_t n, double alpha, int64_t lo,
                            int64_t hi, uint64_t seed, int64_t *rowptr,
                            int nthreads) {
  if (m < 0 || n < 0 || lo < 0 || hi < lo || !rowptr)
    return -1;
  std::vector<double> cdf((size_t)(hi - lo + 1));
  long double acc = 0;
  for (int64_t k = lo; k <= hi; k++) {
    acc += std::pow((long double)std::max<int64_t>(k, 1), -(long double)alpha);
    cdf[(size_t)(k - lo)] = (double)acc;
  }
  for (auto &c : cdf)
    c /= (double)acc;
  const int nth = pick_threads(nthreads);
  parallel_chunks(m, 1 << 16, nth, [&](int64_t r0, int64_t r1) {
    for (int64_t r = r0; r < r1; r++) {
      Rng g(seed, 1, (uint64_t)r);
      const double u = g.uniform01();
      const int64_t k = lo + (int64_t)(std::upper_bound(cdf.begin(), cdf.end(), u) - cdf.begin());
      rowptr[r + 1] = std::min<int64_t>(std::min(k, hi), n);
    }
  });
  rowptr[0] = 0;
  for (int64_t r = 0; r < m; r++)
    rowptr[r + 1] += rowptr[r];
  return rowptr[m];
}

int64_t drb_gen_rowptr_uniform(int64_t m, int64_t n, int64_t lo, int64_t hi,
                               uint64_t seed, int64_t *rowptr, int nthreads) {
  if (m < 0 || n < 0 || lo < 0 || hi < lo || !rowptr)
    return -1;
  const int nth = pick_threads(nthreads);
  parallel_chunks(m, 1 << 16, nth, [&](int64_t r0, int64_t r1) {
    for (int64_t r = r0; r < r1; r++) {
      Rng g(seed, 1, (uint64_t)r);
      const int64_t k = lo + (int64_t)g.below_incl((uint64_t)(hi - lo));
      rowptr[r + 1] = std::min<int64_t>(k, n);
    }
  });
  rowptr[0] = 0;
  for (int64_t r = 0; r < m; r++)
    rowptr[r + 1] += rowptr[r];
  return rowptr[m];
}

int64_t drb_gen_rowptr_fixed(int64_t m, int64_t n, int64_t len,
                             int64_t *rowptr) {
  if (m < 0 || len < 0 || len > n || !rowptr)
    return -1;
  for (int64_t r = 0; r <= m; r++)
    rowptr[r] = r * len;
  return m * len;
}

int drb_gen_fill_uniform(int64_t m, int64_t n, const int64_t *rowptr,
                         uint64_t seed, int itype, void *colind, int vtype,
                         void *values, int dist, int nthreads) {
  if (m < 0 || n < 0 || !rowptr || (itype != 0 && itype != 1) ||
      (vtype != 0 && vtype != 1))
    return 1;
  const int nth = pick_threads(nthreads);
  int bad = 0;
  parallel_chunks(m, 4096, nth, [&](int64_t r0, int64_t r1) {
    std::vector<int64_t> cols;
    for (int64_t r = r0; r < r1; r++) {
      const int64_t p0 = rowptr[r], L = rowptr[r + 1] - p0;
      if (L <= 0)
        continue;
      if (L > n) {
        bad = 1;
        continue;
      }
      Rng g(seed, 2, (uint64_t)r);
      cols.resize((size_t)L);
      if (L == n) {
        for (int64_t i = 0; i < L; i++)
          cols[i] = i;
      } else {
        // L sorted draws from [0, n-L] plus their rank: distinct, ascending,
        // covering [0, n).
        for (int64_t i = 0; i < L; i++)
          cols[i] = (int64_t)g.below_incl((uint64_t)(n - L));
        std::sort(cols.begin(), cols.end());
        for (int64_t i = 0; i < L; i++)
          cols[i] += i;
      }
      const double scale =
          dist == DRB_GEN_NORMAL_ROWSCALE ? std::pow(10.0, 6.0 * g.uniform01() - 3.0) : 1.0;
      for (int64_t i = 0; i < L; i++) {
        if (itype == 0)
          ((int32_t *)colind)[p0 + i] = (int32_t)cols[i];
        else
          ((int64_t *)colind)[p0 + i] = cols[i];
        const double v = draw_value(g, dist, scale);
        if (vtype == 0)
          ((float *)values)[p0 + i] = (float)v;
        else
          ((double *)values)[p0 + i] = v;
      }
    }
  });
  return bad;
}

int64_t drb_gen_laplacian2d(int64_t g, int64_t *rowptr, int itype,
                            void *colind, int vtype, void *values) {
  if (g <= 0)
    return -1;
  const int64_t m = g * g;
  const int64_t nnz = 5 * m - 4 * g;
  if (!rowptr || !colind || !values)
    return nnz;
  int64_t c = 0;
  rowptr[0] = 0;
  auto put = [&](int64_t col, double v) {
    if (itype == 0)
      ((int32_t *)colind)[c] = (int32_t)col;
    else
      ((int64_t *)colind)[c] = col;
    if (vtype == 0)
      ((float *)values)[c] = (float)v;
    else
      ((double *)values)[c] = v;
    c++;
  };
  for (int64_t i = 0; i < m; i++) {
    const int64_t a = i / g, b = i % g;
    if (a > 0)
      put(i - g, -1.0);
    if (b > 0)
      put(i - 1, -1.0);
    put(i, 4.0);
    if (b < g - 1)
      put(i + 1, -1.0);
    if (a < g - 1)
      put(i + g, -1.0);
    rowptr[i + 1] = c;
  }
  return nnz;
}

int drb_gen_values(int64_t count, uint64_t seed, int vtype, void *out,
                   int dist, int nthreads) {
  if (count < 0 || !out || (vtype != 0 && vtype != 1))
    return 1;
  const int nth = pick_threads(nthreads);
  const int64_t B = 1024;
  const int64_t nb = (count + B - 1) / B;
  parallel_chunks(nb, 64, nth, [&](int64_t b0, int64_t b1) {
    for (int64_t b = b0; b < b1; b++) {
      Rng g(seed, 3, (uint64_t)b);
      const double scale =
          dist == DRB_GEN_NORMAL_ROWSCALE ? std::pow(10.0, 6.0 * g.uniform01() - 3.0) : 1.0;
      for (int64_t i = b * B; i < std::min(count, (b + 1) * B); i++) {
        const double v = draw_value(g, dist, scale);
        if (vtype == 0)
          ((float *)out)[i] = (float)v;
        else
          ((double *)out)[i] = v;
      }
    }
  });
  return 0;
}

} // extern "C"
