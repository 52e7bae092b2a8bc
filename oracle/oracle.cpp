// oracle.cpp -- CPU restatement of the Distributed Ranges gemv hot path.
//
// TEST INFRASTRUCTURE ONLY: the checker for the CUDA path (tests/, smoke(),
// and bench.py's CPU-baseline leg).  The product never calls it.
//
// Compiled with -ffp-contract=off so every multiply and add rounds exactly as
// the reference's scalar loop does (no fused multiply-add contraction).
#include "oracle.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <thread>
#include <unordered_set>
#include <utility>
#include <vector>

namespace {

struct pair_hash_u {
  template <class I> std::size_t operator()(const std::pair<I, I> &v) const {
    // Any hash works: membership only; entry order comes from the sort below.
    return std::hash<unsigned long long>()((unsigned long long)v.first *
                                               1000003ull ^
                                           (unsigned long long)v.second);
  }
};

template <class T> struct value_dist {
  using type = std::uniform_real_distribution<T>;
};

// --- generate_random_csr (generate_csr.hpp:40-103) -----------------------
template <class T, class I>
void gen_random(int64_t m, int64_t n, double density, uint32_t seed,
                I *rowptr, I *colind, T *vals) {
  // generate_csr.hpp:48: nnz = size_t(density * shape[0] * shape[1]),
  // evaluated left to right in double.
  std::size_t nnz = (std::size_t)(density * (I)m * (I)n);
  std::unordered_set<std::pair<I, I>, pair_hash_u> seen;
  std::vector<std::pair<std::pair<I, I>, T>> entries;
  entries.reserve(nnz);
  // generate_csr.hpp:51-55: one mt19937 engine drives row, column and value.
  std::mt19937 gen(seed);
  std::uniform_int_distribution<I> row((I)0, (I)m - 1);
  std::uniform_int_distribution<I> col((I)0, (I)n - 1);
  typename value_dist<T>::type value_gen(0, 1);
  // generate_csr.hpp:57-65: draw row, then column; a value is drawn only for
  // a pair not seen before.
  while (seen.size() < nnz) {
    I i = row(gen);
    I j = col(gen);
    if (seen.find({i, j}) == seen.end()) {
      T v = value_gen(gen);
      seen.insert({i, j});
      entries.push_back({{i, j}, v});
    }
  }
  // generate_csr.hpp:74: keys are unique, so the sorted order is total.
  std::sort(entries.begin(), entries.end());
  // generate_csr.hpp:70-100: CSR fill with a row cursor.
  rowptr[0] = 0;
  std::size_t r = 0, c = 0;
  for (auto &e : entries) {
    I i = e.first.first;
    vals[c] = e.second;
    colind[c] = e.first.second;
    while (r < (std::size_t)i) {
      rowptr[r + 1] = (I)c;
      r++;
    }
    c++;
  }
  for (; r < (std::size_t)m; r++)
    rowptr[r + 1] = (I)nnz;
}

// --- generate_band_csr (generate_csr.hpp:108-153) -------------------------
template <class T, class I>
void gen_band(int64_t size, int64_t up, int64_t down, I *rowptr, I *colind,
              T *vals) {
  rowptr[0] = 0;
  std::size_t c = 0;
  for (int64_t i = 0; i < size; i++) {
    for (int64_t j = std::max<int64_t>(i - down, 0); j < i; j++) {
      vals[c] = 1;
      colind[c] = (I)j;
      c++;
    }
    vals[c] = 1;
    colind[c] = (I)i;
    c++;
    for (int64_t j = i + 1; j <= i + up; j++) {
      if (j >= size)
        continue;
      vals[c] = 1;
      colind[c] = (I)j;
      c++;
    }
    rowptr[i + 1] = (I)c;
  }
}

template <class Acc, class T> struct acc_out {
  using type = double;
};
template <class T> struct acc_out<T, T> {
  using type = T;
};

// --- csr_row_distribution::local_gemv CPU branch + gather -----------------
// csr_row_distribution.hpp:116-133 (loop), :159-204 (gather), :234-262
// (segment nnz ranges), distributed_vector.hpp:310 (segment size ceil(m/P)).
template <class T, class I, class Acc, class Out>
void gemv_row_segment(int64_t m, int64_t n, const I *rowptr, const I *colind,
                      const T *vals, const T *x, int64_t k, int64_t seg,
                      int64_t rank, Acc *partial /* seg*k, zeroed */) {
  if (m <= seg * rank)
    return;
  int64_t size = std::min(seg, m - seg * rank);
  const I *local_rows = rowptr + seg * rank; // the rank's rowptr slice
  int64_t first = seg * rank;
  int64_t lower = (int64_t)rowptr[first];
  int64_t higher =
      (seg * (rank + 1) < m) ? (int64_t)rowptr[seg * (rank + 1)] : (int64_t)rowptr[m];
  int64_t val_count = higher - lower;
  int64_t row_i = 0;
  int64_t position = lower;
  int64_t current_row_position = size > 1 ? (int64_t)local_rows[1] : 0;
  for (int64_t i = 0; i < val_count; i++) {
    while (row_i + 1 < size && position + i >= current_row_position) {
      row_i++;
      current_row_position = (int64_t)local_rows[row_i + 1];
    }
    for (int64_t j = 0; j < k; j++) {
      partial[row_i + j * seg] +=
          (Acc)vals[lower + i] * (Acc)x[(int64_t)colind[lower + i] + j * n];
    }
  }
}

template <class T, class I, class Acc, class Out>
void gemv_row(int64_t m, int64_t n, const I *rowptr, const I *colind,
              const T *vals, const T *x, int64_t k, Out *y, int nseg) {
  int64_t P = std::max(nseg, 1);
  int64_t seg = (m + P - 1) / P;
  std::vector<Acc> partial;
  for (int64_t r = 0; r < P; r++) {
    partial.assign((size_t)std::max<int64_t>(seg * k, 1), (Acc)0);
    gemv_row_segment<T, I, Acc, Out>(m, n, rowptr, colind, vals, x, k, seg, r,
                                     partial.data());
    if (r * seg >= m)
      break;
    int64_t cnt = std::min(seg, m - r * seg);
    for (int64_t j = 0; j < k; j++)
      for (int64_t i = 0; i < cnt; i++)
        y[m * j + r * seg + i] = (Out)partial[i + j * seg];
  }
}

// --- csr_eq_distribution::local_gemv CPU branch + gather ------------------
// csr_eq_distribution.hpp:112-130 (loop), :159-216 (gather with split-row
// add), :253-272 (row ranges by upper_bound over rowptr[0..m)).
template <class T, class I, class Acc, class Out>
void gemv_eq(int64_t m, int64_t n, const I *rowptr, const I *colind,
             const T *vals, const T *x, int64_t k, Out *y, int nseg) {
  int64_t P = std::max(nseg, 1);
  int64_t nnz = (int64_t)rowptr[m];
  int64_t seg = (nnz + P - 1) / P; // distributed_vector<T>(nnz) segment size
  std::vector<int64_t> row_off(P), row_sz(P);
  for (int64_t r = 0; r < P; r++) {
    uint64_t first_index = (uint64_t)(seg * r);
    uint64_t last_index = (uint64_t)(seg * (r + 1)) - 1; // may wrap when seg=0
    auto ub = [&](uint64_t v) {
      int64_t lo = 0, hi = m; // upper_bound over rowptr[0..m)
      while (lo < hi) {
        int64_t mid = (lo + hi) / 2;
        if ((uint64_t)rowptr[mid] <= v)
          lo = mid + 1;
        else
          hi = mid;
      }
      return lo;
    };
    int64_t lower = ub(first_index) - 1;
    int64_t higher = ub(last_index);
    row_off[r] = lower;
    row_sz[r] = higher - lower;
  }
  for (int64_t i = 0; i < m * k; i++)
    y[i] = (Out)0; // rng::fill(res, 0) (:185)
  std::vector<Acc> partial;
  for (int64_t r = 0; r < P; r++) {
    int64_t size = row_sz[r];
    partial.assign((size_t)std::max<int64_t>(size * k, 1), (Acc)0);
    if (!(nnz <= seg * r)) {
      const I *rows_data = rowptr + row_off[r];
      int64_t row_i = -1;
      int64_t position = seg * r;
      int64_t elem_count = std::min(seg, nnz - seg * r);
      int64_t current_row_position = (int64_t)rows_data[0];
      for (int64_t i = 0; i < elem_count; i++) {
        while (row_i + 1 < size && position + i >= current_row_position) {
          row_i++;
          // rows_data[size] is read past the segment's rowptr slice when
          // row_i + 1 == size; its value is never compared (the loop
          // condition's first clause fails), so any in-bounds value is
          // equivalent.
          current_row_position =
              (row_off[r] + row_i + 1 <= m) ? (int64_t)rows_data[row_i + 1] : 0;
        }
        for (int64_t j = 0; j < k; j++)
          partial[row_i + j * size] += (Acc)vals[position + i] *
                                       (Acc)x[(int64_t)colind[position + i] + j * n];
      }
    }
    // gather: add the first row, copy the others (:193-202)
    for (int64_t j = 0; j < k; j++) {
      int64_t first_row = row_off[r], last_row = row_off[r] + size;
      if (first_row < last_row)
        y[first_row + j * m] = (Out)((Acc)y[first_row + j * m] + partial[j * size]);
      for (int64_t q = 1; q < last_row - first_row; q++)
        y[first_row + q + j * m] = (Out)partial[j * size + q];
    }
  }
}

template <class T, class I>
int dispatch_acc(int acc, int eq, int64_t m, int64_t n, const void *rp,
                 const void *ci, const void *v, const void *x, int64_t k,
                 void *y, int nseg) {
  auto R = (const I *)rp;
  auto C = (const I *)ci;
  auto V = (const T *)v;
  auto X = (const T *)x;
  if (acc == ORC_ACC_T) {
    if (eq)
      gemv_eq<T, I, T, T>(m, n, R, C, V, X, k, (T *)y, nseg);
    else
      gemv_row<T, I, T, T>(m, n, R, C, V, X, k, (T *)y, nseg);
  } else if (acc == ORC_ACC_F64) {
    if (eq)
      gemv_eq<T, I, double, double>(m, n, R, C, V, X, k, (double *)y, nseg);
    else
      gemv_row<T, I, double, double>(m, n, R, C, V, X, k, (double *)y, nseg);
  } else if (acc == ORC_ACC_LD) {
    if (eq)
      gemv_eq<T, I, long double, double>(m, n, R, C, V, X, k, (double *)y, nseg);
    else
      gemv_row<T, I, long double, double>(m, n, R, C, V, X, k, (double *)y,
                                          nseg);
  } else {
    return 1;
  }
  return 0;
}

#define ORC_DISPATCH(vtype, itype, ...)                                       \
  do {                                                                         \
    if (vtype == ORC_F32 && itype == ORC_I32) {                                \
      using T = float;                                                         \
      using I = int32_t;                                                       \
      __VA_ARGS__;                                                                  \
    } else if (vtype == ORC_F32 && itype == ORC_I64) {                         \
      using T = float;                                                         \
      using I = int64_t;                                                       \
      __VA_ARGS__;                                                                  \
    } else if (vtype == ORC_F32 && itype == ORC_U64) {                         \
      using T = float;                                                         \
      using I = unsigned long;                                                 \
      __VA_ARGS__;                                                                  \
    } else if (vtype == ORC_F64 && itype == ORC_I32) {                         \
      using T = double;                                                        \
      using I = int32_t;                                                       \
      __VA_ARGS__;                                                                  \
    } else if (vtype == ORC_F64 && itype == ORC_I64) {                         \
      using T = double;                                                        \
      using I = int64_t;                                                       \
      __VA_ARGS__;                                                                  \
    } else if (vtype == ORC_F64 && itype == ORC_U64) {                         \
      using T = double;                                                        \
      using I = unsigned long;                                                 \
      __VA_ARGS__;                                                                  \
    } else {                                                                   \
      return 1;                                                                \
    }                                                                          \
  } while (0)

} // namespace

extern "C" {

int64_t orc_random_csr_nnz(int64_t m, int64_t n, double density) {
  return (int64_t)(std::size_t)(density * (unsigned long)m * (unsigned long)n);
}

int orc_gen_random_csr(int vtype, int itype, int64_t m, int64_t n,
                       double density, uint32_t seed, void *rowptr,
                       void *colind, void *vals) {
  if (m <= 0 || n <= 0 || !(density >= 0.0 && density < 1.0))
    return 1;
  ORC_DISPATCH(vtype, itype,
               gen_random<T, I>(m, n, density, seed, (I *)rowptr, (I *)colind,
                                (T *)vals));
  return 0;
}

int64_t orc_band_csr_nnz(int64_t size, int64_t up, int64_t down) {
  return (1 + up + down) * size - (up * (up + 1) / 2) - (down * (down + 1) / 2);
}

int orc_gen_band_csr(int vtype, int itype, int64_t size, int64_t up,
                     int64_t down, void *rowptr, void *colind, void *vals) {
  if (size <= 0 || up < 0 || down < 0)
    return 1;
  ORC_DISPATCH(vtype, itype,
               gen_band<T, I>(size, up, down, (I *)rowptr, (I *)colind,
                              (T *)vals));
  return 0;
}

int orc_csr_gemv_row(int vtype, int itype, int acc, int64_t m, int64_t n,
                     const void *rowptr, const void *colind, const void *vals,
                     const void *x, int64_t k, void *y, int nseg) {
  if (m < 0 || n < 0 || k < 1)
    return 1;
  ORC_DISPATCH(vtype, itype,
               return dispatch_acc<T, I>(acc, 0, m, n, rowptr, colind, vals, x,
                                         k, y, nseg));
}

int orc_csr_gemv_eq(int vtype, int itype, int acc, int64_t m, int64_t n,
                    const void *rowptr, const void *colind, const void *vals,
                    const void *x, int64_t k, void *y, int nseg) {
  if (m <= 0 || n < 0 || k < 1)
    return 1;
  ORC_DISPATCH(vtype, itype,
               return dispatch_acc<T, I>(acc, 1, m, n, rowptr, colind, vals, x,
                                         k, y, nseg));
}

int orc_csr_gemv_row_threads(int vtype, int itype, int64_t m, int64_t n,
                             const void *rowptr, const void *colind,
                             const void *vals, const void *x, int64_t k,
                             void *y, int nthreads, double *t_local,
                             double *t_gather) {
  if (m < 0 || k < 1 || nthreads < 1)
    return 1;
  ORC_DISPATCH(vtype, itype, {
    int64_t P = nthreads;
    int64_t seg = (m + P - 1) / P;
    std::vector<std::vector<T>> partial(P);
    auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> th;
    for (int64_t r = 0; r < P; r++) {
      th.emplace_back([&, r] {
        // Each "rank" allocates and zero-fills its partial result
        // (csr_row_distribution.hpp:141-146) and runs the CPU loop.
        partial[r].assign((size_t)std::max<int64_t>(seg * k, 1), (T)0);
        gemv_row_segment<T, I, T, T>(m, n, (const I *)rowptr,
                                     (const I *)colind, (const T *)vals,
                                     (const T *)x, k, seg, r, partial[r].data());
      });
    }
    for (auto &t : th)
      t.join();
    auto t1 = std::chrono::steady_clock::now();
    T *Y = (T *)y;
    for (int64_t r = 0; r < P; r++) {
      if (r * seg >= m)
        break;
      int64_t cnt = std::min(seg, m - r * seg);
      for (int64_t j = 0; j < k; j++)
        std::memcpy(Y + m * j + r * seg, partial[r].data() + j * seg,
                    sizeof(T) * cnt);
    }
    auto t2 = std::chrono::steady_clock::now();
    if (t_local)
      *t_local = std::chrono::duration<double>(t1 - t0).count();
    if (t_gather)
      *t_gather = std::chrono::duration<double>(t2 - t1).count();
  });
  return 0;
}

int orc_csr_absdot(int vtype, int itype, int64_t m, int64_t n,
                   const void *rowptr, const void *colind, const void *vals,
                   const void *x, int64_t k, double *d) {
  ORC_DISPATCH(vtype, itype, {
    auto R = (const I *)rowptr;
    auto C = (const I *)colind;
    auto V = (const T *)vals;
    auto X = (const T *)x;
    for (int64_t j = 0; j < k; j++)
      for (int64_t r = 0; r < m; r++) {
        long double s = 0;
        for (int64_t p = (int64_t)R[r]; p < (int64_t)R[r + 1]; p++)
          s += std::fabs((long double)V[p] * (long double)X[(int64_t)C[p] + j * n]);
        d[r + j * m] = (double)s;
      }
  });
  return 0;
}

int orc_cg(int vtype, int itype, int64_t n, const void *rowptr,
           const void *colind, const void *vals, const double *b, double *x,
           int64_t max_iters, double rtol, int64_t *iters, double *rnorm,
           double *bnorm, int *status, double *hist) {
  if (n < 0 || max_iters < 0)
    return 1;
  ORC_DISPATCH(vtype, itype, {
    auto R = (const I *)rowptr;
    auto Cc = (const I *)colind;
    auto V = (const T *)vals;
    std::vector<double> r(n), p(n), q(n);
    auto matvec = [&](const std::vector<double> &in, std::vector<double> &out) {
      for (int64_t i = 0; i < n; i++) {
        double sum = 0;
        for (int64_t k = (int64_t)R[i]; k < (int64_t)R[i + 1]; k++)
          sum += (double)V[k] * in[(int64_t)Cc[k]];
        out[i] = sum;
      }
    };
    auto dot = [&](const std::vector<double> &a, const std::vector<double> &c) {
      double s = 0;
      for (int64_t i = 0; i < n; i++)
        s += a[i] * c[i];
      return s;
    };
    std::vector<double> xv(x, x + n), bv(b, b + n);
    matvec(xv, q);
    for (int64_t i = 0; i < n; i++)
      r[i] = p[i] = bv[i] - q[i];
    double rr = dot(r, r);
    const double bb = dot(bv, bv);
    const double tol2 = rtol * rtol * bb;
    int64_t it = 0;
    int st = rr <= tol2 ? 1 : (max_iters <= 0 ? 3 : 0);
    if (hist)
      hist[0] = std::sqrt(rr);
    while (st == 0) {
      matvec(p, q);
      const double pq = dot(p, q);
      const double alpha = rr / pq;
      if (!(pq > 0) || !std::isfinite(alpha)) {
        st = 2;
        break;
      }
      for (int64_t i = 0; i < n; i++) {
        xv[i] += alpha * p[i];
        r[i] -= alpha * q[i];
      }
      const double rr1 = dot(r, r);
      it++;
      if (hist)
        hist[it] = std::sqrt(rr1);
      const double beta = rr1 / rr;
      rr = rr1;
      st = rr1 <= tol2 ? 1 : (it >= max_iters ? 3 : 0);
      if (st == 0)
        for (int64_t i = 0; i < n; i++)
          p[i] = r[i] + beta * p[i];
    }
    std::copy(xv.begin(), xv.end(), x);
    *iters = it;
    *rnorm = std::sqrt(rr);
    *bnorm = std::sqrt(bb);
    *status = st;
  });
  return 0;
}

int orc_dense_gemv(int vtype, int acc, int64_t m, int64_t n, const void *A,
                   int64_t lda, const void *x, int64_t k, void *y) {
  auto run = [&](auto tag, auto acc_tag) {
    using T = decltype(tag);
    using Acc = decltype(acc_tag);
    auto a = (const T *)A;
    auto X = (const T *)x;
    for (int64_t j = 0; j < k; j++)
      for (int64_t r = 0; r < m; r++) {
        Acc s = 0;
        for (int64_t c = 0; c < n; c++)
          s += (Acc)a[r * lda + c] * (Acc)X[c + j * n];
        if (acc == ORC_ACC_T)
          ((T *)y)[r + j * m] = (T)s;
        else
          ((double *)y)[r + j * m] = (double)s;
      }
  };
  if (vtype == ORC_F32) {
    if (acc == ORC_ACC_T)
      run(float(), float());
    else if (acc == ORC_ACC_F64)
      run(float(), double());
    else
      run(float(), (long double)0);
  } else if (vtype == ORC_F64) {
    if (acc == ORC_ACC_LD)
      run(double(), (long double)0);
    else
      run(double(), double());
  } else {
    return 1;
  }
  return 0;
}

int orc_csr_transpose(int vtype, int itype, int64_t m, int64_t n,
                      const void *rowptr, const void *colind, const void *vals,
                      void *colptr, void *rowidx, void *vals_t) {
  ORC_DISPATCH(vtype, itype, {
    auto R = (const I *)rowptr;
    auto C = (const I *)colind;
    auto V = (const T *)vals;
    auto CP = (I *)colptr;
    auto RI = (I *)rowidx;
    auto VT = (T *)vals_t;
    int64_t nnz = (int64_t)R[m];
    std::vector<int64_t> cnt(n + 1, 0);
    for (int64_t p = 0; p < nnz; p++)
      cnt[(int64_t)C[p] + 1]++;
    for (int64_t c = 0; c < n; c++)
      cnt[c + 1] += cnt[c];
    for (int64_t c = 0; c <= n; c++)
      CP[c] = (I)cnt[c];
    for (int64_t r = 0; r < m; r++)
      for (int64_t p = (int64_t)R[r]; p < (int64_t)R[r + 1]; p++) {
        int64_t q = cnt[(int64_t)C[p]]++;
        RI[q] = (I)r;
        VT[q] = V[p];
      }
  });
  return 0;
}

int orc_csr_abar(int vtype, int itype, int64_t m, const void *rowptr,
                 const void *colind, const void *ybar, const void *x,
                 double *abar) {
  ORC_DISPATCH(vtype, itype, {
    auto R = (const I *)rowptr;
    auto C = (const I *)colind;
    auto YB = (const T *)ybar;
    auto X = (const T *)x;
    for (int64_t r = 0; r < m; r++)
      for (int64_t p = (int64_t)R[r]; p < (int64_t)R[r + 1]; p++)
        abar[p] = (double)YB[r] * (double)X[(int64_t)C[p]];
  });
  return 0;
}

double orc_dot(int vtype, int64_t n, const void *a, const void *b) {
  long double s = 0;
  if (vtype == ORC_F32) {
    auto A = (const float *)a;
    auto B = (const float *)b;
    for (int64_t i = 0; i < n; i++)
      s += (long double)A[i] * (long double)B[i];
  } else {
    auto A = (const double *)a;
    auto B = (const double *)b;
    for (int64_t i = 0; i < n; i++)
      s += (long double)A[i] * (long double)B[i];
  }
  return (double)s;
}

void orc_f32_to_bf16(int64_t n, const float *in, uint16_t *out) {
  for (int64_t i = 0; i < n; i++) {
    uint32_t u;
    std::memcpy(&u, &in[i], 4);
    if ((u & 0x7f800000u) == 0x7f800000u && (u & 0x007fffffu)) {
      out[i] = (uint16_t)((u >> 16) | 0x0040u); // quiet NaN
    } else {
      uint32_t lsb = (u >> 16) & 1u;
      out[i] = (uint16_t)((u + 0x7fffu + lsb) >> 16);
    }
  }
}

void orc_bf16_to_f32(int64_t n, const uint16_t *in, float *out) {
  for (int64_t i = 0; i < n; i++) {
    uint32_t u = (uint32_t)in[i] << 16;
    std::memcpy(&out[i], &u, 4);
  }
}


// ---- Matrix Market ingest --------------------------------------------------

static int mm_fail(char *err, int errlen, int code, const char *msg,
                   const char *path) {
  if (err && errlen > 0)
    std::snprintf(err, (size_t)errlen, "%s: %s", path, msg);
  return code;
}

int orc_read_matrix_market(const char *path, int one_indexed, int64_t *m,
                           int64_t *n, int64_t *nnz, int64_t **rowptr,
                           int64_t **colind, double **values, char *err,
                           int errlen) {
  FILE *f = std::fopen(path, "r");
  if (!f)
    return mm_fail(err, errlen, 1, "mmread: cannot open", path);
  std::vector<char> line(1 << 16);
  auto getline = [&](void) -> bool {
    return std::fgets(line.data(), (int)line.size(), f) != nullptr;
  };
  // header: five whitespace-separated tokens
  char t[5][64] = {};
  if (!getline() ||
      std::sscanf(line.data(), "%63s %63s %63s %63s %63s", t[0], t[1], t[2],
                  t[3], t[4]) < 3 ||
      std::strcmp(t[0], "%%MatrixMarket") != 0 ||
      std::strcmp(t[1], "matrix") != 0 || std::strcmp(t[2], "coordinate") != 0) {
    std::fclose(f);
    return mm_fail(err, errlen, 2, "could not be parsed as a Matrix Market file.",
                   path);
  }
  const bool pattern = std::strcmp(t[3], "pattern") == 0;
  bool symmetric;
  if (std::strcmp(t[4], "general") == 0)
    symmetric = false;
  else if (std::strcmp(t[4], "symmetric") == 0)
    symmetric = true;
  else {
    std::fclose(f);
    return mm_fail(err, errlen, 3, "has an unsupported matrix type", path);
  }
  // comments, then the size line
  bool have = false;
  while (getline()) {
    if (line[0] != '%') {
      have = true;
      break;
    }
  }
  long long mm = 0, nn = 0, declared = 0;
  if (!have || std::sscanf(line.data(), "%lld %lld %lld", &mm, &nn, &declared) != 3 ||
      mm < 0 || nn < 0 || declared < 0) {
    std::fclose(f);
    return mm_fail(err, errlen, 6, "malformed size line", path);
  }
  // entries, per row in file order (mirrored entries right after theirs)
  std::vector<std::vector<std::pair<int64_t, double>>> rows((size_t)mm);
  long long count = 0;
  while (getline()) {
    const char *p = line.data();
    while (*p == ' ' || *p == '\t' || *p == '\r' || *p == '\n')
      p++;
    if (*p == 0)
      continue; // blank line
    long long i = 0, j = 0;
    double v = 1.0;
    const int got = pattern ? std::sscanf(p, "%lld %lld", &i, &j)
                            : std::sscanf(p, "%lld %lld %lf", &i, &j, &v);
    if (got != (pattern ? 2 : 3)) {
      std::fclose(f);
      return mm_fail(err, errlen, 6, "malformed entry line", path);
    }
    if (one_indexed) {
      i--;
      j--;
    }
    if (i < 0 || j < 0 || i >= mm || j >= nn) {
      std::fclose(f);
      return mm_fail(err, errlen, 4, "read_MatrixMarket: file has nonzero out of bounds.", path);
    }
    rows[(size_t)i].push_back({j, v});
    if (symmetric && i != j)
      rows[(size_t)j].push_back({i, v});
    if (++count > declared) {
      std::fclose(f);
      return mm_fail(err, errlen, 5,
                     "read_MatrixMarket: error reading Matrix Market "
                     "file, file has more nonzeros than reported.", path);
    }
  }
  std::fclose(f);
  int64_t total = 0;
  for (auto &r : rows) {
    std::stable_sort(r.begin(), r.end(), [](const auto &a, const auto &b) {
      return a.first < b.first;
    });
    total += (int64_t)r.size();
  }
  *m = mm;
  *n = nn;
  *nnz = total;
  *rowptr = (int64_t *)std::malloc(sizeof(int64_t) * (size_t)(mm + 1));
  *colind = (int64_t *)std::malloc(sizeof(int64_t) * (size_t)std::max<int64_t>(total, 1));
  *values = (double *)std::malloc(sizeof(double) * (size_t)std::max<int64_t>(total, 1));
  int64_t c = 0;
  (*rowptr)[0] = 0;
  for (int64_t r = 0; r < mm; r++) {
    for (auto &e : rows[(size_t)r]) {
      (*colind)[c] = e.first;
      (*values)[c] = e.second;
      c++;
    }
    (*rowptr)[r + 1] = c;
  }
  return 0;
}

void orc_free(void *p) { std::free(p); }

} // extern "C"

// ---- parity statistics ------------------------------------------------------
namespace {

inline long double elem(int t, const void *p, int64_t i) {
  switch (t) {
  case ORC_F32:
    return ((const float *)p)[i];
  case ORC_F64:
    return ((const double *)p)[i];
  default: {
    uint32_t u = (uint32_t)((const uint16_t *)p)[i] << 16;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
  }
  }
}

inline bool type_ok(int t) { return t == ORC_F32 || t == ORC_F64 || t == ORC_BF16; }

struct BinStats {
  std::vector<double> mx, sm;
  std::vector<int64_t> cnt;
  double worst = -1.0;
  int64_t worst_row = -1;
  explicit BinStats(int nb) : mx(nb, 0.0), sm(nb, 0.0), cnt(nb, 0) {}
  void add(int b, double e, int64_t row) {
    if (!(e == e)) // NaN: counts as infinite
      e = INFINITY;
    if (b >= 0) {
      mx[b] = std::max(mx[b], e);
      sm[b] += e;
      cnt[b]++;
    }
    if (e > worst) {
      worst = e;
      worst_row = row;
    }
  }
  void merge(const BinStats &o) {
    for (size_t b = 0; b < mx.size(); b++) {
      mx[b] = std::max(mx[b], o.mx[b]);
      sm[b] += o.sm[b];
      cnt[b] += o.cnt[b];
    }
    if (o.worst > worst || (o.worst == worst && o.worst_row < worst_row)) {
      worst = o.worst;
      worst_row = o.worst_row;
    }
  }
};

inline double row_err(long double yv, long double ref, long double d) {
  const long double diff = std::fabs(yv - ref);
  return (double)(d > 0 ? diff / d : diff);
}

// Rows [0, m) in blocks of 4096 taken from an atomic counter by `nthreads`
// threads; f(r0, r1, stats) accumulates into the thread's stats.
template <class F>
void parallel_rows(int64_t m, int nthreads, int nbins, BinStats &out, F f) {
  const int64_t blk = 4096;
  std::atomic<int64_t> next{0};
  const int nt = std::max(1, nthreads);
  std::vector<BinStats> part(nt, BinStats(std::max(nbins, 1)));
  std::vector<std::thread> th;
  for (int t = 0; t < nt; t++)
    th.emplace_back([&, t] {
      for (;;) {
        const int64_t r0 = next.fetch_add(blk);
        if (r0 >= m)
          break;
        f(r0, std::min(m, r0 + blk), part[t]);
      }
    });
  for (auto &t : th)
    t.join();
  for (auto &p : part)
    out.merge(p);
}

} // namespace

extern "C" {

int orc_csr_check(int vtype, int xtype, int itype, int ytype, int64_t m,
                  int64_t n, const void *rowptr, const void *colind,
                  const void *vals, const void *x, int64_t k, const void *y,
                  int nthreads, const int64_t *edges, int nbins, double *bmax,
                  double *bsum, int64_t *bcount, double *worst,
                  int64_t *worst_row) {
  if (!type_ok(vtype) || !type_ok(xtype) || (ytype != ORC_F32 && ytype != ORC_F64) ||
      (itype != ORC_I32 && itype != ORC_I64) || m < 0 || n < 0 || k < 1 || nbins < 0)
    return 1;
  auto idx = [&](const void *p, int64_t i) -> int64_t {
    return itype == ORC_I32 ? (int64_t)((const int32_t *)p)[i] : ((const int64_t *)p)[i];
  };
  auto bin_of = [&](int64_t len) -> int {
    for (int b = 0; b < nbins; b++)
      if (len >= edges[b] && len < edges[b + 1])
        return b;
    return -1;
  };
  BinStats all(std::max(nbins, 1));
  parallel_rows(m, nthreads, nbins, all, [&](int64_t r0, int64_t r1, BinStats &st) {
    for (int64_t r = r0; r < r1; r++) {
      const int64_t p0 = idx(rowptr, r), p1 = idx(rowptr, r + 1);
      const int b = bin_of(p1 - p0);
      for (int64_t j = 0; j < k; j++) {
        long double s = 0, d = 0;
        for (int64_t p = p0; p < p1; p++) {
          const long double t = elem(vtype, vals, p) * elem(xtype, x, idx(colind, p) + j * n);
          s += t;
          d += std::fabs(t);
        }
        st.add(nbins > 0 ? b : -1, row_err(elem(ytype, y, r + j * m), s, d), r);
      }
    }
  });
  for (int b = 0; b < nbins; b++) {
    bmax[b] = all.mx[b];
    bsum[b] = all.sm[b];
    bcount[b] = all.cnt[b];
  }
  if (worst)
    *worst = std::max(0.0, all.worst);
  if (worst_row)
    *worst_row = all.worst_row;
  return 0;
}

int orc_dense_check(int atype, int xtype, int ytype, int64_t m, int64_t n,
                    const void *A, int64_t lda, const void *x, int64_t k,
                    const void *y, int nthreads, double *max, double *sum,
                    int64_t *count) {
  if (!type_ok(atype) || !type_ok(xtype) || (ytype != ORC_F32 && ytype != ORC_F64) ||
      m < 0 || n < 0 || k < 1 || lda < n)
    return 1;
  BinStats all(1);
  parallel_rows(m, nthreads, 1, all, [&](int64_t r0, int64_t r1, BinStats &st) {
    for (int64_t r = r0; r < r1; r++)
      for (int64_t j = 0; j < k; j++) {
        long double s = 0, d = 0;
        for (int64_t c = 0; c < n; c++) {
          const long double t = elem(atype, A, r * lda + c) * elem(xtype, x, c + j * n);
          s += t;
          d += std::fabs(t);
        }
        st.add(0, row_err(elem(ytype, y, r + j * m), s, d), r);
      }
  });
  *max = all.mx[0];
  *sum = all.sm[0];
  *count = all.cnt[0];
  return 0;
}

} // extern "C"
