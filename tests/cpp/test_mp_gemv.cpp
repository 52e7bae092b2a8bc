// C++ drop-in check: the reference's gemv test cases (test/gtest/mp/gemv.cpp
// and test/gtest/mp/sparse_matrix.cpp), written against the dr::mp names
// through include/drb/dr_mp.hpp, run on the GPU through the C ABI.
// Prints one line per case and exits non-zero on any failure.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <limits>
#include <numeric>
#include <string>
#include <vector>

#include "drb/dr_mp.hpp"

static int failures = 0;
#define CHECK(cond, name)                                                      \
  do {                                                                         \
    if (cond) {                                                                \
      std::printf("PASS %s\n", name);                                          \
    } else {                                                                   \
      std::printf("FAIL %s (%s:%d)\n", name, __FILE__, __LINE__);              \
      failures++;                                                              \
    }                                                                          \
  } while (0)

// fp_equal of test/gtest/include/common-tests.hpp:82-111
template <class T> bool fp_equal(T a, T b) {
  if (a == b)
    return true;
  const T eps = 128 * std::numeric_limits<T>::epsilon();
  const T diff = std::abs(a - b);
  const T norm = std::min<T>(std::abs(a) + std::abs(b), std::numeric_limits<float>::max());
  return diff < std::max(std::numeric_limits<T>::min(), eps * norm);
}
template <class T> bool fp_equal(const std::vector<T> &a, const std::vector<T> &b) {
  if (a.size() != b.size())
    return false;
  for (std::size_t i = 0; i < a.size(); i++)
    if (!fp_equal(a[i], b[i]))
      return false;
  return true;
}

template <class M> bool gemv_case(std::size_t m, std::size_t k, M &a) {
  std::vector<float> base_b(k, 1.f), c(m, 0.f);
  dr::mp::broadcasted_vector<float> b;
  b.broadcast_data(k, 0, base_b, dr::mp::default_comm());
  dr::mp::gemv(c, a, b);
  std::vector<float> c_ref(m, 0.f);
  for (auto &&[index, v] : a) {
    auto &&[i, kk] = index;
    c_ref[i] += v;
  }
  b.destroy_data();
  return fp_equal(c_ref, c);
}

template <class M>
bool gemm_case(std::size_t m, std::size_t n, M &a, std::size_t width) {
  std::vector<float> base_b(n * width), c(m * width, 0.f);
  for (std::size_t i = 0; i < n * width; i++)
    base_b[i] = (float)i;
  dr::mp::broadcasted_slim_matrix<float> b;
  b.broadcast_data(n, width, 0, base_b, dr::mp::default_comm());
  dr::mp::gemv(c, a, b);
  std::vector<float> c_ref(m * width, 0.f);
  for (auto &&[index, v] : a) {
    auto &&[i, kk] = index;
    for (std::size_t j = 0; j < width; j++)
      c_ref[i + j * m] += v * base_b[kk + j * n];
  }
  b.destroy_data();
  return fp_equal(c_ref, c);
}

using Row = dr::mp::csr_row_distribution<float, unsigned long, dr::mp::MpiBackend>;
using Eq = dr::mp::csr_eq_distribution<float, unsigned long, dr::mp::MpiBackend>;
template <class D>
using Mat = dr::mp::distributed_sparse_matrix<float, unsigned long, dr::mp::MpiBackend, D>;

template <class D> void run_shapes(const char *tag, int nseg) {
  const std::size_t shapes[3][2] = {{100, 100}, {1000, 10}, {10, 1000}};
  for (auto &s : shapes) {
    auto csr = dr::generate_random_csr({s[0], s[1]}, 0.1f);
    Mat<D> a(csr, 0, dr::mp::distribution(), nseg);
    char name[96];
    std::snprintf(name, sizeof name, "Gemv%s_%zux%zu_seg%d", tag, s[0], s[1], nseg);
    CHECK(gemv_case(s[0], s[1], a), name);
    std::snprintf(name, sizeof name, "Gemm%s_%zux%zu_seg%d", tag, s[0], s[1], nseg);
    CHECK(gemm_case(s[0], s[1], a, 20), name);
    dr::__detail::destroy_csr_matrix_view(csr, std::allocator<float>{});
  }
}

template <class D> void iter_case(const char *tag) {
  // IterRow / IterEq / ReduceRow (test/gtest/mp/sparse_matrix.cpp)
  auto csr = dr::generate_random_csr({100, 100}, 0.1f);
  Mat<D> a(csr, 0, dr::mp::distribution(), 3);
  auto ref = csr.entries();
  bool ok = a.size() == ref.size();
  double sum = 0, sum_ref = 0;
  std::size_t i = 0;
  for (auto e : a) {
    ok = ok && i < ref.size() && e == ref[i];
    sum += e.value();
    sum_ref += ref[i].value();
    i++;
  }
  char name[64];
  std::snprintf(name, sizeof name, "Iter%s", tag);
  CHECK(ok, name);
  std::snprintf(name, sizeof name, "Reduce%s", tag);
  CHECK(sum == sum_ref, name);
  std::size_t seg_total = 0;
  for (auto &s : a.segments())
    seg_total += s.size();
  std::snprintf(name, sizeof name, "Segments%s", tag);
  CHECK(seg_total == a.size(), name);
  dr::__detail::destroy_csr_matrix_view(csr, std::allocator<float>{});
}

void band_exact() {
  // examples/mp/sparse_matrix.cpp:84-102: double/long, x[i] = i, exact
  auto csr = dr::generate_band_csr<double, long>(1000, 20, 20);
  dr::mp::distributed_sparse_matrix<double, long, dr::mp::MpiBackend,
                                    dr::mp::csr_eq_distribution<double, long>>
      m(csr, 0, dr::mp::distribution(), 4);
  std::vector<double> a(1000), res(1000), ref(1000, 0.0);
  for (int i = 0; i < 1000; i++)
    a[i] = i;
  dr::mp::broadcasted_vector<double> x;
  x.broadcast_data(1000, 0, a, dr::mp::default_comm());
  dr::mp::gemv(0, res, m, x);
  for (long r = 0; r < 1000; r++)
    for (long p = csr.rowptr_data()[r]; p < csr.rowptr_data()[r + 1]; p++)
      ref[r] += csr.colind_data()[p] * csr.values_data()[p];
  bool ok = true;
  for (int i = 0; i < 1000; i++)
    ok = ok && res[i] == ref[i];
  CHECK(ok, "BandExactF64");
  x.destroy_data();
  dr::__detail::destroy_csr_matrix_view(csr, std::allocator<double>{});
}

// The reference's reduce tests (test/gtest/common/reduce.cpp,
// test/gtest/mp/reduce.cpp): Ops1 ops(10) -- a distributed_vector<int> filled
// by iota(dist_vec, 100) -- against std::reduce on the local copy.
void reduce_cases() {
  dr::mp::distributed_vector<int> dv(10, dr::mp::distribution(), 3);
  dr::mp::iota(dv, 100);
  std::vector<int> vec(10);
  std::iota(vec.begin(), vec.end(), 100);
  auto mx = [](double x, double y) { return std::max(x, y); };
  CHECK(dr::mp::reduce(0, dv, 0, std::plus{}) ==
            std::reduce(vec.begin(), vec.end(), 0, std::plus{}),
        "ReduceMP.RootRange");
  CHECK(dr::mp::reduce(0, dv.begin() + 1, dv.end() - 1, 0, std::plus{}) ==
            std::reduce(vec.begin() + 1, vec.end() - 1, 0, std::plus{}),
        "ReduceMP.RootIterators");
  CHECK(dr::mp::reduce(dv, 3, dr::mp::ops::max{}) == std::reduce(vec.begin(), vec.end(), 3, mx),
        "Reduce.Range");
  CHECK(dr::mp::reduce(dv, 3, std::plus{}) ==
            std::reduce(vec.begin(), vec.end(), 3, std::plus{}),
        "Reduce.Max");
  CHECK(dr::mp::reduce(dv.begin(), dv.end(), 3, std::plus{}) ==
            std::reduce(vec.begin(), vec.end(), 3, std::plus{}),
        "Reduce.Iterators");
  CHECK(dr::mp::reduce(dv, 3) == std::reduce(vec.begin(), vec.end(), 3),
        "Reduce.RangeDefaultOp");
  CHECK(dr::mp::reduce(dv.begin(), dv.end(), 3) == std::reduce(vec.begin(), vec.end(), 3),
        "Reduce.IteratorsDefaultOp");
  CHECK(dr::mp::reduce(dv) == std::reduce(vec.begin(), vec.end()), "Reduce.RangeDefaultInit");
  CHECK(dr::mp::reduce(dv.begin(), dv.end()) == std::reduce(vec.begin(), vec.end()),
        "Reduce.IteratorsDefaultInit");
  // ReduceMP.TransformReduce: transform(+1) then reduce(root, ., 1, min)
  dr::mp::distributed_vector<int> added(10);
  dr::mp::iota(added, 101);
  CHECK(dr::mp::reduce(0, added, 1, dr::mp::ops::min{}) == 1, "ReduceMP.TransformReduce");
  dr::mp::fill(dv.begin() + 2, dv.end(), 7);
  CHECK(dv[0] == 100 && dv[1] == 101 && dv[2] == 7 && dv[9] == 7, "FillIterators");
  auto segs = dv.segments();
  CHECK(segs.size() == 3 && segs[0].size() == 4 && segs[2].begin() == 8 && segs[2].end() == 10,
        "VectorSegments");
}

// CG on the 1-D Laplacian tridiag(-1, 2, -1), n = 1000, b = 1.
void cg_case() {
  const long n = 1000;
  std::vector<long> rp(n + 1), ci;
  std::vector<double> v;
  for (long i = 0; i < n; i++) {
    rp[i] = (long)ci.size();
    for (long j = i - 1; j <= i + 1; j++)
      if (j >= 0 && j < n) {
        ci.push_back(j);
        v.push_back(j == i ? 2.0 : -1.0);
      }
  }
  rp[n] = (long)ci.size();
  dr::views::csr_matrix_view<double, long> view(v.data(), rp.data(), ci.data(),
                                                {(long)n, (long)n}, ci.size(), 0);
  dr::mp::distributed_sparse_matrix<double, long, dr::mp::MpiBackend,
                                    dr::mp::csr_row_distribution<double, long>>
      a(view, 0);
  dr::mp::distributed_vector<double> b(n, 1.0), x(n, 0.0);
  auto info = dr::mp::conjugate_gradient(a, b, x, 2000, 1e-10);
  // exact solution of tridiag(-1, 2, -1) x = 1: x_i = (i+1)(n-i)/2
  double err = 0, nx = 0;
  for (long i = 0; i < n; i++) {
    const double xe = 0.5 * (double)(i + 1) * (double)(n - i);
    err = std::max(err, std::abs(x[i] - xe));
    nx = std::max(nx, xe);
  }
  CHECK(info.converged && info.iterations <= n && err <= 1e-6 * nx, "ConjugateGradient1D");
}

// `dump-random m n seed out.bin`: write generate_random_csr<float, unsigned
// long>({m, n}, 0.1f, seed) in oracle/_ref/ref_gen's layout (no GPU needed),
// so a CPU test can compare the mirror's generator with the reference's.
static int dump_random(int argc, char **argv) {
  if (argc != 6)
    return 2;
  const unsigned long m = std::strtoul(argv[2], nullptr, 10);
  const unsigned long n = std::strtoul(argv[3], nullptr, 10);
  const unsigned seed = (unsigned)std::strtoul(argv[4], nullptr, 10);
  auto v = dr::generate_random_csr({m, n}, 0.1f, seed);
  FILE *f = std::fopen(argv[5], "wb");
  if (!f)
    return 3;
  int64_t hdr[3] = {(int64_t)m, (int64_t)n, (int64_t)v.size()};
  std::fwrite(hdr, sizeof hdr, 1, f);
  std::fwrite(v.rowptr_data(), sizeof(unsigned long), m + 1, f);
  std::fwrite(v.colind_data(), sizeof(unsigned long), v.size(), f);
  std::fwrite(v.values_data(), sizeof(float), v.size(), f);
  std::fclose(f);
  dr::__detail::destroy_csr_matrix_view(v, std::allocator<float>{});
  return 0;
}

// `dump-mtx file.mtx out.bin`: dr::read_csr<double, long>(file) written in
// oracle/_ref/ref_mmread's layout (no GPU needed); a read error prints the
// message and returns 3, as ref_mmread does.
static int dump_mtx(int argc, char **argv) {
  if (argc != 4)
    return 2;
  try {
    auto v = dr::read_csr<double, long>(argv[2]);
    FILE *f = std::fopen(argv[3], "wb");
    if (!f)
      return 2;
    int64_t hdr[3] = {(int64_t)v.shape()[0], (int64_t)v.shape()[1],
                      (int64_t)v.size()};
    std::fwrite(hdr, sizeof hdr, 1, f);
    std::fwrite(v.rowptr_data(), sizeof(long), hdr[0] + 1, f);
    std::fwrite(v.colind_data(), sizeof(long), hdr[2], f);
    std::fwrite(v.values_data(), sizeof(double), hdr[2], f);
    std::fclose(f);
    dr::__detail::destroy_csr_matrix_view(v, std::allocator<double>{});
  } catch (const std::exception &e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 3;
  }
  return 0;
}

int main(int argc, char **argv) {
  if (argc > 1 && std::string(argv[1]) == "dump-random")
    return dump_random(argc, argv);
  if (argc > 1 && std::string(argv[1]) == "dump-mtx")
    return dump_mtx(argc, argv);
  for (int nseg : {1, 2, 4}) {
    run_shapes<Row>("Row", nseg);
    run_shapes<Eq>("Eq", nseg);
  }
  iter_case<Row>("Row");
  iter_case<Eq>("Eq");
  band_exact();
  reduce_cases();
  cg_case();
  try {
    auto bad = dr::generate_random_csr({10, 10}, 0.2f);
    bad.rowptr_data()[3] = 1000; // not monotone: rejected by the C ABI
    Mat<Row> a(bad, 0);
    CHECK(false, "BadCsrRejected");
  } catch (const drb::error &e) {
    CHECK(e.status == DRB_ERR_BAD_CSR, "BadCsrRejected");
  }
  std::printf("%s: %d failure(s)\n", failures ? "FAILED" : "OK", failures);
  return failures ? 1 : 0;
}
