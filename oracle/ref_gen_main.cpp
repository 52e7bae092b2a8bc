// ref_gen: runs the REFERENCE's own generators (include/dr/detail/
// generate_csr.hpp, compiled from the reference tree by oracle/Makefile) and
// writes the CSR arrays as raw little-endian binary, so that tests/golden/
// fixtures come from the reference code itself.
//
// usage: ref_gen random <f32|f64> <u64|i64|i32> m n density seed out.bin
//        ref_gen band   <f32|f64> <u64|i64|i32> size up down out.bin
// out.bin layout: int64 m, n, nnz; rowptr[m+1]; colind[nnz]; values[nnz]
// (index and value types as requested).
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include <dr/detail/generate_csr.hpp>

template <class View> static int dump(const View &v, const char *path) {
  FILE *f = std::fopen(path, "wb");
  if (!f)
    return 2;
  int64_t hdr[3] = {(int64_t)v.shape()[0], (int64_t)v.shape()[1],
                    (int64_t)v.size()};
  std::fwrite(hdr, sizeof hdr, 1, f);
  std::fwrite(v.rowptr_data(), sizeof(*v.rowptr_data()), hdr[0] + 1, f);
  std::fwrite(v.colind_data(), sizeof(*v.colind_data()), hdr[2], f);
  std::fwrite(v.values_data(), sizeof(*v.values_data()), hdr[2], f);
  std::fclose(f);
  delete[] v.values_data();
  delete[] v.rowptr_data();
  delete[] v.colind_data();
  return 0;
}

template <class T, class I> static int run(int argc, char **argv) {
  std::string kind = argv[1];
  if (kind == "random" && argc == 9) {
    I m = (I)std::strtoll(argv[4], nullptr, 10);
    I n = (I)std::strtoll(argv[5], nullptr, 10);
    double density = std::strtod(argv[6], nullptr);
    unsigned seed = (unsigned)std::strtoul(argv[7], nullptr, 10);
    auto v = dr::generate_random_csr<T, I>(dr::index<I>(m, n), density, seed);
    return dump(v, argv[8]);
  }
  if (kind == "band" && argc == 8) {
    I size = (I)std::strtoll(argv[4], nullptr, 10);
    std::size_t up = std::strtoull(argv[5], nullptr, 10);
    std::size_t down = std::strtoull(argv[6], nullptr, 10);
    auto v = dr::generate_band_csr<T, I>(size, up, down);
    return dump(v, argv[7]);
  }
  return 1;
}

int main(int argc, char **argv) {
  if (argc < 4) {
    std::fprintf(stderr, "usage: see source header\n");
    return 1;
  }
  std::string t = argv[2], i = argv[3];
  if (t == "f32" && i == "u64") return run<float, unsigned long>(argc, argv);
  if (t == "f32" && i == "i64") return run<float, long>(argc, argv);
  if (t == "f32" && i == "i32") return run<float, int>(argc, argv);
  if (t == "f64" && i == "u64") return run<double, unsigned long>(argc, argv);
  if (t == "f64" && i == "i64") return run<double, long>(argc, argv);
  if (t == "f64" && i == "i32") return run<double, int>(argc, argv);
  return 1;
}
