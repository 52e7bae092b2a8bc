// ref_mmread: runs the REFERENCE's own Matrix Market reader (include/dr/
// detail/matrix_io.hpp, dr::read_csr<double, long>, compiled from the
// reference tree by oracle/Makefile with the stand-in csr_matrix_view of
// oracle/ref_shim) and writes the CSR arrays as raw little-endian binary, so
// that tests/golden/ fixtures for the ingest path come from the reference
// code itself.  Test infrastructure only.
//
// usage: ref_mmread file.mtx out.bin
// out.bin layout: int64 m, n, nnz; rowptr[m+1] int64; colind[nnz] int64;
// values[nnz] f64.  A reader exception prints its message to stderr and
// exits with status 3.
#include <cstdint>
#include <cstdio>
#include <exception>
#include <string>

#include <dr/detail/matrix_io.hpp>

int main(int argc, char **argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: ref_mmread file.mtx out.bin\n");
    return 1;
  }
  try {
    auto v = dr::read_csr<double, long>(argv[1]);
    FILE *f = std::fopen(argv[2], "wb");
    if (!f)
      return 2;
    int64_t hdr[3] = {(int64_t)v.shape()[0], (int64_t)v.shape()[1],
                      (int64_t)v.size()};
    std::fwrite(hdr, sizeof hdr, 1, f);
    for (int64_t i = 0; i <= hdr[0]; i++) {
      int64_t r = v.rowptr_data()[i];
      std::fwrite(&r, 8, 1, f);
    }
    for (int64_t i = 0; i < hdr[2]; i++) {
      int64_t c = v.colind_data()[i];
      std::fwrite(&c, 8, 1, f);
    }
    std::fwrite(v.values_data(), sizeof(double), hdr[2], f);
    std::fclose(f);
  } catch (const std::exception &e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 3;
  }
  return 0;
}
