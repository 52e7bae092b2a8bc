// mmio.cpp -- Matrix Market ingest: drb_read_matrix_market.
//
// Replaces dr::read_csr<T, I>(path, one_indexed) (include/dr/detail/
// matrix_io.hpp:120-256 with read_csr_matrix_base and
// convert_csr_base_to_csr): header "%%MatrixMarket matrix coordinate <field>
// <general|symmetric>", '%' comment lines, the "m n nnz" size line, then one
// "i j [v]" entry per line (1-based when one_indexed; field "pattern" gives
// value 1); an off-diagonal entry of a symmetric file is stored at (i, j) and
// (j, i); rows are sorted by column.  The same inputs are rejected, with the
// reference's messages: not a coordinate Matrix Market file, unsupported
// symmetry, an entry out of bounds, more entries than the size line declares
// (the first such error in file order is reported, as a sequential read
// would).  Two deliberate differences: blank lines are skipped (the
// reference has no case for them) and a line that does not parse is an
// error; entries with equal (row, column) keep their file order (the
// reference's unstable sort leaves it unspecified).
//
// The file is read whole and its entry lines are parsed by one thread per
// core, each on a newline-aligned chunk; entries are then bucketed by row in
// file order and each row is stably sorted by column.
#include <algorithm>
#include <charconv>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "drb.h"

namespace drb {
void set_error(const char *fmt, ...);
void clear_error();
} // namespace drb

namespace {

struct Entry {
  int64_t i, j;
  double v;
};

struct Chunk {
  std::vector<Entry> entries;
  int64_t bad_at = -1;   // index (within the chunk) of the first bad entry
  int bad_kind = 0;      // 1 out of bounds, 2 malformed
};

const char *skip_ws(const char *p, const char *e) {
  while (p < e && (*p == ' ' || *p == '\t' || *p == '\r'))
    p++;
  return p;
}

bool parse_i64(const char *&p, const char *e, int64_t &out) {
  p = skip_ws(p, e);
  if (p < e && *p == '+')
    p++;
  auto r = std::from_chars(p, e, out);
  if (r.ec != std::errc())
    return false;
  p = r.ptr;
  return true;
}

bool parse_f64(const char *&p, const char *e, double &out) {
  p = skip_ws(p, e);
  if (p < e && *p == '+')
    p++;
  auto r = std::from_chars(p, e, out);
  if (r.ec != std::errc())
    return false;
  p = r.ptr;
  return true;
}

// Parse entry lines in [b, e) (whole lines).  Stops at the first bad line.
void parse_chunk(const char *b, const char *e, bool pattern, bool one_indexed,
                 int64_t m, int64_t n, Chunk &out) {
  const char *p = b;
  while (p < e) {
    const char *eol = static_cast<const char *>(std::memchr(p, '\n', e - p));
    if (!eol)
      eol = e;
    const char *q = skip_ws(p, eol);
    if (q < eol) { // not blank
      int64_t i, j;
      double v = 1.0;
      bool ok = parse_i64(q, eol, i) && parse_i64(q, eol, j);
      if (ok && !pattern)
        ok = parse_f64(q, eol, v);
      if (!ok) {
        out.bad_at = (int64_t)out.entries.size();
        out.bad_kind = 2;
        return;
      }
      if (one_indexed) {
        i--;
        j--;
      }
      if (i < 0 || j < 0 || i >= m || j >= n) {
        out.bad_at = (int64_t)out.entries.size();
        out.bad_kind = 1;
        return;
      }
      out.entries.push_back({i, j, v});
    }
    p = eol + 1;
  }
}

drb_status io_error(const char *path, const char *what, drb_status st) {
  drb::set_error("%s: %s", path, what);
  return st;
}

} // namespace

extern "C" {

drb_status drb_read_matrix_market(const char *path, int one_indexed,
                                  drb_csr_host *out) {
  drb::clear_error();
  if (!path || !out) {
    drb::set_error("invalid argument: path or out is NULL");
    return DRB_ERR_INVALID_ARG;
  }
  std::memset(out, 0, sizeof(*out));
  FILE *f = std::fopen(path, "rb");
  if (!f)
    return io_error(path, "mmread: cannot open", DRB_ERR_IO);
  std::fseek(f, 0, SEEK_END);
  const long size = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  std::string buf(size > 0 ? (size_t)size : 0, '\0');
  const size_t got = size > 0 ? std::fread(&buf[0], 1, (size_t)size, f) : 0;
  std::fclose(f);
  if (size < 0 || got != (size_t)std::max<long>(size, 0))
    return io_error(path, "mmread: read failed", DRB_ERR_IO);
  const char *p = buf.data(), *end = buf.data() + buf.size();
  auto next_line = [&](const char *&b, const char *&e) -> bool {
    if (p >= end)
      return false;
    b = p;
    const char *nl = static_cast<const char *>(std::memchr(p, '\n', end - p));
    e = nl ? nl : end;
    p = nl ? nl + 1 : end;
    return true;
  };
  // header tokens
  const char *lb, *le;
  if (!next_line(lb, le))
    return io_error(path, "could not be parsed as a Matrix Market file.",
                    DRB_ERR_IO);
  std::vector<std::string> tok;
  for (const char *q = lb; q < le;) {
    q = skip_ws(q, le);
    const char *s = q;
    while (q < le && *q != ' ' && *q != '\t' && *q != '\r')
      q++;
    if (q > s)
      tok.emplace_back(s, q);
  }
  if (tok.size() < 3 || tok[0] != "%%MatrixMarket" || tok[1] != "matrix" ||
      tok[2] != "coordinate")
    return io_error(path, "could not be parsed as a Matrix Market file.",
                    DRB_ERR_IO);
  const bool pattern = tok.size() > 3 && tok[3] == "pattern";
  bool symmetric;
  if (tok.size() > 4 && tok[4] == "general")
    symmetric = false;
  else if (tok.size() > 4 && tok[4] == "symmetric")
    symmetric = true;
  else
    return io_error(path, "has an unsupported matrix type", DRB_ERR_UNSUPPORTED);
  // comment lines, then the size line
  bool have = false;
  while (next_line(lb, le)) {
    if (lb == le || *lb != '%') {
      have = true;
      break;
    }
  }
  int64_t m = 0, n = 0, declared = 0;
  {
    const char *q = lb;
    if (!have || !parse_i64(q, le, m) || !parse_i64(q, le, n) ||
        !parse_i64(q, le, declared) || m < 0 || n < 0 || declared < 0)
      return io_error(path, "malformed size line", DRB_ERR_IO);
  }
  // entry lines, parsed in newline-aligned chunks
  const int64_t bytes = end - p;
  int nth = (int)std::min<int64_t>(std::max(1u, std::thread::hardware_concurrency()),
                                   std::max<int64_t>(1, bytes >> 20));
  std::vector<const char *> cut(nth + 1);
  cut[0] = p;
  cut[nth] = end;
  for (int t = 1; t < nth; t++) {
    const char *c = p + bytes * t / nth;
    c = std::max(c, cut[t - 1]);
    const char *nl = static_cast<const char *>(std::memchr(c, '\n', end - c));
    cut[t] = nl ? nl + 1 : end;
  }
  std::vector<Chunk> chunks(nth);
  {
    std::vector<std::thread> pool;
    for (int t = 0; t < nth; t++)
      pool.emplace_back([&, t] {
        parse_chunk(cut[t], cut[t + 1], pattern, one_indexed != 0, m, n,
                    chunks[t]);
      });
    for (auto &th : pool)
      th.join();
  }
  // the first error in file order, as a sequential read reports it
  int64_t before = 0;
  for (int t = 0; t < nth; t++) {
    const Chunk &c = chunks[t];
    const int64_t upto = c.bad_at >= 0 ? c.bad_at : (int64_t)c.entries.size();
    if (before + upto > declared)
      return io_error(path,
                      "read_MatrixMarket: error reading Matrix Market file, file "
                      "has more nonzeros than reported.",
                      DRB_ERR_BAD_CSR);
    if (c.bad_at >= 0)
      return c.bad_kind == 1
                 ? io_error(path,
                            "read_MatrixMarket: file has nonzero out of bounds.",
                            DRB_ERR_BAD_CSR)
                 : io_error(path, "malformed entry line", DRB_ERR_IO);
    before += upto;
  }
  // bucket by row in file order (a mirrored entry right after its own)
  std::vector<int64_t> rowptr((size_t)m + 1, 0);
  for (const Chunk &c : chunks)
    for (const Entry &e : c.entries) {
      rowptr[e.i + 1]++;
      if (symmetric && e.i != e.j)
        rowptr[e.j + 1]++;
    }
  for (int64_t r = 0; r < m; r++)
    rowptr[r + 1] += rowptr[r];
  const int64_t nnz = rowptr[m];
  int64_t *rp = static_cast<int64_t *>(std::malloc(sizeof(int64_t) * (m + 1)));
  int64_t *ci = static_cast<int64_t *>(std::malloc(sizeof(int64_t) * std::max<int64_t>(nnz, 1)));
  double *vv = static_cast<double *>(std::malloc(sizeof(double) * std::max<int64_t>(nnz, 1)));
  if (!rp || !ci || !vv) {
    std::free(rp), std::free(ci), std::free(vv);
    drb::set_error("%s: out of host memory", path);
    return DRB_ERR_OOM;
  }
  std::vector<int64_t> fill(rowptr.begin(), rowptr.end() - 1);
  for (const Chunk &c : chunks)
    for (const Entry &e : c.entries) {
      int64_t k = fill[e.i]++;
      ci[k] = e.j;
      vv[k] = e.v;
      if (symmetric && e.i != e.j) {
        k = fill[e.j]++;
        ci[k] = e.i;
        vv[k] = e.v;
      }
    }
  chunks.clear();
  // stable sort of every row by column, rows split over threads
  {
    const int sth = (int)std::max<int64_t>(1, std::min<int64_t>(
        std::max(1u, std::thread::hardware_concurrency()), m / 4096));
    std::vector<std::thread> pool;
    for (int t = 0; t < sth; t++)
      pool.emplace_back([&, t] {
        std::vector<std::pair<int64_t, double>> tmp;
        for (int64_t r = m * t / sth; r < m * (t + 1) / sth; r++) {
          const int64_t a = rowptr[r], b = rowptr[r + 1];
          bool sorted = true;
          for (int64_t k = a + 1; k < b && sorted; k++)
            sorted = ci[k - 1] <= ci[k];
          if (sorted)
            continue;
          tmp.clear();
          for (int64_t k = a; k < b; k++)
            tmp.push_back({ci[k], vv[k]});
          std::stable_sort(tmp.begin(), tmp.end(),
                           [](const auto &x, const auto &y) {
                             return x.first < y.first;
                           });
          for (int64_t k = a; k < b; k++) {
            ci[k] = tmp[k - a].first;
            vv[k] = tmp[k - a].second;
          }
        }
      });
    for (auto &th : pool)
      th.join();
  }
  std::memcpy(rp, rowptr.data(), sizeof(int64_t) * (m + 1));
  out->m = m;
  out->n = n;
  out->nnz = nnz;
  out->rowptr = rp;
  out->colind = ci;
  out->values = vv;
  return DRB_OK;
}

void drb_csr_host_free(drb_csr_host *h) {
  if (!h)
    return;
  std::free(h->rowptr);
  std::free(h->colind);
  std::free(h->values);
  h->rowptr = nullptr;
  h->colind = nullptr;
  h->values = nullptr;
}

} // extern "C"
