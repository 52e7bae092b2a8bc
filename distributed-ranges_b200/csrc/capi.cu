// capi.cu -- the extern "C" entry points declared in include/drb.h.
//
// The handle (drb_csr_t) plays the role of the reference's
// distributed_sparse_matrix + csr_row_distribution / csr_eq_distribution:
// it owns device copies of the CSR arrays (csr_row_distribution.hpp:205-318
// copies each rank's slice into MPI-window memory; here all slices are one
// device allocation), the row-block plan, and the segment table that
// segments() reports.  No exception crosses the ABI.
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <thread>

#include "drb_internal.cuh"

namespace drb {

int plan_group(int vbytes, int cbytes);

std::atomic<uint64_t> g_launch_count{0};
thread_local int g_count_pause = 0;

namespace {
thread_local std::string t_error;

drb_status invalid(const char *msg) {
  set_error("invalid argument: %s", msg);
  return DRB_ERR_INVALID_ARG;
}

// Device checks are cached per device: cudaGetDeviceProperties costs tens of
// microseconds, too much for every call of a sub-millisecond kernel.
constexpr int kMaxDevices = 64;
std::atomic<int> g_dev_ok[kMaxDevices];

drb_status check_device(int *dev) {
  if (cudaGetDevice(dev) == cudaSuccess && *dev >= 0 && *dev < kMaxDevices &&
      g_dev_ok[*dev].load(std::memory_order_relaxed) == 1)
    return DRB_OK;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    set_error("no CUDA device available (%s)",
              e == cudaSuccess ? "count 0" : cudaGetErrorString(e));
    return DRB_ERR_NO_DEVICE;
  }
  DRB_CUDA_TRY(cudaGetDevice(dev));
  cudaDeviceProp prop;
  DRB_CUDA_TRY(cudaGetDeviceProperties(&prop, *dev));
  if (prop.major != 10 || prop.minor != 0) {
    set_error("device %d is sm_%d%d; this library is built for sm_100a (B200)",
              *dev, prop.major, prop.minor);
    return DRB_ERR_NO_DEVICE;
  }
  if (*dev >= 0 && *dev < kMaxDevices)
    g_dev_ok[*dev].store(1, std::memory_order_relaxed);
  return DRB_OK;
}

template <class I>
drb_status validate_rowptr(const I *rp, int64_t m, int64_t nnz) {
  if ((int64_t)rp[0] != 0) {
    set_error("bad CSR: rowptr[0] = %lld, expected 0", (long long)rp[0]);
    return DRB_ERR_BAD_CSR;
  }
  for (int64_t i = 0; i < m; i++) {
    if (rp[i + 1] < rp[i]) {
      set_error("bad CSR: rowptr decreases at row %lld", (long long)i);
      return DRB_ERR_BAD_CSR;
    }
  }
  if ((int64_t)rp[m] != nnz) {
    set_error("bad CSR: rowptr[m] = %lld but nnz = %lld", (long long)rp[m],
              (long long)nnz);
    return DRB_ERR_BAD_CSR;
  }
  return DRB_OK;
}

template <class I>
drb_status validate_cols(const I *ci, int64_t nnz, int64_t n) {
  const int64_t nth =
      nnz > (1 << 22) ? std::min<int64_t>(16, std::max(1u, std::thread::hardware_concurrency())) : 1;
  std::vector<int64_t> bad(nth, -1);
  auto work = [&](int64_t t) {
    const int64_t lo = nnz * t / nth, hi = nnz * (t + 1) / nth;
    for (int64_t p = lo; p < hi; p++) {
      const int64_t c = (int64_t)ci[p];
      if (c < 0 || c >= n) {
        bad[t] = p;
        return;
      }
    }
  };
  if (nth == 1) {
    work(0);
  } else {
    std::vector<std::thread> th;
    for (int64_t t = 0; t < nth; t++)
      th.emplace_back(work, t);
    for (auto &t : th)
      t.join();
  }
  for (int64_t t = 0; t < nth; t++)
    if (bad[t] >= 0) {
      set_error("bad CSR: column index %lld at nnz %lld is outside [0, %lld)",
                (long long)ci[bad[t]], (long long)bad[t], (long long)n);
      return DRB_ERR_BAD_CSR;
    }
  return DRB_OK;
}

int64_t rp_at(const void *rp, int ib, int64_t i) {
  return ib == 8 ? ((const int64_t *)rp)[i] : (int64_t)((const int32_t *)rp)[i];
}

// Upload `count` elements of width in_b to dst (width out_b), narrowing or
// widening on the device through a temporary when the widths differ.
drb_status upload(void *dst, int out_b, const void *src, int in_b,
                  int64_t count, bool src_on_device, bool to_bf16,
                  cudaStream_t s) {
  if (count == 0)
    return DRB_OK;
  const cudaMemcpyKind kind =
      src_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  if (in_b == out_b && !to_bf16) {
    DRB_CUDA_TRY(cudaMemcpyAsync(dst, src, (size_t)in_b * count, kind, s));
    return DRB_OK;
  }
  const void *dsrc = src;
  DevBuf tmp;
  if (!src_on_device) {
    DRB_TRY(tmp.alloc((size_t)in_b * count));
    DRB_CUDA_TRY(cudaMemcpyAsync(tmp.p, src, (size_t)in_b * count, kind, s));
    dsrc = tmp.p;
  }
  DRB_TRY(convert_launch(dsrc, in_b, dst, out_b, count, to_bf16, s));
  DRB_CUDA_TRY(cudaStreamSynchronize(s)); // tmp is freed on return
  return DRB_OK;
}

void compute_segments(Csr &A, const void *rp, int ib) {
  const int64_t P = A.nseg, m = A.m, nnz = A.nnz;
  A.seg_row0.assign(P, 0);
  A.seg_row1.assign(P, 0);
  A.seg_nz0.assign(P, 0);
  A.seg_nz1.assign(P, 0);
  if (A.part == DRB_PART_ROW) {
    // distributed_vector<I>(m) segment size ceil(m/P)
    // (distributed_vector.hpp:310); nnz ranges per
    // csr_row_distribution.hpp:234-252.
    const int64_t seg = (m + P - 1) / P;
    for (int64_t r = 0; r < P; r++) {
      const int64_t r0 = std::min(m, r * seg), r1 = std::min(m, (r + 1) * seg);
      A.seg_row0[r] = r0;
      A.seg_row1[r] = r1;
      A.seg_nz0[r] = rp_at(rp, ib, r0);
      A.seg_nz1[r] = rp_at(rp, ib, r1);
    }
  } else {
    // distributed_vector<T>(nnz) segment size ceil(nnz/P); the rows a
    // segment touches come from upper_bound over rowptr[0..m)
    // (csr_eq_distribution.hpp:253-272).
    const int64_t seg = (nnz + P - 1) / P;
    auto ub = [&](int64_t v) {
      int64_t lo = 0, hi = m;
      while (lo < hi) {
        const int64_t mid = (lo + hi) / 2;
        if (rp_at(rp, ib, mid) <= v)
          lo = mid + 1;
        else
          hi = mid;
      }
      return lo;
    };
    for (int64_t r = 0; r < P; r++) {
      const int64_t z0 = std::min(nnz, r * seg), z1 = std::min(nnz, (r + 1) * seg);
      A.seg_nz0[r] = z0;
      A.seg_nz1[r] = z1;
      if (z0 >= z1) {
        A.seg_row0[r] = A.seg_row1[r] = m;
        continue;
      }
      A.seg_row0[r] = std::max<int64_t>(0, ub(z0) - 1);
      A.seg_row1[r] = ub(z1 - 1);
    }
  }
}

} // namespace

void set_error(const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  t_error = buf;
}
void clear_error() { t_error.clear(); }

drb_status DevBuf::alloc(size_t nbytes) {
  release();
  if (nbytes == 0)
    nbytes = 16;
  cudaError_t e = cudaMalloc(&p, nbytes);
  if (e != cudaSuccess) {
    p = nullptr;
    set_error("cudaMalloc(%zu) failed: %s", nbytes, cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? DRB_ERR_OOM : DRB_ERR_CUDA;
  }
  bytes = nbytes;
  return DRB_OK;
}

drb_status DevBuf::ensure(size_t nbytes) {
  if (p && bytes >= nbytes)
    return DRB_OK;
  return alloc(nbytes);
}

void DevBuf::release() {
  if (p)
    cudaFree(p);
  p = nullptr;
  bytes = 0;
}

Csr::~Csr() {
  for (cudaEvent_t e : seg_done)
    cudaEventDestroy(e);
  if (copy_stream)
    cudaStreamDestroy(copy_stream);
}

} // namespace drb

using namespace drb;

extern "C" {

const char *drb_last_error(void) { return t_error.c_str(); }

const char *drb_version(void) { return "drb 0.1 (sm_100a)"; }

uint64_t drb_launch_count(void) { return g_launch_count.load(); }

drb_status drb_csr_create(drb_csr_t *out, int64_t m, int64_t n, int64_t nnz,
                          const void *rowptr, const void *colind,
                          const void *values, drb_itype index_type,
                          drb_dtype value_type, drb_dtype storage,
                          int nsegments, drb_partition partition,
                          uint32_t flags, void *stream) {
  clear_error();
  if (!out)
    return invalid("out is NULL");
  *out = nullptr;
  if (m < 0 || n < 0 || nnz < 0)
    return invalid("negative m, n or nnz");
  if (m >= 0x7fffffff) {
    set_error("m = %lld rows: at most 2^31-2 rows per handle", (long long)m);
    return DRB_ERR_UNSUPPORTED;
  }
  if (!rowptr)
    return invalid("rowptr is NULL");
  if (nnz > 0 && (!colind || !values))
    return invalid("colind or values is NULL");
  if (index_type != DRB_I32 && index_type != DRB_I64)
    return invalid("index_type");
  if (value_type != DRB_F32 && value_type != DRB_F64)
    return invalid("value_type must be DRB_F32 or DRB_F64");
  if (!(storage == value_type || (storage == DRB_BF16 && value_type == DRB_F32)))
    return invalid("storage must equal value_type, or be DRB_BF16 for F32");
  if (nsegments < 1)
    return invalid("nsegments < 1");
  if (partition != DRB_PART_ROW && partition != DRB_PART_EQ)
    return invalid("partition");
  if (index_type == DRB_I32 && (nnz > 0x7fffffff || n > 0x7fffffff))
    return invalid("int32 indices cannot address nnz or n >= 2^31");
  int dev = 0;
  DRB_TRY(check_device(&dev));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const bool on_dev = flags & DRB_FLAG_DEVICE_INPUT;
  const int ib = index_type == DRB_I64 ? 8 : 4;

  std::vector<char> rp_copy;
  const void *rp_h = rowptr;
  if (on_dev) {
    rp_copy.resize((size_t)ib * (m + 1));
    DRB_CUDA_TRY(cudaMemcpy(rp_copy.data(), rowptr, rp_copy.size(),
                            cudaMemcpyDeviceToHost));
    rp_h = rp_copy.data();
  }
  if (!(flags & DRB_FLAG_SKIP_VALIDATE)) {
    if (ib == 8)
      DRB_TRY(validate_rowptr((const int64_t *)rp_h, m, nnz));
    else
      DRB_TRY(validate_rowptr((const int32_t *)rp_h, m, nnz));
    if (!on_dev) {
      if (ib == 8)
        DRB_TRY(validate_cols((const int64_t *)colind, nnz, n));
      else
        DRB_TRY(validate_cols((const int32_t *)colind, nnz, n));
    }
  } else if (rp_at(rp_h, ib, m) != nnz) {
    set_error("bad CSR: rowptr[m] != nnz");
    return DRB_ERR_BAD_CSR;
  }

  auto A = std::make_unique<drb_csr_matrix>();
  A->device = dev;
  A->m = m;
  A->n = n;
  A->nnz = nnz;
  A->value_type = value_type;
  A->storage = storage;
  A->nseg = nsegments;
  A->part = partition;
  A->flags = flags;
  A->cbytes = (ib == 8 && ((flags & DRB_FLAG_KEEP_INDEX64) || n > 0x7fffffff)) ? 8 : 4;
  A->rbytes = (ib == 8 && ((flags & DRB_FLAG_KEEP_INDEX64) || nnz > 0x7fffffff)) ? 8 : 4;
  const int vb_in = dtype_bytes(value_type), vb = dtype_bytes(storage);
  const int64_t pad = ((nnz + kPadElems - 1) / kPadElems + 1) * kPadElems;
  DRB_TRY(A->rowptr.alloc((size_t)A->rbytes * (m + 1 + kRowptrPad)));
  DRB_CUDA_TRY(cudaMemsetAsync(A->rowptr.p, 0, A->rowptr.bytes, s));
  DRB_TRY(A->colind.alloc((size_t)A->cbytes * pad));
  DRB_TRY(A->vals.alloc((size_t)vb * pad));
  DRB_CUDA_TRY(cudaMemsetAsync(A->colind.p, 0, A->colind.bytes, s));
  DRB_CUDA_TRY(cudaMemsetAsync(A->vals.p, 0, A->vals.bytes, s));
  DRB_TRY(upload(A->rowptr.p, A->rbytes, rowptr, ib, m + 1, on_dev, false, s));
  DRB_TRY(upload(A->colind.p, A->cbytes, colind, ib, nnz, on_dev, false, s));
  DRB_TRY(upload(A->vals.p, vb, values, vb_in, nnz, on_dev,
                 storage == DRB_BF16, s));
  DRB_CUDA_TRY(cudaStreamSynchronize(s));
  for (int64_t i = 0; i < m; i++)
    A->max_row = std::max(A->max_row, rp_at(rp_h, ib, i + 1) - rp_at(rp_h, ib, i));
  DRB_TRY(build_plan(A->plan, m, rp_h, ib, plan_group(vb, A->cbytes), 0, 0, 0));
  DRB_TRY(build_pipe_plan(A->pipe, m, rp_h, ib, plan_group(vb, A->cbytes), 0, 0));
  DRB_TRY(sell_build(*A, rp_h, ib, s));
  compute_segments(*A, rp_h, ib);
  if (flags & DRB_FLAG_ADJOINT) {
    DRB_TRY(adjoint_build(*A, s));
    DRB_CUDA_TRY(cudaStreamSynchronize(s));
  }
  if ((flags & DRB_FLAG_AUTOTUNE) && storage != DRB_BF16 && nnz > 0) {
    DRB_TRY(autotune_pipe(*A, s, nullptr));
    if (A->tr)
      DRB_TRY(autotune_pipe(*A->tr, s, nullptr));
  }
  // a column-blocked copy when x would not stay in L2 (after the autotuner,
  // whose item variant it starts from)
  DRB_TRY(colsplit_build(*A, s));
  if (A->tr)
    DRB_TRY(colsplit_build(*A->tr, s));
  if (flags & DRB_FLAG_AUTOTUNE) {
    DRB_TRY(colsplit_tune(*A, s));
    if (A->tr)
      DRB_TRY(colsplit_tune(*A->tr, s));
  }
  DRB_CUDA_TRY(cudaStreamSynchronize(s));
  *out = A.release();
  return DRB_OK;
}

drb_status drb_csr_destroy(drb_csr_t A) {
  clear_error();
  if (!A)
    return DRB_OK;
  DeviceGuard g(A->device);
  cudaDeviceSynchronize();
  delete A;
  return DRB_OK;
}

drb_status drb_csr_shape(drb_csr_t A, int64_t *m, int64_t *n, int64_t *nnz) {
  if (!A)
    return invalid("A is NULL");
  if (m)
    *m = A->m;
  if (n)
    *n = A->n;
  if (nnz)
    *nnz = A->nnz;
  return DRB_OK;
}

drb_status drb_csr_storage(drb_csr_t A, int *value_bytes, int *col_bytes,
                           int *rowptr_bytes) {
  if (!A)
    return invalid("A is NULL");
  if (value_bytes)
    *value_bytes = dtype_bytes(A->storage);
  if (col_bytes)
    *col_bytes = A->cbytes;
  if (rowptr_bytes)
    *rowptr_bytes = A->rbytes;
  return DRB_OK;
}

drb_status drb_csr_num_segments(drb_csr_t A, int *nsegments) {
  if (!A || !nsegments)
    return invalid("NULL argument");
  *nsegments = A->nseg;
  return DRB_OK;
}

drb_status drb_csr_segment(drb_csr_t A, int seg, int64_t *row_begin,
                           int64_t *row_end, int64_t *nnz_begin,
                           int64_t *nnz_end) {
  if (!A)
    return invalid("A is NULL");
  if (seg < 0 || seg >= A->nseg)
    return invalid("segment index out of range");
  if (row_begin)
    *row_begin = A->seg_row0[seg];
  if (row_end)
    *row_end = A->seg_row1[seg];
  if (nnz_begin)
    *nnz_begin = A->seg_nz0[seg];
  if (nnz_end)
    *nnz_end = A->seg_nz1[seg];
  return DRB_OK;
}

drb_status drb_csr_get_entries(drb_csr_t A, int64_t offset, int64_t count,
                               int64_t *rows, int64_t *cols, double *values) {
  clear_error();
  if (!A)
    return invalid("A is NULL");
  if (offset < 0 || count < 0 || offset + count > A->nnz)
    return invalid("entry range outside [0, nnz)");
  if (count == 0)
    return DRB_OK;
  DeviceGuard g(A->device);
  if (rows) {
    if (A->rowptr_h.empty()) {
      std::vector<char> raw((size_t)A->rbytes * (A->m + 1));
      DRB_CUDA_TRY(cudaMemcpy(raw.data(), A->rowptr.p, raw.size(),
                              cudaMemcpyDeviceToHost));
      A->rowptr_h.resize(A->m + 1);
      for (int64_t i = 0; i <= A->m; i++)
        A->rowptr_h[i] = rp_at(raw.data(), A->rbytes, i);
    }
    const auto &rp = A->rowptr_h;
    int64_t r = std::upper_bound(rp.begin(), rp.end(), offset) - rp.begin() - 1;
    for (int64_t i = 0; i < count; i++) {
      while (rp[r + 1] <= offset + i)
        r++;
      rows[i] = r;
    }
  }
  if (cols) {
    std::vector<char> raw((size_t)A->cbytes * count);
    DRB_CUDA_TRY(cudaMemcpy(raw.data(),
                            (const char *)A->colind.p + (size_t)A->cbytes * offset,
                            raw.size(), cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < count; i++)
      cols[i] = rp_at(raw.data(), A->cbytes, i);
  }
  if (values) {
    const int vb = dtype_bytes(A->storage);
    std::vector<char> raw((size_t)vb * count);
    DRB_CUDA_TRY(cudaMemcpy(raw.data(),
                            (const char *)A->vals.p + (size_t)vb * offset,
                            raw.size(), cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < count; i++) {
      if (A->storage == DRB_F64) {
        values[i] = ((const double *)raw.data())[i];
      } else if (A->storage == DRB_F32) {
        values[i] = ((const float *)raw.data())[i];
      } else {
        uint32_t u = (uint32_t)((const uint16_t *)raw.data())[i] << 16;
        float f;
        std::memcpy(&f, &u, 4);
        values[i] = f;
      }
    }
  }
  return DRB_OK;
}

drb_status drb_csr_gemv(drb_csr_t A, const void *x, void *y, int64_t k,
                        drb_layout layout, void *stream) {
  clear_error();
  if (!A)
    return invalid("A is NULL");
  if (k < 1)
    return invalid("k < 1");
  if (layout != DRB_COL_MAJOR && layout != DRB_ROW_MAJOR)
    return invalid("layout");
  if ((A->m > 0 && !y) || (A->n > 0 && A->nnz > 0 && !x))
    return invalid("x or y is NULL");
  if (A->m == 0)
    return DRB_OK;
  DeviceGuard g(A->device);
  return spmv_launch(*A, x, y, k, layout, static_cast<cudaStream_t>(stream));
}

} // extern "C"

namespace drb {
namespace {

constexpr int kHostSegments = 6;          // row segments of a host-pointer gemv
constexpr int64_t kSegmentMinNnz = 1 << 22; // below this, one launch
// Each segment holds this fraction of the previous one's nonzeros, so each
// segment's copy back over PCIe ends about when the next segment's compute
// does and the small last segment leaves a short tail.  Measured on a 16.8M-row
// power-law matrix (64 MB of y, 1.18 ms D2H against 1.55 ms of SpMV): 6
// segments at 0.6 / 0.7 / 0.8: 3.14 / 3.08 / 3.11 ms per call; 8 to 16
// segments 3.12 to 3.43 ms (each launch adds a ramp and a tail).
constexpr double kSegmentRatio = 0.7;

// Segment count of a host-pointer gemv: DRB_HOST_SEGMENTS (1..64) when set,
// read when a handle first runs one.
int host_segments() {
  const char *e = std::getenv("DRB_HOST_SEGMENTS");
  if (!e || !*e)
    return kHostSegments;
  return std::min(64, std::max(1, std::atoi(e)));
}

// Ratio of consecutive segments' nnz: DRB_HOST_SEGMENT_RATIO (0.2..1) when
// set, read with the segment count.
double segment_ratio() {
  const char *e = std::getenv("DRB_HOST_SEGMENT_RATIO");
  if (!e || !*e)
    return kSegmentRatio;
  return std::min(1.0, std::max(0.2, std::atof(e)));
}

// Orders the single-RHS items by row and cuts them into at most `target` row
// segments of geometrically shrinking nnz; a chunked row never straddles two
// segments.
drb_status build_row_segments(Csr &A, int target) {
  PipePlan &P = A.pipe;
  std::vector<Item> it((size_t)P.nitems);
  DRB_CUDA_TRY(cudaMemcpy(it.data(), P.items.p, sizeof(Item) * it.size(),
                          cudaMemcpyDeviceToHost));
  std::stable_sort(it.begin(), it.end(), [](const Item &a, const Item &b) {
    return a.r0 < b.r0;
  });
  int64_t total = 0;
  for (const Item &t : it)
    total += t.len;
  // cut[j]: running nnz at which segment j + 1 may start
  std::vector<double> cut;
  const double ratio = segment_ratio();
  double w = 1.0, wsum = 0.0;
  for (int j = 0; j < target; j++, w *= ratio)
    wsum += w;
  w = 1.0;
  for (double acc = 0.0; (int)cut.size() < target - 1; w *= ratio) {
    acc += w;
    cut.push_back((double)total * acc / wsum);
  }
  P.seg_i0.assign(1, 0);
  P.seg_r0.assign(1, 0);
  int64_t acc = 0;
  for (size_t i = 0; i < it.size(); i++) {
    const size_t j = P.seg_i0.size() - 1;
    // cut before item i when the running nnz passed the next target and item
    // i starts a new row (a whole-row item, or the first chunk of its row)
    if (i > 0 && j < cut.size() && (double)acc >= cut[j] &&
        (it[i].nrows > 0 || it[i].r0 != it[i - 1].r0)) {
      P.seg_i0.push_back((int64_t)i);
      P.seg_r0.push_back(it[i].r0);
    }
    acc += it[i].len;
  }
  P.seg_i0.push_back((int64_t)it.size());
  P.seg_r0.push_back(A.m);
  // chunks are numbered in row order and a split row stays in one segment,
  // so segment g's chunks are the contiguous range [seg_c0[g], seg_c0[g+1])
  P.seg_c0.assign(1, 0);
  for (size_t g = 0; g + 1 < P.seg_i0.size(); g++) {
    int64_t cend = P.seg_c0.back();
    for (int64_t i = P.seg_i0[g]; i < P.seg_i0[g + 1]; i++)
      if (it[(size_t)i].nrows == 0)
        cend = std::max<int64_t>(cend, (int64_t)it[(size_t)i].chunk + 1);
    P.seg_c0.push_back(cend);
  }
  DRB_TRY(P.seg_items.alloc(sizeof(Item) * std::max<size_t>(it.size(), 1)));
  DRB_CUDA_TRY(cudaMemcpy(P.seg_items.p, it.data(), sizeof(Item) * it.size(),
                          cudaMemcpyHostToDevice));
  return DRB_OK;
}

// The same geometric cut for the sliced-ELL copy: slice ranges, by padded
// elements.
void build_slice_segments(Csr &A, int target) {
  const std::vector<int64_t> &off = A.sell.off_h;
  const int64_t nsl = A.sell.nslices, total = off[nsl];
  const double ratio = segment_ratio();
  double w = 1.0, wsum = 0.0;
  for (int j = 0; j < target; j++, w *= ratio)
    wsum += w;
  A.sell.seg_s0.assign(1, 0);
  w = 1.0;
  double acc = 0.0;
  for (int j = 0; j < target - 1; j++, w *= ratio) {
    acc += w;
    const double cut = (double)total * acc / wsum;
    int64_t sl = std::lower_bound(off.begin(), off.end(), (int64_t)cut) - off.begin();
    sl = std::min(sl, nsl);
    if (sl > A.sell.seg_s0.back() && sl < nsl)
      A.sell.seg_s0.push_back(sl);
  }
  A.sell.seg_s0.push_back(nsl);
}

// y = A x for one right-hand side with host x and y: x goes up, then each row
// segment runs while the rows of the previous ones copy back on a second
// stream.  The segment launches run the same kernel on a subset of the items,
// so y is bit-identical to drb_csr_gemv's.
drb_status gemv_host_segmented(Csr &A, const void *x_host, void *y_host,
                               size_t xb, size_t yb, cudaStream_t s) {
  PipePlan &P = A.pipe;
  const bool sell = A.sell.on;
  if (sell && A.sell.seg_s0.empty())
    build_slice_segments(A, host_segments());
  if (!sell && P.seg_i0.empty())
    DRB_TRY(build_row_segments(A, host_segments()));
  const int nseg = sell ? (int)A.sell.seg_s0.size() - 1 : (int)P.seg_i0.size() - 1;
  // rows of segment g: [row0(g), row0(g + 1))
  auto row0 = [&](int g) -> int64_t {
    return sell ? std::min(A.m, A.sell.seg_s0[g] * 32) : P.seg_r0[g];
  };
  if (!A.copy_stream)
    DRB_CUDA_TRY(cudaStreamCreateWithFlags(&A.copy_stream, cudaStreamNonBlocking));
  while ((int)A.seg_done.size() < nseg + 1) {
    cudaEvent_t e;
    DRB_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    A.seg_done.push_back(e);
  }
  DRB_CUDA_TRY(cudaMemcpyAsync(A.xh_dev.p, x_host, xb * A.n,
                               cudaMemcpyHostToDevice, s));
  // the kernel reads P.items / P.nitems: point them at one segment at a time
  void *items0 = P.items.p;
  const int64_t n0 = P.nitems;
  drb_status st = DRB_OK;
  // all segment launches first (a copy into pageable host memory would block
  // this thread), then the copies, each behind its segment's event
  for (int g = 0; g < nseg && st == DRB_OK; g++) {
    if (sell) {
      st = sell_launch(A, A.xh_dev.p, A.yh_dev.p, nullptr, A.sell.seg_s0[g],
                       A.sell.seg_s0[g + 1], s);
    } else {
      P.items.p = P.seg_items.as<Item>() + P.seg_i0[g];
      P.nitems = P.seg_i0[g + 1] - P.seg_i0[g];
      P.fin_c0 = P.seg_c0[g];
      P.fin_c1 = P.seg_c0[g + 1];
      st = spmv_pipe_launch(A, A.xh_dev.p, A.yh_dev.p, s);
      P.items.p = items0;
      P.nitems = n0;
      P.fin_c0 = 0;
      P.fin_c1 = -1;
    }
    if (st == DRB_OK && cudaEventRecord(A.seg_done[g], s) != cudaSuccess)
      st = DRB_ERR_CUDA;
  }
  DRB_TRY(st);
  for (int g = 0; g < nseg; g++) {
    DRB_CUDA_TRY(cudaStreamWaitEvent(A.copy_stream, A.seg_done[g], 0));
    const int64_t r0 = row0(g), r1 = row0(g + 1);
    if (r1 > r0)
      DRB_CUDA_TRY(cudaMemcpyAsync(static_cast<char *>(y_host) + yb * r0,
                                   A.yh_dev.as<char>() + yb * r0,
                                   yb * (r1 - r0), cudaMemcpyDeviceToHost,
                                   A.copy_stream));
  }
  DRB_CUDA_TRY(cudaEventRecord(A.seg_done[nseg], A.copy_stream));
  DRB_CUDA_TRY(cudaStreamWaitEvent(s, A.seg_done[nseg], 0));
  DRB_CUDA_TRY(cudaStreamSynchronize(s));
  return DRB_OK;
}

} // namespace
} // namespace drb

extern "C" {

drb_status drb_csr_gemv_host(drb_csr_t A, const void *x_host, void *y_host,
                             int64_t k, drb_layout layout, void *stream) {
  clear_error();
  if (!A)
    return invalid("A is NULL");
  if (k < 1)
    return invalid("k < 1");
  if ((A->m > 0 && !y_host) || (A->n > 0 && !x_host))
    return invalid("x or y is NULL");
  if (A->m == 0)
    return DRB_OK;
  DeviceGuard g(A->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t xb = (size_t)(A->storage == DRB_BF16
                                 ? ((A->flags & DRB_FLAG_BF16_X_F32) ? 4 : 2)
                                 : dtype_bytes(A->storage));
  const size_t yb = (size_t)(A->storage == DRB_BF16 ? 4 : dtype_bytes(A->storage));
  DRB_TRY(A->xh_dev.ensure(xb * A->n * k));
  DRB_TRY(A->yh_dev.ensure(yb * A->m * k));
  // (both pipelines run the device call's items and sums: y is the same as
  // drb_csr_gemv's, bit for bit)
  if (k == 1 && A->csplit && !A->sell.on)
    return colsplit_gemv_host(*A, x_host, y_host, xb, yb, s);
  if (k == 1 && A->nnz >= kSegmentMinNnz && (A->pipe.nitems > 0 || A->sell.on))
    return gemv_host_segmented(*A, x_host, y_host, xb, yb, s);
  if (A->n > 0)
    DRB_CUDA_TRY(cudaMemcpyAsync(A->xh_dev.p, x_host, xb * A->n * k,
                                 cudaMemcpyHostToDevice, s));
  DRB_TRY(spmv_launch(*A, A->xh_dev.p, A->yh_dev.p, k, layout, s));
  DRB_CUDA_TRY(cudaMemcpyAsync(y_host, A->yh_dev.p, yb * A->m * k,
                               cudaMemcpyDeviceToHost, s));
  DRB_CUDA_TRY(cudaStreamSynchronize(s));
  return DRB_OK;
}

drb_status drb_csr_residual_norm2(drb_csr_t A, const void *x, const void *b,
                                  void *y, double *out, void *stream) {
  clear_error();
  if (!A || !out || (A->m > 0 && !b) || (A->nnz > 0 && !x))
    return invalid("NULL argument");
  if (A->storage == DRB_BF16)
    return invalid("residual_norm2 takes F32 or F64 storage");
  DeviceGuard g(A->device);
  return residual_launch(*A, x, b, y, out, static_cast<cudaStream_t>(stream));
}

drb_status drb_csr_gemv_backward(drb_csr_t A, const void *ybar, const void *x,
                                 void *xbar, void *abar, void *stream) {
  clear_error();
  if (!A)
    return invalid("A is NULL");
  if (!A->has_adjoint) {
    set_error("gemv_backward needs a handle created with DRB_FLAG_ADJOINT");
    return DRB_ERR_INVALID_ARG;
  }
  if (!ybar && (xbar || abar))
    return invalid("ybar is NULL");
  if (abar && !x)
    return invalid("x is NULL but abar requested");
  DeviceGuard g(A->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (xbar && A->n > 0)
    DRB_TRY(spmv_t_launch(*A, ybar, xbar, s));
  if (abar && A->nnz > 0)
    DRB_TRY(abar_launch(*A, ybar, x, abar, s));
  return DRB_OK;
}

drb_status drb_csr_variant(drb_csr_t A, int *variant) {
  if (!A || !variant)
    return invalid("NULL argument");
  // a column-split handle's gemv runs the plan of its block-major copy
  const PipePlan &P = (A->csplit && !A->sell.on) ? A->csplit->pipe : A->pipe;
  *variant = A->sell.on ? kVariantSell : P.tile | (P.skew ? 1 : 0) | (P.two_slot ? 2 : 0);
  return DRB_OK;
}

drb_status drb_csr_column_blocks(drb_csr_t A, int *nblocks, int64_t *block_width) {
  clear_error();
  if (!A)
    return invalid("A is NULL");
  if (nblocks)
    *nblocks = (A->csplit && !A->sell.on) ? A->csplit_nblk : 1;
  if (block_width)
    *block_width = (A->csplit && !A->sell.on) ? A->cbounds[1] - A->cbounds[0] : A->n;
  return DRB_OK;
}

drb_status drb_csr_autotune(drb_csr_t A, int *variant, void *stream) {
  clear_error();
  if (!A)
    return invalid("A is NULL");
  DeviceGuard g(A->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int v = 0;
  DRB_TRY(autotune_pipe(*A, s, &v));
  if (A->tr)
    DRB_TRY(autotune_pipe(*A->tr, s, nullptr));
  DRB_TRY(colsplit_tune(*A, s));
  if (A->tr)
    DRB_TRY(colsplit_tune(*A->tr, s));
  if (variant)
    *variant = v;
  return DRB_OK;
}

drb_status drb_csr_check(drb_csr_t A, void *stream) {
  clear_error();
  if (!A)
    return invalid("A is NULL");
  DeviceGuard g(A->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  DRB_TRY(pipe_check(*A, s));
  if (A->tr)
    DRB_TRY(pipe_check(*A->tr, s));
  return DRB_OK;
}

drb_status drb_csr_update_values(drb_csr_t A, const void *values,
                                 void *stream) {
  clear_error();
  if (!A || (A->nnz > 0 && !values))
    return invalid("NULL argument");
  DeviceGuard g(A->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (A->nnz == 0)
    return DRB_OK;
  DRB_CUDA_TRY(cudaMemcpyAsync(A->vals.p, values,
                               (size_t)dtype_bytes(A->storage) * A->nnz,
                               cudaMemcpyDeviceToDevice, s));
  DRB_TRY(sell_pack_values(*A, s));
  DRB_TRY(colsplit_refresh_values(*A, s));
  DRB_TRY(adjoint_refresh_values(*A, s));
  if (A->tr)
    DRB_TRY(colsplit_refresh_values(*A->tr, s));
  return DRB_OK;
}

drb_status drb_dense_gemv(int64_t m, int64_t n, const void *Am, int64_t lda,
                          const void *x, void *y, int64_t k, drb_layout layout,
                          drb_dtype dtype, void *stream) {
  clear_error();
  if (m < 0 || n < 0 || k < 1 || lda < n)
    return invalid("sizes (need m, n >= 0, k >= 1, lda >= n)");
  if ((m > 0 && n > 0 && (!Am || !x)) || (m > 0 && !y))
    return invalid("NULL pointer");
  if (layout != DRB_COL_MAJOR && layout != DRB_ROW_MAJOR)
    return invalid("layout");
  int dev = 0;
  DRB_TRY(check_device(&dev));
  return dense_launch(m, n, Am, lda, x, y, k, layout, dtype,
                      static_cast<cudaStream_t>(stream));
}

drb_status drb_dot_noalloc(int64_t n, const void *a, const void *b,
                           drb_dtype dtype, double *out, void *stream) {
  clear_error();
  if (n < 0 || !out || (n > 0 && (!a || !b)))
    return invalid("NULL pointer or negative n");
  if (n > dot_noalloc_max_n()) {
    set_error("invalid argument: drb_dot_noalloc: n = %lld exceeds the maximum %lld "
              "elements that its static scratch covers; use drb_dot",
              (long long)n, (long long)dot_noalloc_max_n());
    return DRB_ERR_INVALID_ARG;
  }
  int dev = 0;
  DRB_TRY(check_device(&dev));
  return dot_noalloc_launch(n, a, b, dtype, out, static_cast<cudaStream_t>(stream));
}

drb_status drb_malloc(void **ptr, size_t bytes) {
  clear_error();
  if (!ptr)
    return invalid("ptr is NULL");
  *ptr = nullptr;
  int dev = 0;
  DRB_TRY(check_device(&dev));
  DRB_CUDA_TRY(cudaMalloc(ptr, bytes ? bytes : 16));
  return DRB_OK;
}

drb_status drb_free(void *ptr) {
  clear_error();
  if (ptr)
    DRB_CUDA_TRY(cudaFree(ptr));
  return DRB_OK;
}

drb_status drb_memcpy(void *dst, const void *src, size_t bytes, int kind,
                      void *stream) {
  clear_error();
  if (bytes == 0)
    return DRB_OK;
  if (!dst || !src)
    return invalid("NULL pointer");
  cudaMemcpyKind k;
  switch (kind) {
  case 0:
    k = cudaMemcpyHostToDevice;
    break;
  case 1:
    k = cudaMemcpyDeviceToHost;
    break;
  case 2:
    k = cudaMemcpyDeviceToDevice;
    break;
  default:
    return invalid("memcpy kind");
  }
  DRB_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, k, static_cast<cudaStream_t>(stream)));
  return DRB_OK;
}

drb_status drb_memset(void *dst, int value, size_t bytes, void *stream) {
  clear_error();
  if (bytes == 0)
    return DRB_OK;
  if (!dst)
    return invalid("NULL pointer");
  DRB_CUDA_TRY(cudaMemsetAsync(dst, value, bytes, static_cast<cudaStream_t>(stream)));
  return DRB_OK;
}

drb_status drb_stream_synchronize(void *stream) {
  clear_error();
  DRB_CUDA_TRY(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
  return DRB_OK;
}

drb_status drb_reduce(int64_t n, const void *x, drb_dtype dtype, drb_reduce_op op,
                      const void *init, void *out, void *stream) {
  clear_error();
  if (n < 0 || !out || (n > 0 && !x))
    return invalid("NULL pointer or negative n");
  if (!elementwise_dtype(dtype))
    return invalid("dtype must be F32, F64, INT32 or INT64");
  if (op != DRB_REDUCE_SUM && op != DRB_REDUCE_MIN && op != DRB_REDUCE_MAX)
    return invalid("op must be DRB_REDUCE_SUM, _MIN or _MAX");
  int dev = 0;
  DRB_TRY(check_device(&dev));
  return reduce_launch(n, x, dtype, op, init, out, static_cast<cudaStream_t>(stream));
}

drb_status drb_iota(int64_t n, void *x, drb_dtype dtype, int64_t start, void *stream) {
  clear_error();
  if (n < 0 || (n > 0 && !x))
    return invalid("NULL pointer or negative n");
  if (!elementwise_dtype(dtype))
    return invalid("dtype must be F32, F64, INT32 or INT64");
  int dev = 0;
  DRB_TRY(check_device(&dev));
  return iota_launch(n, x, dtype, start, static_cast<cudaStream_t>(stream));
}

drb_status drb_fill(int64_t n, void *x, drb_dtype dtype, const void *value, void *stream) {
  clear_error();
  if (n < 0 || !value || (n > 0 && !x))
    return invalid("NULL pointer or negative n");
  if (!elementwise_dtype(dtype))
    return invalid("dtype must be F32, F64, INT32 or INT64");
  int dev = 0;
  DRB_TRY(check_device(&dev));
  return fill_launch(n, x, dtype, value, static_cast<cudaStream_t>(stream));
}

drb_status drb_csr_cg(drb_csr_t A, const void *b, void *x, int64_t max_iters, double rtol,
                      drb_cg_info *info, void *stream) {
  clear_error();
  if (!A)
    return invalid("A is NULL");
  if (A->m != A->n)
    return invalid("drb_csr_cg needs a square matrix");
  if (max_iters < 0 || !(rtol >= 0.0))
    return invalid("max_iters < 0 or rtol not >= 0");
  if (A->m > 0 && (!b || !x))
    return invalid("x or b is NULL");
  if (A->storage != DRB_F32 && A->storage != DRB_F64) {
    set_error("drb_csr_cg: F32 or F64 storage required (BF16 storage is not supported)");
    return DRB_ERR_UNSUPPORTED;
  }
  if (A->m == 0) {
    if (info)
      *info = drb_cg_info{0, 0.0, 0.0, 1, 0};
    return DRB_OK;
  }
  DeviceGuard g(A->device);
  return cg_solve(*A, b, x, max_iters, rtol, info, static_cast<cudaStream_t>(stream));
}

drb_status drb_dot(int64_t n, const void *a, const void *b, drb_dtype dtype,
                   double *out, void *stream) {
  clear_error();
  if (n < 0 || !out || (n > 0 && (!a || !b)))
    return invalid("NULL pointer or negative n");
  int dev = 0;
  DRB_TRY(check_device(&dev));
  return dot_launch(n, a, b, dtype, out, static_cast<cudaStream_t>(stream));
}

} // extern "C"
