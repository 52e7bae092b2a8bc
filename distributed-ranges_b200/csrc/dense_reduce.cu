// dense_reduce.cu -- dense row-major gemv and the deterministic dot/norm
// reduction.
//
// Dense gemv has no dr::mp counterpart (dr::mp::gemv only takes
// distributed_sparse_matrix, include/dr/mp/algorithms/matrix/gemv.hpp:16-71);
// it is shaped after the sparse call over a row-major matrix, the layout of
// dr::sp::distributed_dense_matrix tiles
// (include/dr/sp/containers/distributed_dense_matrix.hpp:205-219).
// The dot product replaces mp::reduce over zip(a, b) | transform(mul)
// (include/dr/mp/algorithms/reduce.hpp:58-107,
// benchmarks/gbench/common/dot_product.cpp:33-52) with one launch and a
// fixed summation order.
#include <algorithm>
#include <mutex>

#include <cuda.h> // CUcontext, CUresult: types only; the library does not link libcuda

#include "drb_internal.cuh"

namespace drb {
namespace {

constexpr int kDenseNT = 256;

template <class V> __device__ __forceinline__ V warp_sum_d(V v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1)
    v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

// One warp owns RPW consecutive rows at a time and streams them with 16-byte
// loads (evict-first); x is read through L1 once per column step and reused
// for the RPW rows and KB right-hand sides.  x is column-major (x[c + j*n]).
template <class V, int KB, int RPW, bool VEC>
__global__ void __launch_bounds__(kDenseNT)
    dense_gemv_kernel(int64_t m, int64_t n, const V *__restrict__ A,
                      int64_t lda, const V *__restrict__ x,
                      V *__restrict__ y, int64_t kb_count, int64_t y_ld,
                      int64_t y_js) {
  constexpr int PER = 16 / sizeof(V);
  const uint64_t pol_s = ptx::policy_evict_first();
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * kDenseNT + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * kDenseNT) >> 5;
  const int64_t nvec = VEC ? (n / PER) * PER : 0;
  for (int64_t row0 = warp * RPW; row0 < m; row0 += nwarps * RPW) {
    V acc[RPW][KB];
#pragma unroll
    for (int r = 0; r < RPW; r++)
#pragma unroll
      for (int j = 0; j < KB; j++)
        acc[r][j] = 0;
    if (VEC) {
      for (int64_t c = (int64_t)lane * PER; c < nvec; c += 32 * PER) {
        V a[RPW][PER];
#pragma unroll
        for (int r = 0; r < RPW; r++) {
          union {
            uint4 u;
            V t[PER];
          } w;
          w.u = make_uint4(0, 0, 0, 0);
          if (row0 + r < m)
            w.u = ptx::ld_stream16(A + (row0 + r) * lda + c, pol_s);
#pragma unroll
          for (int i = 0; i < PER; i++)
            a[r][i] = w.t[i];
        }
#pragma unroll
        for (int j = 0; j < KB; j++) {
          union {
            uint4 u;
            V t[PER];
          } xv;
          xv.u = __ldg(reinterpret_cast<const uint4 *>(x + j * n + c));
#pragma unroll
          for (int r = 0; r < RPW; r++)
#pragma unroll
            for (int i = 0; i < PER; i++)
              acc[r][j] += a[r][i] * xv.t[i];
        }
      }
    }
    for (int64_t c = nvec + lane; c < n; c += 32) {
#pragma unroll
      for (int j = 0; j < KB; j++) {
        const V xv = __ldg(x + j * n + c);
#pragma unroll
        for (int r = 0; r < RPW; r++)
          if (row0 + r < m)
            acc[r][j] += A[(row0 + r) * lda + c] * xv;
      }
    }
#pragma unroll
    for (int r = 0; r < RPW; r++)
#pragma unroll
      for (int j = 0; j < KB; j++) {
        const V s = warp_sum_d(acc[r][j]);
        if (lane == 0 && row0 + r < m && j < kb_count)
          y[(row0 + r) * y_ld + j * y_js] = s;
      }
  }
}

// Balanced 16-byte path.  The work is cut into units of one row x one column
// slab (slab_groups<V>() 16-byte groups: 32 KB of an f32 row, 16 KB of an
// f64 row); warp w of W takes the contiguous unit range
// [units*w/W, units*(w+1)/W), so every warp gets the same number of units
// (+-1) whatever the shape -- tall, square or wide.  A unit's sums go to y
// directly when a row is one slab, else to part[(row * ns + slab) * KB + j],
// which dense_slab_sum adds in slab order (deterministic).  Each lane keeps
// U consecutive 16-byte groups of its row in flight, so a warp reads
// 512*U contiguous bytes per step: one row per warp with U = 4 (f32) / 16
// (f64) measured 6.9 TB/s on 32768^2, against 4.9 TB/s (f32) for four rows
// per warp with one group each (page locality, not occupancy, decides).
template <class V> constexpr int64_t slab_groups() { return sizeof(V) == 4 ? 2048 : 1024; }
template <class V, int KB> constexpr int slab_unroll() {
  return KB == 1 ? (sizeof(V) == 4 ? 4 : 16) : (KB <= 4 ? 2 : 1);
}

template <class V, int KB>
__global__ void __launch_bounds__(kDenseNT)
    dense_slab_kernel(int64_t m, int64_t ng, const V *__restrict__ A, int64_t lda,
                      const V *__restrict__ x, int64_t n, V *__restrict__ y, int64_t kbc,
                      int64_t y_ld, int64_t y_js, V *__restrict__ part, int64_t ns,
                      int64_t units) {
  constexpr int PER = 16 / sizeof(V);
  constexpr int U = slab_unroll<V, KB>();
  constexpr int64_t SG = slab_groups<V>();
  const uint64_t pol_s = ptx::policy_evict_first();
  const int lane = threadIdx.x & 31;
  const int64_t w = ((int64_t)blockIdx.x * kDenseNT + threadIdx.x) >> 5;
  const int64_t W = ((int64_t)gridDim.x * kDenseNT) >> 5;
  // units * W stays far below 2^63 (units <= m * n / 1024, W < 2^17)
  const int64_t u0 = units * w / W;
  const int64_t u1 = units * (w + 1) / W;
  for (int64_t u = u0; u < u1; u++) {
    const int64_t row = u / ns, sl = u - row * ns;
    const int64_t g0 = sl * SG;
    const int64_t g1 = min(g0 + SG, ng);
    const V *Ar = A + row * lda;
    V acc[KB];
#pragma unroll
    for (int j = 0; j < KB; j++)
      acc[j] = 0;
    for (int64_t gb = g0 + lane; gb < g1; gb += 32 * U) {
      union G16 {
        uint4 u;
        V t[PER];
      };
      G16 a[U];
#pragma unroll
      for (int q = 0; q < U; q++) {
        a[q].u = make_uint4(0, 0, 0, 0);
        if (gb + 32 * q < g1)
          a[q].u = ptx::ld_stream16(Ar + (gb + 32 * q) * PER, pol_s);
      }
#pragma unroll
      for (int q = 0; q < U; q++) {
        const int64_t g = gb + 32 * q;
        if (g < g1) {
#pragma unroll
          for (int j = 0; j < KB; j++) {
            G16 xv;
            xv.u = __ldg(reinterpret_cast<const uint4 *>(x + j * n) + g);
#pragma unroll
            for (int i = 0; i < PER; i++)
              acc[j] += a[q].t[i] * xv.t[i];
          }
        }
      }
    }
#pragma unroll
    for (int j = 0; j < KB; j++) {
      const V t = warp_sum_d(acc[j]);
      if (lane == 0 && j < kbc) {
        if (ns == 1)
          y[row * y_ld + j * y_js] = t;
        else
          part[(row * ns + sl) * KB + j] = t;
      }
    }
  }
}

// y[r, j] = sum over slabs of part[(r * ns + s) * KB + j], in slab order.
template <class V, int KB>
__global__ void dense_slab_sum(int64_t m, int64_t ns, const V *__restrict__ part,
                               V *__restrict__ y, int64_t kbc, int64_t y_ld, int64_t y_js) {
  const int64_t nth = (int64_t)gridDim.x * blockDim.x;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < m * kbc; t += nth) {
    const int64_t r = t / kbc, j = t - r * kbc;
    const V *p = part + r * ns * KB + j;
    V s = 0;
    for (int64_t q = 0; q < ns; q++)
      s += p[q * KB];
    y[r * y_ld + j * y_js] = s;
  }
}

template <class V, int KB>
drb_status dense_slab_call(cudaStream_t s, int64_t m, int64_t n, const V *A, int64_t lda,
                           const V *x, V *y, int64_t kbc, int64_t y_ld, int64_t y_js) {
  constexpr int PER = 16 / sizeof(V);
  constexpr int64_t SG = slab_groups<V>();
  static int grid_cache[64] = {0};
  int dev = 0;
  DRB_CUDA_TRY(cudaGetDevice(&dev));
  int &grid = grid_cache[dev < 64 ? dev : 0];
  if (grid == 0) {
    int occ = 0, sms = 0;
    DRB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &occ, dense_slab_kernel<V, KB>, kDenseNT, 0));
    DRB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    grid = std::max(1, occ) * sms;
  }
  const int64_t ng = n / PER;
  const int64_t ns = std::max<int64_t>(1, (ng + SG - 1) / SG);
  const int64_t units = m * ns;
  V *part = nullptr;
  if (ns > 1)
    DRB_TRY(scratch_alloc(reinterpret_cast<void **>(&part), sizeof(V) * (size_t)m * ns * KB, s));
  const int64_t need = (units + 7) / 8; // 8 warps per CTA
  const unsigned g = (unsigned)std::max<int64_t>(1, std::min<int64_t>(grid, need));
  dense_slab_kernel<V, KB><<<g, kDenseNT, 0, s>>>(m, ng, A, lda, x, n, y, kbc, y_ld, y_js,
                                                  part, ns, units);
  note_launch();
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess && ns > 1) {
    const unsigned sg = (unsigned)std::max<int64_t>(
        1, std::min<int64_t>(148 * 16, (m * kbc + 255) / 256));
    dense_slab_sum<V, KB><<<sg, 256, 0, s>>>(m, ns, part, y, kbc, y_ld, y_js);
    note_launch();
    e = cudaGetLastError();
  }
  if (part)
    scratch_free(part, s);
  if (e != cudaSuccess) {
    set_error("dense gemv launch: %s", cudaGetErrorString(e));
    return DRB_ERR_CUDA;
  }
  return DRB_OK;
}

template <class V, int KB, int RPW>
drb_status dense_call(bool vec, unsigned grid, cudaStream_t s, int64_t m, int64_t n,
                      const V *A, int64_t lda, const V *x, V *y, int64_t kbc,
                      int64_t y_ld, int64_t y_js) {
  if (vec)
    return dense_slab_call<V, KB>(s, m, n, A, lda, x, y, kbc, y_ld, y_js);
  dense_gemv_kernel<V, KB, RPW, false><<<grid, kDenseNT, 0, s>>>(
      m, n, A, lda, x, y, kbc, y_ld, y_js);
  note_launch();
  return DRB_OK;
}

template <class V>
drb_status dense_typed(int64_t m, int64_t n, const V *A, int64_t lda,
                       const V *x, V *y, int64_t k, drb_layout layout,
                       cudaStream_t s) {
  constexpr int PER = 16 / sizeof(V);
  // x as column-major: a row-major k > 1 block is transposed first.
  const V *xc = x;
  void *tmp = nullptr;
  if (layout == DRB_ROW_MAJOR && k > 1) {
    DRB_TRY(scratch_alloc(&tmp, sizeof(V) * n * k, s));
    drb_status st = transpose_launch(x, tmp, n, k, sizeof(V), s);
    if (st != DRB_OK) {
      scratch_free(tmp, s);
      return st;
    }
    xc = static_cast<const V *>(tmp);
  }
  const bool vec = (reinterpret_cast<uintptr_t>(A) % 16 == 0) &&
                   (reinterpret_cast<uintptr_t>(xc) % 16 == 0) &&
                   (lda % PER == 0) && (n % PER == 0);
  const unsigned grid = 148 * 8;
  // y address of (row r, rhs j): r*y_ld + j*y_js
  const int64_t y_ld = layout == DRB_ROW_MAJOR ? k : 1;
  const int64_t y_js = layout == DRB_ROW_MAJOR ? 1 : m;
  for (int64_t jb = 0; jb < k;) {
    const int64_t left = k - jb;
    const V *xj = xc + jb * n;
    V *yj = y + jb * y_js;
    drb_status st;
    if (left >= 8) {
      st = dense_call<V, 8, 1>(vec, grid, s, m, n, A, lda, xj, yj, 8, y_ld, y_js);
      jb += 8;
    } else if (left >= 4) {
      st = dense_call<V, 4, 2>(vec, grid, s, m, n, A, lda, xj, yj, 4, y_ld, y_js);
      jb += 4;
    } else if (left >= 2) {
      st = dense_call<V, 2, 2>(vec, grid, s, m, n, A, lda, xj, yj, 2, y_ld, y_js);
      jb += 2;
    } else {
      st = dense_call<V, 1, 4>(vec, grid, s, m, n, A, lda, xj, yj, 1, y_ld, y_js);
      jb += 1;
    }
    if (st != DRB_OK) {
      if (tmp)
        scratch_free(tmp, s);
      return st;
    }
  }
  cudaError_t e = cudaGetLastError();
  if (tmp)
    scratch_free(tmp, s);
  if (e != cudaSuccess) {
    set_error("dense gemv launch: %s", cudaGetErrorString(e));
    return DRB_ERR_CUDA;
  }
  return DRB_OK;
}

// ---- dot -------------------------------------------------------------------------
constexpr int kDotNT = 256;
constexpr int kDotGrid = 592; // fixed: the summation order must not vary
constexpr int kDotUnroll = 4; // 16-byte loads in flight per vector per thread

template <class V>
__global__ void __launch_bounds__(kDotNT)
    dot_kernel(int64_t n, const V *__restrict__ a, const V *__restrict__ b,
               double *partials, int *ticket, double *out) {
  __shared__ double s_red[kDotNT / 32];
  __shared__ int s_last;
  constexpr int PER = 16 / sizeof(V);
  const uint64_t pol_s = ptx::policy_evict_first();
  double acc = 0.0;
  const int64_t tid = (int64_t)blockIdx.x * kDotNT + threadIdx.x;
  const int64_t nth = (int64_t)gridDim.x * kDotNT;
  const bool vec = (reinterpret_cast<uintptr_t>(a) % 16 == 0) &&
                   (reinterpret_cast<uintptr_t>(b) % 16 == 0);
  int64_t done = 0;
  if (vec) {
    union W {
      uint4 u;
      V t[PER];
    };
    const int64_t nv = n / PER;
    int64_t i = tid;
    // kDotUnroll grid-strided vectors per trip, all loads issued first
    for (; i + (kDotUnroll - 1) * nth < nv; i += kDotUnroll * nth) {
      W wa[kDotUnroll], wb[kDotUnroll];
#pragma unroll
      for (int u = 0; u < kDotUnroll; u++)
        wa[u].u = ptx::ld_stream16(a + (i + u * nth) * PER, pol_s);
#pragma unroll
      for (int u = 0; u < kDotUnroll; u++)
        wb[u].u = (a == b) ? wa[u].u : ptx::ld_stream16(b + (i + u * nth) * PER, pol_s);
#pragma unroll
      for (int u = 0; u < kDotUnroll; u++)
#pragma unroll
        for (int q = 0; q < PER; q++)
          acc += (double)wa[u].t[q] * (double)wb[u].t[q];
    }
    for (; i < nv; i += nth) {
      W wa, wb;
      wa.u = ptx::ld_stream16(a + i * PER, pol_s);
      wb.u = (a == b) ? wa.u : ptx::ld_stream16(b + i * PER, pol_s);
#pragma unroll
      for (int q = 0; q < PER; q++)
        acc += (double)wa.t[q] * (double)wb.t[q];
    }
    done = nv * PER;
  }
  for (int64_t i = done + tid; i < n; i += nth)
    acc += (double)a[i] * (double)b[i];
  // block reduction
  acc = warp_sum_d(acc);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0)
    s_red[warp] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < kDotNT / 32; w++)
      s += s_red[w];
    partials[blockIdx.x] = s;
    __threadfence();
    s_last = atomicAdd(ticket, 1) == (int)gridDim.x - 1;
  }
  __syncthreads();
  if (s_last) {
    // the last CTA adds the partials with all threads in a fixed order
    __threadfence();
    double s = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += kDotNT)
      s += __ldcg(&partials[i]);
    s = warp_sum_d(s);
    __syncthreads();
    if (lane == 0)
      s_red[warp] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < kDotNT / 32; w++)
        t += s_red[w];
      *out = t;
      *ticket = 0;
    }
  }
}

// ---- dot without allocation --------------------------------------------------
// Scratch of drb_dot_noalloc: one f64 partial per CTA plus the ticket, in a
// file-scope device array that every GPU loading the library keeps until
// process exit (kNoAllocSlots * 8 bytes + 256 = 512.25 KiB).  Each CTA covers
// kNoAllocBlock elements, so the largest vector is kNoAllocSlots *
// kNoAllocBlock elements.
constexpr int kNoAllocBlock = kDotNT * 32;   // 8192 elements per CTA
constexpr int kNoAllocSlots = 65536;         // partials (one per CTA)
constexpr int64_t kNoAllocMaxN = (int64_t)kNoAllocBlock * kNoAllocSlots; // 2^29
static __device__ __align__(256) double g_dot_noalloc_scratch[kNoAllocSlots + 32];

std::mutex g_noalloc_mu;
struct NoAllocAddr {
  unsigned long long ctx = 0; // id of the context the address belongs to
  void *addr = nullptr;
};
NoAllocAddr g_noalloc_addr[64];

// The driver's context queries, through the runtime's entry-point lookup (the
// library does not link libcuda itself).
typedef CUresult (*CtxCurrentFn)(CUcontext *);
typedef CUresult (*CtxIdFn)(CUcontext, unsigned long long *);

// Id of the calling thread's current context (unique for the life of the
// process: a context created again, e.g. after cudaDeviceReset, gets a new
// id), or 0 when none is current.  Called with g_noalloc_mu held.
drb_status current_ctx_id(unsigned long long *id) {
  static CtxCurrentFn cur = nullptr;
  static CtxIdFn get_id = nullptr;
  if (!cur || !get_id) {
    void *f1 = nullptr, *f2 = nullptr;
    cudaDriverEntryPointQueryResult q1, q2;
    DRB_CUDA_TRY(cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f1, 12000,
                                                  cudaEnableDefault, &q1));
    DRB_CUDA_TRY(cudaGetDriverEntryPointByVersion("cuCtxGetId", &f2, 12000,
                                                  cudaEnableDefault, &q2));
    if (q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess || !f1 ||
        !f2) {
      set_error("drb_dot_noalloc: the driver does not provide cuCtxGetCurrent/cuCtxGetId");
      return DRB_ERR_CUDA;
    }
    cur = reinterpret_cast<CtxCurrentFn>(f1);
    get_id = reinterpret_cast<CtxIdFn>(f2);
  }
  CUcontext c = nullptr;
  *id = 0;
  if (cur(&c) != CUDA_SUCCESS || !c)
    return DRB_OK;
  if (get_id(c, id) != CUDA_SUCCESS)
    *id = 0;
  return DRB_OK;
}

// Device address of the scratch array in the current device's context.  Host
// code only sees a host-side stand-in under that name, so the address is
// looked up with cudaGetSymbolAddress on the first call in each context (the
// first call on a device, and the first after its context was destroyed and
// created again) and cached under the context's id.
drb_status noalloc_scratch(double **out) {
  int dev = 0;
  DRB_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) {
    set_error("drb_dot_noalloc: device %d out of range", dev);
    return DRB_ERR_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  unsigned long long id = 0;
  DRB_TRY(current_ctx_id(&id));
  NoAllocAddr &e = g_noalloc_addr[dev];
  if (id == 0 || e.ctx != id || !e.addr) {
    void *p = nullptr;
    DRB_CUDA_TRY(cudaGetSymbolAddress(&p, g_dot_noalloc_scratch)); // makes the context
    DRB_TRY(current_ctx_id(&id));
    e.ctx = id;
    e.addr = p;
  }
  *out = static_cast<double *>(e.addr);
  return DRB_OK;
}

} // namespace

int64_t dot_noalloc_max_n() { return kNoAllocMaxN; }

drb_status dot_noalloc_launch(int64_t n, const void *a, const void *b,
                              drb_dtype dt, double *out, cudaStream_t s) {
  if (n > kNoAllocMaxN) {
    set_error("drb_dot_noalloc: n = %lld exceeds the maximum %lld elements that its "
              "static scratch covers; use drb_dot",
              (long long)n, (long long)kNoAllocMaxN);
    return DRB_ERR_INVALID_ARG;
  }
  if (dt != DRB_F32 && dt != DRB_F64) {
    set_error("drb_dot_noalloc: dtype %d not supported", (int)dt);
    return DRB_ERR_UNSUPPORTED;
  }
  double *scratch = nullptr;
  DRB_TRY(noalloc_scratch(&scratch));
  int *ticket = reinterpret_cast<int *>(scratch + kNoAllocSlots);
  // the array keeps the previous call's contents: the ticket must start at 0
  DRB_CUDA_TRY(cudaMemsetAsync(ticket, 0, sizeof(int), s));
  const int64_t grid = std::max<int64_t>(1, (n + kNoAllocBlock - 1) / kNoAllocBlock);
  if (dt == DRB_F32)
    dot_kernel<float><<<(unsigned)grid, kDotNT, 0, s>>>(
        n, (const float *)a, (const float *)b, scratch, ticket, out);
  else
    dot_kernel<double><<<(unsigned)grid, kDotNT, 0, s>>>(
        n, (const double *)a, (const double *)b, scratch, ticket, out);
  note_launch();
  DRB_CUDA_TRY(cudaGetLastError());
  return DRB_OK;
}

drb_status dense_launch(int64_t m, int64_t n, const void *A, int64_t lda,
                        const void *x, void *y, int64_t k, drb_layout layout,
                        drb_dtype dt, cudaStream_t s) {
  if (m == 0 || k == 0)
    return DRB_OK;
  if (n == 0) {
    DRB_CUDA_TRY(cudaMemsetAsync(y, 0, (size_t)dtype_bytes(dt) * m * k, s));
    return DRB_OK;
  }
  if (dt == DRB_F32)
    return dense_typed<float>(m, n, (const float *)A, lda, (const float *)x,
                              (float *)y, k, layout, s);
  if (dt == DRB_F64)
    return dense_typed<double>(m, n, (const double *)A, lda, (const double *)x,
                               (double *)y, k, layout, s);
  set_error("dense gemv: dtype %d not supported", (int)dt);
  return DRB_ERR_UNSUPPORTED;
}

drb_status dot_launch(int64_t n, const void *a, const void *b, drb_dtype dt,
                      double *out, cudaStream_t s) {
  if (dt != DRB_F32 && dt != DRB_F64) {
    set_error("dot: dtype %d not supported", (int)dt);
    return DRB_ERR_UNSUPPORTED;
  }
  void *scratch = nullptr;
  const size_t bytes = sizeof(double) * kDotGrid + 16;
  DRB_TRY(scratch_alloc(&scratch, bytes, s));
  double *partials = static_cast<double *>(scratch);
  int *ticket = reinterpret_cast<int *>(partials + kDotGrid);
  cudaError_t e = cudaMemsetAsync(ticket, 0, sizeof(int), s);
  if (e == cudaSuccess) {
    if (dt == DRB_F32)
      dot_kernel<float><<<kDotGrid, kDotNT, 0, s>>>(
          n, (const float *)a, (const float *)b, partials, ticket, out);
    else
      dot_kernel<double><<<kDotGrid, kDotNT, 0, s>>>(
          n, (const double *)a, (const double *)b, partials, ticket, out);
    note_launch();
    e = cudaGetLastError();
  }
  scratch_free(scratch, s);
  if (e != cudaSuccess) {
    set_error("dot launch: %s", cudaGetErrorString(e));
    return DRB_ERR_CUDA;
  }
  return DRB_OK;
}

} // namespace drb
