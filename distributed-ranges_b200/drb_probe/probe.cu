// probe.cu -- a measured floor for gather-bound sparse products.
//
// A CSR SpMV with uniformly random columns is not bound by HBM: every x
// element it gathers costs one L1-to-crossbar request, and the SM issues about
// one such request per clock.  drb_csr_gather_probe measures that floor on a
// handle's own pattern: it streams the column indices (and, with
// with_values, the values) with the row-block kernel's 16-byte evict-first
// loads and gathers x at every column with its evict-last loads -- the reads
// of an SpMV without its rows, row sums or y.  No kernel that reads the
// nonzeros and fetches x element by element through the SM can take less
// time, so its time is the roofline a gather-bound product is measured
// against.  Nothing is written unless the running sum hits a sentinel no
// finite input reaches (which keeps the loads live).
//
// Built into its own library (lib/libdrb_probe.so, linked against
// libdrb.so for the handle's storage and error reporting), used by the bench
// and its test only: it is not part of the C ABI of include/drb.h.
#include "drb_probe.h"
#include "spmv_warp.cuh"

namespace drb {
namespace {

using warpk::AccOf;
using warpk::ld_group;
using warpk::ld_x;
using warpk::to_acc;

constexpr int kProbeNT = 256;

template <class V, class CI, bool VALS>
__global__ void __launch_bounds__(kProbeNT)
    gather_probe(int64_t nnz, const CI *__restrict__ colind, const V *__restrict__ vals,
                 const V *__restrict__ x, typename AccOf<V>::type *out) {
  using Acc = typename AccOf<V>::type;
  // G nonzeros per group: one 16-byte load of the narrower array
  constexpr int G = 16 / (sizeof(V) < sizeof(CI) ? sizeof(V) : sizeof(CI));
  constexpr int U = G >= 8 ? 1 : 8 / G; // 8 gathers in flight per thread
  const uint64_t pol_s = ptx::policy_evict_first(), pol_x = ptx::policy_evict_last();
  const int64_t nth = (int64_t)gridDim.x * kProbeNT;
  const int64_t tid = (int64_t)blockIdx.x * kProbeNT + threadIdx.x;
  const int64_t ng = nnz / G;
  Acc acc = Acc(0);
  int64_t g = tid;
  for (; g + (U - 1) * nth < ng; g += U * nth) {
    CI c[U][G];
    V v[U][G];
#pragma unroll
    for (int u = 0; u < U; u++) {
      ld_group<CI, G>(colind + (g + u * nth) * G, c[u], pol_s);
      if (VALS)
        ld_group<V, G>(vals + (g + u * nth) * G, v[u], pol_s);
    }
    Acc xv[U][G];
#pragma unroll
    for (int u = 0; u < U; u++)
#pragma unroll
      for (int i = 0; i < G; i++)
        xv[u][i] = ld_x(x + c[u][i], pol_x);
#pragma unroll
    for (int u = 0; u < U; u++)
#pragma unroll
      for (int i = 0; i < G; i++)
        acc += VALS ? to_acc(v[u][i]) * xv[u][i] : xv[u][i];
  }
  for (; g < ng; g += nth) {
    CI c[G];
    V v[G];
    ld_group<CI, G>(colind + g * G, c, pol_s);
    if (VALS)
      ld_group<V, G>(vals + g * G, v, pol_s);
#pragma unroll
    for (int i = 0; i < G; i++) {
      const Acc xi = ld_x(x + c[i], pol_x);
      acc += VALS ? to_acc(v[i]) * xi : xi;
    }
  }
  for (int64_t p = ng * G + tid; p < nnz; p += nth) {
    const Acc xi = ld_x(x + colind[p], pol_x);
    acc += VALS ? to_acc(vals[p]) * xi : xi;
  }
  if (acc == Acc(-3.0e38)) // unreachable for finite inputs of this size
    *out = acc;
}

// The row form (k right-hand sides, X row-major): every nonzero gathers its
// X row -- KP 16-byte vectors, one per lane of a group of KP lanes, with the
// read-only loads of the batched SpMM -- while the column indices (and
// values) stream, four nonzeros in flight per lane.  Consecutive groups of a
// warp take consecutive nonzeros, so the index loads coalesce as the SpMM's
// staged ones do.
template <class V, class CI, bool VALS>
__global__ void __launch_bounds__(kProbeNT)
    gather_rows_probe(int64_t nnz, const CI *__restrict__ colind, const V *__restrict__ vals,
                      const uint4 *__restrict__ X, int64_t ldv, int lkp,
                      typename AccOf<V>::type *out) {
  using Acc = typename AccOf<V>::type;
  constexpr int PER = 16 / sizeof(V); // elements of one 16-byte vector
  constexpr int U = 4;
  const int64_t t = (int64_t)blockIdx.x * kProbeNT + threadIdx.x;
  const int part = (int)(t & ((1 << lkp) - 1));
  const int64_t ns = ((int64_t)gridDim.x * kProbeNT) >> lkp;
  auto words = [](const uint4 &w, Acc a, Acc v) {
    const V *e = reinterpret_cast<const V *>(&w);
#pragma unroll
    for (int i = 0; i < PER; i++)
      a += VALS ? v * to_acc(e[i]) : to_acc(e[i]);
    return a;
  };
  Acc acc = Acc(0);
  int64_t p = t >> lkp;
  for (; p + (U - 1) * ns < nnz; p += U * ns) {
    CI c[U];
    Acc v[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      c[u] = __ldg(colind + p + u * ns);
      v[u] = VALS ? to_acc(__ldg(vals + p + u * ns)) : Acc(1);
    }
    uint4 w[U];
#pragma unroll
    for (int u = 0; u < U; u++)
      w[u] = __ldg(X + (int64_t)c[u] * ldv + part);
#pragma unroll
    for (int u = 0; u < U; u++)
      acc = words(w[u], acc, v[u]);
  }
  for (; p < nnz; p += ns) {
    const CI c = __ldg(colind + p);
    const Acc v = VALS ? to_acc(__ldg(vals + p)) : Acc(1);
    acc = words(__ldg(X + (int64_t)c * ldv + part), acc, v);
  }
  if (acc == Acc(-3.0e38)) // unreachable for finite inputs of this size
    *out = acc;
}

template <class V, class CI>
drb_status rows_probe_typed(Csr &A, const void *X, int64_t ldv, int lkp, bool with_values,
                            void *out, cudaStream_t s) {
  using Acc = typename AccOf<V>::type;
  auto kern = with_values ? gather_rows_probe<V, CI, true> : gather_rows_probe<V, CI, false>;
  int occ = 0, sms = 0;
  DRB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kProbeNT, 0));
  DRB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, A.device));
  const int grid = std::max(1, occ) * sms;
  kern<<<grid, kProbeNT, 0, s>>>(A.nnz, A.colind.as<CI>(), A.vals.as<V>(),
                                 static_cast<const uint4 *>(X), ldv, lkp,
                                 static_cast<Acc *>(out));
  note_launch();
  DRB_CUDA_TRY(cudaGetLastError());
  return DRB_OK;
}

template <class V, class CI>
drb_status probe_typed(Csr &A, const void *x, bool with_values, void *out, cudaStream_t s) {
  using Acc = typename AccOf<V>::type;
  auto kern = with_values ? gather_probe<V, CI, true> : gather_probe<V, CI, false>;
  int occ = 0, sms = 0;
  DRB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kProbeNT, 0));
  DRB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, A.device));
  const int grid = std::max(1, occ) * sms;
  kern<<<grid, kProbeNT, 0, s>>>(A.nnz, A.colind.as<CI>(), A.vals.as<V>(),
                                 static_cast<const V *>(x), static_cast<Acc *>(out));
  note_launch();
  DRB_CUDA_TRY(cudaGetLastError());
  return DRB_OK;
}

} // namespace
} // namespace drb

extern "C" drb_status drb_csr_gather_probe(drb_csr_t A, const void *x, int with_values,
                                           void *stream) {
  using namespace drb;
  clear_error();
  if (!A || (A->nnz > 0 && !x)) {
    set_error("invalid argument: A or x is NULL");
    return DRB_ERR_INVALID_ARG;
  }
  if (A->nnz == 0)
    return DRB_OK;
  if (A->storage != DRB_F32 && A->storage != DRB_F64) {
    set_error("gather probe: F32 or F64 storage only");
    return DRB_ERR_UNSUPPORTED;
  }
  DeviceGuard g(A->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  void *out = nullptr;
  DRB_TRY(scratch_alloc(&out, 16, s));
  const bool wv = with_values != 0;
  drb_status st;
  if (A->storage == DRB_F32)
    st = A->cbytes == 4 ? probe_typed<float, int32_t>(*A, x, wv, out, s)
                        : probe_typed<float, int64_t>(*A, x, wv, out, s);
  else
    st = A->cbytes == 4 ? probe_typed<double, int32_t>(*A, x, wv, out, s)
                        : probe_typed<double, int64_t>(*A, x, wv, out, s);
  scratch_free(out, s);
  return st;
}

extern "C" drb_status drb_csr_gather_rows_probe(drb_csr_t A, const void *X, int64_t ldx,
                                                int64_t k, int with_values, void *stream) {
  using namespace drb;
  clear_error();
  if (!A || (A->nnz > 0 && !X)) {
    set_error("invalid argument: A or X is NULL");
    return DRB_ERR_INVALID_ARG;
  }
  if (A->storage != DRB_F32 && A->storage != DRB_F64) {
    set_error("gather rows probe: F32 or F64 storage only");
    return DRB_ERR_UNSUPPORTED;
  }
  const int64_t es = A->storage == DRB_F32 ? 4 : 8;
  const int64_t kp = k * es / 16;
  if (k < 1 || ldx < k || (k * es) % 16 != 0 || (ldx * es) % 16 != 0 || kp > 32 ||
      (kp & (kp - 1)) != 0) {
    set_error("gather rows probe: k * element size must be 16, 32, ..., 512 bytes (a power "
              "of two) and ldx >= k a multiple of 16 bytes");
    return DRB_ERR_UNSUPPORTED;
  }
  if (reinterpret_cast<uintptr_t>(X) % 16 != 0) {
    set_error("invalid argument: X must be 16-byte aligned");
    return DRB_ERR_INVALID_ARG;
  }
  if (A->nnz == 0)
    return DRB_OK;
  int lkp = 0;
  while ((1 << lkp) < kp)
    lkp++;
  DeviceGuard g(A->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  void *out = nullptr;
  DRB_TRY(scratch_alloc(&out, 16, s));
  const bool wv = with_values != 0;
  const int64_t ldv = ldx * es / 16;
  drb_status st;
  if (A->storage == DRB_F32)
    st = A->cbytes == 4 ? rows_probe_typed<float, int32_t>(*A, X, ldv, lkp, wv, out, s)
                        : rows_probe_typed<float, int64_t>(*A, X, ldv, lkp, wv, out, s);
  else
    st = A->cbytes == 4 ? rows_probe_typed<double, int32_t>(*A, X, ldv, lkp, wv, out, s)
                        : rows_probe_typed<double, int64_t>(*A, X, ldv, lkp, wv, out, s);
  scratch_free(out, s);
  return st;
}
