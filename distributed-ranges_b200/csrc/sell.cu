// sell.cu -- sliced-ELL (SELL-32) copy of a CSR matrix whose rows are short
// and regular, and the single-right-hand-side SpMV over it.
//
// The row-block kernel (spmv_warp.cuh) stages products in shared memory and
// sums each row with a segmented reduction; for rows of a handful of
// nonzeros (a 5-point stencil) that bookkeeping costs more than the bytes it
// moves.  Here rows are grouped in slices of 32 consecutive rows; slice s is
// padded to its longest row, w_s, and stored k-major: element k of row
// 32*s + lane sits at off[s] + 32*k + lane.  A warp runs one slice (two for
// f32) per step with lane = row, so every load of values and column indices
// is one coalesced 128/256-byte line, and x gathers of a banded matrix (neighbouring rows,
// neighbouring columns) coalesce too.  Each row is summed by its own lane in
// k order, so results are deterministic.  Padding entries carry value 0 and
// the row's last column (x stays in a cached line).
//
// A handle gets the copy when its rows are short and regular enough that the
// padding is small (sell_build); the CSR arrays stay for every other path.
// The kernel carries the same fused row reductions as the row-block kernel
// (warpk::WarpResid: ||Ax - b||^2, or sum y_i w_i for conjugate gradients,
// and the stop word) and runs over any slice range, which the host-pointer
// gemv uses to stream y back in row segments.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "spmv_warp.cuh"

namespace drb {
namespace {

using warpk::AccOf;
using warpk::WarpResid;
constexpr int kSellNT = 256;
constexpr int kSellWarps = kSellNT / 32;
constexpr int kSellMaxWidth = 64;  // longest row a SELL copy accepts
constexpr double kSellMaxPad = 1.2; // padded elements / nnz

__device__ __forceinline__ float ld_stream(const float *p, uint64_t pol) {
  float r;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;"
      : "=f"(r) : "l"(p), "l"(pol));
  return r;
}
__device__ __forceinline__ double ld_stream(const double *p, uint64_t pol) {
  double r;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;"
      : "=d"(r) : "l"(p), "l"(pol));
  return r;
}
__device__ __forceinline__ int ld_stream(const int *p, uint64_t pol) {
  int r;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.b32 %0, [%1], %2;"
      : "=r"(r) : "l"(p), "l"(pol));
  return r;
}

// One thread per row of the padded slices: copies the row's entries into
// the k-major slots and pads to the slice width.  With cols_too == false
// only the values are rewritten (drb_csr_update_values).
template <class V, class RI>
__global__ void sell_pack(int64_t m, int64_t nrows_padded, const RI *__restrict__ rowptr,
                          const int *__restrict__ colind, const V *__restrict__ vals,
                          const int64_t *__restrict__ off, V *__restrict__ svals,
                          int *__restrict__ scols, bool cols_too) {
  const int64_t nth = (int64_t)gridDim.x * blockDim.x;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < nrows_padded;
       r += nth) {
    const int64_t sl = r >> 5;
    const int lane = (int)(r & 31);
    const int64_t o = off[sl];
    const int w = (int)((off[sl + 1] - o) >> 5);
    int64_t p0 = 0, len = 0;
    if (r < m) {
      p0 = (int64_t)rowptr[r];
      len = (int64_t)rowptr[r + 1] - p0;
    }
    const int padc = len > 0 ? colind[p0 + len - 1] : 0;
    for (int k = 0; k < w; k++) {
      const int64_t d = o + 32 * (int64_t)k + lane;
      svals[d] = k < len ? vals[p0 + k] : V(0);
      if (cols_too)
        scols[d] = k < len ? colind[p0 + k] : padc;
    }
  }
}

template <class V, bool RESID, int NS, int K>
__global__ void __launch_bounds__(kSellNT)
    sell_spmv(const V *__restrict__ vals, const int *__restrict__ cols,
              const int64_t *__restrict__ off, int64_t s0, int64_t s1, int64_t m,
              const V *__restrict__ x, typename AccOf<V>::type *__restrict__ y,
              WarpResid ra) {
  using Acc = typename AccOf<V>::type;
  __shared__ double s_red[kSellWarps];
  __shared__ int s_last;
  if (RESID && ra.stop && *static_cast<const volatile int *>(ra.stop))
    return; // uniform: every CTA reads the same word, written by an earlier launch
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t w = (int64_t)blockIdx.x * kSellWarps + warp;
  const int64_t W = (int64_t)gridDim.x * kSellWarps;
  const int64_t ns = s1 - s0;
  const int64_t a = s0 + ns * w / W, b = s0 + ns * (w + 1) / W;
  const uint64_t pol_s = ptx::policy_evict_first();
  const uint64_t pol_x = ptx::policy_evict_last();
  const Acc *bvec = static_cast<const Acc *>(ra.b);
  double r2 = 0.0;
  for (int64_t sl = a; sl < b; sl += NS) {
    int64_t o[NS];
    int wd[NS];
    int wmax = 0;
#pragma unroll
    for (int j = 0; j < NS; j++) {
      wd[j] = 0;
      o[j] = 0;
      if (sl + j < b) {
        o[j] = __ldg(off + sl + j);
        wd[j] = (int)((__ldg(off + sl + j + 1) - o[j]) >> 5);
      }
      wmax = max(wmax, wd[j]);
    }
    Acc acc[NS];
#pragma unroll
    for (int j = 0; j < NS; j++)
      acc[j] = 0;
    for (int k0 = 0; k0 < wmax; k0 += K) {
      V v[NS][K];
      int c[NS][K];
#pragma unroll
      for (int j = 0; j < NS; j++)
#pragma unroll
        for (int q = 0; q < K; q++) {
          v[j][q] = V(0);
          c[j][q] = 0;
          if (k0 + q < wd[j]) {
            const int64_t e = o[j] + 32 * (k0 + q) + lane;
            v[j][q] = ld_stream(vals + e, pol_s);
            c[j][q] = ld_stream(cols + e, pol_s);
          }
        }
      Acc xv[NS][K];
#pragma unroll
      for (int j = 0; j < NS; j++)
#pragma unroll
        for (int q = 0; q < K; q++)
          xv[j][q] = k0 + q < wd[j] ? warpk::ld_x(x + c[j][q], pol_x) : Acc(0);
#pragma unroll
      for (int j = 0; j < NS; j++)
#pragma unroll
        for (int q = 0; q < K; q++)
          if (k0 + q < wd[j])
            acc[j] += (Acc)v[j][q] * xv[j][q];
    }
#pragma unroll
    for (int j = 0; j < NS; j++) {
      const int64_t row = (sl + j) * 32 + lane;
      if (sl + j < b && row < m) {
        y[row] = acc[j];
        if (RESID) {
          if (ra.dot) {
            r2 += (double)acc[j] * (double)bvec[row];
          } else {
            const double dd = (double)acc[j] - (double)bvec[row];
            r2 += dd * dd;
          }
        }
      }
    }
  }
  if (!RESID)
    return;
  // Per-CTA partial in a fixed order, then the last CTA (ticket) adds the
  // partials in CTA order.
  const double t = warpk::wsum(r2);
  if (lane == 0)
    s_red[warp] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    double cta = 0.0;
    for (int i = 0; i < kSellWarps; i++)
      cta += s_red[i];
    ra.partials[blockIdx.x] = cta;
    __threadfence();
    s_last = atomicAdd(ra.ticket, 1) == (int)gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last)
    return;
  __threadfence();
  double sum = 0.0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += kSellNT)
    sum += __ldcg(&ra.partials[i]);
  sum = warpk::wsum(sum);
  __syncthreads();
  if (lane == 0)
    s_red[warp] = sum;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0.0;
    for (int i = 0; i < kSellWarps; i++)
      tot += s_red[i];
    *ra.out = tot;
    *ra.ticket = 0;
  }
}

template <class V, bool RESID, int NS, int K> int sell_grid(int dev) {
  static int cache[64] = {0};
  int &g = cache[dev < 64 ? dev : 0];
  if (g == 0) {
    int occ = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, sell_spmv<V, RESID, NS, K>, kSellNT, 0) !=
            cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      return 148;
    g = std::max(1, occ) * sms;
  }
  return g;
}

template <class V, int NS, int K>
drb_status sell_run(Csr &A, const void *x, void *y, const WarpResid *ra, int64_t s0,
                    int64_t s1, cudaStream_t s) {
  using Acc = typename AccOf<V>::type;
  const Sell &S = A.sell;
  const int64_t need = (s1 - s0 + kSellWarps * NS - 1) / (kSellWarps * NS);
  WarpResid r{};
  if (ra) {
    r = *ra;
    const int g = (int)std::min<int64_t>(sell_grid<V, true, NS, K>(A.device), need);
    sell_spmv<V, true, NS, K><<<g, kSellNT, 0, s>>>(S.vals.as<V>(), S.cols.as<int>(),
                                                   S.off.as<int64_t>(), s0, s1, A.m,
                                                   static_cast<const V *>(x),
                                                   static_cast<Acc *>(y), r);
  } else {
    const int g = (int)std::min<int64_t>(sell_grid<V, false, NS, K>(A.device), need);
    sell_spmv<V, false, NS, K><<<g, kSellNT, 0, s>>>(S.vals.as<V>(), S.cols.as<int>(),
                                                    S.off.as<int64_t>(), s0, s1, A.m,
                                                    static_cast<const V *>(x),
                                                    static_cast<Acc *>(y), r);
  }
  note_launch();
  DRB_CUDA_TRY(cudaGetLastError());
  return DRB_OK;
}

// Slices per warp step and row elements per load step, per element type:
// measured on the 2048^2 Laplacian, f64 is best with one slice of 8 (56 us;
// two slices 58-87 us: the extra registers cost occupancy), f32 with two
// slices of 6 (39.5 us against 42 us for one of 8).
template <class V>
drb_status sell_typed(Csr &A, const void *x, void *y, const WarpResid *ra, int64_t s0,
                      int64_t s1, cudaStream_t s) {
  if (s1 <= s0)
    return DRB_OK;
  if constexpr (sizeof(V) == 4)
    return sell_run<V, 2, 6>(A, x, y, ra, s0, s1, s);
  else
    return sell_run<V, 1, 8>(A, x, y, ra, s0, s1, s);
}

template <class V, class RI>
drb_status pack_typed(Csr &A, bool cols_too, cudaStream_t s) {
  const int64_t rows = A.sell.nslices * 32;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(148 * 8, (rows + 255) / 256));
  sell_pack<V, RI><<<grid, 256, 0, s>>>(A.m, rows, A.rowptr.as<RI>(), A.colind.as<int>(),
                                        A.vals.as<V>(), A.sell.off.as<int64_t>(),
                                        A.sell.vals.as<V>(), A.sell.cols.as<int>(), cols_too);
  note_launch();
  DRB_CUDA_TRY(cudaGetLastError());
  return DRB_OK;
}

drb_status pack(Csr &A, bool cols_too, cudaStream_t s) {
  const bool r8 = A.rbytes == 8;
  if (A.storage == DRB_F32)
    return r8 ? pack_typed<float, int64_t>(A, cols_too, s)
              : pack_typed<float, int32_t>(A, cols_too, s);
  return r8 ? pack_typed<double, int64_t>(A, cols_too, s)
            : pack_typed<double, int32_t>(A, cols_too, s);
}

} // namespace

void sell_release(Csr &A) {
  A.sell.vals.release();
  A.sell.cols.release();
  A.sell.off.release();
  A.sell.built = A.sell.on = false;
  A.sell.nslices = A.sell.padded = 0;
  A.sell.off_h.clear();
  A.sell.seg_s0.clear();
}

drb_status sell_build(Csr &A, const void *rowptr_host, int rbytes, cudaStream_t s) {
  sell_release(A);
  if ((A.storage != DRB_F32 && A.storage != DRB_F64) || A.cbytes != 4 ||
      (A.flags & DRB_FLAG_COMPENSATED) || A.m == 0 || A.nnz == 0)
    return DRB_OK;
  auto RP = [&](int64_t i) -> int64_t {
    return rbytes == 4 ? (int64_t)((const int32_t *)rowptr_host)[i]
                       : ((const int64_t *)rowptr_host)[i];
  };
  const int64_t nsl = (A.m + 31) / 32;
  std::vector<int64_t> off((size_t)nsl + 1, 0);
  int maxw = 0;
  for (int64_t sl = 0; sl < nsl; sl++) {
    int64_t w = 0;
    const int64_t r1 = std::min(A.m, (sl + 1) * 32);
    for (int64_t r = sl * 32; r < r1; r++)
      w = std::max(w, RP(r + 1) - RP(r));
    if (w > kSellMaxWidth)
      return DRB_OK; // a long row: the row-block kernel's case
    maxw = std::max(maxw, (int)w);
    off[sl + 1] = off[sl] + 32 * w;
  }
  const int64_t padded = off[nsl];
  if ((double)padded > kSellMaxPad * (double)A.nnz)
    return DRB_OK;
  const size_t vb = (size_t)dtype_bytes(A.storage);
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess ||
      (double)free_b < 2.0 * (double)padded * (double)(vb + 4))
    return DRB_OK; // keep the memory for the caller
  DRB_TRY(A.sell.off.alloc(sizeof(int64_t) * off.size()));
  DRB_TRY(A.sell.vals.alloc(vb * (size_t)std::max<int64_t>(padded, 1)));
  DRB_TRY(A.sell.cols.alloc(sizeof(int) * (size_t)std::max<int64_t>(padded, 1)));
  DRB_CUDA_TRY(cudaMemcpyAsync(A.sell.off.p, off.data(), sizeof(int64_t) * off.size(),
                               cudaMemcpyHostToDevice, s));
  DRB_CUDA_TRY(cudaStreamSynchronize(s)); // off is moved below
  A.sell.nslices = nsl;
  A.sell.padded = padded;
  A.sell.off_h = std::move(off);
  A.sell.maxw = maxw;
  A.sell.built = true;
  DRB_TRY(pack(A, true, s));
  DRB_CUDA_TRY(cudaStreamSynchronize(s));
  // used by default; DRB_SPMV_VARIANT naming a row-block variant keeps it off
  const char *e = std::getenv("DRB_SPMV_VARIANT");
  A.sell.on = !(e && std::strcmp(e, "sell") != 0);
  return DRB_OK;
}

drb_status sell_pack_values(Csr &A, cudaStream_t s) {
  if (!A.sell.built)
    return DRB_OK;
  return pack(A, false, s);
}

drb_status sell_launch(Csr &A, const void *x, void *y, const warpk::WarpResid *ra,
                       int64_t s0, int64_t s1, cudaStream_t s) {
  if (A.storage == DRB_F32)
    return sell_typed<float>(A, x, y, ra, s0, s1, s);
  if (A.storage == DRB_F64)
    return sell_typed<double>(A, x, y, ra, s0, s1, s);
  set_error("sliced-ELL SpMV: storage type not handled");
  return DRB_ERR_UNSUPPORTED;
}

} // namespace drb
