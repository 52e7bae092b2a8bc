// adjoint.cu -- gemv_backward: xbar = A^T ybar and abar = ybar_i * x_j on the
// sparsity pattern.  No reference counterpart (the reference has no adjoint).
//
// Plan (built once, DRB_FLAG_ADJOINT): a stable device radix sort of the
// column indices (CUB DeviceRadixSort on (col, nnz id) pairs) gives the CSC
// permutation perm[q] = CSR position of the q-th entry in column-major order.
// From it: colptr (column boundaries of the sorted keys), rowidx_t (the row of
// each entry) and vals_t (values in CSC order).  A^T is then an ordinary CSR
// matrix of shape n x m, so xbar uses the same row-block SpMV kernel as the
// forward product: no atomics, fixed summation order.
// abar needs each entry's row without an expanded row-index array: short
// rows (at most 64 nonzeros) find it by a warp-wide search over 32 row starts
// (abar_rows), longer rows run on the forward product's work items
// (abar_items).
#include <cub/device/device_radix_sort.cuh>

#include <memory>
#include <vector>

#include "spmv_warp.cuh"

namespace drb {

int plan_group(int vbytes, int cbytes);

namespace {

template <class RI>
__device__ __forceinline__ int64_t row_of(const RI *rowptr, int64_t m,
                                          int64_t p) {
  // upper_bound(rowptr[0..m], p) - 1
  int64_t lo = 0, hi = m + 1;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if ((int64_t)rowptr[mid] <= p)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo - 1;
}

template <class K, class RI>
__global__ void csc_boundaries(const K *__restrict__ keys, int64_t nnz,
                               int64_t n, RI *__restrict__ colptr) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p <= nnz;
       p += (int64_t)gridDim.x * blockDim.x) {
    const int64_t prev = p == 0 ? -1 : (int64_t)keys[p - 1];
    const int64_t cur = p == nnz ? n : (int64_t)keys[p];
    for (int64_t c = prev + 1; c <= cur; c++)
      colptr[c] = (RI)p;
  }
}

template <class PI, class RI, class CI>
__global__ void csc_rows(const PI *__restrict__ perm, const RI *__restrict__ rowptr,
                         int64_t m, int64_t nnz, CI *__restrict__ rowidx_t) {
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < nnz;
       q += (int64_t)gridDim.x * blockDim.x)
    rowidx_t[q] = (CI)row_of(rowptr, m, (int64_t)perm[q]);
}

template <class PI, class V>
__global__ void gather_vals(const PI *__restrict__ perm, const V *__restrict__ vals,
                            int64_t nnz, V *__restrict__ vals_t) {
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < nnz;
       q += (int64_t)gridDim.x * blockDim.x)
    vals_t[q] = vals[(int64_t)perm[q]];
}

template <class T>
__global__ void iota_kernel(T *out, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (T)i;
}

// abar on the forward product's work items (the persistent SpMV's plan),
// one item ahead: while an item's x gathers are in flight, the warp loads the
// next item's descriptor, column indices, row starts and ybar values.  The
// row of every position comes from stamps: each non-empty row writes its
// index (a byte; at most 64 rows an item) at its first position of a zeroed
// per-warp buffer, and a running max over positions -- row indices only grow
// along an item -- fills the rest: within a lane over its G positions, then
// across lanes by a warp max-scan, in registers.  ybar of the item's rows
// sits in shared memory, abar goes out with 16-byte streaming stores.  Pure
// element-wise products: no sums, no order to keep.  (The previous form --
// no look-ahead, the row scan through shared memory and ybar loaded per
// element -- took 1.76 ms on a 16.8M-row power-law matrix with 336M
// nonzeros, against 1.25 ms for streaming the column indices and values and
// gathering x alone.)
constexpr int kAbWarps = 8;

template <class V, class CI, int TILE> struct AbSlot {
  static constexpr int G = 16 / (sizeof(V) < sizeof(CI) ? sizeof(V) : sizeof(CI));
  static constexpr int NG = TILE / (G * 32);
  CI c[NG][G];
  Item d;
  int64_t a0;
  int rp0, rp1, rp2; // rowptr[r0 + lane], [r0 + lane + 32], [r0 + 64], relative to a0
  V y0, y1;          // ybar[r0 + lane], ybar[r0 + lane + 32] (a chunk: ybar[r0])
  bool valid;
};

template <class V, class CI, class RI, int TILE>
__global__ void __launch_bounds__(kAbWarps * 32)
    abar_items(const RI *__restrict__ rowptr, const CI *__restrict__ colind,
               const V *__restrict__ ybar, const V *__restrict__ x, V *__restrict__ abar,
               const Item *__restrict__ items, int64_t nitems, unsigned *counter, bool vec) {
  using S = AbSlot<V, CI, TILE>;
  constexpr int G = S::G, NG = S::NG;
  constexpr int VPER = 16 / sizeof(V);
  static_assert(G == 2 || G == 4, "abar_items: 2 or 4 positions per group");
  static_assert(TILE % 128 == 0, "abar_items: TILE a multiple of 128");
  __shared__ __align__(16) uint8_t s_row[kAbWarps][TILE];
  __shared__ V s_y[kAbWarps][warpk::kRows];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint8_t *srow = s_row[warp];
  V *sy = s_y[warp];
  const uint64_t pol_s = ptx::policy_evict_first();
  const uint64_t pol_x = ptx::policy_evict_last();
  constexpr unsigned kFull = 0xffffffffu;
  constexpr int kBatch = 8;
  int64_t base = 0;
  int k = 0;
  auto grab = [&]() -> int64_t {
    unsigned v = 0;
    if (lane == 0)
      v = atomicAdd(counter, (unsigned)kBatch);
    return (int64_t)__shfl_sync(kFull, v, 0);
  };
  auto advance = [&]() -> int64_t {
    if (++k == kBatch) {
      base = grab();
      k = 0;
    }
    return base + k;
  };
  auto fetch = [&](S &sl, int64_t i) {
    sl.valid = i < nitems;
    if (!sl.valid)
      return;
    sl.d = warpk::load_item(items, i);
    sl.a0 = sl.d.p0 & ~(int64_t)(G - 1);
    const int ng = (int)((sl.d.p0 + sl.d.len - sl.a0 + G - 1) / G);
#pragma unroll
    for (int j = 0; j < NG; j++) {
      const int g = lane + 32 * j;
      if (g < ng)
        warpk::ld_group<CI, G>(colind + sl.a0 + (int64_t)g * G, sl.c[j], pol_s);
    }
    const int64_t r0 = sl.d.r0;
    const int nr = sl.d.nrows;
    sl.rp0 = sl.rp1 = sl.rp2 = 0;
    if (nr > 0) {
      if (lane <= nr)
        sl.rp0 = (int)((int64_t)rowptr[r0 + lane] - sl.a0);
      if (lane + 32 <= nr)
        sl.rp1 = (int)((int64_t)rowptr[r0 + lane + 32] - sl.a0);
      if (lane == 0 && 64 <= nr)
        sl.rp2 = (int)((int64_t)rowptr[r0 + 64] - sl.a0);
      sl.y0 = lane < nr ? ybar[r0 + lane] : V(0);
      sl.y1 = lane + 32 < nr ? ybar[r0 + lane + 32] : V(0);
    } else {
      sl.y0 = ybar[r0]; // one chunk of a long row
      sl.y1 = V(0);
    }
  };
  // gathers of x for the item in sl (zeros outside it)
  auto gather = [&](const S &sl, V (&xv)[NG][G]) {
    const int off = (int)(sl.d.p0 - sl.a0), end = off + sl.d.len;
#pragma unroll
    for (int j = 0; j < NG; j++) {
      const int g = lane + 32 * j;
#pragma unroll
      for (int i = 0; i < G; i++) {
        const int q = g * G + i;
        xv[j][i] = (q >= off && q < end) ? ptx::ld_keep(x + sl.c[j][i], pol_x) : V(0);
      }
    }
  };
  // abar of the item in cur, whose x values are in xv (the next item's loads
  // were issued just before)
  auto step = [&](const S &cur, V (&xv)[NG][G]) {
    const int off = (int)(cur.d.p0 - cur.a0), end = off + cur.d.len;
    const int nr = cur.d.nrows;
    if (nr > 0) {
#pragma unroll
      for (int w = lane; w < TILE / 4; w += 32)
        reinterpret_cast<uint32_t *>(srow)[w] = 0u;
      // next row's start for the lane's rows r = lane and r = lane + 32
      const int rp32 = __shfl_sync(kFull, cur.rp1, 0);
      const int rp64 = __shfl_sync(kFull, cur.rp2, 0);
      int nx0 = __shfl_down_sync(kFull, cur.rp0, 1);
      int nx1 = __shfl_down_sync(kFull, cur.rp1, 1);
      if (lane == 31) {
        nx0 = rp32;
        nx1 = rp64;
      }
      __syncwarp();
      if (lane < nr && nx0 > cur.rp0)
        srow[cur.rp0] = (uint8_t)lane;
      if (lane + 32 < nr && nx1 > cur.rp1)
        srow[cur.rp1] = (uint8_t)(lane + 32);
      if (lane < nr)
        sy[lane] = cur.y0;
      if (lane + 32 < nr)
        sy[lane + 32] = cur.y1;
    }
    __syncwarp();
    int carry = 0; // row of the last position of the previous group
#pragma unroll
    for (int j = 0; j < NG; j++) {
      const int g = lane + 32 * j, q0 = g * G;
      int row[G];
      if (nr > 0) {
        uint32_t w;
        if (G == 4)
          w = *reinterpret_cast<const uint32_t *>(srow + q0);
        else
          w = *reinterpret_cast<const uint16_t *>(srow + q0);
        int run = 0;
#pragma unroll
        for (int i = 0; i < G; i++) {
          run = max(run, (int)((w >> (8 * i)) & 0xffu));
          row[i] = run;
        }
        int inc = run;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int u = __shfl_up_sync(kFull, inc, o);
          if (lane >= o)
            inc = max(inc, u);
        }
        int before = __shfl_up_sync(kFull, inc, 1);
        before = lane == 0 ? carry : max(before, carry);
        carry = max(carry, __shfl_sync(kFull, inc, 31));
#pragma unroll
        for (int i = 0; i < G; i++)
          row[i] = max(row[i], before);
      }
      V out[G];
#pragma unroll
      for (int i = 0; i < G; i++) {
        const int q = q0 + i;
        const V yr = nr > 0 ? sy[row[i]] : cur.y0;
        out[i] = (q >= off && q < end) ? yr * xv[j][i] : V(0);
      }
      V *dst = abar + cur.a0 + q0;
      if (vec && q0 >= off && q0 + G <= end) {
#pragma unroll
        for (int h = 0; h < G / VPER; h++) {
          warpk::Vec16<V> wv;
#pragma unroll
          for (int i = 0; i < VPER; i++)
            wv.t[i] = out[h * VPER + i];
          __stcs(reinterpret_cast<uint4 *>(dst + h * VPER), wv.u);
        }
      } else {
#pragma unroll
        for (int i = 0; i < G; i++)
          if (q0 + i >= off && q0 + i < end)
            __stcs(dst + i, out[i]);
      }
    }
    __syncwarp(); // the stamps and ybar of the next item overwrite these
  };
  base = grab();
  S A, B;
  V xv[NG][G];
  fetch(A, base);
  while (A.valid) {
    gather(A, xv);
    fetch(B, advance());
    step(A, xv);
    if (!B.valid)
      break;
    gather(B, xv);
    fetch(A, advance());
    step(B, xv);
  }
}

unsigned grid1(int64_t n) {
  int64_t g = (n + 255) / 256;
  if (g > 148 * 16)
    g = 148 * 16;
  return (unsigned)(g < 1 ? 1 : g);
}

template <class K, class PI>
drb_status sort_columns(const K *keys_in, int64_t nnz, int64_t n, K *keys_out,
                        PI *perm, cudaStream_t s) {
  DevBuf ids;
  DRB_TRY(ids.alloc(sizeof(PI) * std::max<int64_t>(nnz, 1)));
  iota_kernel<PI><<<grid1(nnz), 256, 0, s>>>(ids.as<PI>(), nnz);
  note_launch();
  int bits = 1;
  while (bits < 63 && ((int64_t)1 << bits) < n)
    bits++;
  size_t tmp_bytes = 0;
  DRB_CUDA_TRY(cub::DeviceRadixSort::SortPairs(
      nullptr, tmp_bytes, keys_in, keys_out, ids.as<PI>(), perm, nnz, 0, bits,
      s));
  DevBuf tmp;
  DRB_TRY(tmp.alloc(std::max<size_t>(tmp_bytes, 16)));
  DRB_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp.p, tmp_bytes, keys_in,
                                               keys_out, ids.as<PI>(), perm,
                                               nnz, 0, bits, s));
  note_launch();
  DRB_CUDA_TRY(cudaStreamSynchronize(s));
  ids.release();
  tmp.release();
  return DRB_OK;
}

template <class V, class CI, class RI>
drb_status build_typed(Csr &A, cudaStream_t s) {
  // A^T stored as a CSR handle of shape n x m sharing the index widths.
  auto &T = *A.tr;
  T.device = A.device;
  T.m = A.n;
  T.n = A.m;
  T.nnz = A.nnz;
  T.value_type = A.value_type;
  T.storage = A.storage;
  T.cbytes = A.cbytes;
  T.rbytes = A.rbytes;
  const int64_t nnz = A.nnz, pad = ((nnz + kPadElems - 1) / kPadElems + 1) * kPadElems;
  DRB_TRY(T.rowptr.alloc(sizeof(RI) * (A.n + 1 + kRowptrPad)));
  DRB_CUDA_TRY(cudaMemsetAsync(T.rowptr.p, 0, T.rowptr.bytes, s));
  DRB_TRY(T.colind.alloc(sizeof(CI) * pad));
  DRB_TRY(T.vals.alloc(sizeof(V) * pad));
  DRB_CUDA_TRY(cudaMemsetAsync(T.colind.p, 0, T.colind.bytes, s));
  DRB_CUDA_TRY(cudaMemsetAsync(T.vals.p, 0, T.vals.bytes, s));
  DRB_TRY(A.perm.alloc(sizeof(int64_t) * std::max<int64_t>(nnz, 1)));
  DevBuf keys_out;
  DRB_TRY(keys_out.alloc(sizeof(CI) * std::max<int64_t>(nnz, 1)));
  const bool perm32 = nnz < 0x7fffffff;
  if (nnz > 0) {
    if (perm32)
      DRB_TRY(sort_columns<CI, int32_t>(A.colind.as<CI>(), nnz, A.n,
                                        keys_out.as<CI>(), A.perm.as<int32_t>(),
                                        s));
    else
      DRB_TRY(sort_columns<CI, int64_t>(A.colind.as<CI>(), nnz, A.n,
                                        keys_out.as<CI>(), A.perm.as<int64_t>(),
                                        s));
  }
  A.perm_bytes = perm32 ? 4 : 8;
  csc_boundaries<CI, RI><<<grid1(nnz + 1), 256, 0, s>>>(
      keys_out.as<CI>(), nnz, A.n, T.rowptr.as<RI>());
  note_launch();
  if (nnz > 0) {
    if (perm32) {
      csc_rows<int32_t, RI, CI><<<grid1(nnz), 256, 0, s>>>(
          A.perm.as<int32_t>(), A.rowptr.as<RI>(), A.m, nnz, T.colind.as<CI>());
    } else {
      csc_rows<int64_t, RI, CI><<<grid1(nnz), 256, 0, s>>>(
          A.perm.as<int64_t>(), A.rowptr.as<RI>(), A.m, nnz, T.colind.as<CI>());
    }
    note_launch();
  }
  DRB_CUDA_TRY(cudaGetLastError());
  DRB_TRY(adjoint_refresh_values(A, s));
  std::vector<char> cp((size_t)sizeof(RI) * (A.n + 1));
  DRB_CUDA_TRY(cudaMemcpyAsync(cp.data(), T.rowptr.p, cp.size(),
                               cudaMemcpyDeviceToHost, s));
  DRB_CUDA_TRY(cudaStreamSynchronize(s));
  keys_out.release();
  DRB_TRY(build_plan(T.plan, T.m, cp.data(), sizeof(RI),
                     plan_group(dtype_bytes(T.storage), T.cbytes), 0, 0, 0));
  DRB_TRY(build_pipe_plan(T.pipe, T.m, cp.data(), sizeof(RI),
                          plan_group(dtype_bytes(T.storage), T.cbytes), 0, 0));
  // A^T of a short-row matrix (a stencil) has short rows too: x-bar then
  // runs on its sliced-ELL copy, as the forward product does
  DRB_TRY(sell_build(T, cp.data(), sizeof(RI), s));
  return DRB_OK;
}

template <class V>
drb_status build_v(Csr &A, cudaStream_t s) {
  if (A.cbytes == 4 && A.rbytes == 4)
    return build_typed<V, int32_t, int32_t>(A, s);
  if (A.cbytes == 4 && A.rbytes == 8)
    return build_typed<V, int32_t, int64_t>(A, s);
  if (A.cbytes == 8 && A.rbytes == 4)
    return build_typed<V, int64_t, int32_t>(A, s);
  return build_typed<V, int64_t, int64_t>(A, s);
}

// Abar for short rows (at most kAbRowsMaxLen nonzeros): a warp takes 32
// consecutive rows; lane l holds rowptr[r0 + l] (relative to the group's
// first nonzero) and ybar[r0 + l].  The warp walks the group's nonzeros 32
// at a time: each lane loads its position's column (coalesced), gathers x,
// finds the position's row by a 5-step binary search over the lanes' row
// starts (shuffles) and takes that row's ybar with one more shuffle, then
// stores abar (coalesced).  No shared memory and no per-item bookkeeping, so
// rows of a handful of nonzeros (a stencil) stream at close to HBM speed.
constexpr int kAbRowsNT = 256;
constexpr int kAbRowsMaxLen = 64; // a group spans at most 32 * 64 nonzeros

template <class V, class CI, class RI>
__global__ void __launch_bounds__(kAbRowsNT)
    abar_rows(int64_t m, const RI *__restrict__ rowptr, const CI *__restrict__ colind,
              const V *__restrict__ ybar, const V *__restrict__ x, V *__restrict__ abar) {
  // U positions per lane per trip with all loads first; the last partial
  // trip goes 32 positions at a time (a masked U-wide trip measured slower:
  // 2048^2 Laplacian FP32 0.064 against 0.0485 ms)
  constexpr int U = 4;
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * kAbRowsNT) >> 5;
  const uint64_t pol_x = ptx::policy_evict_last();
  for (int64_t r0 = (((int64_t)blockIdx.x * kAbRowsNT + threadIdx.x) >> 5) * 32; r0 < m;
       r0 += nw * 32) {
    const int64_t r = r0 + lane;
    const int64_t pbeg = (int64_t)rowptr[r0];
    const int64_t pend = (int64_t)rowptr[r0 + 32 < m ? r0 + 32 : m];
    // rows past m start at the group's end: never selected
    const int rs = (int)((int64_t)rowptr[r < m ? r : m] - pbeg);
    const V yb = r < m ? ybar[r] : V(0);
    const int len = (int)(pend - pbeg);
    auto row_lane = [&](int q) {
      int lo = 0;
#pragma unroll
      for (int step = 16; step > 0; step >>= 1) {
        const int v = __shfl_sync(0xffffffffu, rs, lo + step);
        if (v <= q)
          lo += step;
      }
      return lo;
    };
    int q0 = 0;
    for (; q0 + 32 * U <= len; q0 += 32 * U) {
      CI c[U];
      V xv[U];
#pragma unroll
      for (int u = 0; u < U; u++)
        c[u] = __ldcs(colind + pbeg + q0 + lane + 32 * u);
#pragma unroll
      for (int u = 0; u < U; u++)
        xv[u] = ptx::ld_keep(x + c[u], pol_x);
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int q = q0 + lane + 32 * u;
        const V yr = __shfl_sync(0xffffffffu, yb, row_lane(q));
        __stcs(abar + pbeg + q, yr * xv[u]);
      }
    }
    for (; q0 < len; q0 += 32) {
      const int q = q0 + lane;
      const bool in = q < len;
      const CI c = in ? __ldcs(colind + pbeg + q) : CI(0);
      const V xv = in ? ptx::ld_keep(x + c, pol_x) : V(0);
      const V yr = __shfl_sync(0xffffffffu, yb, row_lane(q));
      if (in)
        __stcs(abar + pbeg + q, yr * xv);
    }
  }
}

template <class V, class CI, class RI>
drb_status abar_rows_launch(Csr &A, const V *ybar, const V *x, V *abar, cudaStream_t s) {
  static int grid_cache[64] = {0};
  int &grid = grid_cache[A.device < 64 ? A.device : 0];
  if (grid == 0) {
    int occ = 0, sms = 0;
    DRB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &occ, abar_rows<V, CI, RI>, kAbRowsNT, 0));
    DRB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, A.device));
    grid = std::max(1, occ) * sms;
  }
  const int64_t groups = (A.m + 31) / 32;
  const int g = (int)std::max<int64_t>(
      1, std::min<int64_t>(grid, (groups + kAbRowsNT / 32 - 1) / (kAbRowsNT / 32)));
  abar_rows<V, CI, RI><<<g, kAbRowsNT, 0, s>>>(A.m, A.rowptr.as<RI>(), A.colind.as<CI>(),
                                               ybar, x, abar);
  note_launch();
  DRB_CUDA_TRY(cudaGetLastError());
  return DRB_OK;
}

// Rows short enough for abar_rows (2048-entry 32-row groups at most, so a
// static share of groups stays balanced).  Longer rows use the forward
// product's work items (a 16.8M-row power-law matrix with rows up to 16384:
// 1.73 ms on the items, 2.02 ms on 32-row groups).
bool abar_short_rows(const Csr &A) { return A.max_row <= kAbRowsMaxLen; }

template <class V, class CI, class RI, int TILE>
drb_status abar_tile(Csr &A, const V *ybar, const V *x, V *abar, cudaStream_t s) {
  static int grid_cache[64] = {0};
  int &grid = grid_cache[A.device < 64 ? A.device : 0];
  if (grid == 0) {
    int occ = 0, sms = 0;
    DRB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &occ, abar_items<V, CI, RI, TILE>, kAbWarps * 32, 0));
    DRB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, A.device));
    grid = std::max(1, occ) * sms;
  }
  const PipePlan &P = A.pipe;
  const int g = (int)std::min<int64_t>(grid, (P.nitems + kAbWarps - 1) / kAbWarps);
  const bool vec = reinterpret_cast<uintptr_t>(abar) % 16 == 0;
  DRB_CUDA_TRY(cudaMemsetAsync(P.counters.p, 0, sizeof(unsigned), s)); // work counter
  abar_items<V, CI, RI, TILE><<<g, kAbWarps * 32, 0, s>>>(
      A.rowptr.as<RI>(), A.colind.as<CI>(), ybar, x, abar, P.items.as<Item>(), P.nitems,
      P.counters.as<unsigned>(), vec);
  note_launch();
  DRB_CUDA_TRY(cudaGetLastError());
  return DRB_OK;
}

template <class V, class CI, class RI>
drb_status abar_typed(Csr &A, const V *ybar, const V *x, V *abar,
                      cudaStream_t s) {
  if (A.nnz == 0)
    return DRB_OK;
  if (abar_short_rows(A))
    return abar_rows_launch<V, CI, RI>(A, ybar, x, abar, s);
  if (A.pipe.nitems == 0)
    return DRB_OK;
  if (A.pipe.tile == 512)
    return abar_tile<V, CI, RI, 512>(A, ybar, x, abar, s);
  if constexpr (AbSlot<V, CI, 256>::G * 32 <= 128) {
    if (A.pipe.tile == 128)
      return abar_tile<V, CI, RI, 128>(A, ybar, x, abar, s);
  }
  return abar_tile<V, CI, RI, 256>(A, ybar, x, abar, s);
}

template <class V>
drb_status abar_v(Csr &A, const void *ybar, const void *x, void *abar,
                  cudaStream_t s) {
  auto yb = (const V *)ybar;
  auto xx = (const V *)x;
  auto ab = (V *)abar;
  if (A.cbytes == 4 && A.rbytes == 4)
    return abar_typed<V, int32_t, int32_t>(A, yb, xx, ab, s);
  if (A.cbytes == 4 && A.rbytes == 8)
    return abar_typed<V, int32_t, int64_t>(A, yb, xx, ab, s);
  if (A.cbytes == 8 && A.rbytes == 4)
    return abar_typed<V, int64_t, int32_t>(A, yb, xx, ab, s);
  return abar_typed<V, int64_t, int64_t>(A, yb, xx, ab, s);
}

} // namespace

drb_status adjoint_build(Csr &A, cudaStream_t s) {
  A.tr = std::make_unique<Csr>();
  drb_status st;
  if (A.storage == DRB_F32)
    st = build_v<float>(A, s);
  else if (A.storage == DRB_F64)
    st = build_v<double>(A, s);
  else {
    set_error("adjoint: storage type not supported");
    st = DRB_ERR_UNSUPPORTED;
  }
  if (st != DRB_OK) {
    A.tr.reset();
    return st;
  }
  A.has_adjoint = true;
  return DRB_OK;
}

drb_status adjoint_refresh_values(Csr &A, cudaStream_t s) {
  if (!A.tr)
    return DRB_OK;
  const int64_t nnz = A.nnz;
  if (nnz == 0)
    return DRB_OK;
  if (A.storage == DRB_F32) {
    if (A.perm_bytes == 4)
      gather_vals<int32_t, float><<<grid1(nnz), 256, 0, s>>>(
          A.perm.as<int32_t>(), A.vals.as<float>(), nnz, A.tr->vals.as<float>());
    else
      gather_vals<int64_t, float><<<grid1(nnz), 256, 0, s>>>(
          A.perm.as<int64_t>(), A.vals.as<float>(), nnz, A.tr->vals.as<float>());
  } else {
    if (A.perm_bytes == 4)
      gather_vals<int32_t, double><<<grid1(nnz), 256, 0, s>>>(
          A.perm.as<int32_t>(), A.vals.as<double>(), nnz,
          A.tr->vals.as<double>());
    else
      gather_vals<int64_t, double><<<grid1(nnz), 256, 0, s>>>(
          A.perm.as<int64_t>(), A.vals.as<double>(), nnz,
          A.tr->vals.as<double>());
  }
  note_launch();
  DRB_CUDA_TRY(cudaGetLastError());
  return sell_pack_values(*A.tr, s);
}

drb_status spmv_t_launch(Csr &A, const void *ybar, void *xbar, cudaStream_t s) {
  return spmv_launch(*A.tr, ybar, xbar, 1, DRB_COL_MAJOR, s);
}

drb_status abar_launch(Csr &A, const void *ybar, const void *x, void *abar,
                       cudaStream_t s) {
  if (A.storage == DRB_F32)
    return abar_v<float>(A, ybar, x, abar, s);
  if (A.storage == DRB_F64)
    return abar_v<double>(A, ybar, x, abar, s);
  set_error("abar: storage type not supported");
  return DRB_ERR_UNSUPPORTED;
}

} // namespace drb
