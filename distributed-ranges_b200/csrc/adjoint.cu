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
// abar walks the forward plan's row blocks so each entry's row is known
// without an expanded row-index array.
#include <cub/device/device_radix_sort.cuh>

#include <memory>
#include <vector>

#include "drb_internal.cuh"

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

constexpr int kAbarNT = 256;
constexpr int kAbarSpan = 2048; // nonzeros of a row-block tile (the plan's tile)

// abar[p] = ybar[row(p)] * x[col(p)], one CTA per forward row block.
template <class V, class CI, class RI>
__global__ void __launch_bounds__(kAbarNT)
    abar_kernel(const RI *__restrict__ rowptr, const CI *__restrict__ colind,
                const V *__restrict__ ybar, const V *__restrict__ x,
                V *__restrict__ abar, const int2 *__restrict__ blocks,
                const Chunk *__restrict__ chunks) {
  __shared__ int64_t s_rp[kAbarSpan + 1];
  __shared__ uint16_t s_row[kAbarSpan]; // row (within the block) of each nonzero
  __shared__ unsigned s_wmax[kAbarNT / 32];
  const int2 blk = blocks[blockIdx.x];
  const uint64_t pol_x = ptx::policy_evict_last();
  if (blk.y > 0) {
    // a tile of whole rows: rows stamp their nonzeros' row ids into shared
    // memory, then all threads stream the nonzeros coalesced
    const int r0 = blk.x, nrows = blk.y - blk.x;
    for (int i = threadIdx.x; i <= nrows; i += kAbarNT)
      s_rp[i] = (int64_t)rowptr[r0 + i];
    __syncthreads();
    const int64_t p0 = s_rp[0], p1 = s_rp[nrows];
    const bool stamped = p1 - p0 <= kAbarSpan && nrows <= 65536;
    if (stamped) {
      // Every row writes its id at its first nonzero, then a block-wide
      // running-max scan (row ids only grow along the nonzeros) gives every
      // nonzero its row: 8 entries per thread whatever the row lengths
      // (writing each row's ids by one thread serialised long rows).
      constexpr int PER = kAbarSpan / kAbarNT;
      const int span = (int)(p1 - p0);
      for (int q = threadIdx.x; q < span; q += kAbarNT)
        s_row[q] = 0;
      __syncthreads();
      for (int i = threadIdx.x; i < nrows; i += kAbarNT)
        if (s_rp[i + 1] > s_rp[i])
          s_row[s_rp[i] - p0] = (uint16_t)i;
      __syncthreads();
      const int q0 = threadIdx.x * PER;
      unsigned v[PER];
      unsigned run = 0;
#pragma unroll
      for (int k = 0; k < PER; k++) {
        if (q0 + k < span)
          run = max(run, (unsigned)s_row[q0 + k]);
        v[k] = run;
      }
      // the running max of all threads before this one
      const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
      unsigned inc = run;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o)
          inc = max(inc, t);
      }
      if (lane == 31)
        s_wmax[wid] = inc;
      __syncthreads();
      unsigned before = __shfl_up_sync(0xffffffffu, inc, 1);
      if (lane == 0)
        before = 0;
      for (int w = 0; w < wid; w++)
        before = max(before, s_wmax[w]);
#pragma unroll
      for (int k = 0; k < PER; k++)
        if (q0 + k < span)
          s_row[q0 + k] = (uint16_t)max(v[k], before);
    }
    __syncthreads();
    if (stamped) {
      // all of this thread's nonzeros (at most kAbarSpan / kAbarNT) at once:
      // column loads, then x gathers, then the products
      constexpr int U = kAbarSpan / kAbarNT;
      CI col[U];
      V xv[U];
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int64_t p = p0 + threadIdx.x + (int64_t)u * kAbarNT;
        col[u] = p < p1 ? colind[p] : CI(0);
      }
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int64_t p = p0 + threadIdx.x + (int64_t)u * kAbarNT;
        xv[u] = p < p1 ? ptx::ld_keep(x + col[u], pol_x) : V(0);
      }
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int64_t p = p0 + threadIdx.x + (int64_t)u * kAbarNT;
        if (p < p1)
          abar[p] = ybar[r0 + s_row[p - p0]] * xv[u];
      }
      return;
    }
    for (int64_t p = p0 + threadIdx.x; p < p1; p += kAbarNT) {
      int lo = 0, hi = nrows; // last i with s_rp[i] <= p
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (s_rp[mid] <= p)
          lo = mid;
        else
          hi = mid;
      }
      abar[p] = ybar[r0 + lo] * ptx::ld_keep(x + colind[p], pol_x);
    }
    return;
  }
  int64_t row, lo, hi;
  if (blk.y == -1) {
    row = blk.x;
    lo = (int64_t)rowptr[row];
    hi = (int64_t)rowptr[row + 1];
  } else {
    const Chunk ch = chunks[-blk.y - 2];
    row = ch.row;
    lo = ch.p0;
    hi = ch.p1;
  }
  const V yb = ybar[row];
  for (int64_t p = lo + threadIdx.x; p < hi; p += kAbarNT)
    abar[p] = yb * ptx::ld_keep(x + colind[p], pol_x);
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

template <class V, class CI, class RI>
drb_status abar_typed(Csr &A, const V *ybar, const V *x, V *abar,
                      cudaStream_t s) {
  if (A.plan.nblocks == 0)
    return DRB_OK;
  abar_kernel<V, CI, RI><<<(unsigned)A.plan.nblocks, kAbarNT, 0, s>>>(
      A.rowptr.as<RI>(), A.colind.as<CI>(), ybar, x, abar,
      A.plan.blocks.as<int2>(), A.plan.chunks.as<Chunk>());
  note_launch();
  DRB_CUDA_TRY(cudaGetLastError());
  return DRB_OK;
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
