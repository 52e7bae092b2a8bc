// colsplit.cu -- column-blocked plan of the single-RHS SpMV, for matrices
// whose x does not stay in L2.
//
// A randomly gathered x stays L2-resident on B200 only up to about 48 MB
// while the matrix streams past it: on a 16.8M-row power-law pattern (336M
// nonzeros, uniform columns) the SpMV takes the same time for an x of 8 to
// 48 MB (FP32 1.39-1.40 ms, FP64 1.68 ms) and degrades beyond it (FP32 1.53 ms
// at 64 MB; FP64 2.03 / 2.91 / 3.69 ms at 64 / 96 / 128 MB).
//
// So when x is larger than kSplitAbove, the handle keeps a second copy of its
// nonzeros grouped by column block, as one "virtual" CSR matrix: its row
// b*(m+1) + r holds the nonzeros of row r whose columns lie in block b
// ([c_b, c_{b+1}), columns kept global, each row's order kept), and its
// rows b*(m+1) + m are empty separators.  The unchanged persistent SpMV runs
// over it in ONE launch into a block-major scratch y; its work counter hands
// out items in order, so at any time nearly all warps work inside one block
// and only that block's slice of x is hot in L2.  A last small pass adds the
// blocks' row sums into y in block order (deterministic).  The scratch costs
// nblk * (m + 1) partial sums, written once and read once.  Measured on that
// pattern: FP32 (x = 64 MB) 1.470 ms in two blocks against 1.525 ms unsplit,
// FP64 (x = 128 MB) 1.90 ms in three blocks against 3.57 ms.
//
// The regrouping runs on the device at plan time: a warp per row counts its
// nonzeros per block with ballots, a scan per block gives the blocks' row
// starts (offset by the blocks before them), and a second warp-per-row pass
// scatters the nonzeros (a ballot per block gives each lane its place), so
// rows need not be sorted.
//
// The host-pointer gemv (colsplit_gemv_host) pipelines over the blocks: x
// goes up slice by slice on a copy stream, each block's items start as soon
// as its slice is on the device, and the last block runs in row segments
// whose combined rows copy back while the next segments compute -- so most of
// the SpMV hides behind x's upload and most of y's download behind the last
// block.  The segments run the same items, chunk sums and combine as the one
// launch: y is bit-identical to the device-pointer call.
#include <algorithm>
#include <cstdlib>
#include <vector>

#include <cub/cub.cuh>

#include "drb_internal.cuh"

namespace drb {
namespace {

constexpr int kMaxBlocks = 8;
constexpr int64_t kSplitAbove = 48ll << 20; // split when x is larger than this
constexpr int64_t kSplitBlock = 48ll << 20; // and give each block at most this

struct BlockOffsets {
  int64_t off[kMaxBlocks]; // first nonzero of each block in the regrouped arrays
};

// First column of each block (c[0] = 0); blocks past nblk unused.
struct Bounds {
  int64_t c[kMaxBlocks];
  int nblk;
};

__device__ __forceinline__ int block_of(int64_t col, const Bounds &B) {
  int b = 0;
#pragma unroll
  for (int j = 1; j < kMaxBlocks; j++)
    b += (j < B.nblk && col >= B.c[j]) ? 1 : 0;
  return b;
}

// cnt[b * (m + 1) + r] = nonzeros of row r in column block b (a warp per row);
// cnt[b * (m + 1) + m] stays 0.
template <class CI, class RI>
__global__ void __launch_bounds__(256)
    split_count(const RI *__restrict__ rp, const CI *__restrict__ ci, int64_t m,
                Bounds B, RI *__restrict__ cnt) {
  const int nblk = B.nblk;
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < m; r += nw) {
    const int64_t p0 = (int64_t)rp[r], p1 = (int64_t)rp[r + 1];
    int c[kMaxBlocks];
#pragma unroll
    for (int bb = 0; bb < kMaxBlocks; bb++)
      c[bb] = 0;
    for (int64_t base = p0; base < p1; base += 32) {
      const int64_t p = base + lane;
      const int b = p < p1 ? block_of((int64_t)ci[p], B) : -1;
#pragma unroll
      for (int bb = 0; bb < kMaxBlocks; bb++)
        if (bb < nblk)
          c[bb] += __popc(__ballot_sync(0xffffffffu, b == bb));
    }
    if (lane == 0)
      for (int bb = 0; bb < nblk; bb++)
        cnt[(int64_t)bb * (m + 1) + r] = (RI)c[bb];
  }
}

// rp[b * (m + 1) + r] += off[b]: each block's row starts, counted from 0 by
// its scan, become positions in the regrouped arrays.
template <class RI>
__global__ void split_offsets(RI *__restrict__ rp, int64_t m, int nblk, BlockOffsets o) {
  const int64_t total = (int64_t)nblk * (m + 1);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x)
    rp[i] += (RI)o.off[i / (m + 1)];
}

// Copies every row's nonzeros into its blocks' rows of the virtual matrix,
// in row order (a warp per row: for each block, a ballot marks the lanes
// whose nonzero falls in it and the lane's rank among them is its place
// after the ones already copied).  Columns stay global.
template <class CI, class RI, class V>
__global__ void __launch_bounds__(256)
    split_scatter(const RI *__restrict__ rp, const CI *__restrict__ ci,
                  const V *__restrict__ v, int64_t m, Bounds B,
                  const RI *__restrict__ rpv, CI *__restrict__ civ, V *__restrict__ vv) {
  const int nblk = B.nblk;
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < m; r += nw) {
    const int64_t p0 = (int64_t)rp[r], p1 = (int64_t)rp[r + 1];
    // lane bb < nblk holds the start of row r's copy in block bb
    const int64_t my_base = lane < nblk ? (int64_t)rpv[(int64_t)lane * (m + 1) + r] : 0;
    int run[kMaxBlocks];
#pragma unroll
    for (int bb = 0; bb < kMaxBlocks; bb++)
      run[bb] = 0;
    for (int64_t base = p0; base < p1; base += 32) {
      const int64_t p = base + lane;
      const bool on = p < p1;
      const CI col = on ? ci[p] : CI(0);
      const V val = on ? v[p] : V(0);
      const int b = on ? block_of((int64_t)col, B) : -1;
#pragma unroll
      for (int bb = 0; bb < kMaxBlocks; bb++) {
        if (bb < nblk) {
          const unsigned mk = __ballot_sync(0xffffffffu, b == bb);
          const int64_t start = __shfl_sync(0xffffffffu, my_base, bb);
          if (b == bb) {
            const int64_t q = start + run[bb] + __popc(mk & lt);
            civ[q] = col;
            vv[q] = val;
          }
          run[bb] += __popc(mk);
        }
      }
    }
  }
}

// Row sums over the blocks of four grid-stride rows at once (their loads
// first, so each thread keeps 4 * nblk loads in flight): t[u] = sum over
// blocks b (in order) of ys[b * (m + 1) + row u]; rows at or past r1 give 0.
constexpr int kCombineRows = 4;

template <class Acc>
__device__ __forceinline__ void combine4(const Acc *__restrict__ ys, int64_t m, int64_t r,
                                         int64_t stride, int64_t r1, int nblk,
                                         Acc (&t)[kCombineRows]) {
#pragma unroll
  for (int u = 0; u < kCombineRows; u++)
    t[u] = r + u * stride < r1 ? ys[r + u * stride] : Acc(0);
  for (int b = 1; b < nblk; b++) {
    Acc a[kCombineRows];
#pragma unroll
    for (int u = 0; u < kCombineRows; u++)
      a[u] = r + u * stride < r1 ? ys[(int64_t)b * (m + 1) + r + u * stride] : Acc(0);
#pragma unroll
    for (int u = 0; u < kCombineRows; u++)
      t[u] += a[u];
  }
}

// y[r] = sum over blocks b (in order) of ys[b * (m + 1) + r], rows [r0, r1).
template <class Acc>
__global__ void split_combine(const Acc *__restrict__ ys, Acc *__restrict__ y, int64_t m,
                              int64_t r0, int64_t r1, int nblk) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t r = r0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < r1;
       r += kCombineRows * stride) {
    Acc t[kCombineRows];
    combine4(ys, m, r, stride, r1, nblk, t);
#pragma unroll
    for (int u = 0; u < kCombineRows; u++)
      if (r + u * stride < r1)
        y[r + u * stride] = t[u];
  }
}

// split_combine with the residual ||y - b||^2 folded in: each thread adds the
// terms (y_r - b_r)^2 of its grid-stride rows in row order (in double), a CTA's
// threads in a fixed tree into slots[blockIdx.x], and the last CTA (ticket)
// adds the slots in index order into *out and resets the ticket.  The grid is
// a function of m, so the grouping is fixed and the result repeats bit for
// bit.
template <class Acc>
__global__ void __launch_bounds__(256)
    split_combine_resid(const Acc *__restrict__ ys, Acc *__restrict__ y,
                        const Acc *__restrict__ b, int64_t m, int nblk, double *slots,
                        int *ticket, double *out) {
  __shared__ double s_red[8];
  __shared__ int s_last;
  double sum = 0.0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < m;
       r += kCombineRows * stride) {
    Acc t[kCombineRows], bb[kCombineRows];
#pragma unroll
    for (int u = 0; u < kCombineRows; u++)
      bb[u] = r + u * stride < m ? b[r + u * stride] : Acc(0);
    combine4(ys, m, r, stride, m, nblk, t);
#pragma unroll
    for (int u = 0; u < kCombineRows; u++)
      if (r + u * stride < m) {
        y[r + u * stride] = t[u];
        const double d = (double)t[u] - (double)bb[u];
        sum += d * d;
      }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    sum += __shfl_xor_sync(0xffffffffu, sum, o);
  if (lane == 0)
    s_red[warp] = sum;
  __syncthreads();
  if (threadIdx.x == 0) {
    double c = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++)
      c += s_red[w];
    slots[blockIdx.x] = c;
    __threadfence();
    s_last = atomicAdd(ticket, 1) == (int)gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last)
    return;
  __threadfence();
  double t = 0.0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x)
    t += __ldcg(&slots[i]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    t += __shfl_xor_sync(0xffffffffu, t, o);
  __syncthreads(); // s_red is reused
  if (lane == 0)
    s_red[warp] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    double c = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++)
      c += s_red[w];
    *out = c;
    *ticket = 0;
  }
}

unsigned warp_grid(int64_t rows) {
  const int64_t g = (rows + 7) / 8; // 8 warps per 256-thread CTA
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(g, 148 * 32));
}

unsigned flat_grid(int64_t n) {
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 16));
}

// Number of column blocks for A's single-RHS gemv (0: no split).
// DRB_COLSPLIT=<n> overrides it for handles created afterwards (0 or 1: off).
int split_blocks(const Csr &A) {
  if (A.storage != DRB_F32 && A.storage != DRB_F64)
    return 0;
  if (A.sell.on) // short regular rows (a stencil): the sliced-ELL kernel's gathers are local
    return 0;
  if (A.m == 0 || A.n < 2 || A.nnz == 0)
    return 0;
  if (const char *e = std::getenv("DRB_COLSPLIT")) {
    const int nb = std::atoi(e);
    return nb >= 2 ? (int)std::min<int64_t>({(int64_t)nb, (int64_t)kMaxBlocks, A.n}) : 0;
  }
  const int64_t xbytes = A.n * (int64_t)dtype_bytes(A.storage);
  if (xbytes <= kSplitAbove || A.nnz < 2 * A.n)
    return 0; // x stays in L2, or too little reuse of x for hits to matter
  return (int)std::min<int64_t>(kMaxBlocks, (xbytes + kSplitBlock - 1) / kSplitBlock);
}

// Share of the columns in the first of two blocks.  The host-pointer gemv
// starts block 0 when its slice of x has arrived; its compute should end as
// the last slice lands, so that the last block's rows can start their copy
// back at once: f * (upload + compute) = upload, with PCIe at ~55 GB/s
// (1.21 ms for a 64 MB x) and ~1.47 ms of SpMV on a 16.8M-row power-law
// matrix, f = 0.45 (measured: block 0 done 0.02 ms after the last slice
// against 0.15 ms with halves; 2.66 against 2.75 ms per call).  The device
// call does not care (1.478 against 1.470 ms).
constexpr double kFirstOfTwo = 0.45;

// First column of each of nblk blocks, plus n: equal widths, except a first
// block of kFirstOfTwo * n columns when there are two; DRB_COLSPLIT_FIRST=<f>
// (0 < f < 1) sets the first block's share for any count, any other value
// asks for equal widths.  Empty blocks are dropped.
std::vector<int64_t> block_bounds(int64_t n, int nblk) {
  double first = nblk == 2 ? kFirstOfTwo : 0.0;
  if (const char *e = std::getenv("DRB_COLSPLIT_FIRST"))
    first = std::atof(e);
  std::vector<int64_t> c(1, 0);
  if (first > 0.0 && first < 1.0) {
    const int64_t c1 = std::min(n - 1, std::max<int64_t>(1, (int64_t)(first * (double)n)));
    c.push_back(c1);
    const int64_t w = (n - c1 + nblk - 2) / (nblk - 1);
    for (int b = 2; b < nblk; b++)
      c.push_back(std::min(n, c1 + (b - 1) * w));
  } else {
    const int64_t w = (n + nblk - 1) / nblk;
    for (int b = 1; b < nblk; b++)
      c.push_back(std::min(n, b * w));
  }
  c.push_back(n);
  c.erase(std::unique(c.begin(), c.end()), c.end()); // drop empty blocks
  return c;
}

Bounds device_bounds(const std::vector<int64_t> &c) {
  Bounds B{};
  B.nblk = (int)c.size() - 1;
  for (int b = 0; b < B.nblk; b++)
    B.c[b] = c[b];
  return B;
}

template <class V, class CI, class RI>
drb_status scatter_typed(Csr &A, cudaStream_t s) {
  const Csr &S = *A.csplit;
  split_scatter<CI, RI, V><<<warp_grid(A.m), 256, 0, s>>>(
      A.rowptr.as<RI>(), A.colind.as<CI>(), A.vals.as<V>(), A.m, device_bounds(A.cbounds),
      S.rowptr.as<RI>(), S.colind.as<CI>(), S.vals.as<V>());
  note_launch();
  DRB_CUDA_TRY(cudaGetLastError());
  return DRB_OK;
}

template <class V, class CI, class RI>
drb_status build_typed(Csr &A, int nblk, int tile, cudaStream_t s) {
  const int64_t m = A.m;
  const std::vector<int64_t> bounds = block_bounds(A.n, nblk);
  nblk = (int)bounds.size() - 1; // every block holds at least one column
  if (nblk < 2)
    return DRB_OK;
  const int64_t mv = (int64_t)nblk * (m + 1) - 1; // rows of the virtual matrix
  if (mv >= 0x7fffffff)
    return DRB_OK; // work items index rows with 32 bits
  // device memory: the regrouped copy, its row starts, the count table and
  // the scratch y; keep 1 GB free beside them
  const int vb = dtype_bytes(A.storage), ab = A.storage == DRB_F64 ? 8 : 4;
  const int64_t pad = ((A.nnz + kPadElems - 1) / kPadElems + 1) * kPadElems;
  const size_t need = (size_t)pad * (vb + sizeof(CI)) +
                      (size_t)2 * (mv + 1 + kRowptrPad) * sizeof(RI) + (size_t)(mv + 1) * ab;
  size_t free_b = 0, total_b = 0;
  DRB_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
  if (need + ((size_t)1 << 30) > free_b)
    return DRB_OK; // not enough room: the handle runs unsplit
  auto S = std::make_unique<Csr>();
  S->device = A.device;
  S->m = mv;
  S->n = A.n;
  S->nnz = A.nnz;
  S->value_type = A.value_type;
  S->storage = A.storage;
  S->cbytes = A.cbytes;
  S->rbytes = A.rbytes;
  S->flags = A.flags & ~(DRB_FLAG_ADJOINT | DRB_FLAG_AUTOTUNE);
  S->max_row = A.max_row;
  DRB_TRY(S->rowptr.alloc(sizeof(RI) * (mv + 1 + kRowptrPad)));
  DRB_CUDA_TRY(cudaMemsetAsync(S->rowptr.p, 0, S->rowptr.bytes, s));
  {
    DevBuf cnt;
    DRB_TRY(cnt.alloc(sizeof(RI) * (mv + 1)));
    DRB_CUDA_TRY(cudaMemsetAsync(cnt.p, 0, cnt.bytes, s));
    split_count<CI, RI><<<warp_grid(m), 256, 0, s>>>(A.rowptr.as<RI>(), A.colind.as<CI>(),
                                                     m, device_bounds(bounds), cnt.as<RI>());
    note_launch();
    DRB_CUDA_TRY(cudaGetLastError());
    size_t tmp_bytes = 0;
    DRB_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, cnt.as<RI>(),
                                               S->rowptr.as<RI>(), m + 1, s));
    DevBuf tmp;
    DRB_TRY(tmp.alloc(std::max<size_t>(tmp_bytes, 16)));
    BlockOffsets o{};
    int64_t acc = 0;
    for (int b = 0; b < nblk; b++) {
      size_t tb = tmp_bytes;
      RI *seg = S->rowptr.as<RI>() + (int64_t)b * (m + 1);
      DRB_CUDA_TRY(cub::DeviceScan::ExclusiveSum(tmp.p, tb, cnt.as<RI>() + (int64_t)b * (m + 1),
                                                 seg, m + 1, s));
      note_launch();
      RI tot = 0;
      DRB_CUDA_TRY(cudaMemcpyAsync(&tot, seg + m, sizeof(RI), cudaMemcpyDeviceToHost, s));
      DRB_CUDA_TRY(cudaStreamSynchronize(s));
      o.off[b] = acc;
      acc += (int64_t)tot;
    }
    if (acc != A.nnz) {
      set_error("column split: regrouped %lld of %lld nonzeros", (long long)acc,
                (long long)A.nnz);
      return DRB_ERR_CUDA;
    }
    split_offsets<RI><<<flat_grid(mv + 1), 256, 0, s>>>(S->rowptr.as<RI>(), m, nblk, o);
    note_launch();
    DRB_CUDA_TRY(cudaGetLastError());
  }
  DRB_TRY(S->colind.alloc(sizeof(CI) * pad));
  DRB_TRY(S->vals.alloc((size_t)vb * pad));
  DRB_CUDA_TRY(cudaMemsetAsync(S->colind.p, 0, S->colind.bytes, s));
  DRB_CUDA_TRY(cudaMemsetAsync(S->vals.p, 0, S->vals.bytes, s));
  DRB_TRY(A.csplit_y.alloc((size_t)(mv + 1) * ab));
  A.csplit = std::move(S);
  A.csplit_nblk = nblk;
  A.cbounds = bounds;
  DRB_TRY(scatter_typed<V, CI, RI>(A, s));
  std::vector<RI> rp_h(mv + 1);
  DRB_CUDA_TRY(cudaMemcpyAsync(rp_h.data(), A.csplit->rowptr.p, sizeof(RI) * (mv + 1),
                               cudaMemcpyDeviceToHost, s));
  DRB_CUDA_TRY(cudaStreamSynchronize(s));
  return build_pipe_plan(A.csplit->pipe, mv, rp_h.data(), sizeof(RI),
                         plan_group(vb, A.cbytes), tile, 0);
}

template <class V>
drb_status build_v(Csr &A, int nblk, int tile, cudaStream_t s) {
  if (A.cbytes == 4 && A.rbytes == 4)
    return build_typed<V, int32_t, int32_t>(A, nblk, tile, s);
  if (A.cbytes == 4 && A.rbytes == 8)
    return build_typed<V, int32_t, int64_t>(A, nblk, tile, s);
  if (A.cbytes == 8 && A.rbytes == 4)
    return build_typed<V, int64_t, int32_t>(A, nblk, tile, s);
  return build_typed<V, int64_t, int64_t>(A, nblk, tile, s);
}

template <class V>
drb_status scatter_v(Csr &A, cudaStream_t s) {
  if (A.cbytes == 4 && A.rbytes == 4)
    return scatter_typed<V, int32_t, int32_t>(A, s);
  if (A.cbytes == 4 && A.rbytes == 8)
    return scatter_typed<V, int32_t, int64_t>(A, s);
  if (A.cbytes == 8 && A.rbytes == 4)
    return scatter_typed<V, int64_t, int32_t>(A, s);
  return scatter_typed<V, int64_t, int64_t>(A, s);
}

} // namespace

drb_status colsplit_build(Csr &A, cudaStream_t s) {
  A.csplit.reset();
  A.csplit_y.release();
  A.csplit_nblk = 0;
  A.cbounds.clear();
  const int nblk = split_blocks(A);
  if (nblk < 2)
    return DRB_OK;
  const int tile = A.pipe.tile | (A.pipe.skew ? 1 : 0) | (A.pipe.two_slot ? 2 : 0);
  return A.storage == DRB_F64 ? build_v<double>(A, nblk, tile, s)
                              : build_v<float>(A, nblk, tile, s);
}

drb_status colsplit_refresh_values(Csr &A, cudaStream_t s) {
  if (!A.csplit)
    return DRB_OK;
  return A.storage == DRB_F64 ? scatter_v<double>(A, s) : scatter_v<float>(A, s);
}

namespace {
// y[r0, r1) from the blocks' partial sums.
drb_status combine_rows(Csr &A, void *y, int64_t r0, int64_t r1, cudaStream_t s) {
  if (r1 <= r0)
    return DRB_OK;
  const unsigned g = flat_grid(r1 - r0);
  if (A.storage == DRB_F64)
    split_combine<double><<<g, 256, 0, s>>>(A.csplit_y.as<double>(), static_cast<double *>(y),
                                            A.m, r0, r1, A.csplit_nblk);
  else
    split_combine<float><<<g, 256, 0, s>>>(A.csplit_y.as<float>(), static_cast<float *>(y),
                                           A.m, r0, r1, A.csplit_nblk);
  note_launch();
  DRB_CUDA_TRY(cudaGetLastError());
  return DRB_OK;
}
} // namespace

drb_status colsplit_launch(Csr &A, const void *x, void *y, cudaStream_t s) {
  DRB_TRY(spmv_pipe_launch(*A.csplit, x, A.csplit_y.p, s));
  return combine_rows(A, y, 0, A.m, s);
}

drb_status colsplit_residual(Csr &A, const void *x, const void *b, void *y, double *out,
                             cudaStream_t s) {
  DRB_TRY(spmv_pipe_launch(*A.csplit, x, A.csplit_y.p, s));
  // per-CTA slots and the ticket: the fused-reduction scratch of A's own plan
  // (sms * 32 doubles, then the ticket), used by one launch at a time
  DRB_TRY(fused_scratch(A));
  int sms = 0;
  DRB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, A.device));
  const unsigned g = std::min<unsigned>(flat_grid(A.m), (unsigned)sms * 32);
  double *slots = A.pipe.red.as<double>();
  int *ticket = reinterpret_cast<int *>(slots + (size_t)sms * 32);
  if (A.storage == DRB_F64)
    split_combine_resid<double><<<g, 256, 0, s>>>(A.csplit_y.as<double>(),
                                                  static_cast<double *>(y),
                                                  static_cast<const double *>(b), A.m,
                                                  A.csplit_nblk, slots, ticket, out);
  else
    split_combine_resid<float><<<g, 256, 0, s>>>(A.csplit_y.as<float>(), static_cast<float *>(y),
                                                 static_cast<const float *>(b), A.m,
                                                 A.csplit_nblk, slots, ticket, out);
  note_launch();
  DRB_CUDA_TRY(cudaGetLastError());
  return DRB_OK;
}

namespace {

constexpr int kSplitHostSegments = 6; // row segments of the last block
// Each of the last block's segments holds this multiple of the previous one's
// nonzeros: the last block computes about as fast as its rows copy back over
// PCIe, so a smaller first segment starts the copy earlier while the later,
// larger ones still finish before the copy reaches them.  Measured on a
// 16.8M-row power-law matrix (FP32 in two blocks, FP64 in three; ms per call,
// pinned buffers): 2 to 6 segments at growth 0.8 / 1.0 / 1.25: FP32 3.16 /
// 3.09 / 3.06 (2) ... 2.93 / 2.86 / 2.84 (6), FP64 5.77 / 5.73 / 5.69 (2) ...
// 5.54 / 5.45 / 5.37 (6); growth 1.5 and 2.0 lost on FP32 (+1-2 %, +8 %).
constexpr double kSplitSegmentGrowth = 1.25;

int split_host_segments() {
  const char *e = std::getenv("DRB_HOST_SEGMENTS");
  if (!e || !*e)
    return kSplitHostSegments;
  return std::min(64, std::max(1, std::atoi(e)));
}

// DRB_HOST_SPLIT_GROWTH (0.2..5) overrides the growth, read with the count.
double split_segment_growth() {
  const char *e = std::getenv("DRB_HOST_SPLIT_GROWTH");
  if (!e || !*e)
    return kSplitSegmentGrowth;
  return std::min(5.0, std::max(0.2, std::atof(e)));
}

// Orders the virtual matrix's items by row and cuts them for the host-pointer
// gemv.  An item belongs to the block of its last row (an item may run from
// one block's last rows over the empty separator into the next block's first
// rows; the x slices arrive in order, so it waits for the later one).  Every
// block but the last is one segment; the last is cut into `target` row
// segments whose nonzeros grow by `growth`, each cut before a whole-row item
// or a row's first chunk, so a split row never straddles two segments.
drb_status build_host_segments(Csr &A, int target, double growth) {
  Csr &S = *A.csplit;
  PipePlan &P = S.pipe;
  const int nb = A.csplit_nblk;
  const int64_t stride = A.m + 1;
  std::vector<Item> it((size_t)P.nitems);
  DRB_CUDA_TRY(cudaMemcpy(it.data(), P.items.p, sizeof(Item) * it.size(),
                          cudaMemcpyDeviceToHost));
  std::stable_sort(it.begin(), it.end(),
                   [](const Item &a, const Item &b) { return a.r0 < b.r0; });
  auto blk = [&](const Item &t) {
    const int64_t last = (int64_t)t.r0 + std::max<int64_t>(t.nrows, 1) - 1;
    return (int)std::min<int64_t>(nb - 1, last / stride);
  };
  // the last block's first item and its nonzeros
  size_t lb = 0;
  while (lb < it.size() && blk(it[lb]) < nb - 1)
    lb++;
  int64_t total = 0;
  for (size_t i = lb; i < it.size(); i++)
    total += it[i].len;
  std::vector<double> cut; // running nnz (within the last block) of each later segment's start
  {
    double w = 1.0, wsum = 0.0;
    for (int j = 0; j < target; j++, w *= growth)
      wsum += w;
    w = 1.0;
    for (double acc = 0.0; (int)cut.size() < target - 1; w *= growth) {
      acc += w;
      cut.push_back((double)total * acc / wsum);
    }
  }
  P.seg_i0.assign(1, 0);
  P.seg_r0.assign(1, 0);
  P.seg_blk.assign(1, it.empty() ? nb - 1 : blk(it[0]));
  int64_t acc = 0;
  size_t j = 0;
  for (size_t i = 1; i < it.size(); i++) {
    const int b = blk(it[i]);
    if (i > lb)
      acc += it[i - 1].len;
    const bool new_row = it[i].nrows > 0 || it[i].r0 != it[i - 1].r0;
    bool cut_here = b != blk(it[i - 1]); // a new block (never inside a split row)
    if (!cut_here && b == nb - 1 && i > lb && j < cut.size() && (double)acc >= cut[j] &&
        new_row) {
      cut_here = true;
      j++;
    }
    if (cut_here) {
      P.seg_i0.push_back((int64_t)i);
      P.seg_r0.push_back(it[i].r0);
      P.seg_blk.push_back(b);
    }
  }
  P.seg_i0.push_back((int64_t)it.size());
  P.seg_r0.push_back(S.m + 1);
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
  if (!it.empty())
    DRB_CUDA_TRY(cudaMemcpy(P.seg_items.p, it.data(), sizeof(Item) * it.size(),
                            cudaMemcpyHostToDevice));
  return DRB_OK;
}

} // namespace

drb_status colsplit_gemv_host(Csr &A, const void *x_host, void *y_host, size_t xb,
                              size_t yb, cudaStream_t s) {
  Csr &S = *A.csplit;
  PipePlan &P = S.pipe;
  const int nb = A.csplit_nblk;
  if (P.seg_i0.empty() || P.seg_blk.size() + 1 != P.seg_i0.size())
    DRB_TRY(build_host_segments(A, split_host_segments(), split_segment_growth()));
  const int nseg = (int)P.seg_i0.size() - 1;
  const int64_t base = (int64_t)(nb - 1) * (A.m + 1); // first virtual row of the last block
  if (!A.copy_stream)
    DRB_CUDA_TRY(cudaStreamCreateWithFlags(&A.copy_stream, cudaStreamNonBlocking));
  // events: [start][x block 0 .. nb-1][segment 0 .. nseg-1][end]
  while ((int)A.seg_done.size() < nseg + nb + 2) {
    cudaEvent_t e;
    DRB_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    A.seg_done.push_back(e);
  }
  cudaEvent_t *ev = A.seg_done.data();
  // the copies follow the work already queued on s
  DRB_CUDA_TRY(cudaEventRecord(ev[0], s));
  DRB_CUDA_TRY(cudaStreamWaitEvent(A.copy_stream, ev[0], 0));
  for (int b = 0; b < nb; b++) {
    const int64_t c0 = A.cbounds[b], c1 = A.cbounds[b + 1];
    DRB_CUDA_TRY(cudaMemcpyAsync(A.xh_dev.as<char>() + xb * c0,
                                 static_cast<const char *>(x_host) + xb * c0, xb * (c1 - c0),
                                 cudaMemcpyHostToDevice, A.copy_stream));
    DRB_CUDA_TRY(cudaEventRecord(ev[1 + b], A.copy_stream));
  }
  // real rows of segment g (the last block's segments; empty for the others)
  auto rows = [&](int g, int64_t &r0, int64_t &r1) {
    r0 = std::min(A.m, std::max<int64_t>(0, P.seg_r0[g] - base));
    r1 = g + 1 == nseg ? A.m : std::min(A.m, std::max<int64_t>(0, P.seg_r0[g + 1] - base));
    if (P.seg_blk[g] != nb - 1)
      r0 = r1 = 0;
  };
  // the kernel reads P.items / P.nitems: point them at one segment at a time;
  // all launches first (a copy into pageable host memory would block this
  // thread), then the copies back, each behind its segment's event
  void *items0 = P.items.p;
  const int64_t n0 = P.nitems;
  drb_status st = DRB_OK;
  int waited = -1;
  for (int g = 0; g < nseg && st == DRB_OK; g++) {
    for (; waited < P.seg_blk[g] && st == DRB_OK; waited++)
      if (cudaStreamWaitEvent(s, ev[2 + waited], 0) != cudaSuccess)
        st = DRB_ERR_CUDA;
    if (st != DRB_OK)
      break;
    P.items.p = P.seg_items.as<Item>() + P.seg_i0[g];
    P.nitems = P.seg_i0[g + 1] - P.seg_i0[g];
    P.fin_c0 = P.seg_c0[g];
    P.fin_c1 = P.seg_c0[g + 1];
    st = spmv_pipe_launch(S, A.xh_dev.p, A.csplit_y.p, s);
    P.items.p = items0;
    P.nitems = n0;
    P.fin_c0 = 0;
    P.fin_c1 = -1;
    int64_t r0, r1;
    rows(g, r0, r1);
    if (st == DRB_OK)
      st = combine_rows(A, A.yh_dev.p, r0, r1, s);
    if (st == DRB_OK && cudaEventRecord(ev[1 + nb + g], s) != cudaSuccess)
      st = DRB_ERR_CUDA;
  }
  DRB_TRY(st);
  for (int g = 0; g < nseg; g++) {
    int64_t r0, r1;
    rows(g, r0, r1);
    if (r1 <= r0)
      continue;
    DRB_CUDA_TRY(cudaStreamWaitEvent(A.copy_stream, ev[1 + nb + g], 0));
    DRB_CUDA_TRY(cudaMemcpyAsync(static_cast<char *>(y_host) + yb * r0,
                                 A.yh_dev.as<char>() + yb * r0, yb * (r1 - r0),
                                 cudaMemcpyDeviceToHost, A.copy_stream));
  }
  DRB_CUDA_TRY(cudaEventRecord(ev[nseg + nb + 1], A.copy_stream));
  DRB_CUDA_TRY(cudaStreamWaitEvent(s, ev[nseg + nb + 1], 0));
  DRB_CUDA_TRY(cudaStreamSynchronize(s));
  return DRB_OK;
}

drb_status colsplit_tune(Csr &A, cudaStream_t s) {
  if (!A.csplit)
    return DRB_OK;
  Csr &S = *A.csplit;
  const int vb = dtype_bytes(A.storage);
  const int group = plan_group(vb, A.cbytes);
  std::vector<int> variants = {256 | 1, 256, 256 | 3};
  if (group <= 4) {
    variants.push_back(128 | 1);
    variants.push_back(128);
    variants.push_back(128 | 3);
  }
  DevBuf xb, yb;
  DRB_TRY(xb.alloc((size_t)vb * (A.n + 1)));
  DRB_TRY(yb.alloc((size_t)vb * (A.m + 1)));
  DRB_CUDA_TRY(cudaMemsetAsync(xb.p, 0, xb.bytes, s));
  std::vector<char> rp((size_t)S.rbytes * (S.m + 1));
  DRB_CUDA_TRY(cudaMemcpy(rp.data(), S.rowptr.p, rp.size(), cudaMemcpyDeviceToHost));
  cudaEvent_t e0, e1;
  DRB_CUDA_TRY(cudaEventCreate(&e0));
  DRB_CUDA_TRY(cudaEventCreate(&e1));
  std::vector<float> best(variants.size(), 3.4e38f);
  drb_status st = DRB_OK;
  for (int round = 0; round < 2 && st == DRB_OK; round++)
    for (size_t i = 0; i < variants.size() && st == DRB_OK; i++) {
      if ((st = build_pipe_plan(S.pipe, S.m, rp.data(), S.rbytes, group, variants[i], 0)) !=
          DRB_OK)
        break;
      for (int w = 0; w < 2 && st == DRB_OK; w++)
        st = colsplit_launch(A, xb.p, yb.p, s);
      for (int r = 0; r < 5 && st == DRB_OK; r++) { // the fastest of five launches
        cudaEventRecord(e0, s);
        st = colsplit_launch(A, xb.p, yb.p, s);
        cudaEventRecord(e1, s);
        float ms = 0.f;
        if (st != DRB_OK || cudaEventSynchronize(e1) != cudaSuccess ||
            cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
          if (st == DRB_OK)
            st = DRB_ERR_CUDA;
          break;
        }
        best[i] = std::min(best[i], ms);
      }
    }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  DRB_TRY(st);
  const size_t pick = std::min_element(best.begin(), best.end()) - best.begin();
  return build_pipe_plan(S.pipe, S.m, rp.data(), S.rbytes, group, variants[pick], 0);
}

} // namespace drb
