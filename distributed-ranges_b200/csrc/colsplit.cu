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
// ([b*bw, (b+1)*bw), columns kept global, each row's order kept), and its
// rows b*(m+1) + m are empty separators.  The unchanged persistent SpMV runs
// over it in ONE launch into a block-major scratch y; its work counter hands
// out items in order, so at any time nearly all warps work inside one block
// and only that block's slice of x is hot in L2.  A last small pass adds the
// blocks' row sums into y in block order (deterministic).  The scratch costs
// nblk * (m + 1) partial sums, written once and read once.
//
// The regrouping runs on the device at plan time: a warp per row counts its
// nonzeros per block with ballots, a scan per block gives the blocks' row
// starts (offset by the blocks before them), and a second warp-per-row pass
// scatters the nonzeros (a ballot per block gives each lane its place), so
// rows need not be sorted.
#include <algorithm>
#include <cstdlib>
#include <vector>

#include <cub/cub.cuh>

#include "drb_internal.cuh"

namespace drb {
namespace {

constexpr int kMaxBlocks = 8;
constexpr int64_t kSplitAbove = 64ll << 20; // split when x is larger than this
constexpr int64_t kSplitBlock = 48ll << 20; // and give each block at most this

struct BlockOffsets {
  int64_t off[kMaxBlocks]; // first nonzero of each block in the regrouped arrays
};

__device__ __forceinline__ int block_of(int64_t col, int64_t bw, int nblk) {
  return (int)min(col / bw, (int64_t)nblk - 1);
}

// cnt[b * (m + 1) + r] = nonzeros of row r in column block b (a warp per row);
// cnt[b * (m + 1) + m] stays 0.
template <class CI, class RI>
__global__ void __launch_bounds__(256)
    split_count(const RI *__restrict__ rp, const CI *__restrict__ ci, int64_t m,
                int64_t bw, int nblk, RI *__restrict__ cnt) {
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
      const int b = p < p1 ? block_of((int64_t)ci[p], bw, nblk) : -1;
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
                  const V *__restrict__ v, int64_t m, int64_t bw, int nblk,
                  const RI *__restrict__ rpv, CI *__restrict__ civ, V *__restrict__ vv) {
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
      const int b = on ? block_of((int64_t)col, bw, nblk) : -1;
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

// y[r] = sum over blocks b (in order) of ys[b * (m + 1) + r].
template <class Acc>
__global__ void split_combine(const Acc *__restrict__ ys, Acc *__restrict__ y, int64_t m,
                              int nblk) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < m;
       r += (int64_t)gridDim.x * blockDim.x) {
    Acc t = ys[r];
    for (int b = 1; b < nblk; b++)
      t += ys[(int64_t)b * (m + 1) + r];
    y[r] = t;
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

template <class V, class CI, class RI>
drb_status scatter_typed(Csr &A, cudaStream_t s) {
  const Csr &S = *A.csplit;
  split_scatter<CI, RI, V><<<warp_grid(A.m), 256, 0, s>>>(
      A.rowptr.as<RI>(), A.colind.as<CI>(), A.vals.as<V>(), A.m, A.cbw, A.csplit_nblk,
      S.rowptr.as<RI>(), S.colind.as<CI>(), S.vals.as<V>());
  note_launch();
  DRB_CUDA_TRY(cudaGetLastError());
  return DRB_OK;
}

template <class V, class CI, class RI>
drb_status build_typed(Csr &A, int nblk, int tile, cudaStream_t s) {
  const int64_t m = A.m;
  const int64_t bw = (A.n + nblk - 1) / nblk;
  nblk = (int)((A.n + bw - 1) / bw); // every block holds at least one column
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
                                                     m, bw, nblk, cnt.as<RI>());
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
  A.cbw = bw;
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
  A.cbw = 0;
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

drb_status colsplit_launch(Csr &A, const void *x, void *y, cudaStream_t s) {
  DRB_TRY(spmv_pipe_launch(*A.csplit, x, A.csplit_y.p, s));
  if (A.storage == DRB_F64)
    split_combine<double><<<flat_grid(A.m), 256, 0, s>>>(A.csplit_y.as<double>(),
                                                         static_cast<double *>(y), A.m,
                                                         A.csplit_nblk);
  else
    split_combine<float><<<flat_grid(A.m), 256, 0, s>>>(A.csplit_y.as<float>(),
                                                        static_cast<float *>(y), A.m,
                                                        A.csplit_nblk);
  note_launch();
  DRB_CUDA_TRY(cudaGetLastError());
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
