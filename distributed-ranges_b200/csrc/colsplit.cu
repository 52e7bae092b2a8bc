// colsplit.cu -- column-blocked plan of the single-RHS SpMV, for matrices
// whose x does not stay in L2.
//
// A randomly gathered x stays L2-resident on B200 only up to about 48 MB:
// on a 16.8M-row power-law pattern (336M nonzeros, uniform columns) the SpMV
// takes the same time for an x of 8 to 48 MB (FP32 1.39-1.40 ms, FP64 1.68 ms)
// and degrades beyond it (FP64 2.03 / 2.91 / 3.69 ms at 64 / 96 / 128 MB).
// So when x is larger than kSplitAbove, the handle keeps a second copy of its
// nonzeros grouped by column block: block b holds, for every row, the
// nonzeros whose columns lie in [b*bw, (b+1)*bw) (columns rebased to b*bw,
// each row's order kept), as a CSR matrix of its own with its own work items.
// A single-RHS gemv then runs one launch per block over its slice of x: the
// first writes y, the later ones add their row sums to it, in block order,
// so the result is deterministic (each row's sum is grouped by block).  The
// 16.8M-row FP64 product with three blocks of 42.7 MB: 3.69 -> 2.16 ms.  An
// x of 48-64 MB stays unsplit: the second launch's ramp and tail cost what
// the hits save (the FP32 bench matrix: 1.53 ms whole, 1.54 ms in halves).
//
// The regrouping runs on the device at plan time: a warp per row counts its
// nonzeros per block with ballots, a scan per block gives the blocks' row
// pointers, and a second warp-per-row pass scatters the nonzeros (a ballot
// per block gives each lane its place), so rows need not be sorted.
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

template <class CI, class RI, class V> struct SplitDst {
  RI *rp[kMaxBlocks];
  CI *ci[kMaxBlocks];
  V *v[kMaxBlocks];
};

__device__ __forceinline__ int block_of(int64_t col, int64_t bw, int nblk) {
  return (int)min(col / bw, (int64_t)nblk - 1);
}

// cnt[b * (m + 1) + r] = nonzeros of row r in column block b (a warp per row).
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

// Copies every row's nonzeros into its blocks, in row order (a warp per row:
// for each block, a ballot marks the lanes whose nonzero falls in it and the
// lane's rank among them is its place after the ones already copied).
template <class CI, class RI, class V>
__global__ void __launch_bounds__(256)
    split_scatter(const RI *__restrict__ rp, const CI *__restrict__ ci,
                  const V *__restrict__ v, int64_t m, int64_t bw, int nblk,
                  SplitDst<CI, RI, V> d) {
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < m; r += nw) {
    const int64_t p0 = (int64_t)rp[r], p1 = (int64_t)rp[r + 1];
    RI my_base = 0; // lane bb < nblk holds block bb's row start
#pragma unroll
    for (int bb = 0; bb < kMaxBlocks; bb++)
      if (bb < nblk && lane == bb)
        my_base = d.rp[bb][r];
    int run[kMaxBlocks];
#pragma unroll
    for (int bb = 0; bb < kMaxBlocks; bb++)
      run[bb] = 0;
    for (int64_t base = p0; base < p1; base += 32) {
      const int64_t p = base + lane;
      const bool on = p < p1;
      const int64_t col = on ? (int64_t)ci[p] : 0;
      const V val = on ? v[p] : V(0);
      const int b = on ? block_of(col, bw, nblk) : -1;
#pragma unroll
      for (int bb = 0; bb < kMaxBlocks; bb++) {
        if (bb < nblk) {
          const unsigned mk = __ballot_sync(0xffffffffu, b == bb);
          const int64_t start = (int64_t)__shfl_sync(0xffffffffu, my_base, bb);
          if (b == bb) {
            const int64_t q = start + run[bb] + __popc(mk & lt);
            d.ci[bb][q] = (CI)(col - (int64_t)bb * bw);
            d.v[bb][q] = val;
          }
          run[bb] += __popc(mk);
        }
      }
    }
  }
}

unsigned warp_grid(int64_t rows) {
  const int64_t g = (rows + 7) / 8; // 8 warps per 256-thread CTA
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(g, 148 * 32));
}

// Number of column blocks for A's single-RHS gemv (0: no split).
// DRB_COLSPLIT=<n> overrides it for handles created afterwards (0 or 1: off).
int split_blocks(const Csr &A) {
  if (A.storage != DRB_F32 && A.storage != DRB_F64)
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
  SplitDst<CI, RI, V> d{};
  const int nblk = (int)A.cblk.size();
  for (int b = 0; b < nblk; b++) {
    d.rp[b] = A.cblk[b]->rowptr.as<RI>();
    d.ci[b] = A.cblk[b]->colind.as<CI>();
    d.v[b] = A.cblk[b]->vals.as<V>();
  }
  split_scatter<CI, RI, V><<<warp_grid(A.m), 256, 0, s>>>(
      A.rowptr.as<RI>(), A.colind.as<CI>(), A.vals.as<V>(), A.m, A.cbw, nblk, d);
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
  // device memory: the blocks' copies (values, columns, row pointers) plus
  // the count table; keep 1 GB free beside them
  const int vb = dtype_bytes(A.storage);
  const size_t need = (size_t)A.nnz * (vb + sizeof(CI)) +
                      (size_t)(2 * nblk + 1) * (m + 1 + kRowptrPad) * sizeof(RI) +
                      (size_t)nblk * 2 * kPadElems * (vb + sizeof(CI));
  size_t free_b = 0, total_b = 0;
  DRB_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
  if (need + ((size_t)1 << 30) > free_b)
    return DRB_OK; // not enough room: the handle runs unsplit
  DevBuf cnt;
  DRB_TRY(cnt.alloc(sizeof(RI) * nblk * (m + 1)));
  DRB_CUDA_TRY(cudaMemsetAsync(cnt.p, 0, cnt.bytes, s));
  split_count<CI, RI><<<warp_grid(m), 256, 0, s>>>(A.rowptr.as<RI>(), A.colind.as<CI>(), m,
                                                   bw, nblk, cnt.as<RI>());
  note_launch();
  DRB_CUDA_TRY(cudaGetLastError());
  std::vector<std::unique_ptr<Csr>> blk;
  size_t tmp_bytes = 0;
  DRB_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, cnt.as<RI>(),
                                             cnt.as<RI>(), m + 1, s));
  DevBuf tmp;
  DRB_TRY(tmp.alloc(std::max<size_t>(tmp_bytes, 16)));
  std::vector<int64_t> nnzb(nblk);
  for (int b = 0; b < nblk; b++) {
    auto B = std::make_unique<Csr>();
    B->device = A.device;
    B->m = m;
    B->n = std::min(bw, A.n - (int64_t)b * bw);
    B->value_type = A.value_type;
    B->storage = A.storage;
    B->cbytes = A.cbytes;
    B->rbytes = A.rbytes;
    B->flags = A.flags & ~(DRB_FLAG_ADJOINT | DRB_FLAG_AUTOTUNE);
    B->max_row = A.max_row;
    DRB_TRY(B->rowptr.alloc(sizeof(RI) * (m + 1 + kRowptrPad)));
    DRB_CUDA_TRY(cudaMemsetAsync(B->rowptr.p, 0, B->rowptr.bytes, s));
    size_t tb = tmp_bytes;
    DRB_CUDA_TRY(cub::DeviceScan::ExclusiveSum(tmp.p, tb, cnt.as<RI>() + (int64_t)b * (m + 1),
                                               B->rowptr.as<RI>(), m + 1, s));
    note_launch();
    RI total = 0;
    DRB_CUDA_TRY(cudaMemcpyAsync(&total, B->rowptr.as<RI>() + m, sizeof(RI),
                                 cudaMemcpyDeviceToHost, s));
    DRB_CUDA_TRY(cudaStreamSynchronize(s));
    B->nnz = nnzb[b] = (int64_t)total;
    const int64_t pad = ((B->nnz + kPadElems - 1) / kPadElems + 1) * kPadElems;
    DRB_TRY(B->colind.alloc(sizeof(CI) * pad));
    DRB_TRY(B->vals.alloc((size_t)vb * pad));
    DRB_CUDA_TRY(cudaMemsetAsync(B->colind.p, 0, B->colind.bytes, s));
    DRB_CUDA_TRY(cudaMemsetAsync(B->vals.p, 0, B->vals.bytes, s));
    blk.push_back(std::move(B));
  }
  cnt.release();
  tmp.release();
  A.cblk = std::move(blk);
  A.cbw = bw;
  DRB_TRY(scatter_typed<V, CI, RI>(A, s));
  DRB_CUDA_TRY(cudaStreamSynchronize(s));
  std::vector<RI> rp_h(m + 1);
  for (int b = 0; b < nblk; b++) {
    Csr &B = *A.cblk[b];
    DRB_CUDA_TRY(cudaMemcpy(rp_h.data(), B.rowptr.p, sizeof(RI) * (m + 1),
                            cudaMemcpyDeviceToHost));
    DRB_TRY(build_pipe_plan(B.pipe, m, rp_h.data(), sizeof(RI),
                            plan_group(vb, A.cbytes), tile, 0));
    B.pipe.accum = b > 0;
  }
  return DRB_OK;
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
  A.cblk.clear();
  A.cbw = 0;
  const int nblk = split_blocks(A);
  if (nblk < 2)
    return DRB_OK;
  // the blocks' rows are shorter than A's (about 1/nblk of each row)
  const int tile = A.pipe.tile | (A.pipe.skew ? 1 : 0) | (A.pipe.two_slot ? 2 : 0);
  return A.storage == DRB_F64 ? build_v<double>(A, nblk, tile, s)
                              : build_v<float>(A, nblk, tile, s);
}

drb_status colsplit_refresh_values(Csr &A, cudaStream_t s) {
  if (A.cblk.empty())
    return DRB_OK;
  return A.storage == DRB_F64 ? scatter_v<double>(A, s) : scatter_v<float>(A, s);
}

drb_status colsplit_launch(Csr &A, const void *x, void *y, cudaStream_t s) {
  const size_t xb = (size_t)dtype_bytes(A.storage);
  for (size_t b = 0; b < A.cblk.size(); b++) {
    const void *xs = static_cast<const char *>(x) + xb * A.cbw * b;
    DRB_TRY(spmv_pipe_launch(*A.cblk[b], xs, y, s));
  }
  return DRB_OK;
}

drb_status colsplit_tune(Csr &A, cudaStream_t s) {
  if (A.cblk.empty())
    return DRB_OK;
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
  DRB_CUDA_TRY(cudaMemsetAsync(yb.p, 0, yb.bytes, s));
  std::vector<std::vector<char>> rps(A.cblk.size());
  for (size_t b = 0; b < A.cblk.size(); b++) {
    rps[b].resize((size_t)A.rbytes * (A.m + 1));
    DRB_CUDA_TRY(cudaMemcpy(rps[b].data(), A.cblk[b]->rowptr.p, rps[b].size(),
                            cudaMemcpyDeviceToHost));
  }
  auto rebuild = [&](int v) -> drb_status {
    for (size_t b = 0; b < A.cblk.size(); b++) {
      DRB_TRY(build_pipe_plan(A.cblk[b]->pipe, A.m, rps[b].data(), A.rbytes, group, v, 0));
      A.cblk[b]->pipe.accum = b > 0;
    }
    return DRB_OK;
  };
  cudaEvent_t e0, e1;
  DRB_CUDA_TRY(cudaEventCreate(&e0));
  DRB_CUDA_TRY(cudaEventCreate(&e1));
  std::vector<float> best(variants.size(), 3.4e38f);
  drb_status st = DRB_OK;
  for (int round = 0; round < 2 && st == DRB_OK; round++)
    for (size_t i = 0; i < variants.size() && st == DRB_OK; i++) {
      if ((st = rebuild(variants[i])) != DRB_OK)
        break;
      for (int w = 0; w < 3 && st == DRB_OK; w++)
        st = colsplit_launch(A, xb.p, yb.p, s);
      cudaEventRecord(e0, s);
      for (int r = 0; r < 3 && st == DRB_OK; r++)
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
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  DRB_TRY(st);
  const size_t pick = std::min_element(best.begin(), best.end()) - best.begin();
  return rebuild(variants[pick]);
}

} // namespace drb
