// spmv.cu -- multi-RHS CSR SpMM of one handle, its row-block plan, and the
// gemv / residual entry dispatch.
//
// Replaces the segment loop of csr_row_distribution::local_gemv
// (include/dr/mp/containers/matrix_formats/csr_row_distribution.hpp:63-134)
// and csr_eq_distribution::local_gemv (csr_eq_distribution.hpp:54-131): all
// segments of the matrix are resident on one GPU and one launch covers them.
// One right-hand side (k = 1) and the fused residual run the persistent warp
// kernel (spmv_warp.cu); k > 1 runs the batched SpMM kernel on a batch of the
// one handle (batch.cu), or, for what a batch does not take (64-bit indices,
// misaligned row-major X), spmm_rowblocks below over CTA work items ("row
// blocks", built once per matrix):
//   * rows   : consecutive short rows, one warp per row;
//   * long   : one row longer than a tile: the whole CTA loops over it;
//   * chunk  : a row longer than long_max is split into chunks; each CTA
//              writes its partial, and the CTA that finishes last (ticket
//              counter) adds the partials in chunk order.
// No atomics touch y, and every sum has a fixed order, so results are
// deterministic run to run.
#include <algorithm>
#include <cstring>

#include "drb_internal.cuh"

namespace drb {
namespace {

constexpr int kNT = 256;     // threads per CTA
constexpr int kTile = 2048;  // nnz span of a tile
constexpr int kRowsMax = 2048;
constexpr int kLongMax = 65536; // longer rows are chunked

// ---- multi-RHS: X row-major [n][k], one warp per row --------------------------
// Lanes are split into S = 32/KP slots of KP lanes; a slot takes one nonzero
// and its KP lanes read KP consecutive right-hand sides of x's row (one
// coalesced 4*KP-byte gather), so each nonzero's column and value are loaded
// once for all k right-hand sides.
template <class V, class CI>
__device__ __forceinline__ V warp_range_rhs(const CI *__restrict__ colind,
                                            const V *__restrict__ vals,
                                            const V *__restrict__ X, int64_t k,
                                            int64_t jb, int64_t lo, int64_t hi,
                                            int64_t first, int64_t stride,
                                            int KP, uint64_t pol_x) {
  const int lane = threadIdx.x & 31;
  const int S = 32 / KP, slot = lane / KP, jj = lane % KP;
  const bool jok = jb + jj < k;
  V acc = 0;
  for (int64_t base = lo + first; base < hi; base += stride) {
    const int cnt = (int)min((int64_t)32, hi - base);
    CI my_c = 0;
    V my_v = 0;
    if (lane < cnt) {
      my_c = colind[base + lane];
      my_v = vals[base + lane];
    }
    for (int t = 0; t < cnt; t += S) {
      const int src = t + slot;
      const CI c = __shfl_sync(0xffffffffu, my_c, src & 31);
      const V v = __shfl_sync(0xffffffffu, my_v, src & 31);
      if (src < cnt && jok)
        acc += v * ptx::ld_keep(X + (int64_t)c * k + jb + jj, pol_x);
    }
  }
  for (int off = KP; off < 32; off <<= 1)
    acc += __shfl_xor_sync(0xffffffffu, acc, off);
  return acc;
}

template <class V, class CI, class RI, int NT>
__global__ void __launch_bounds__(NT)
    spmm_rowblocks(const RI *__restrict__ rowptr, const CI *__restrict__ colind,
                   const V *__restrict__ vals, const V *__restrict__ X,
                   V *__restrict__ Y, int64_t m, int64_t k, int y_row_major,
                   const int2 *__restrict__ blocks,
                   const Chunk *__restrict__ chunks, V *partials,
                   int *counters) {
  constexpr int NW = NT / 32;
  __shared__ V s_part[NW][32];
  __shared__ int s_last;
  const uint64_t pol_x = ptx::policy_evict_last();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int KP = 1;
  while (KP < 32 && KP < k)
    KP <<= 1;
  const int jj = lane % KP, slot = lane / KP;
  auto store = [&](int64_t r, int64_t j, V v) {
    if (y_row_major)
      Y[r * k + j] = v;
    else
      Y[r + j * m] = v;
  };
  const int2 blk = blocks[blockIdx.x];
  if (blk.y > 0) {
    for (int64_t r = blk.x + warp; r < blk.y; r += NW) {
      const int64_t p0 = (int64_t)rowptr[r], p1 = (int64_t)rowptr[r + 1];
      for (int64_t jb = 0; jb < k; jb += KP) {
        const V acc =
            warp_range_rhs<V, CI>(colind, vals, X, k, jb, p0, p1, 0, 32, KP,
                                  pol_x);
        if (slot == 0 && jb + jj < k)
          store(r, jb + jj, acc);
      }
    }
    return;
  }
  int64_t lo, hi, row;
  int ci = -1;
  Chunk ch{};
  if (blk.y == -1) {
    row = blk.x;
    lo = (int64_t)rowptr[row];
    hi = (int64_t)rowptr[row + 1];
  } else {
    ci = -blk.y - 2;
    ch = chunks[ci];
    row = ch.row;
    lo = ch.p0;
    hi = ch.p1;
  }
  for (int64_t jb = 0; jb < k; jb += KP) {
    V acc = warp_range_rhs<V, CI>(colind, vals, X, k, jb, lo, hi,
                                  (int64_t)warp * 32, (int64_t)NW * 32, KP,
                                  pol_x);
    __syncthreads();
    if (slot == 0)
      s_part[warp][jj] = acc;
    __syncthreads();
    if (warp == 0 && lane < KP && jb + lane < k) {
      V s = 0;
      for (int w = 0; w < NW; w++)
        s += s_part[w][lane];
      if (ci < 0)
        store(row, jb + lane, s);
      else
        partials[(int64_t)ci * k + jb + lane] = s;
    }
  }
  if (ci >= 0) {
    __threadfence(); // every lane that wrote a partial publishes it
    __syncthreads();
    if (threadIdx.x == 0) {
      const int t = atomicAdd(&counters[ch.counter], 1);
      s_last = (t == ch.count - 1);
    }
    __syncthreads();
    if (s_last) {
      __threadfence();
      for (int64_t j = threadIdx.x; j < k; j += NT) {
        V s = 0;
        for (int i = 0; i < ch.count; i++)
          s += *(volatile V *)&partials[(int64_t)(ch.first + i) * k + j];
        store(row, j, s);
      }
      __syncthreads();
      if (threadIdx.x == 0)
        counters[ch.counter] = 0;
    }
  }
}

template <class V, class CI, class RI>
drb_status launch_typed(Csr &A, const V *x, V *y, int64_t k, drb_layout layout,
                        cudaStream_t s) {
  Plan &P = A.plan;
  if (P.nblocks == 0)
    return DRB_OK;
  const RI *rp = A.rowptr.as<RI>();
  const CI *ci = A.colind.as<CI>();
  const V *va = A.vals.as<V>();
  auto blocks = P.blocks.as<int2>();
  auto chunks = P.chunks.as<Chunk>();
  // k > 1: gather from a row-major copy of X.
  const V *Xr = x;
  if (layout == DRB_COL_MAJOR) {
    DRB_TRY(A.xs.ensure(sizeof(V) * (size_t)A.n * k));
    DRB_TRY(transpose_launch(x, A.xs.p, k, A.n, sizeof(V), s));
    Xr = A.xs.as<V>();
  }
  DRB_TRY(P.partials.ensure(sizeof(V) * std::max<int64_t>(P.nchunks * k, 1)));
  spmm_rowblocks<V, CI, RI, kNT><<<(unsigned)P.nblocks, kNT, 0, s>>>(
      rp, ci, va, Xr, y, A.m, k, layout == DRB_ROW_MAJOR ? 1 : 0, blocks,
      chunks, P.partials.as<V>(), P.counters.as<int>());
  note_launch();
  DRB_CUDA_TRY(cudaGetLastError());
  return DRB_OK;
}

template <class V>
drb_status dispatch_idx(Csr &A, const void *x, void *y, int64_t k,
                        drb_layout layout, cudaStream_t s) {
  auto X = static_cast<const V *>(x);
  auto Y = static_cast<V *>(y);
  if (A.cbytes == 4 && A.rbytes == 4)
    return launch_typed<V, int32_t, int32_t>(A, X, Y, k, layout, s);
  if (A.cbytes == 4 && A.rbytes == 8)
    return launch_typed<V, int32_t, int64_t>(A, X, Y, k, layout, s);
  if (A.cbytes == 8 && A.rbytes == 4)
    return launch_typed<V, int64_t, int32_t>(A, X, Y, k, layout, s);
  return launch_typed<V, int64_t, int64_t>(A, X, Y, k, layout, s);
}

} // namespace

int plan_group(int vbytes, int cbytes) {
  return 16 / std::min(vbytes, cbytes);
}

drb_status build_plan(Plan &plan, int64_t m, const void *rowptr_host,
                      int rbytes, int group, int tile, int rows_max,
                      int long_max) {
  if (tile <= 0)
    tile = kTile;
  if (rows_max <= 0)
    rows_max = kRowsMax;
  if (long_max <= 0)
    long_max = kLongMax;
  rows_max = std::min(rows_max, kRowsMax);
  plan.tile = tile;
  plan.rows_max = rows_max;
  plan.long_max = long_max;
  plan.group = group;
  auto RP = [&](int64_t i) -> int64_t {
    return rbytes == 4 ? (int64_t)((const int32_t *)rowptr_host)[i]
                       : ((const int64_t *)rowptr_host)[i];
  };
  const int64_t G = group;
  const int64_t CH = (long_max / G) * G; // chunk span, multiple of G
  std::vector<int2> longb, tiles;
  std::vector<Chunk> chunks;
  int64_t nsplit = 0;
  int64_t r = 0;
  while (r < m) {
    const int64_t p0 = RP(r), a0 = p0 & ~(G - 1), p1 = RP(r + 1);
    if (p1 - a0 > tile) {
      if (p1 - p0 <= long_max) {
        longb.push_back(make_int2((int)r, -1));
      } else {
        const int64_t nch = (p1 - a0 + CH - 1) / CH;
        const int first = (int)chunks.size();
        for (int64_t i = 0; i < nch; i++) {
          Chunk c;
          c.p0 = std::max(p0, a0 + i * CH);
          c.p1 = std::min(p1, a0 + (i + 1) * CH);
          c.row = (int32_t)r;
          c.first = first;
          c.count = (int32_t)nch;
          c.counter = (int32_t)nsplit;
          chunks.push_back(c);
          longb.push_back(make_int2((int)r, -(first + (int)i) - 2));
        }
        nsplit++;
      }
      r++;
      continue;
    }
    int64_t r1 = r + 1;
    while (r1 < m && r1 - r < rows_max && RP(r1 + 1) - a0 <= tile)
      r1++;
    tiles.push_back(make_int2((int)r, (int)r1));
    r = r1;
  }
  // Long rows first: they are the longest-running CTAs.
  std::vector<int2> all;
  all.reserve(longb.size() + tiles.size());
  all.insert(all.end(), longb.begin(), longb.end());
  all.insert(all.end(), tiles.begin(), tiles.end());
  plan.nblocks = (int64_t)all.size();
  plan.nchunks = (int64_t)chunks.size();
  plan.nsplit = nsplit;
  if (plan.nblocks > 0x7fffffff) {
    set_error("plan has too many row blocks (%lld)", (long long)plan.nblocks);
    return DRB_ERR_UNSUPPORTED;
  }
  if (plan.nblocks) {
    DRB_TRY(plan.blocks.alloc(sizeof(int2) * all.size()));
    DRB_CUDA_TRY(cudaMemcpy(plan.blocks.p, all.data(), sizeof(int2) * all.size(),
                            cudaMemcpyHostToDevice));
  }
  DRB_TRY(plan.chunks.alloc(sizeof(Chunk) * std::max<size_t>(chunks.size(), 1)));
  if (!chunks.empty())
    DRB_CUDA_TRY(cudaMemcpy(plan.chunks.p, chunks.data(),
                            sizeof(Chunk) * chunks.size(),
                            cudaMemcpyHostToDevice));
  DRB_TRY(plan.counters.alloc(sizeof(int) * std::max<int64_t>(nsplit, 1)));
  DRB_CUDA_TRY(cudaMemset(plan.counters.p, 0, plan.counters.bytes));
  return DRB_OK;
}

drb_status spmv_launch(Csr &A, const void *x, void *y, int64_t k,
                       drb_layout layout, cudaStream_t s) {
  if (k == 1)
    return (A.csplit && !A.sell.on) ? colsplit_launch(A, x, y, s)
                                    : spmv_pipe_launch(A, x, y, s);
  // k > 1: the batched SpMM kernel on a batch of this one handle (2.0-2.3x
  // the row-block kernel below at k = 2..20 on 4M-row and 16.8M-row
  // matrices); the row-block kernel covers what a batch does not take
  bool used = false;
  DRB_TRY(multi_rhs_batch_launch(A, x, y, k, layout, s, &used));
  if (used)
    return DRB_OK;
  switch (A.storage) {
  case DRB_F32:
    return dispatch_idx<float>(A, x, y, k, layout, s);
  case DRB_F64:
    return dispatch_idx<double>(A, x, y, k, layout, s);
  default:
    set_error("multi-RHS gemv with 64-bit indices or a misaligned row-major x takes F32 or "
              "F64 storage");
    return DRB_ERR_UNSUPPORTED;
  }
}

drb_status residual_launch(Csr &A, const void *x, const void *b, void *y,
                           double *out, cudaStream_t s) {
  if (!y) {
    DRB_TRY(A.ys.ensure((size_t)dtype_bytes(A.storage) * A.m));
    y = A.ys.p;
  }
  if (A.csplit && !A.sell.on && A.m > 0)
    return colsplit_residual(A, x, b, y, out, s);
  return residual_pipe_launch(A, x, b, y, out, s);
}

} // namespace drb
