// spmv.cu -- CSR SpMV / SpMM kernels for sm_100a and their execution plan.
//
// Replaces the segment loop of csr_row_distribution::local_gemv
// (include/dr/mp/containers/matrix_formats/csr_row_distribution.hpp:63-134)
// and csr_eq_distribution::local_gemv (csr_eq_distribution.hpp:54-131): all
// segments of the matrix are resident on one GPU and one launch covers them.
//
// The reference's GPU kernel gives each (row, rhs) a 32-item work-group that
// strides the row and atomically adds its partial into y.  Here the rows are
// binned by length into CTA work items ("row blocks", built once per matrix):
//   * tile   : consecutive short rows whose nnz span fits TILE elements.  The
//              CTA streams the span with 16-byte vector loads of colind and
//              values (evict-first), gathers x (L2 evict-last), stages the
//              products in shared memory and reduces each row with a group of
//              1..32 lanes sized to the row count (shuffle reduction);
//   * long   : one row longer than a tile: the whole CTA loops over it and
//              reduces with warp shuffles and shared memory;
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

template <class T> union Vec16 {
  uint4 u;
  T t[16 / sizeof(T)];
};

template <class T, int G>
__device__ __forceinline__ void load_group(const T *p, T (&out)[G],
                                           uint64_t pol) {
  constexpr int PER = 16 / sizeof(T);
  constexpr int NV = G / PER;
#pragma unroll
  for (int v = 0; v < NV; v++) {
    Vec16<T> r;
    r.u = ptx::ld_stream16(p + v * PER, pol);
#pragma unroll
    for (int i = 0; i < PER; i++)
      out[v * PER + i] = r.t[i];
  }
}

template <class V> __device__ __forceinline__ V warp_sum(V v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1)
    v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

// Sum over the CTA; the result is valid in thread 0.
template <class V, int NT> __device__ __forceinline__ V block_sum(V v, V *s_red) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0)
    s_red[warp] = v;
  __syncthreads();
  V t = 0;
  if (warp == 0) {
    t = lane < NT / 32 ? s_red[lane] : V(0);
    t = warp_sum(t);
  }
  return t;
}

// Products of one range [lo, hi) of a row (G-aligned group walk), summed per
// thread in a fixed order.
template <class V, class CI, int NT, int G, int U>
__device__ __forceinline__ V range_dot(const CI *__restrict__ colind,
                                       const V *__restrict__ vals,
                                       const V *__restrict__ x, int64_t lo,
                                       int64_t hi, uint64_t pol_s,
                                       uint64_t pol_x) {
  const int64_t a0 = lo & ~(int64_t)(G - 1);
  const int64_t ng = (hi - a0 + G - 1) / G;
  V acc = 0;
  for (int64_t gb = 0; gb < ng; gb += (int64_t)U * NT) {
    V v[U][G];
    CI c[U][G];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int64_t g = gb + threadIdx.x + (int64_t)u * NT;
      if (g < ng) {
        load_group<V, G>(vals + a0 + g * G, v[u], pol_s);
        load_group<CI, G>(colind + a0 + g * G, c[u], pol_s);
      }
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int64_t g = gb + threadIdx.x + (int64_t)u * NT;
      if (g < ng) {
#pragma unroll
        for (int i = 0; i < G; i++) {
          const int64_t q = a0 + g * G + i;
          if (q >= lo && q < hi)
            acc += v[u][i] * ptx::ld_keep(x + c[u][i], pol_x);
        }
      }
    }
  }
  return acc;
}

struct ResidArgs {
  const void *b = nullptr;   // right-hand side b (value type)
  double *partials = nullptr; // one per CTA
  int *ticket = nullptr;
  double *out = nullptr;
};

template <class V, class CI, class RI, int NT, int TILE, bool RESID>
__global__ void __launch_bounds__(NT)
    spmv_rowblocks(const RI *__restrict__ rowptr, const CI *__restrict__ colind,
                   const V *__restrict__ vals, const V *__restrict__ x,
                   V *__restrict__ y, const int2 *__restrict__ blocks,
                   const Chunk *__restrict__ chunks, V *partials,
                   int *counters, ResidArgs ra) {
  constexpr int G = 16 / (sizeof(V) < sizeof(CI) ? sizeof(V) : sizeof(CI));
  constexpr int U = TILE / (G * NT);
  static_assert(U >= 1 && TILE % (G * NT) == 0, "tile/group mismatch");
  __shared__ V s_prod[TILE];
  __shared__ int s_rp[kRowsMax + 1];
  __shared__ V s_red[NT / 32];
  __shared__ double s_red_d[NT / 32];
  __shared__ int s_last;

  const uint64_t pol_s = ptx::policy_evict_first();
  const uint64_t pol_x = ptx::policy_evict_last();
  const int tid = threadIdx.x;
  const int2 blk = blocks[blockIdx.x];
  double r2 = 0.0;
  const V *bvec = static_cast<const V *>(ra.b);

  if (blk.y > 0) {
    // ---- tile of short rows ----
    const int r0 = blk.x, nrows = blk.y - blk.x;
    const int64_t p0 = (int64_t)rowptr[r0];
    const int64_t a0 = p0 & ~(int64_t)(G - 1);
    const int64_t p1 = (int64_t)rowptr[blk.y];
    for (int i = tid; i <= nrows; i += NT)
      s_rp[i] = (int)((int64_t)rowptr[r0 + i] - a0);
    const int ng = (int)((p1 - a0 + G - 1) / G);
    V v[U][G];
    CI c[U][G];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int g = tid + u * NT;
      if (g < ng) {
        load_group<V, G>(vals + a0 + (int64_t)g * G, v[u], pol_s);
        load_group<CI, G>(colind + a0 + (int64_t)g * G, c[u], pol_s);
      }
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int g = tid + u * NT;
      if (g < ng) {
#pragma unroll
        for (int i = 0; i < G; i++) {
          const int64_t q = a0 + (int64_t)g * G + i;
          V prod = 0;
          if (q >= p0 && q < p1)
            prod = v[u][i] * ptx::ld_keep(x + c[u][i], pol_x);
          s_prod[g * G + i] = prod;
        }
      }
    }
    __syncthreads();
    int tpr = 1;
    while (tpr < 32 && tpr * 2 * nrows <= NT)
      tpr <<= 1;
    const int ngroups = NT / tpr, gid = tid / tpr, lane = tid & (tpr - 1);
    const int iters = (nrows + ngroups - 1) / ngroups;
    for (int it = 0; it < iters; it++) {
      const int r = gid + it * ngroups;
      V acc = 0;
      if (r < nrows) {
        const int b = s_rp[r], e = s_rp[r + 1];
        for (int q = b + lane; q < e; q += tpr)
          acc += s_prod[q];
      }
      for (int off = tpr >> 1; off > 0; off >>= 1)
        acc += __shfl_down_sync(0xffffffffu, acc, off, tpr);
      if (r < nrows && lane == 0) {
        y[r0 + r] = acc;
        if (RESID) {
          const double d = (double)acc - (double)bvec[r0 + r];
          r2 += d * d;
        }
      }
    }
  } else if (blk.y == -1) {
    // ---- one long row, whole CTA ----
    const int row = blk.x;
    const int64_t p0 = (int64_t)rowptr[row], p1 = (int64_t)rowptr[row + 1];
    V acc = range_dot<V, CI, NT, G, U>(colind, vals, x, p0, p1, pol_s, pol_x);
    acc = block_sum<V, NT>(acc, s_red);
    if (tid == 0) {
      y[row] = acc;
      if (RESID) {
        const double d = (double)acc - (double)bvec[row];
        r2 += d * d;
      }
    }
  } else {
    // ---- one chunk of a very long row ----
    const int ci = -blk.y - 2;
    const Chunk ch = chunks[ci];
    V acc = range_dot<V, CI, NT, G, U>(colind, vals, x, ch.p0, ch.p1, pol_s,
                                       pol_x);
    acc = block_sum<V, NT>(acc, s_red);
    if (tid == 0) {
      partials[ci] = acc;
      __threadfence();
      const int t = atomicAdd(&counters[ch.counter], 1);
      if (t == ch.count - 1) {
        __threadfence();
        V s = 0;
        for (int i = 0; i < ch.count; i++)
          s += *(volatile V *)&partials[ch.first + i];
        y[ch.row] = s;
        counters[ch.counter] = 0; // ready for the next launch
        if (RESID) {
          const double d = (double)s - (double)bvec[ch.row];
          r2 += d * d;
        }
      }
    }
  }

  if (RESID) {
    // Deterministic two-level reduction of the squared residual: one partial
    // per CTA, summed in CTA order by the CTA that finishes last.
    r2 = block_sum<double, NT>(r2, s_red_d);
    if (tid == 0) {
      ra.partials[blockIdx.x] = r2;
      __threadfence();
      const int t = atomicAdd(ra.ticket, 1);
      s_last = (t == (int)gridDim.x - 1);
    }
    __syncthreads();
    if (s_last) {
      __threadfence();
      double s = 0.0;
      for (int i = tid; i < (int)gridDim.x; i += NT)
        s += *(volatile double *)&ra.partials[i];
      s = block_sum<double, NT>(s, s_red_d);
      if (tid == 0) {
        *ra.out = s;
        *ra.ticket = 0;
      }
    }
  }
}

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
                        const ResidArgs *ra, cudaStream_t s) {
  Plan &P = A.plan;
  if (P.nblocks == 0)
    return DRB_OK;
  const RI *rp = A.rowptr.as<RI>();
  const CI *ci = A.colind.as<CI>();
  const V *va = A.vals.as<V>();
  auto blocks = P.blocks.as<int2>();
  auto chunks = P.chunks.as<Chunk>();
  if (k == 1) {
    DRB_TRY(P.partials.ensure(sizeof(V) * std::max<int64_t>(P.nchunks, 1)));
    if (ra) {
      spmv_rowblocks<V, CI, RI, kNT, kTile, true><<<(unsigned)P.nblocks, kNT, 0, s>>>(
          rp, ci, va, x, y, blocks, chunks, P.partials.as<V>(),
          P.counters.as<int>(), *ra);
    } else {
      spmv_rowblocks<V, CI, RI, kNT, kTile, false><<<(unsigned)P.nblocks, kNT, 0, s>>>(
          rp, ci, va, x, y, blocks, chunks, P.partials.as<V>(),
          P.counters.as<int>(), ResidArgs{});
    }
    note_launch();
    DRB_CUDA_TRY(cudaGetLastError());
    return DRB_OK;
  }
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
                        drb_layout layout, const ResidArgs *ra,
                        cudaStream_t s) {
  auto X = static_cast<const V *>(x);
  auto Y = static_cast<V *>(y);
  if (A.cbytes == 4 && A.rbytes == 4)
    return launch_typed<V, int32_t, int32_t>(A, X, Y, k, layout, ra, s);
  if (A.cbytes == 4 && A.rbytes == 8)
    return launch_typed<V, int32_t, int64_t>(A, X, Y, k, layout, ra, s);
  if (A.cbytes == 8 && A.rbytes == 4)
    return launch_typed<V, int64_t, int32_t>(A, X, Y, k, layout, ra, s);
  return launch_typed<V, int64_t, int64_t>(A, X, Y, k, layout, ra, s);
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
    return spmv_pipe_launch(A, x, y, s);
  switch (A.storage) {
  case DRB_F32:
    return dispatch_idx<float>(A, x, y, k, layout, nullptr, s);
  case DRB_F64:
    return dispatch_idx<double>(A, x, y, k, layout, nullptr, s);
  default:
    set_error("storage type not handled by spmv_launch");
    return DRB_ERR_UNSUPPORTED;
  }
}

drb_status residual_launch(Csr &A, const void *x, const void *b, void *y,
                           double *out, cudaStream_t s) {
  if (A.storage == DRB_F32 || A.storage == DRB_F64) {
    void *yt = y;
    if (!yt) {
      DRB_TRY(A.ys.ensure((size_t)dtype_bytes(A.storage) * A.m));
      yt = A.ys.p;
    }
    return residual_pipe_launch(A, x, b, yt, out, s);
  }
  Plan &P = A.plan;
  if (P.nblocks == 0) {
    DRB_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(double), s));
    return DRB_OK;
  }
  if (!P.red.p) {
    DRB_TRY(P.red.alloc(sizeof(double) * P.nblocks + 16));
    DRB_CUDA_TRY(cudaMemset(P.red.p, 0, P.red.bytes));
  }
  void *ytmp = y;
  if (!ytmp) {
    DRB_TRY(A.ys.ensure((size_t)dtype_bytes(A.storage) * A.m));
    ytmp = A.ys.p;
  }
  ResidArgs ra;
  ra.b = b;
  ra.partials = P.red.as<double>();
  ra.ticket = reinterpret_cast<int *>(P.red.as<double>() + P.nblocks);
  ra.out = out;
  switch (A.storage) {
  case DRB_F32:
    return dispatch_idx<float>(A, x, ytmp, 1, DRB_COL_MAJOR, &ra, s);
  case DRB_F64:
    return dispatch_idx<double>(A, x, ytmp, 1, DRB_COL_MAJOR, &ra, s);
  default:
    set_error("storage type not handled by residual_launch");
    return DRB_ERR_UNSUPPORTED;
  }
}

} // namespace drb
