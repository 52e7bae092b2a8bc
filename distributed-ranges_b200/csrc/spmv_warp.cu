// spmv_warp.cu -- persistent warp-granular CSR SpMV (one right-hand side).
//
// The matrix is cut once (build_pipe_plan) into work items of at most TILE
// nonzeros counted from a 16-byte aligned start: up to kRows whole short rows,
// or one fixed-size chunk of a long row.  Every warp of the grid owns the items
// w, w + W, w + 2W, ... (W = warps in the grid) and runs them with no CTA-wide
// barrier, so warps progress independently.
//
// For its current item every lane holds TILE/32 nonzeros in registers
// (16-byte vector loads of colind and values, evict-first L2 policy), gathers
// x for all of them at once (evict-last L2 policy keeps x resident), stores
// the products to its warp's shared-memory slice, and immediately reloads the
// registers with its next item; the current item's rows are then summed from
// shared memory while the next item's loads are in flight.  Products are stored skewed
// (element q at q + q/32) so lanes that sum different rows hit different
// banks; rows are summed by 1..32 lanes each (shuffles).
//
// On B200 the random x gathers are bounded by the SM's L1-to-crossbar request
// rate (about one request per SM per clock); the design keeps many gathers in
// flight per warp and as many warps as registers allow.
//
// A chunked long row writes one partial per chunk; the warp that completes
// the last chunk (ticket counter) adds the partials in chunk order.  Every sum
// has a fixed order, so results are deterministic.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "drb_internal.cuh"

namespace drb {
namespace {

constexpr int kRows = 64;  // rows of a whole-row item (<= 64: three rowptr regs)
constexpr int kWarps = 8;  // warps per CTA
constexpr int kThreads = kWarps * 32;

template <class T> union Vec16 {
  uint4 u;
  T t[16 / sizeof(T)];
};

template <class T, int G>
__device__ __forceinline__ void ld_group(const T *p, T (&out)[G], uint64_t pol) {
  constexpr int PER = 16 / sizeof(T);
#pragma unroll
  for (int v = 0; v < G / PER; v++) {
    Vec16<T> r;
    r.u = ptx::ld_stream16(p + v * PER, pol);
#pragma unroll
    for (int i = 0; i < PER; i++)
      out[v * PER + i] = r.t[i];
  }
}

template <class V> __device__ __forceinline__ V wsum(V v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1)
    v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

__device__ __forceinline__ Item load_item(const Item *items, int64_t i) {
  const int4 *p = reinterpret_cast<const int4 *>(items + i);
  const int4 a = __ldg(p), b = __ldg(p + 1);
  Item d;
  d.p0 = (int64_t)(((uint64_t)(uint32_t)a.y << 32) | (uint32_t)a.x);
  d.len = a.z;
  d.r0 = a.w;
  d.nrows = b.x;
  d.chunk = b.y;
  d.pad0 = d.pad1 = 0;
  return d;
}

__device__ __forceinline__ int skew(int q) { return q + (q >> 5); }

// Fused ||A x - b||^2: whole rows add into a per-CTA partial; a chunked row's
// square goes to its own slot because which warp finishes it varies run to
// run.  The last CTA sums partials[0..grid) then rowres[0..nsplit) in order.
struct WarpResid {
  const void *b = nullptr;
  double *partials = nullptr;
  double *rowres = nullptr;
  int64_t nsplit = 0;
  int *ticket = nullptr;
  double *out = nullptr;
};

template <class V, class CI, int TILE> struct Slot {
  static constexpr int G = 16 / (sizeof(V) < sizeof(CI) ? sizeof(V) : sizeof(CI));
  static constexpr int NG = TILE / (G * 32);
  static_assert(NG >= 1 && TILE % (G * 32) == 0, "tile/group");
  V v[NG][G];
  CI c[NG][G];
  Item d;
  int64_t a0;
  int rp0, rp1, rp2;
  bool valid;
};

template <class V, class CI, class RI, int TILE, bool SKEW>
struct Kern {
  using S = Slot<V, CI, TILE>;
  static constexpr int G = S::G, NG = S::NG;
  const RI *__restrict__ rowptr;
  const CI *__restrict__ colind;
  const V *__restrict__ vals;
  const V *__restrict__ x;
  V *__restrict__ y;
  const Item *__restrict__ items;
  int64_t nitems;
  const Chunk *__restrict__ chunks;
  V *partials;
  int *counters;
  uint64_t pol_s, pol_x;
  int lane;

  __device__ __forceinline__ void fetch(S &sl, int64_t i) {
    sl.valid = i < nitems;
    if (!sl.valid)
      return;
    sl.d = load_item(items, i);
    sl.a0 = sl.d.p0 & ~(int64_t)(G - 1);
    const int ng = (int)((sl.d.p0 + sl.d.len - sl.a0 + G - 1) / G);
#pragma unroll
    for (int j = 0; j < NG; j++) {
      const int g = lane + 32 * j;
      if (g < ng) {
        ld_group<V, G>(vals + sl.a0 + (int64_t)g * G, sl.v[j], pol_s);
        ld_group<CI, G>(colind + sl.a0 + (int64_t)g * G, sl.c[j], pol_s);
      }
    }
    if (sl.d.nrows > 0) {
      // rowptr[r0 .. r0 + nrows] relative to a0 (nrows <= kRows = 64)
      const int64_t r0 = sl.d.r0;
      if (lane <= sl.d.nrows)
        sl.rp0 = (int)((int64_t)rowptr[r0 + lane] - sl.a0);
      if (lane + 32 <= sl.d.nrows)
        sl.rp1 = (int)((int64_t)rowptr[r0 + lane + 32] - sl.a0);
      if (lane == 0 && 64 <= sl.d.nrows)
        sl.rp2 = (int)((int64_t)rowptr[r0 + 64] - sl.a0);
    }
  }

  // Runs the item in `sl` (index it) and refills the slot with item `refill`.
  template <bool RESID>
  __device__ __forceinline__ void process(S &sl, int64_t refill, V *prod, int *srp,
                                          const V *bvec, double &r2, double *rowres) {
    const Item cur = sl.d;
    const int off = (int)(cur.p0 - sl.a0), end = off + cur.len;
    const int ng = (end + G - 1) / G;
    V xg[NG][G];
#pragma unroll
    for (int j = 0; j < NG; j++) {
      const int g = lane + 32 * j;
#pragma unroll
      for (int i = 0; i < G; i++) {
        const int q = g * G + i;
        xg[j][i] = (g < ng && q >= off && q < end) ? ptx::ld_keep(x + sl.c[j][i], pol_x) : V(0);
      }
    }
    if (cur.nrows == 0) {
      // one chunk of a long row: sum in registers, no shared memory
      V acc = 0;
#pragma unroll
      for (int j = 0; j < NG; j++) {
        const int g = lane + 32 * j;
#pragma unroll
        for (int i = 0; i < G; i++) {
          const int q = g * G + i;
          if (g < ng && q >= off && q < end)
            acc += sl.v[j][i] * xg[j][i];
        }
      }
      fetch(sl, refill);
      acc = wsum(acc);
      if (lane == 0)
        this->template finish_chunk<RESID>(cur, acc, bvec, rowres);
      return;
    }
#pragma unroll
    for (int j = 0; j < NG; j++) {
      const int g = lane + 32 * j;
      if (g < ng) {
        if (SKEW) {
#pragma unroll
          for (int i = 0; i < G; i++)
            prod[skew(g * G + i)] = sl.v[j][i] * xg[j][i];
        } else {
          constexpr int PER = 16 / sizeof(V);
#pragma unroll
          for (int h = 0; h < G / PER; h++) {
            Vec16<V> w;
#pragma unroll
            for (int i = 0; i < PER; i++)
              w.t[i] = sl.v[j][h * PER + i] * xg[j][h * PER + i];
            *reinterpret_cast<uint4 *>(prod + g * G + h * PER) = w.u;
          }
        }
      }
    }
    if (lane <= cur.nrows)
      srp[lane] = sl.rp0;
    if (lane + 32 <= cur.nrows)
      srp[lane + 32] = sl.rp1;
    if (lane == 0 && 64 <= cur.nrows)
      srp[64] = sl.rp2;
    __syncwarp();
    fetch(sl, refill); // the slot's registers are free again

    const int nrows = cur.nrows;
    int tpr = 1;
    while (tpr < 32 && tpr * 2 * nrows <= 32)
      tpr <<= 1;
    const int groups = 32 / tpr, gid = lane / tpr, gl = lane & (tpr - 1);
    for (int base = 0; base < nrows; base += groups) {
      const int r = base + gid;
      V acc = 0;
      if (r < nrows) {
        const int b = srp[r], e = srp[r + 1];
        for (int q = b + gl; q < e; q += tpr)
          acc += prod[SKEW ? skew(q) : q];
      }
      for (int o = tpr >> 1; o > 0; o >>= 1)
        acc += __shfl_down_sync(0xffffffffu, acc, o, tpr);
      if (r < nrows && gl == 0) {
        y[cur.r0 + r] = acc;
        if (RESID) {
          const double dd = (double)acc - (double)bvec[cur.r0 + r];
          r2 += dd * dd;
        }
      }
    }
    __syncwarp(); // the shared slice is rewritten by the next item
  }

  // Lane 0 after a chunk: publish the partial; the last chunk of the row
  // adds all partials in chunk order and writes y.
  template <bool RESID>
  __device__ __forceinline__ void finish_chunk(const Item &cur, V acc, const V *bvec,
                                               double *rowres) {
    const Chunk ch = chunks[cur.chunk];
    partials[cur.chunk] = acc;
    __threadfence();
    const int t = atomicAdd(&counters[ch.counter], 1);
    if (t == ch.count - 1) {
      __threadfence();
      V sum = 0;
      for (int i = 0; i < ch.count; i++)
        sum += *(volatile V *)&partials[ch.first + i];
      y[ch.row] = sum;
      counters[ch.counter] = 0; // re-armed for the next launch
      if (RESID) {
        const double dd = (double)sum - (double)bvec[ch.row];
        rowres[ch.counter] = dd * dd;
      }
    }
  }
};

template <class V, class CI, class RI, int TILE, bool SKEW, bool RESID>
__global__ void __launch_bounds__(kThreads)
    spmv_warp(const RI *__restrict__ rowptr, const CI *__restrict__ colind,
              const V *__restrict__ vals, const V *__restrict__ x,
              V *__restrict__ y, const Item *__restrict__ items, int64_t nitems,
              const Chunk *__restrict__ chunks, V *partials, int *counters,
              WarpResid ra) {
  __shared__ __align__(16) V s_prod[kWarps][TILE + TILE / 32];
  __shared__ int s_rp[kWarps][kRows + 1];
  __shared__ double s_red[kWarps];
  __shared__ int s_last;

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  Kern<V, CI, RI, TILE, SKEW> K{rowptr, colind, vals, x, y, items, nitems, chunks, partials,
                          counters, ptx::policy_evict_first(), ptx::policy_evict_last(),
                          lane};
  const int64_t nw = (int64_t)gridDim.x * kWarps;
  int64_t it = (int64_t)blockIdx.x * kWarps + warp;
  const V *bvec = static_cast<const V *>(ra.b);
  double r2 = 0.0;
  V *prod = s_prod[warp];
  int *srp = s_rp[warp];

  Slot<V, CI, TILE> A;
  K.fetch(A, it);
  while (A.valid) {
    K.template process<RESID>(A, it + nw, prod, srp, bvec, r2, ra.rowres);
    it += nw;
  }

  if (RESID) {
    const double t = wsum(r2);
    if (lane == 0)
      s_red[warp] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
      double cta = 0.0;
      for (int w = 0; w < kWarps; w++)
        cta += s_red[w];
      ra.partials[blockIdx.x] = cta;
      __threadfence();
      s_last = atomicAdd(ra.ticket, 1) == (int)gridDim.x - 1;
    }
    __syncthreads();
    if (s_last) {
      // The last CTA adds the per-CTA partials and the chunked-row slots with
      // all its threads: fixed strided assignment, then a fixed-order tree.
      __threadfence();
      const int64_t total = (int64_t)gridDim.x + ra.nsplit;
      double sum = 0.0;
      for (int64_t i = threadIdx.x; i < total; i += kThreads)
        sum += i < gridDim.x ? __ldcg(&ra.partials[i]) : __ldcg(&ra.rowres[i - gridDim.x]);
      sum = wsum(sum);
      if (lane == 0)
        s_red[warp] = sum;
      __syncthreads();
      if (threadIdx.x == 0) {
        double t2 = 0.0;
        for (int w = 0; w < kWarps; w++)
          t2 += s_red[w];
        *ra.out = t2;
        *ra.ticket = 0;
      }
    }
  }
}

struct Shape {
  int grid = 0;
  bool ready = false;
};

template <class V, class CI, class RI, int TILE, bool SKEW, bool RESID>
drb_status launch_tile(Csr &A, const V *x, V *y, const WarpResid *ra, cudaStream_t s) {
  PipePlan &P = A.pipe;
  static Shape shape[64];
  auto kern = spmv_warp<V, CI, RI, TILE, SKEW, RESID>;
  const int dev = A.device < 64 ? A.device : 0;
  if (!shape[dev].ready) {
    int occ = 0, sms = 0;
    DRB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kThreads, 0));
    DRB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, A.device));
    shape[dev].grid = std::max(1, occ) * sms;
    shape[dev].ready = true;
  }
  const int64_t need = (P.nitems + kWarps - 1) / kWarps;
  const int grid = (int)std::min<int64_t>(shape[dev].grid, need);
  WarpResid r{};
  if (ra)
    r = *ra;
  kern<<<grid, kThreads, 0, s>>>(A.rowptr.as<RI>(), A.colind.as<CI>(), A.vals.as<V>(), x,
                                 y, P.items.as<Item>(), P.nitems, P.chunks.as<Chunk>(),
                                 P.partials.as<V>(), P.counters.as<int>(), r);
  note_launch();
  DRB_CUDA_TRY(cudaGetLastError());
  return DRB_OK;
}

template <class V, class CI, class RI, bool RESID>
drb_status launch_warp(Csr &A, const V *x, V *y, const WarpResid *ra, cudaStream_t s) {
  if (A.pipe.nitems == 0)
    return DRB_OK;
  const bool skew = A.pipe.skew;
  if (A.pipe.tile == 512)
    return skew ? launch_tile<V, CI, RI, 512, true, RESID>(A, x, y, ra, s)
                : launch_tile<V, CI, RI, 512, false, RESID>(A, x, y, ra, s);
  return skew ? launch_tile<V, CI, RI, 256, true, RESID>(A, x, y, ra, s)
              : launch_tile<V, CI, RI, 256, false, RESID>(A, x, y, ra, s);
}

template <class V, bool RESID>
drb_status warp_idx(Csr &A, const void *x, void *y, const WarpResid *ra,
                    cudaStream_t s) {
  auto X = static_cast<const V *>(x);
  auto Y = static_cast<V *>(y);
  if (A.cbytes == 4 && A.rbytes == 4)
    return launch_warp<V, int32_t, int32_t, RESID>(A, X, Y, ra, s);
  if (A.cbytes == 4 && A.rbytes == 8)
    return launch_warp<V, int32_t, int64_t, RESID>(A, X, Y, ra, s);
  if (A.cbytes == 8 && A.rbytes == 4)
    return launch_warp<V, int64_t, int32_t, RESID>(A, X, Y, ra, s);
  return launch_warp<V, int64_t, int64_t, RESID>(A, X, Y, ra, s);
}

} // namespace

// Kernel variant: item span 256 or 512 nonzeros, skewed or plain product
// layout.  Encoded as tile | (skew ? 1 : 0) in build_pipe_plan's `tile`
// argument (0 = choose).  The choice does not change results beyond the
// summation order of a chunked row, which is the same for both layouts.
//
// Heuristic (measured on B200): rows shorter than a warp of lanes per row
// favour 256-nonzero items with the skewed layout (bank-conflict-free row
// sums); matrices whose nonzeros sit mostly in long rows favour 512-nonzero
// items (fewer chunks) with vector product stores.  The environment variable
// DRB_SPMV_VARIANT="tile,skew" (e.g. "512,0") overrides the heuristic for
// handles created afterwards; drb_csr_autotune measures all four instead.
int choose_pipe_variant(int64_t m, const void *rowptr_host, int rbytes) {
  if (const char *e = std::getenv("DRB_SPMV_VARIANT")) {
    const int t = std::atoi(e);
    const char *c = std::strchr(e, ',');
    const int sk = c ? std::atoi(c + 1) : 0;
    if (t == 256 || t == 512)
      return t | (sk ? 1 : 0);
  }
  auto RP = [&](int64_t i) -> int64_t {
    return rbytes == 4 ? (int64_t)((const int32_t *)rowptr_host)[i]
                       : ((const int64_t *)rowptr_host)[i];
  };
  const int64_t nnz = m > 0 ? RP(m) : 0;
  if (nnz == 0)
    return 256 | 1;
  int64_t in_long = 0;
  for (int64_t r = 0; r < m; r++) {
    const int64_t len = RP(r + 1) - RP(r);
    if (len > 256)
      in_long += len;
  }
  return (double)in_long / (double)nnz > 0.3 ? 512 : (256 | 1);
}

drb_status build_pipe_plan(PipePlan &plan, int64_t m, const void *rowptr_host,
                           int rbytes, int group, int tile, int rows) {
  if (tile == 0)
    tile = choose_pipe_variant(m, rowptr_host, rbytes);
  plan.skew = (tile & 1) != 0;
  tile &= ~1;
  if (tile != 256 && tile != 512)
    tile = 256;
  if (rows <= 0 || rows > kRows)
    rows = kRows;
  plan.tile = tile;
  plan.rows = rows;
  plan.group = group;
  auto RP = [&](int64_t i) -> int64_t {
    return rbytes == 4 ? (int64_t)((const int32_t *)rowptr_host)[i]
                       : ((const int64_t *)rowptr_host)[i];
  };
  const int64_t G = group;
  std::vector<Item> longi, tiles;
  std::vector<Chunk> chunks;
  int64_t nsplit = 0;
  int64_t r = 0;
  while (r < m) {
    const int64_t p0 = RP(r), a0 = p0 & ~(G - 1), p1 = RP(r + 1);
    if (p1 - a0 > tile) {
      // a row wider than one item: aligned chunks of `tile` elements
      const int64_t nch = (p1 - a0 + tile - 1) / tile;
      const int first = (int)chunks.size();
      for (int64_t i = 0; i < nch; i++) {
        Chunk c;
        c.p0 = std::max(p0, a0 + i * tile);
        c.p1 = std::min(p1, a0 + (i + 1) * tile);
        c.row = (int32_t)r;
        c.first = first;
        c.count = (int32_t)nch;
        c.counter = (int32_t)nsplit;
        chunks.push_back(c);
        Item it{};
        it.p0 = c.p0;
        it.len = (int32_t)(c.p1 - c.p0);
        it.r0 = (int32_t)r;
        it.nrows = 0;
        it.chunk = first + (int32_t)i;
        longi.push_back(it);
      }
      nsplit++;
      r++;
      continue;
    }
    int64_t r1 = r + 1;
    while (r1 < m && r1 - r < rows && RP(r1 + 1) - a0 <= tile)
      r1++;
    Item it{};
    it.p0 = p0;
    it.len = (int32_t)(RP(r1) - p0);
    it.r0 = (int32_t)r;
    it.nrows = (int32_t)(r1 - r);
    it.chunk = -1;
    tiles.push_back(it);
    r = r1;
  }
  // Interleave chunk items with whole-row items so every warp's share mixes
  // both kinds.
  std::vector<Item> all;
  all.reserve(longi.size() + tiles.size());
  size_t a = 0, b = 0;
  const double ratio = tiles.empty() ? 0.0 : (double)longi.size() / (double)tiles.size();
  double acc = 0.0;
  while (a < longi.size() || b < tiles.size()) {
    if (b < tiles.size()) {
      all.push_back(tiles[b++]);
      acc += ratio;
    }
    while (a < longi.size() && (acc >= 1.0 || b >= tiles.size())) {
      all.push_back(longi[a++]);
      acc -= 1.0;
    }
  }
  plan.nitems = (int64_t)all.size();
  plan.nchunks = (int64_t)chunks.size();
  plan.nsplit = nsplit;
  DRB_TRY(plan.items.alloc(sizeof(Item) * std::max<size_t>(all.size(), 1)));
  if (!all.empty())
    DRB_CUDA_TRY(cudaMemcpy(plan.items.p, all.data(), sizeof(Item) * all.size(),
                            cudaMemcpyHostToDevice));
  DRB_TRY(plan.chunks.alloc(sizeof(Chunk) * std::max<size_t>(chunks.size(), 1)));
  if (!chunks.empty())
    DRB_CUDA_TRY(cudaMemcpy(plan.chunks.p, chunks.data(), sizeof(Chunk) * chunks.size(),
                            cudaMemcpyHostToDevice));
  DRB_TRY(plan.partials.alloc(sizeof(double) * std::max<size_t>(chunks.size(), 1)));
  DRB_TRY(plan.counters.alloc(sizeof(int) * std::max<int64_t>(nsplit, 1)));
  DRB_CUDA_TRY(cudaMemset(plan.counters.p, 0, plan.counters.bytes));
  DRB_TRY(plan.err.alloc(sizeof(int) * 4));
  DRB_CUDA_TRY(cudaMemset(plan.err.p, 0, plan.err.bytes));
  return DRB_OK;
}

drb_status spmv_pipe_launch(Csr &A, const void *x, void *y, cudaStream_t s) {
  if (A.storage == DRB_F32)
    return warp_idx<float, false>(A, x, y, nullptr, s);
  if (A.storage == DRB_F64)
    return warp_idx<double, false>(A, x, y, nullptr, s);
  set_error("spmv: storage type not handled");
  return DRB_ERR_UNSUPPORTED;
}

drb_status residual_pipe_launch(Csr &A, const void *x, const void *b, void *y,
                                double *out, cudaStream_t s) {
  PipePlan &P = A.pipe;
  if (P.nitems == 0) {
    DRB_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(double), s));
    return DRB_OK;
  }
  int sms = 0;
  DRB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, A.device));
  const size_t slots = (size_t)sms * 32 + (size_t)P.nsplit;
  if (!P.red.p) {
    DRB_TRY(P.red.alloc(sizeof(double) * slots + 16));
    DRB_CUDA_TRY(cudaMemset(P.red.p, 0, P.red.bytes));
  }
  WarpResid ra;
  ra.b = b;
  ra.partials = P.red.as<double>();
  ra.rowres = P.red.as<double>() + (size_t)sms * 32;
  ra.nsplit = P.nsplit;
  ra.ticket = reinterpret_cast<int *>(P.red.as<double>() + slots);
  ra.out = out;
  if (A.storage == DRB_F32)
    return warp_idx<float, true>(A, x, y, &ra, s);
  if (A.storage == DRB_F64)
    return warp_idx<double, true>(A, x, y, &ra, s);
  set_error("residual: storage type not handled");
  return DRB_ERR_UNSUPPORTED;
}

int plan_group(int vbytes, int cbytes);

// Times the four single-RHS variants on this matrix's sparsity pattern (x = 0,
// three launches each after one warm-up) and rebuilds the plan with the
// fastest.  Returns the chosen variant (tile | skew) in *chosen.
drb_status autotune_pipe(Csr &A, cudaStream_t s, int *chosen) {
  if (A.storage != DRB_F32 && A.storage != DRB_F64) {
    set_error("autotune: storage type has no tunable kernel");
    return DRB_ERR_UNSUPPORTED;
  }
  const int vb = dtype_bytes(A.storage);
  const int group = plan_group(vb, A.cbytes);
  std::vector<char> rp((size_t)A.rbytes * (A.m + 1));
  if (A.m >= 0)
    DRB_CUDA_TRY(cudaMemcpy(rp.data(), A.rowptr.p, rp.size(), cudaMemcpyDeviceToHost));
  DevBuf xb, yb;
  DRB_TRY(xb.alloc((size_t)vb * (A.n + 1)));
  DRB_TRY(yb.alloc((size_t)vb * (A.m + 1)));
  DRB_CUDA_TRY(cudaMemsetAsync(xb.p, 0, xb.bytes, s));
  cudaEvent_t e0, e1;
  DRB_CUDA_TRY(cudaEventCreate(&e0));
  DRB_CUDA_TRY(cudaEventCreate(&e1));
  const int variants[4] = {256 | 1, 256, 512 | 1, 512};
  int best = variants[0];
  float best_ms = 3.4e38f;
  drb_status st = DRB_OK;
  for (int v : variants) {
    st = build_pipe_plan(A.pipe, A.m, rp.data(), A.rbytes, group, v, 0);
    if (st != DRB_OK)
      break;
    if ((st = spmv_pipe_launch(A, xb.p, yb.p, s)) != DRB_OK)
      break;
    cudaEventRecord(e0, s);
    for (int i = 0; i < 3 && st == DRB_OK; i++)
      st = spmv_pipe_launch(A, xb.p, yb.p, s);
    cudaEventRecord(e1, s);
    if (st != DRB_OK || cudaEventSynchronize(e1) != cudaSuccess)
      break;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best_ms) {
      best_ms = ms;
      best = v;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  DRB_TRY(st);
  DRB_TRY(build_pipe_plan(A.pipe, A.m, rp.data(), A.rbytes, group, best, 0));
  if (chosen)
    *chosen = best;
  return DRB_OK;
}

// Reads and clears the handle's device error word (set by kernels whose
// bounded device-side waits expired).
drb_status pipe_check(Csr &A, cudaStream_t s) {
  if (!A.pipe.err.p)
    return DRB_OK;
  int e = 0;
  DRB_CUDA_TRY(cudaMemcpyAsync(&e, A.pipe.err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  DRB_CUDA_TRY(cudaStreamSynchronize(s));
  if (e != 0) {
    DRB_CUDA_TRY(cudaMemsetAsync(A.pipe.err.p, 0, sizeof(int), s));
    set_error("a device-side wait timed out");
    return DRB_ERR_TIMEOUT;
  }
  return DRB_OK;
}

} // namespace drb
