// spmv_warp.cuh -- persistent warp-granular CSR SpMV (one right-hand side).
//
// The matrix is cut once (build_pipe_plan, spmv_warp.cu) into work items of at
// most TILE nonzeros counted from a 16-byte aligned start: up to kRows whole
// short rows, or one fixed-size chunk of a long row.  Warps take items in
// batches of consecutive indices from a work counter (a fused row reduction:
// items w, w + W, ..., W = warps in the grid) and run them with no CTA-wide
// barrier, so warps progress independently.
//
// For its current item every lane holds TILE/32 nonzeros in registers
// (16-byte vector loads of colind and values, evict-first L2 policy), gathers
// x for all of them at once (evict-last L2 policy keeps x resident), stores
// the products to its warp's shared-memory slice, and immediately reloads the
// registers with its next item; the current item's rows are then summed from
// shared memory while the next item's loads are in flight.  With SKEW the
// products are stored skewed (element q at q + q/32) so lanes that sum
// different rows hit different banks; rows are summed by 1..32 lanes each.
//
// Storage and accumulation types: V is the stored element type of values and
// x (float, double, or bfloat16 bits in uint16_t); products and sums use
// Acc = float for float/bf16 and double for double; y has type Acc.  With
// COMP the sums are two-sum compensated: a running sum plus the rounding
// error of every addition of a block of four products (their plain sum),
// combined at the end, so y carries the products' roundings (none for bf16 x
// bf16), at most 3u of each block's magnitudes and the final rounding.
//
// On B200 the random x gathers are bounded by the SM's L1-to-crossbar request
// rate (about one request per SM per clock); the design keeps many gathers in
// flight per warp and as many warps as registers allow.
//
// A chunked long row writes one partial per chunk; a second small pass
// (chunk_finish, or resid_finish with a fused row reduction) adds each split
// row's partials in chunk order after the main launch.  (Finishing them in
// the main launch -- the warp that completed a row's last chunk, found by an
// atomic ticket -- made every chunk item wait on the ticket's round trip,
// which cost a quarter of the time on long-row matrices.)  Every sum has a
// fixed order, so results are deterministic.
#pragma once

#include <algorithm>
#include <cstdlib>
#include <cstring>

#include "drb_internal.cuh"

namespace drb::warpk {

constexpr int kRows = 64; // rows of a whole-row item (<= 64: three rowptr regs)
constexpr int kWarps = 8; // warps per CTA
constexpr int kThreads = kWarps * 32;

template <class V> struct AccOf {
  using type = float;
};
template <> struct AccOf<double> {
  using type = double;
};

__device__ __forceinline__ float to_acc(float v) { return v; }
__device__ __forceinline__ double to_acc(double v) { return v; }
__device__ __forceinline__ float to_acc(uint16_t v) {
  return __uint_as_float(((uint32_t)v) << 16);
}

__device__ __forceinline__ float ld_x(const float *p, uint64_t pol) {
  return ptx::ld_keep(p, pol);
}
__device__ __forceinline__ double ld_x(const double *p, uint64_t pol) {
  return ptx::ld_keep(p, pol);
}
__device__ __forceinline__ float ld_x(const uint16_t *p, uint64_t pol) {
  return ptx::ld_keep(reinterpret_cast<const __nv_bfloat16 *>(p), pol);
}

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

template <class T> __device__ __forceinline__ T wsum(T v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1)
    v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

// Additions that the compiler may not contract with a preceding multiply
// into a fused multiply-add (an error-free transformation needs each
// operation rounded on its own).
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }

// Knuth's two-sum: s + e == a + b exactly, s = fl(a + b).
template <class T> __device__ __forceinline__ void two_sum(T a, T b, T &s, T &e) {
  s = add_rn(a, b);
  const T bb = sub_rn(s, a);
  e = add_rn(sub_rn(a, sub_rn(s, bb)), sub_rn(b, bb));
}

// Compensated accumulator (running sum and error term).
template <class T> struct CSum {
  T s = 0, c = 0;
  __device__ __forceinline__ void add(T x) {
    T e;
    two_sum(s, x, s, e);
    c += e;
  }
  __device__ __forceinline__ void merge(T s2, T c2) {
    T e;
    two_sum(s, s2, s, e);
    c += c2 + e;
  }
  __device__ __forceinline__ T value() const { return s + c; }
};

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

// Fused row reduction: ||A x - b||^2, or with `dot` set sum_i y_i b_i (b is
// then a weight vector, e.g. p for p.Ap).  The whole rows of work item i add
// into their own slot ipart[i] (whichever warp ran the item).  The finish
// pass completes the chunked rows; its CTA c adds the terms of the split rows
// it completes (a fixed grid-stride share) and a fixed range of ipart into
// partials[c], and its last CTA sums partials[0..grid) in order, so the
// result never depends on the schedule.  (The sliced-ELL kernel writes one
// partial per CTA and combines them itself.)  A non-null `stop` pointing at
// a non-zero word makes the launches return before touching anything (a
// converged iterative loop replaying a captured graph).
struct WarpResid {
  const void *b = nullptr;
  double *partials = nullptr;
  double *ipart = nullptr;
  int *ticket = nullptr;
  double *out = nullptr;
  const int *stop = nullptr;
  int dot = 0;
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

template <class V, class XT, class CI, class RI, int TILE, bool SKEW, bool COMP> struct Kern {
  using Acc = typename AccOf<V>::type;
  using S = Slot<V, CI, TILE>;
  static constexpr int G = S::G, NG = S::NG;
  const RI *__restrict__ rowptr;
  const CI *__restrict__ colind;
  const V *__restrict__ vals;
  const XT *__restrict__ x;
  Acc *__restrict__ y;
  const Item *__restrict__ items;
  int64_t nitems;
  const Chunk *__restrict__ chunks;
  Acc *partials;
  int *counters;
  uint64_t pol_s, pol_x, pol_y;
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

  // Reduce over a group of `tpr` lanes (segments of a warp), plain or
  // compensated.  The result is valid in the group's first lane.
  __device__ __forceinline__ Acc group_sum(Acc s, Acc c, int tpr) {
    if (!COMP) {
      for (int o = tpr >> 1; o > 0; o >>= 1)
        s += __shfl_down_sync(0xffffffffu, s, o, tpr);
      return s;
    }
    CSum<Acc> t;
    t.s = s;
    t.c = c;
    for (int o = tpr >> 1; o > 0; o >>= 1) {
      const Acc s2 = __shfl_down_sync(0xffffffffu, t.s, o, tpr);
      const Acc c2 = __shfl_down_sync(0xffffffffu, t.c, o, tpr);
      t.merge(s2, c2);
    }
    return t.value();
  }

  // Sum of the products of a chunk item held by this lane (registers).  With
  // COMP the products are added in blocks of four -- a plain sum, then one
  // two-sum into the running compensated sum: a block's roundings stay below
  // 3u of its magnitudes (u = 2^-24), far under the input rounding of a bf16
  // operand (2^-8) and the 1e-6 accumulation gate, at a quarter of the
  // two-sums (one per product cost ~9 % on a bf16 single-RHS product).
  __device__ __forceinline__ void chunk_sum(const S &sl, const Acc (&xg)[NG][G], int off,
                                            int end, int ng, CSum<Acc> &acc) const {
    static_assert((NG * G) % 4 == 0, "blocks of four products");
    Acc blk = Acc(0);
#pragma unroll
    for (int j = 0; j < NG; j++) {
      const int g = lane + 32 * j;
#pragma unroll
      for (int i = 0; i < G; i++) {
        const int q = g * G + i;
        const bool in = g < ng && q >= off && q < end;
        if (COMP) {
          const Acc p = in ? to_acc(sl.v[j][i]) * xg[j][i] : Acc(0);
          blk = add_rn(blk, p);
          if ((j * G + i) % 4 == 3) {
            acc.add(blk);
            blk = Acc(0);
          }
        } else if (in) {
          acc.s += to_acc(sl.v[j][i]) * xg[j][i];
        }
      }
    }
  }

  // Sum of positions b + gl, b + gl + tpr, ... < e of the staged products
  // (one lane's share of a row); with COMP in blocks of four as chunk_sum.
  __device__ __forceinline__ void row_sum(const Acc *prod, int b, int e, int gl, int tpr,
                                          CSum<Acc> &acc) const {
    auto at = [&](int q) { return prod[SKEW ? skew(q) : q]; };
    int q = b + gl;
    if (COMP) {
      for (; q + 3 * tpr < e; q += 4 * tpr)
        acc.add(add_rn(add_rn(add_rn(at(q), at(q + tpr)), at(q + 2 * tpr)), at(q + 3 * tpr)));
      Acc rest = Acc(0);
      for (; q < e; q += tpr)
        rest = add_rn(rest, at(q));
      acc.add(rest);
    } else {
      for (; q < e; q += tpr)
        acc.s += at(q);
    }
  }

  // Runs the item in `sl` and refills the slot with item `refill`.
  template <bool RESID>
  __device__ __forceinline__ void process(S &sl, int64_t refill, Acc *prod, int *srp,
                                          const Acc *bvec, double &r2, bool dotw) {
    const Item cur = sl.d;
    const int off = (int)(cur.p0 - sl.a0), end = off + cur.len;
    const int ng = (end + G - 1) / G;
    Acc xg[NG][G];
#pragma unroll
    for (int j = 0; j < NG; j++) {
      const int g = lane + 32 * j;
#pragma unroll
      for (int i = 0; i < G; i++) {
        const int q = g * G + i;
        xg[j][i] = (g < ng && q >= off && q < end) ? ld_x(x + sl.c[j][i], pol_x) : Acc(0);
      }
    }
    if (cur.nrows == 0) {
      // one chunk of a long row: sum in registers, no shared memory
      CSum<Acc> acc;
      chunk_sum(sl, xg, off, end, ng, acc);
      fetch(sl, refill);
      const Acc tot = group_sum(acc.s, acc.c, 32);
      if (lane == 0)
        partials[cur.chunk] = tot; // the row is completed by the finish pass
      return;
    }
#pragma unroll
    for (int j = 0; j < NG; j++) {
      const int g = lane + 32 * j;
      if (g < ng) {
        if (SKEW) {
#pragma unroll
          for (int i = 0; i < G; i++)
            prod[skew(g * G + i)] = to_acc(sl.v[j][i]) * xg[j][i];
        } else {
          constexpr int PER = 16 / sizeof(Acc);
#pragma unroll
          for (int h = 0; h < G / PER; h++) {
            Vec16<Acc> w;
#pragma unroll
            for (int i = 0; i < PER; i++)
              w.t[i] = to_acc(sl.v[j][h * PER + i]) * xg[j][h * PER + i];
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
      CSum<Acc> acc;
      if (r < nrows)
        row_sum(prod, srp[r], srp[r + 1], gl, tpr, acc);
      const Acc tot = group_sum(acc.s, acc.c, tpr);
      if (r < nrows && gl == 0) {
        ptx::st_hint(y + cur.r0 + r, tot, pol_y);
        if (RESID) {
          if (dotw) {
            r2 += (double)tot * (double)bvec[cur.r0 + r];
          } else {
            const double dd = (double)tot - (double)bvec[cur.r0 + r];
            r2 += dd * dd;
          }
        }
      }
    }
    __syncwarp(); // the shared slice is rewritten by the next item
  }

  // ---- the two-slot pipelined form (spmv_warp_pipe) --------------------------
  // Issues the x gathers of the item in `sl` (zeros where masked, or for an
  // empty slot) into xg.
  __device__ __forceinline__ void gather(const S &sl, Acc (&xg)[NG][G]) {
    const int off = sl.valid ? (int)(sl.d.p0 - sl.a0) : 0;
    const int end = sl.valid ? off + sl.d.len : 0;
    const int ng = (end + G - 1) / G;
#pragma unroll
    for (int j = 0; j < NG; j++) {
      const int g = lane + 32 * j;
#pragma unroll
      for (int i = 0; i < G; i++) {
        const int q = g * G + i;
        xg[j][i] = (g < ng && q >= off && q < end) ? ld_x(x + sl.c[j][i], pol_x) : Acc(0);
      }
    }
  }

  // Runs the item in `cur`, whose x values are in xg; meanwhile issues the
  // gathers of `nxt` (loaded one step earlier) into xg and refills `cur`
  // with item `refill`, so a warp keeps one item's gathers in flight while it
  // sums the previous item's rows.
  __device__ __forceinline__ void step(S &cur, const S &nxt, Acc (&xg)[NG][G],
                                       int64_t refill, Acc *prod, int *srp) {
    const Item it = cur.d;
    const int off = (int)(it.p0 - cur.a0), end = off + it.len;
    const int ng = (end + G - 1) / G;
    if (it.nrows == 0) {
      CSum<Acc> acc;
      chunk_sum(cur, xg, off, end, ng, acc);
      gather(nxt, xg);
      fetch(cur, refill);
      const Acc tot = group_sum(acc.s, acc.c, 32);
      if (lane == 0)
        partials[it.chunk] = tot; // the row is completed by the finish pass
      return;
    }
#pragma unroll
    for (int j = 0; j < NG; j++) {
      const int g = lane + 32 * j;
      if (g < ng) {
        if (SKEW) {
#pragma unroll
          for (int i = 0; i < G; i++)
            prod[skew(g * G + i)] = to_acc(cur.v[j][i]) * xg[j][i];
        } else {
          constexpr int PER = 16 / sizeof(Acc);
#pragma unroll
          for (int h = 0; h < G / PER; h++) {
            Vec16<Acc> w;
#pragma unroll
            for (int i = 0; i < PER; i++)
              w.t[i] = to_acc(cur.v[j][h * PER + i]) * xg[j][h * PER + i];
            *reinterpret_cast<uint4 *>(prod + g * G + h * PER) = w.u;
          }
        }
      }
    }
    if (lane <= it.nrows)
      srp[lane] = cur.rp0;
    if (lane + 32 <= it.nrows)
      srp[lane + 32] = cur.rp1;
    if (lane == 0 && 64 <= it.nrows)
      srp[64] = cur.rp2;
    __syncwarp();
    gather(nxt, xg);    // the next item's gathers fly while these rows are summed
    fetch(cur, refill); // and the item after it streams in
    const int nrows = it.nrows;
    int tpr = 1;
    while (tpr < 32 && tpr * 2 * nrows <= 32)
      tpr <<= 1;
    const int groups = 32 / tpr, gid = lane / tpr, gl = lane & (tpr - 1);
    for (int base = 0; base < nrows; base += groups) {
      const int r = base + gid;
      CSum<Acc> acc;
      if (r < nrows)
        row_sum(prod, srp[r], srp[r + 1], gl, tpr, acc);
      const Acc tot = group_sum(acc.s, acc.c, tpr);
      if (r < nrows && gl == 0) {
        ptx::st_hint(y + it.r0 + r, tot, pol_y);
      }
    }
    __syncwarp(); // the shared slice is rewritten by the next item
  }
};

template <class V, class XT, class CI, class RI, int TILE, bool SKEW, bool RESID, bool COMP>
__global__ void __launch_bounds__(kThreads)
    spmv_warp(const RI *__restrict__ rowptr, const CI *__restrict__ colind,
              const V *__restrict__ vals, const XT *__restrict__ x,
              typename AccOf<V>::type *__restrict__ y, const Item *__restrict__ items,
              int64_t nitems, const Chunk *__restrict__ chunks,
              typename AccOf<V>::type *partials, int *counters, WarpResid ra,
              int ypol) {
  using Acc = typename AccOf<V>::type;
  __shared__ __align__(16) Acc s_prod[kWarps][TILE + TILE / 32];
  __shared__ int s_rp[kWarps][kRows + 1];

  if (RESID && ra.stop && *static_cast<const volatile int *>(ra.stop))
    return; // uniform: every CTA reads the same word, written by an earlier launch
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // y is written once: evict-first by default so that it does not push the
  // gathered x out of L2
  Kern<V, XT, CI, RI, TILE, SKEW, COMP> K{rowptr, colind, vals, x, y, items, nitems,
                                      chunks, partials, counters,
                                      ptx::policy_evict_first(), ptx::policy_evict_last(),
                                      ypol ? ptx::policy_evict_normal()
                                           : ptx::policy_evict_first(),
                                      lane};
  const Acc *bvec = static_cast<const Acc *>(ra.b);
  double r2 = 0.0;
  Acc *prod = s_prod[warp];
  int *srp = s_rp[warp];

  // Warps take items in batches of kBatch consecutive indices from a work
  // counter (zeroed before the launch; lane 0 takes the next index one item
  // ahead, so the atomic's round trip overlaps the current item): a fixed
  // round-robin share was sensitive to the exact sequence of item costs (the
  // bench's power-law ran 2.23 ms against 1.61 ms for the same distribution
  // with another seed; batched grabs: 1.53 ms for both).  Which warp runs an
  // item changes neither a row's sum nor an item's reduction slot.
  constexpr int kBatch = 8; // items per grab
  auto grab = [&]() -> int64_t {
    unsigned v = 0;
    if (lane == 0)
      v = atomicAdd(reinterpret_cast<unsigned *>(counters), (unsigned)kBatch);
    return (int64_t)__shfl_sync(0xffffffffu, v, 0);
  };
  int64_t base = grab();
  int k = 0;
  auto advance = [&]() -> int64_t {
    if (++k == kBatch) {
      base = grab();
      k = 0;
    }
    return base + k;
  };
  Slot<V, CI, TILE> A;
  int64_t cur = base;
  K.fetch(A, cur);
  int64_t next = advance();
  while (A.valid) {
    K.template process<RESID>(A, next, prod, srp, bvec, r2, ra.dot != 0);
    if (RESID) {
      // the item's whole rows, in row order within each lane, then a fixed tree
      const double t = wsum(r2);
      if (lane == 0)
        ra.ipart[cur] = t;
      r2 = 0.0;
    }
    cur = next;
    next = advance();
  }
}

// The plain product (no fused reduction) with two item slots per warp: the
// gathers of item t+1 are issued before the rows of item t are summed, and
// item t+2's indices and values load meanwhile, so each item exposes one
// memory latency instead of two (gathers waiting on the indices they need).
// Same items, work counter, products and sums as spmv_warp: the same bits.
template <class V, class XT, class CI, class RI, int TILE, bool SKEW, bool COMP>
__global__ void __launch_bounds__(kThreads, TILE == 128 ? 4 : 2)
    spmv_warp_pipe(const RI *__restrict__ rowptr, const CI *__restrict__ colind,
                   const V *__restrict__ vals, const XT *__restrict__ x,
                   typename AccOf<V>::type *__restrict__ y, const Item *__restrict__ items,
                   int64_t nitems, const Chunk *__restrict__ chunks,
                   typename AccOf<V>::type *partials, int *counters, WarpResid,
                   int ypol) {
  using Acc = typename AccOf<V>::type;
  using Kt = Kern<V, XT, CI, RI, TILE, SKEW, COMP>;
  __shared__ __align__(16) Acc s_prod[kWarps][TILE + TILE / 32];
  __shared__ int s_rp[kWarps][kRows + 1];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  Kt K{rowptr, colind, vals, x, y, items, nitems, chunks, partials, counters,
       ptx::policy_evict_first(), ptx::policy_evict_last(),
       ypol ? ptx::policy_evict_normal() : ptx::policy_evict_first(), lane};
  Acc *prod = s_prod[warp];
  int *srp = s_rp[warp];
  constexpr int kBatch = 8; // items per grab, as spmv_warp
  auto grab = [&]() -> int64_t {
    unsigned v = 0;
    if (lane == 0)
      v = atomicAdd(reinterpret_cast<unsigned *>(counters), (unsigned)kBatch);
    return (int64_t)__shfl_sync(0xffffffffu, v, 0);
  };
  int64_t base = grab();
  int k = 0;
  auto advance = [&]() -> int64_t {
    if (++k == kBatch) {
      base = grab();
      k = 0;
    }
    return base + k;
  };
  Slot<V, CI, TILE> A, B;
  Acc xg[Kt::NG][Kt::G];
  K.fetch(A, base);
  K.fetch(B, advance());
  K.gather(A, xg);
  // a warp's item indices only grow, so once a slot comes back empty every
  // later one would too
  while (A.valid) {
    K.step(A, B, xg, advance(), prod, srp);
    if (!B.valid)
      break;
    K.step(B, A, xg, advance(), prod, srp);
  }
}

// A split row's sum: its chunk partials pp[0, count) added in chunk order.
// The loads go out kBatch at a time: a row of 16384 nonzeros has 128 chunks,
// and one dependent load per chunk made it the finishing pass's critical
// path.
template <class Acc, bool COMP>
__device__ __forceinline__ Acc chunk_row_sum(const Acc *__restrict__ pp, int count) {
  constexpr int kBatch = 16;
  CSum<Acc> sum;
  int i = 0;
  for (; i + kBatch <= count; i += kBatch) {
    Acc p[kBatch];
#pragma unroll
    for (int j = 0; j < kBatch; j++)
      p[j] = pp[i + j];
#pragma unroll
    for (int j = 0; j < kBatch; j++) {
      if (COMP)
        sum.add(p[j]);
      else
        sum.s += p[j];
    }
  }
  for (; i < count; i++) {
    if (COMP)
      sum.add(pp[i]);
    else
      sum.s += pp[i];
  }
  return sum.value();
}

// y of the split rows [s0, s1) (splits[s] = {row, first chunk, chunks}): their
// partials added in chunk order.  (Reading the whole chunk table to find the
// rows' first chunks made this pass read 68 MB on the bench matrix.)
template <class Acc, bool COMP>
__global__ void chunk_finish(const int4 *__restrict__ splits, int64_t s0, int64_t s1,
                             const Acc *__restrict__ partials, Acc *__restrict__ y) {
  const int64_t nth = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = s0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < s1; i += nth) {
    const int4 sp = splits[i];
    y[sp.x] = chunk_row_sum<Acc, COMP>(partials + sp.y, sp.z);
  }
}

// The fused row reduction's second pass: split rows as in chunk_finish; CTA
// c adds the terms of the split rows it completes (split rows c * kThreads +
// t, strided by the grid) and the item slots ipart[c * per, (c + 1) * per) into
// partials[c]; the last CTA (ticket) adds partials[0..grid) in index order
// into *out.  The grid is a function of the plan, so the grouping is fixed.
// Returns at once when the stop word is set.
template <class Acc, bool COMP>
__global__ void __launch_bounds__(kThreads)
    resid_finish(const int4 *__restrict__ splits, int64_t nsplit,
                 const Acc *__restrict__ cpart, Acc *__restrict__ y, WarpResid ra,
                 int64_t nitems) {
  __shared__ double s_red[kWarps];
  __shared__ int s_last;
  if (ra.stop && *static_cast<const volatile int *>(ra.stop))
    return;
  const Acc *bvec = static_cast<const Acc *>(ra.b);
  const int64_t nth = (int64_t)gridDim.x * kThreads;
  double sum = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < nsplit; i += nth) {
    const int4 sp = splits[i];
    const Acc v = chunk_row_sum<Acc, COMP>(cpart + sp.y, sp.z);
    y[sp.x] = v;
    const double dd = (double)v - (double)bvec[sp.x];
    sum += ra.dot ? (double)v * (double)bvec[sp.x] : dd * dd;
  }
  {
    const int64_t per = (nitems + gridDim.x - 1) / gridDim.x;
    const int64_t i0 = (int64_t)blockIdx.x * per, i1 = min(nitems, i0 + per);
    int64_t i = i0 + threadIdx.x;
    for (; i + 3 * kThreads < i1; i += 4 * kThreads) { // four loads in flight
      const double a0 = ra.ipart[i], a1 = ra.ipart[i + kThreads];
      const double a2 = ra.ipart[i + 2 * kThreads], a3 = ra.ipart[i + 3 * kThreads];
      sum += a0;
      sum += a1;
      sum += a2;
      sum += a3;
    }
    for (; i < i1; i += kThreads)
      sum += ra.ipart[i];
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  sum = wsum(sum);
  if (lane == 0)
    s_red[warp] = sum;
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
  if (!s_last)
    return;
  __threadfence();
  double t = 0.0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += kThreads)
    t += __ldcg(&ra.partials[i]);
  t = wsum(t);
  __syncthreads(); // s_red is reused
  if (lane == 0)
    s_red[warp] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t2 = 0.0;
    for (int w = 0; w < kWarps; w++)
      t2 += s_red[w];
    *ra.out = t2;
    *ra.ticket = 0;
  }
}

// Upper bound on resid_finish's grid (its per-CTA partials live in the
// fused-reduction scratch).
constexpr int kResidFinishGrid = 592;

struct Shape {
  int grid = 0;
  bool ready = false;
};

// L2 policy of the y stores: evict-first (0), or evict-normal (1) with
// DRB_Y_STORE=normal, read once per process.
inline int y_store_keep() {
  static const int keep = [] {
    const char *e = std::getenv("DRB_Y_STORE");
    return (e && std::strcmp(e, "normal") == 0) ? 1 : 0;
  }();
  return keep;
}

template <class V, class XT, class CI, class RI, int TILE, bool SKEW, bool RESID, bool COMP,
          bool PIPE = false>
drb_status launch_tile(Csr &A, const void *x, void *y, const WarpResid *ra,
                       cudaStream_t s) {
  using Acc = typename AccOf<V>::type;
  PipePlan &P = A.pipe;
  static Shape shape[64];
  auto kern = [] {
    if constexpr (PIPE)
      return spmv_warp_pipe<V, XT, CI, RI, TILE, SKEW, COMP>;
    else
      return spmv_warp<V, XT, CI, RI, TILE, SKEW, RESID, COMP>;
  }();
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
  DRB_CUDA_TRY(cudaMemsetAsync(P.counters.p, 0, sizeof(unsigned), s)); // work counter
  kern<<<grid, kThreads, 0, s>>>(A.rowptr.as<RI>(), A.colind.as<CI>(), A.vals.as<V>(),
                                 static_cast<const XT *>(x), static_cast<Acc *>(y),
                                 P.items.as<Item>(), P.nitems, P.chunks.as<Chunk>(),
                                 P.partials.as<Acc>(), P.counters.as<int>(), r,
                                 y_store_keep());
  note_launch();
  DRB_CUDA_TRY(cudaGetLastError());
  if (RESID) {
    // a function of the plan only, so the reduction's grouping is fixed
    const int g = (int)std::max<int64_t>(
        1, std::min<int64_t>(kResidFinishGrid,
                             std::max((P.nchunks + kThreads - 1) / kThreads,
                                      (P.nitems + 8191) / 8192)));
    resid_finish<Acc, COMP><<<g, kThreads, 0, s>>>(P.splits.as<int4>(), P.nsplit,
                                                   P.partials.as<Acc>(),
                                                   static_cast<Acc *>(y), r, P.nitems);
    note_launch();
    DRB_CUDA_TRY(cudaGetLastError());
  } else if (P.nsplit > 0) {
    // the split rows whose first chunk lies in [fin_c0, fin_c1) (all with -1)
    const auto &f = P.split_first;
    const int64_t s0 =
        P.fin_c1 >= 0 ? std::lower_bound(f.begin(), f.end(), P.fin_c0) - f.begin() : 0;
    const int64_t s1 =
        P.fin_c1 >= 0 ? std::lower_bound(f.begin(), f.end(), P.fin_c1) - f.begin() : P.nsplit;
    if (s1 > s0) {
      // one split row per thread: each is a short chain of dependent loads,
      // and a thread walking several in turn made the pass latency-bound
      const int g = (int)std::max<int64_t>(1, std::min<int64_t>(1 << 20, (s1 - s0 + 255) / 256));
      chunk_finish<Acc, COMP><<<g, 256, 0, s>>>(P.splits.as<int4>(), s0, s1,
                                                P.partials.as<Acc>(), static_cast<Acc *>(y));
      note_launch();
      DRB_CUDA_TRY(cudaGetLastError());
    }
  }
  return DRB_OK;
}

template <class V, class XT, class CI, class RI, bool RESID, bool COMP>
drb_status launch_variant(Csr &A, const void *x, void *y, const WarpResid *ra,
                          cudaStream_t s) {
  if (A.pipe.nitems == 0)
    return DRB_OK;
  const bool sk = A.pipe.skew;
  if constexpr (!RESID) {
    if (A.pipe.two_slot) { // the pipelined kernel: skewed layout, 128 or 256 nonzeros
      if constexpr (Slot<V, CI, 256>::G * 32 <= 128) {
        if (A.pipe.tile == 128)
          return launch_tile<V, XT, CI, RI, 128, true, false, COMP, true>(A, x, y, ra, s);
      }
      return launch_tile<V, XT, CI, RI, 256, true, false, COMP, true>(A, x, y, ra, s);
    }
  }
  if constexpr (Slot<V, CI, 256>::G * 32 <= 128) {
    if (A.pipe.tile == 128)
      return sk ? launch_tile<V, XT, CI, RI, 128, true, RESID, COMP>(A, x, y, ra, s)
                : launch_tile<V, XT, CI, RI, 128, false, RESID, COMP>(A, x, y, ra, s);
  }
  if (A.pipe.tile == 512)
    return sk ? launch_tile<V, XT, CI, RI, 512, true, RESID, COMP>(A, x, y, ra, s)
              : launch_tile<V, XT, CI, RI, 512, false, RESID, COMP>(A, x, y, ra, s);
  return sk ? launch_tile<V, XT, CI, RI, 256, true, RESID, COMP>(A, x, y, ra, s)
            : launch_tile<V, XT, CI, RI, 256, false, RESID, COMP>(A, x, y, ra, s);
}

// Dispatch on the stored index widths.
template <class V, class XT, bool RESID, bool COMP>
drb_status launch_typed(Csr &A, const void *x, void *y, const WarpResid *ra,
                        cudaStream_t s) {
  if (A.cbytes == 4 && A.rbytes == 4)
    return launch_variant<V, XT, int32_t, int32_t, RESID, COMP>(A, x, y, ra, s);
  if (A.cbytes == 4 && A.rbytes == 8)
    return launch_variant<V, XT, int32_t, int64_t, RESID, COMP>(A, x, y, ra, s);
  if (A.cbytes == 8 && A.rbytes == 4)
    return launch_variant<V, XT, int64_t, int32_t, RESID, COMP>(A, x, y, ra, s);
  return launch_variant<V, XT, int64_t, int64_t, RESID, COMP>(A, x, y, ra, s);
}

} // namespace drb::warpk

namespace drb {
// Per storage type (defined in spmv_warp_f32.cu / _f64.cu / _bf16.cu).
drb_status warp_launch_f32(Csr &A, const void *x, void *y, const warpk::WarpResid *ra,
                           bool comp, cudaStream_t s);
drb_status warp_launch_f64(Csr &A, const void *x, void *y, const warpk::WarpResid *ra,
                           cudaStream_t s);
drb_status warp_launch_bf16(Csr &A, const void *x, void *y, bool x_f32, cudaStream_t s);
} // namespace drb
