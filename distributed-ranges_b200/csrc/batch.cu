// batch.cu -- batched CSR SpMM: Y_i = A_i X_i over many handles in one
// persistent launch, captured once in a CUDA graph.
//
// No reference counterpart: the reference multiplies one matrix per
// dr::mp::gemv call (include/dr/mp/algorithms/matrix/gemv.hpp:29-39, k
// right-hand sides as a broadcasted_slim_matrix, column-major).
//
// Work list.  Every matrix is cut into items of whole rows with at most CAP
// nonzeros and RMAX rows; a row longer than CAP is an item of its own (a
// "long row").  An item is 16 bytes {matrix, first row, rows | nnz << 8,
// first nonzero}; the items of all matrices form one list, and with more
// right-hand sides than one block holds, (item, block) pairs are the units.
// Warps of the persistent grid take units in batches of 8 consecutive indices
// from a work counter (zeroed by a memset node before the kernel in the
// graph); no warp waits on another (no spin anywhere).
//
// Random gathers of X rows bound this kernel.  Every warp runs a software
// pipeline over its units: while unit t computes, the column indices,
// values and row offsets of unit t+1 stream into shared memory (16-byte
// cp.async chunks, no registers held), and the item record of unit t+2 is
// read.  For unit t, groups of G slots (a slot = KP lanes, each lane VEC
// consecutive right-hand sides) share a row and R = S/G rows run at once; a
// lane keeps four 16-byte X gathers in flight (read-only path; k = 16 fp32 is
// one 64-byte row per nonzero), a group's partial sums meet in a fixed
// xor-shuffle tree, and the row sums go to a shared tile that the warp
// stores to Y coalesced, in either layout.  A long row is staged CAP
// nonzeros at a time and summed by all slots.  Every output element is
// summed in a fixed order: results are deterministic and, for a given G,
// independent of CAP for rows of at most 128 nonzeros.
//
// X in column-major layout (the reference's slim matrix) is first packed by a
// batched tiled transpose, in the same graph, into a row-major copy whose
// rows are padded to a multiple of VEC.
#include <algorithm>
#include <cstring>
#include <vector>

#include "drb_internal.cuh"

namespace drb {
namespace {

constexpr int kWarps = 8; // warps per CTA
constexpr int kYBudget = 4096; // bytes of a warp's output tile
constexpr int kRmax = 32;      // rows per item
constexpr int kNumCaps = 3;
constexpr int kCaps[kNumCaps] = {128, 256, 512};

struct BMat { // one per matrix of the batch (64 bytes)
  const int32_t *rowptr;
  const int32_t *colind;
  const void *vals;
  const void *x; // row-major, ldx elements per row
  void *y;
  int64_t m;
  int64_t n;
  int64_t pad;
};
static_assert(sizeof(BMat) == 64, "BMat is 64 bytes");

struct PackEnt {
  const void *src;
  void *dst;
  int64_t n;
  int64_t tile0; // first pack tile of this matrix
};

struct BArgs {
  const BMat *mats;
  const int4 *items;
  int64_t nunits;
  int nkb;       // right-hand-side blocks per item
  int k, ldx;    // right-hand sides; row stride of X (elements)
  int KP, S, KB; // lanes per slot, slots per warp, RHS per block (KP*VEC)
  int G;         // slots per row (power of two dividing S)
  int cap, rmax;
  int row_major;
  int warp_bytes;
  int cols_off, cols_stage, vals_off, vals_stage, rs_off, rs_stage;
  int y_off;
  unsigned long long *counter; // next unit to take (zeroed before each launch)
};

template <class V> struct AccOf {
  using type = float;
};
template <> struct AccOf<double> {
  using type = double;
};

// ---- cp.async (global -> shared, asynchronous, no registers in flight) ----
// Plain forms: the lanes of one instruction that touch the same line are
// served by one request.
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
template <int BYTES>
__device__ __forceinline__ void cp_async(uint32_t dst, const void *src) {
  if constexpr (BYTES == 16) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst),
                 "l"(src)
                 : "memory");
  } else {
    static_assert(BYTES == 4 || BYTES == 8, "4, 8 or 16 bytes");
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(dst),
                 "l"(src), "n"(BYTES)
                 : "memory");
  }
}
__device__ __forceinline__ void cp_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N> __device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}


__device__ __forceinline__ float to_acc(float v) { return v; }
__device__ __forceinline__ double to_acc(double v) { return v; }
__device__ __forceinline__ float to_acc(uint16_t v) {
  return __uint_as_float(((uint32_t)v) << 16);
}


// VEC consecutive X elements from global memory (read-only path) as raw
// 32-bit words, decoded to accumulator values only when used, so gathers in
// flight hold 16 bytes of registers each.
template <class XT, int VEC> struct XWords {
  static constexpr int W = VEC * (int)sizeof(XT) / 4;
  uint32_t w[W];
};
template <class XT, int VEC>
__device__ __forceinline__ void ldg_x(const XT *p, XWords<XT, VEC> &o) {
  constexpr int W = XWords<XT, VEC>::W;
  if constexpr (W == 4) {
    const uint4 u = __ldg(reinterpret_cast<const uint4 *>(p));
    o.w[0] = u.x, o.w[1] = u.y, o.w[2] = u.z, o.w[3] = u.w;
  } else if constexpr (W == 2) {
    const uint2 u = __ldg(reinterpret_cast<const uint2 *>(p));
    o.w[0] = u.x, o.w[1] = u.y;
  } else {
    o.w[0] = __ldg(reinterpret_cast<const uint32_t *>(p));
  }
}
template <class XT, int VEC, class A>
__device__ __forceinline__ A x_at(const XWords<XT, VEC> &o, int t) {
  if constexpr (sizeof(XT) == 4) {
    return __uint_as_float(o.w[t]);
  } else if constexpr (sizeof(XT) == 8) {
    return __hiloint2double((int)o.w[2 * t + 1], (int)o.w[2 * t]);
  } else {
    return (t & 1) ? __uint_as_float(o.w[t >> 1] & 0xffff0000u)
                   : __uint_as_float(o.w[t >> 1] << 16);
  }
}

// 32-bit shared-memory loads at explicit shared addresses.
__device__ __forceinline__ int32_t lds_s32(uint32_t addr) {
  int32_t v;
  asm volatile("ld.shared.b32 %0, [%1];" : "=r"(v) : "r"(addr));
  return v;
}
template <class V> __device__ __forceinline__ V lds_val(uint32_t addr);
template <> __device__ __forceinline__ float lds_val<float>(uint32_t addr) {
  float v;
  asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(addr));
  return v;
}
template <> __device__ __forceinline__ double lds_val<double>(uint32_t addr) {
  double v;
  asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(addr));
  return v;
}
template <>
__device__ __forceinline__ uint16_t lds_val<uint16_t>(uint32_t addr) {
  uint16_t v;
  asm volatile("ld.shared.u16 %0, [%1];" : "=h"(v) : "r"(addr));
  return v;
}

// Copy elements [e0, e0 + cnt) of a 16-byte aligned array to the shared
// address dst in 16-byte chunks from the aligned element below e0 (the
// array's allocation is padded, so the last chunk stays inside it).
template <class T>
__device__ __forceinline__ void copy16s(uint32_t dst, const T *base,
                                        int64_t e0, int cnt, int lane) {
  constexpr int PER = 16 / (int)sizeof(T);
  const int64_t a0 = e0 & ~(int64_t)(PER - 1);
  const int nch = (int)((e0 + cnt - a0 + PER - 1) / PER);
  const T *src = base + a0;
  for (int c = lane; c < nch; c += 32)
    cp_async<16>(dst + 16 * c, src + (int64_t)c * PER);
}

__device__ __forceinline__ int ilog2(int x) { return 31 - __clz(x); }
__device__ __forceinline__ int clog2(int x) {
  return ilog2(x) + ((x & (x - 1)) ? 1 : 0);
}

constexpr int kUnroll = 4; // X gathers in flight per lane

// BF16 storage sums two-sum compensated, per block of the kUnroll products a
// lane has in flight: the block is one chain of fused multiply-adds (at most
// kUnroll roundings, each within u of the block's sum of |a x|), and the
// block sum enters the row's running sum through a two-sum whose exact error
// goes to a compensation term, added when the row completes.  So a row's
// error stays within about (kUnroll + 1) u of sum |a x| however long the row
// (plain f32 sums grow with its length), for about a third of the
// arithmetic of a two-sum per product.  The operations are the _rn
// intrinsics, which the compiler never contracts or reorders.
template <class V> struct Comp {
  static constexpr bool value = sizeof(V) == 2;
};

__device__ __forceinline__ void two_sum_rn(float a, float b, float &s, float &e) {
  s = __fadd_rn(a, b);
  const float bb = __fsub_rn(s, a);
  e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
}

// ---- packed f32 pairs (sm_100's f32x2 arithmetic) -------------------------
// One instruction does the fma / add / sub / mul of two f32 elements, each
// rounded exactly as its scalar form, so a lane's VEC sums take half the
// issue slots (the BF16 kernel is bound by instruction issue).  The pair's
// first element sits in the low 32 bits.
__device__ __forceinline__ uint64_t pk2(float lo, float hi) {
  uint64_t d;
  asm("mov.b64 %0, {%1, %2};" : "=l"(d) : "f"(lo), "f"(hi));
  return d;
}
__device__ __forceinline__ void unpk2(uint64_t d, float &lo, float &hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(d));
}
__device__ __forceinline__ uint64_t fma2(uint64_t a, uint64_t b, uint64_t c) {
  uint64_t d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
__device__ __forceinline__ uint64_t mul2(uint64_t a, uint64_t b) {
  uint64_t d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ uint64_t add2(uint64_t a, uint64_t b) {
  uint64_t d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ uint64_t sub2(uint64_t a, uint64_t b) {
  uint64_t d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
// d = a * b + c for bf16 a and b (bits) and f32 c, one rounding: the bf16
// product is exact in f32, so this is fmaf(float(a), float(b), c) without
// unpacking the bf16 operands first.
__device__ __forceinline__ float fma_bf16(uint16_t a, uint16_t b, float c) {
  float d;
  asm("fma.rn.f32.bf16 %0, %1, %2, %3;" : "=f"(d) : "h"(a), "h"(b), "f"(c));
  return d;
}

// Elements 2p and 2p+1 of a lane's VEC gathered X values as an f32 pair.
template <class XT, int VEC>
__device__ __forceinline__ uint64_t x_pair(const XWords<XT, VEC> &o, int p) {
  if constexpr (sizeof(XT) == 4)
    return pk2(__uint_as_float(o.w[2 * p]), __uint_as_float(o.w[2 * p + 1]));
  else // one 32-bit word holds both bf16 values, the first in its low half
    return pk2(__uint_as_float(o.w[p] << 16), __uint_as_float(o.w[p] & 0xffff0000u));
}

// The nonzeros [b, e) of one row staged at shared addresses colS/valS (byte
// address of stage element 0), this lane's VEC sums (and, compensated, their
// error terms cmp); the lane takes b, b + step, ... with kUnroll gathers in
// flight.  f32 sums of an even VEC run on packed pairs.
template <class V, class XT, int VEC, class A>
__device__ __forceinline__ void row_sums(uint32_t colS, uint32_t valS, int b,
                                         int e, const XT *Xl, int ldx,
                                         int step, A (&acc)[VEC], A (&cmp)[VEC]) {
  if constexpr (sizeof(A) == 4 && VEC % 2 == 0) {
    constexpr int P = VEC / 2;
    uint64_t a2[P], c2[P];
#pragma unroll
    for (int p = 0; p < P; p++) {
      a2[p] = pk2(acc[2 * p], acc[2 * p + 1]);
      c2[p] = pk2(cmp[2 * p], cmp[2 * p + 1]);
    }
    // bf16 values and bf16 X: the block's chains run on the bf16 operands
    constexpr bool kMixed = Comp<V>::value && sizeof(XT) == 2;
    for (int q = b; q < e; q += kUnroll * step) {
      XWords<XT, VEC> xv[kUnroll];
      uint64_t v2[kUnroll];
      uint16_t vb[kUnroll];
#pragma unroll
      for (int u = 0; u < kUnroll; u++) {
        const int qq = min(q + u * step, e - 1); // in range; extra lanes masked
        const int32_t col = lds_s32(colS + 4 * qq);
        const V raw = lds_val<V>(valS + (uint32_t)sizeof(V) * qq);
        const bool in = q + u * step < e;
        if constexpr (kMixed) {
          vb[u] = in ? (uint16_t)raw : (uint16_t)0; // bf16 +0 for masked lanes
        } else {
          const float vm = in ? to_acc(raw) : 0.0f;
          v2[u] = pk2(vm, vm);
        }
        ldg_x<XT, VEC>(Xl + (int64_t)col * ldx, xv[u]);
      }
      if constexpr (kMixed) {
#pragma unroll
        for (int p = 0; p < P; p++) {
          // one 32-bit word holds right-hand sides 2p (low half) and 2p+1
          float lo = fma_bf16(vb[0], (uint16_t)(xv[0].w[p] & 0xffffu), 0.0f);
          float hi = fma_bf16(vb[0], (uint16_t)(xv[0].w[p] >> 16), 0.0f);
#pragma unroll
          for (int u = 1; u < kUnroll; u++) {
            lo = fma_bf16(vb[u], (uint16_t)(xv[u].w[p] & 0xffffu), lo);
            hi = fma_bf16(vb[u], (uint16_t)(xv[u].w[p] >> 16), hi);
          }
          const uint64_t blk = pk2(lo, hi);
          const uint64_t s = add2(a2[p], blk);
          const uint64_t bb = sub2(s, a2[p]);
          const uint64_t err = add2(sub2(a2[p], sub2(s, bb)), sub2(blk, bb));
          a2[p] = s;
          c2[p] = add2(c2[p], err);
        }
      } else if constexpr (Comp<V>::value) {
#pragma unroll
        for (int p = 0; p < P; p++) {
          uint64_t blk = mul2(v2[0], x_pair<XT, VEC>(xv[0], p));
#pragma unroll
          for (int u = 1; u < kUnroll; u++)
            blk = fma2(v2[u], x_pair<XT, VEC>(xv[u], p), blk);
          // two-sum of the pair: s + err == a2 + blk exactly
          const uint64_t s = add2(a2[p], blk);
          const uint64_t bb = sub2(s, a2[p]);
          const uint64_t err = add2(sub2(a2[p], sub2(s, bb)), sub2(blk, bb));
          a2[p] = s;
          c2[p] = add2(c2[p], err);
        }
      } else {
#pragma unroll
        for (int u = 0; u < kUnroll; u++)
#pragma unroll
          for (int p = 0; p < P; p++)
            a2[p] = fma2(v2[u], x_pair<XT, VEC>(xv[u], p), a2[p]);
      }
    }
#pragma unroll
    for (int p = 0; p < P; p++) {
      unpk2(a2[p], acc[2 * p], acc[2 * p + 1]);
      unpk2(c2[p], cmp[2 * p], cmp[2 * p + 1]);
    }
    return;
  }
  for (int q = b; q < e; q += kUnroll * step) {
    XWords<XT, VEC> xv[kUnroll];
    A vv[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; u++) {
      const int qq = min(q + u * step, e - 1); // in range; extra lanes masked
      const int32_t col = lds_s32(colS + 4 * qq);
      const A v = to_acc(lds_val<V>(valS + (uint32_t)sizeof(V) * qq));
      vv[u] = q + u * step < e ? v : A(0);
      ldg_x<XT, VEC>(Xl + (int64_t)col * ldx, xv[u]);
    }
    if constexpr (Comp<V>::value) {
#pragma unroll
      for (int t = 0; t < VEC; t++) {
        float blk = __fmul_rn(vv[0], x_at<XT, VEC, A>(xv[0], t));
#pragma unroll
        for (int u = 1; u < kUnroll; u++)
          blk = __fmaf_rn(vv[u], x_at<XT, VEC, A>(xv[u], t), blk);
        float s, err;
        two_sum_rn(acc[t], blk, s, err);
        acc[t] = s;
        cmp[t] = __fadd_rn(cmp[t], err);
      }
    } else {
#pragma unroll
      for (int u = 0; u < kUnroll; u++) {
#pragma unroll
        for (int t = 0; t < VEC; t++)
          acc[t] = fma(vv[u], (x_at<XT, VEC, A>(xv[u], t)), acc[t]);
      }
    }
  }
}

// acc += other lane's (acc2, cmp2): compensated when the storage is BF16.
template <class V, class A>
__device__ __forceinline__ void merge_sum(A &acc, A &cmp, A acc2, A cmp2) {
  if constexpr (Comp<V>::value) {
    float s, err;
    two_sum_rn(acc, acc2, s, err);
    acc = s;
    cmp = __fadd_rn(cmp, __fadd_rn(cmp2, err));
  } else {
    acc += acc2;
  }
}

template <class V, class XT, int VEC>
__global__ void __launch_bounds__(256, 3) batch_spmm(const BArgs a) {
  using A = typename AccOf<V>::type;
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t wsm = smem_u32(smem) + (uint32_t)(warp * a.warp_bytes);
  A *ytile = reinterpret_cast<A *>(smem + (size_t)warp * a.warp_bytes + a.y_off);
  const int KP = a.KP, S = a.S, KB = a.KB, G = a.G, k = a.k, ldx = a.ldx;
  const int R = S / G;
  const int slot = lane / KP, jj = lane - slot * KP;
  const int grp = slot / G, gs = slot - grp * G; // row group, slot in group
  const bool on = slot < S;
  const bool row_on = on && grp < R; // slots past R*G idle in short units
  const int ystride = KB + 1;
  const int64_t nunits = a.nunits;
  const int nkb = a.nkb;
  constexpr int VOFF_MASK = 16 / (int)sizeof(V) - 1;

  // the warp's units: batches of kGrab consecutive units from the work
  // counter, so the sequence only grows, and which warp runs a unit never
  // changes its rows' sums.  (A static split -- warp w taking units w, w + W,
  // ... -- left warps idle behind unlucky shares: the 512-matrix batch ran
  // 22-26 ms on its best variant, varying run to run; batched grabs: 17.5 ms.)
  constexpr int kGrab = 8;
  int64_t gbase = 0;
  int gk = kGrab;
  auto next_unit = [&]() -> int64_t {
    if (gk == kGrab) {
      unsigned long long v = 0;
      if (lane == 0)
        v = atomicAdd(a.counter, (unsigned long long)kGrab);
      gbase = (int64_t)__shfl_sync(0xffffffffu, v, 0);
      gk = 0;
    }
    return gbase + gk++;
  };
  auto item_of = [&](int64_t uu) -> int64_t {
    return nkb == 1 ? uu : (int64_t)((uint32_t)uu / (uint32_t)nkb);
  };
  int64_t u = next_unit();
  int64_t u1 = next_unit();
  int4 rec = u < nunits ? __ldg(a.items + item_of(u)) : make_int4(0, 0, 0, 0);
  int4 rec_n = u1 < nunits ? __ldg(a.items + item_of(u1)) : make_int4(0, 0, 0, 0);

  // slices (columns, values, row offsets) of a short unit -> stage st
#define DRB_BATCH_PAIRS(REC, VALID, ST)                                          \
  do {                                                                         \
    if ((VALID) && ((REC).z & 0xff) > 0) {                                     \
      const BMat *bm_ = a.mats + (REC).x;                                      \
      const int len_ = (REC).z >> 8, nr_ = (REC).z & 0xff;                     \
      copy16s<int32_t>(wsm + a.cols_off + (ST) * a.cols_stage, bm_->colind,    \
                       (REC).w, len_, lane);                                   \
      copy16s<V>(wsm + a.vals_off + (ST) * a.vals_stage,                       \
                 static_cast<const V *>(bm_->vals), (REC).w, len_, lane);      \
      copy16s<int32_t>(wsm + a.rs_off + (ST) * a.rs_stage, bm_->rowptr,        \
                       (REC).y, nr_ + 1, lane);                                \
    }                                                                          \
    cp_commit();                                                               \
  } while (0)

  DRB_BATCH_PAIRS(rec, u < nunits, 0);
  for (int st = 0; u < nunits; st ^= 1) {
    const int64_t u2 = next_unit();
    const int4 rec_nn = u2 < nunits ? __ldg(a.items + item_of(u2)) : make_int4(0, 0, 0, 0);
    DRB_BATCH_PAIRS(rec_n, u1 < nunits, st ^ 1);
    cp_wait<1>(); // all but the newest group: the slices of unit u
    __syncwarp();

    const BMat *bm = a.mats + rec.x;
    const int jb = nkb == 1 ? 0 : (int)((uint32_t)u % (uint32_t)nkb) * KB;
    const int c0 = jb + jj * VEC;
    const bool con = on && c0 < k;
    const XT *Xl = static_cast<const XT *>(bm->x) + c0;
    A *Y = static_cast<A *>(bm->y);
    const int64_t m = bm->m;
    const int r0 = rec.y, nrows = rec.z & 0xff, p0 = rec.w;
    const uint32_t colS = wsm + a.cols_off + st * a.cols_stage;
    const uint32_t valS = wsm + a.vals_off + st * a.vals_stage;

    if (nrows > 0) {
      // ---- whole rows [r0, r0 + nrows): R rows at a time, G slots each ----
      const uint32_t colP = colS + 4 * (p0 & 3);
      const uint32_t valP = valS + (uint32_t)sizeof(V) * (p0 & VOFF_MASK);
      const uint32_t rsP = wsm + a.rs_off + st * a.rs_stage + 4 * (r0 & 3);
      for (int i0 = 0; i0 < nrows; i0 += R) {
        const int i = i0 + grp;
        A acc[VEC], cmp[VEC];
#pragma unroll
        for (int t = 0; t < VEC; t++)
          acc[t] = cmp[t] = 0;
        if (con && row_on && i < nrows) {
          const int b = lds_s32(rsP + 4 * i) - p0, e = lds_s32(rsP + 4 * i + 4) - p0;
          row_sums<V, XT, VEC, A>(colP, valP, b + gs, e, Xl, ldx, G, acc, cmp);
        }
        for (int dd = 1; dd < G; dd <<= 1) {
#pragma unroll
          for (int t = 0; t < VEC; t++) {
            const A a2 = __shfl_xor_sync(0xffffffffu, acc[t], dd * KP);
            const A c2 = Comp<V>::value ? __shfl_xor_sync(0xffffffffu, cmp[t], dd * KP) : A(0);
            merge_sum<V>(acc[t], cmp[t], a2, c2);
          }
        }
        if (con && row_on && gs == 0 && i < nrows) {
#pragma unroll
          for (int t = 0; t < VEC; t++)
            ytile[i * ystride + jj * VEC + t] = Comp<V>::value ? acc[t] + cmp[t] : acc[t];
        }
      }
      __syncwarp();
      // the tile to Y, coalesced: lanes map (row, column) by powers of two
      const int kbv = min(KB, k - jb);
      if (a.row_major) {
        if (kbv <= 32) {
          const int lc = clog2(kbv);
          const int c = lane & ((1 << lc) - 1);
          for (int i = lane >> lc; i < nrows; i += 32 >> lc)
            if (c < kbv)
              Y[((int64_t)r0 + i) * k + jb + c] = ytile[i * ystride + c];
        } else {
          for (int i = 0; i < nrows; i++)
            for (int c = lane; c < kbv; c += 32)
              Y[((int64_t)r0 + i) * k + jb + c] = ytile[i * ystride + c];
        }
      } else {
        const int lr = clog2(nrows);
        const int i = lane & ((1 << lr) - 1);
        for (int c = lane >> lr; c < kbv; c += 32 >> lr)
          if (i < nrows)
            Y[((int64_t)r0 + i) + (int64_t)(jb + c) * m] = ytile[i * ystride + c];
      }
      __syncwarp();
    } else {
      // ---- one long row, staged cap nonzeros at a time into stage st ----
      const int64_t lo0 = bm->rowptr[r0], hi0 = bm->rowptr[r0 + 1];
      A acc[VEC], cmp[VEC];
#pragma unroll
      for (int t = 0; t < VEC; t++)
        acc[t] = cmp[t] = 0;
      for (int64_t lo = lo0; lo < hi0; lo += a.cap) {
        const int len = (int)min((int64_t)a.cap, hi0 - lo);
        copy16s<int32_t>(colS, bm->colind, lo, len, lane);
        copy16s<V>(valS, static_cast<const V *>(bm->vals), lo, len, lane);
        cp_commit();
        cp_wait<0>();
        __syncwarp();
        if (con)
          row_sums<V, XT, VEC, A>(colS + 4 * (int)(lo & 3),
                                  valS + (uint32_t)sizeof(V) * (int)(lo & VOFF_MASK),
                                  slot, len, Xl, ldx, S, acc, cmp);
        __syncwarp();
      }
      for (int dd = 1; dd < S; dd <<= 1) {
#pragma unroll
        for (int t = 0; t < VEC; t++) {
          const A o = __shfl_down_sync(0xffffffffu, acc[t], dd * KP);
          const A oc = Comp<V>::value ? __shfl_down_sync(0xffffffffu, cmp[t], dd * KP) : A(0);
          if ((slot & (2 * dd - 1)) == 0 && slot + dd < S)
            merge_sum<V>(acc[t], cmp[t], o, oc);
        }
      }
      if (slot == 0 && con) {
#pragma unroll
        for (int t = 0; t < VEC; t++) {
          const int c = c0 + t;
          const A yv = Comp<V>::value ? acc[t] + cmp[t] : acc[t];
          if (c < k) {
            if (a.row_major)
              Y[(int64_t)r0 * k + c] = yv;
            else
              Y[(int64_t)r0 + (int64_t)c * m] = yv;
          }
        }
      }
      __syncwarp();
    }
    rec = rec_n;
    rec_n = rec_nn;
    u = u1;
    u1 = u2;
  }
#undef DRB_BATCH_PAIRS
  cp_wait<0>();
}

// dst[r*ldx + j] = X(r, j) for j < k, 0 for k <= j < ldx, from column-major
// (src[r + j*n]) or row-major (src[r*k + j]) X.  The unit is a tile of 32
// rows x 2^LCW columns, and a persistent grid's warps take tiles w, w + W,
// ...  For a tile every lane loads its row's elements of the tile's columns
// at once (column-major: one coalesced line per column), the warp transposes
// them through its shared buffer (row stride 2^LCW + 1: conflict-free
// writes) and stores the tile's rows -- for a tile of whole packed rows one
// contiguous run -- as 16-byte vectors (scalars when a row piece is not a
// multiple of 16 bytes).  The next tile's loads are issued before the
// current tile is stored, so a warp always has a tile's lines in flight.
// (A CTA moving one 512-row tile through shared memory kept one or two loads
// per thread in flight and packed at 0.4 of HBM speed; this form runs at
// 0.85.)  A tile is
// mapped to its matrix by binary search of the tile offsets; no CTA
// barrier, each warp is independent.
constexpr int kPackWarps = 4;

template <class T> struct PackTile {
  const T *in;    // this lane's first source element (column cb of its row)
  int64_t stride; // elements between a row's consecutive source columns
  T *out;         // the tile's first packed element (row r0, column cb)
  int nr, nc, kc; // rows, packed columns, source columns of the tile
};

template <class T, bool COLMAJOR, int CW>
__global__ void __launch_bounds__(kPackWarps * 32)
    batch_pack(const PackEnt *__restrict__ ents, int count, int64_t k, int64_t ldx, int lcw,
               int ctiles, int64_t ntiles) {
  extern __shared__ __align__(16) unsigned char pack_smem[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int cw = 1 << lcw, bs = cw + 1;
  T *buf = reinterpret_cast<T *>(pack_smem) + wid * 32 * bs;
  auto locate = [&](int64_t t) {
    int lo = 0, hi = count - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (ents[mid].tile0 <= t)
        lo = mid;
      else
        hi = mid - 1;
    }
    const PackEnt e = ents[lo];
    const int lt = (int)(t - e.tile0); // tiles of a batch < 2^31 (checked at build)
    const int64_t r0 = (int64_t)(lt / ctiles) << 5, cb = (int64_t)(lt % ctiles) << lcw;
    PackTile<T> d;
    const int64_t row = min(r0 + lane, e.n - 1); // rows past the end load nothing
    d.in = static_cast<const T *>(e.src) + (COLMAJOR ? cb * e.n + row : row * k + cb);
    d.stride = COLMAJOR ? e.n : 1;
    d.out = static_cast<T *>(e.dst) + r0 * ldx + cb;
    d.nr = (int)min((int64_t)32, e.n - r0);
    d.nc = (int)min((int64_t)cw, ldx - cb);
    d.kc = (int)max((int64_t)0, min((int64_t)cw, k - cb));
    return d;
  };
  auto load = [&](const PackTile<T> &d, T (&v)[CW]) {
#pragma unroll
    for (int j = 0; j < CW; j++) {
      v[j] = T(0);
      if (j < d.kc && lane < d.nr)
        v[j] = __ldg(d.in + j * d.stride);
    }
  };
  auto store = [&](const PackTile<T> &d, const T (&v)[CW]) {
    __syncwarp(); // the previous tile's reads of buf are done
#pragma unroll
    for (int j = 0; j < CW; j++)
      if (j < d.nc)
        buf[lane * bs + j] = v[j];
    __syncwarp();
    constexpr int VW = 16 / (int)sizeof(T);
    T *out = d.out;
    if (d.nc % VW == 0 && ldx % VW == 0) { // 16-byte row pieces (dst 16-byte aligned)
      const int vpr = d.nc / VW;
      for (int q = lane; q < d.nr * vpr; q += 32) {
        const int i = q / vpr, c = (q - i * vpr) * VW;
        union {
          uint4 u;
          T w[VW];
        } w;
#pragma unroll
        for (int x = 0; x < VW; x++)
          w.w[x] = buf[i * bs + c + x];
        *reinterpret_cast<uint4 *>(out + i * ldx + c) = w.u;
      }
    } else {
      for (int q = lane; q < d.nr * d.nc; q += 32) {
        const int i = q / d.nc, c = q - i * d.nc;
        out[i * ldx + c] = buf[i * bs + c];
      }
    }
  };
  const int64_t W = (int64_t)gridDim.x * kPackWarps;
  int64_t t = (int64_t)blockIdx.x * kPackWarps + wid;
  if (t >= ntiles)
    return; // whole warp
  PackTile<T> a = locate(t);
  T va[CW];
  load(a, va);
  for (;;) {
    t += W;
    const bool more = t < ntiles; // warp-uniform
    PackTile<T> b;
    T vb[CW];
    if (more) {
      b = locate(t);
      load(b, vb);
    }
    store(a, va);
    if (!more)
      break;
    a = b;
#pragma unroll
    for (int j = 0; j < CW; j++)
      va[j] = vb[j];
  }
}

using PackFn = void (*)(const PackEnt *, int, int64_t, int64_t, int, int, int64_t);

template <class T, bool COLMAJOR> PackFn pack_for_width(int lcw) {
  if (lcw <= 2)
    return batch_pack<T, COLMAJOR, 4>;
  if (lcw == 3)
    return batch_pack<T, COLMAJOR, 8>;
  if (lcw == 4)
    return batch_pack<T, COLMAJOR, 16>;
  return batch_pack<T, COLMAJOR, 32>;
}

PackFn pick_pack(int xbytes, bool colmajor, int lcw) {
  if (xbytes == 4)
    return colmajor ? pack_for_width<uint32_t, true>(lcw) : pack_for_width<uint32_t, false>(lcw);
  if (xbytes == 2)
    return colmajor ? pack_for_width<uint16_t, true>(lcw) : pack_for_width<uint16_t, false>(lcw);
  return colmajor ? pack_for_width<uint64_t, true>(lcw) : pack_for_width<uint64_t, false>(lcw);
}

using KernelFn = void (*)(const BArgs);

template <class V, class XT> KernelFn pick_vec(int vec) {
  if constexpr (sizeof(XT) == 2) {
    switch (vec) {
    case 2: return batch_spmm<V, XT, 2>;
    case 4: return batch_spmm<V, XT, 4>;
    case 8: return batch_spmm<V, XT, 8>;
    }
  } else if constexpr (sizeof(XT) == 4) {
    switch (vec) {
    case 1: return batch_spmm<V, XT, 1>;
    case 2: return batch_spmm<V, XT, 2>;
    case 4: return batch_spmm<V, XT, 4>;
    }
  } else {
    switch (vec) {
    case 1: return batch_spmm<V, XT, 1>;
    case 2: return batch_spmm<V, XT, 2>;
    }
  }
  return nullptr;
}

KernelFn pick_kernel(drb_dtype storage, bool x_f32, int vec) {
  switch (storage) {
  case DRB_F32:
    return pick_vec<float, float>(vec);
  case DRB_F64:
    return pick_vec<double, double>(vec);
  case DRB_BF16:
    return x_f32 ? pick_vec<uint16_t, float>(vec)
                 : pick_vec<uint16_t, uint16_t>(vec);
  }
  return nullptr;
}

template <class... Args>
drb_status fail(drb_status st, const char *fmt, Args... args) {
  set_error(fmt, args...);
  return st;
}

int round16(int64_t b) { return (int)((b + 15) / 16 * 16); }

} // namespace

struct Batch {
  int device = 0;
  int count = 0;
  drb_dtype storage = DRB_F32;
  bool x_f32 = false;
  int64_t k = 1;
  drb_layout layout = DRB_COL_MAJOR;
  bool xy_row_major = false; // X and Y are addressed row-major
  int vbytes = 4, xbytes = 4, abytes = 4;
  int vec = 1, ldx = 1, KP = 1, S = 32, KB = 1, nkb = 1;
  bool pack = false;
  int variant = -1, cap = 0, G = 1, rmax = kRmax;
  double avg_row = 0;
  int64_t nitems = 0;
  int grid = 0, warps = 0;
  BArgs args{};
  int64_t pack_tiles = 0;
  int pack_lcw = 0, pack_ctiles = 1;
  PackFn pack_fn = nullptr; // the pack kernel, its persistent grid and shared memory
  unsigned pack_grid = 0;
  size_t pack_smem = 0;
  std::vector<Csr *> mats;
  std::vector<BMat> hmats;
  std::vector<PackEnt> hpack;
  DevBuf dmats, items, xpack, dpack, counter;
  bool bound = false;
  bool use_graph = true;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  KernelFn kernel = nullptr;
  int nkernels = 0;
  ~Batch() {
    if (exec)
      cudaGraphExecDestroy(exec);
    if (graph)
      cudaGraphDestroy(graph);
  }
};

namespace {

// Cut every matrix into items of whole rows (<= cap nonzeros, <= rmax rows).
drb_status build_items(Batch &B, int cap) {
  std::vector<int4> items;
  std::vector<int32_t> rp;
  int64_t rows = 0, nnz = 0;
  for (int b = 0; b < B.count; b++) {
    const Csr &A = *B.mats[b];
    if (A.m == 0)
      continue;
    rp.resize(A.m + 1);
    DRB_CUDA_TRY(cudaMemcpy(rp.data(), A.rowptr.p, sizeof(int32_t) * (A.m + 1),
                            cudaMemcpyDeviceToHost));
    rows += A.m;
    nnz += rp[A.m];
    // Column-major Y larger than L2 holds while the matrix streams (64 MB),
    // with m a multiple of the rows in a 32-byte sector: items end on such a
    // multiple where they can, so that every Y column's sector is written by
    // one item.  (A sector two items share is half-written until the later
    // one runs, and L2 may evict and refill it in between: 8.91 -> 8.67 ms at
    // k = 16 on a 16.8M-row matrix.  A small Y stays in L2 meanwhile, and the
    // shorter items only cost: the 512-matrix batch ran 3% slower aligned.)
    const int se = 32 / B.abytes;
    const bool align = !B.xy_row_major && A.m % se == 0 &&
                       A.m * B.k * B.abytes > (int64_t)64 << 20;
    int64_t r = 0;
    while (r < A.m) {
      const int32_t lo = rp[r];
      if (rp[r + 1] - lo > cap) {
        items.push_back(make_int4(b, (int)r, 0, lo));
        r++;
        continue;
      }
      int64_t r1 = r + 1;
      while (r1 < A.m && r1 - r < B.rmax && rp[r1 + 1] - lo <= cap)
        r1++;
      if (align && r1 < A.m && r1 / se * se > r)
        r1 = r1 / se * se;
      items.push_back(
          make_int4(b, (int)r, (int)(r1 - r) | ((rp[r1] - lo) << 8), lo));
      r = r1;
    }
  }
  B.cap = cap;
  B.avg_row = rows ? (double)nnz / rows : 0;
  B.nitems = (int64_t)items.size();
  DRB_TRY(B.items.ensure(std::max<size_t>(1, items.size()) * sizeof(int4)));
  if (!items.empty())
    DRB_CUDA_TRY(cudaMemcpy(B.items.p, items.data(),
                            items.size() * sizeof(int4),
                            cudaMemcpyHostToDevice));
  return DRB_OK;
}

// Shared-memory layout, warps per CTA and grid for the current items and G
// slots per row; fills B.args.
drb_status configure(Batch &B, int G) {
  B.G = G;
  BArgs &a = B.args;
  const int cap = B.cap;
  a.cap = cap;
  a.rmax = B.rmax;
  // two stages (unit t and t+1), each a slice copied from the 16-byte
  // boundary below its start, and the output tile
  a.cols_off = 0;
  a.cols_stage = round16((int64_t)(cap + 8) * 4);
  a.vals_off = 2 * a.cols_stage;
  a.vals_stage = round16((int64_t)(cap + 16) * B.vbytes);
  a.rs_off = a.vals_off + 2 * a.vals_stage;
  a.rs_stage = round16((int64_t)(B.rmax + 8) * 4);
  a.y_off = a.rs_off + 2 * a.rs_stage;
  a.warp_bytes = round16(a.y_off + (int64_t)B.rmax * (B.KB + 1) * B.abytes);
  int optin = 0, sms = 0;
  DRB_CUDA_TRY(cudaDeviceGetAttribute(
      &optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, B.device));
  DRB_CUDA_TRY(
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, B.device));
  const int w = std::min(kWarps, (optin - 1024) / a.warp_bytes);
  if (w < 1)
    return fail(DRB_ERR_UNSUPPORTED,
                "batch: one warp needs %d bytes of shared memory",
                a.warp_bytes);
  B.warps = w;
  const int smem = w * a.warp_bytes;
  DRB_CUDA_TRY(cudaFuncSetAttribute(
      B.kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  int per_sm = 0;
  DRB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, B.kernel,
                                                             w * 32, smem));
  if (per_sm < 1)
    return fail(DRB_ERR_UNSUPPORTED, "batch kernel does not fit an SM");
  const int64_t units = B.nitems * B.nkb;
  const int64_t want = (units + w - 1) / w;
  B.grid = (int)std::max<int64_t>(
      1, std::min<int64_t>((int64_t)per_sm * sms, want));
  a.nunits = units;
  if (!B.counter.p)
    DRB_TRY(B.counter.alloc(16));
  a.counter = B.counter.as<unsigned long long>();
  a.nkb = B.nkb;
  a.k = (int)B.k;
  a.ldx = B.ldx;
  a.KP = B.KP;
  a.S = B.S;
  a.KB = B.KB;
  a.G = G;
  a.row_major = B.xy_row_major;
  a.mats = B.dmats.as<BMat>();
  a.items = B.items.as<int4>();
  return DRB_OK;
}

int encode_variant(int cap_idx, int G) { return (cap_idx << 4) | G; }

drb_status set_variant(Batch &B, int variant) {
  const int ci = variant >> 4, G = variant & 15;
  // xor trees over slots need a power-of-two slot width unless G == 1
  if (ci < 0 || ci >= kNumCaps || G < 1 || G > B.S || (G & (G - 1)) ||
      (G > 1 && (B.KP & (B.KP - 1))))
    return fail(DRB_ERR_INVALID_ARG, "invalid argument: batch variant %d",
                variant);
  if (B.cap != kCaps[ci])
    DRB_TRY(build_items(B, kCaps[ci]));
  DRB_TRY(configure(B, G));
  B.variant = variant;
  return DRB_OK;
}

// Pack (when needed) and the SpMM kernel: the sequence the graph holds.
drb_status enqueue(Batch &B, cudaStream_t s, bool count) {
  int n = 0;
  if (B.pack && B.pack_tiles > 0) {
    const int64_t k = B.k, ldx = B.ldx;
    const PackEnt *ents = B.dpack.as<PackEnt>();
    B.pack_fn<<<B.pack_grid, kPackWarps * 32, B.pack_smem, s>>>(
        ents, B.count, k, ldx, B.pack_lcw, B.pack_ctiles, B.pack_tiles);
    DRB_CUDA_TRY(cudaGetLastError());
    n++;
  }
  if (B.args.nunits > 0) {
    DRB_CUDA_TRY(cudaMemsetAsync(B.args.counter, 0, sizeof(unsigned long long), s));
    B.kernel<<<B.grid, B.warps * 32, (size_t)B.warps * B.args.warp_bytes, s>>>(
        B.args);
    DRB_CUDA_TRY(cudaGetLastError());
    n++;
  }
  B.nkernels = n;
  if (count)
    note_launch(n);
  return DRB_OK;
}

drb_status capture(Batch &B) {
  if (B.exec) {
    cudaGraphExecDestroy(B.exec);
    B.exec = nullptr;
  }
  if (B.graph) {
    cudaGraphDestroy(B.graph);
    B.graph = nullptr;
  }
  cudaStream_t cs;
  DRB_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  drb_status st = DRB_OK;
  cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    st = enqueue(B, cs, false);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(cs, &g);
    if (e == cudaSuccess && st == DRB_OK) {
      B.graph = g;
      e = cudaGraphInstantiate(&B.exec, g, 0);
    } else if (g) {
      cudaGraphDestroy(g);
    }
  }
  cudaStreamDestroy(cs);
  if (st != DRB_OK)
    return st;
  DRB_CUDA_TRY(e);
  return DRB_OK;
}

drb_status launch(Batch &B, cudaStream_t s) {
  if (!B.bound)
    return fail(DRB_ERR_INVALID_ARG,
                "invalid argument: batch has no x/y bound (drb_batch_bind)");
  if (B.use_graph && B.exec) {
    DRB_CUDA_TRY(cudaGraphLaunch(B.exec, s));
    note_launch(B.nkernels);
    return DRB_OK;
  }
  return enqueue(B, s, true);
}

drb_status make_batch(Batch &B, int32_t count, Csr *const *handles,
                      int64_t k, drb_layout layout, uint32_t flags) {
  if (count < 1)
    return fail(DRB_ERR_INVALID_ARG, "invalid argument: count < 1");
  if (!handles)
    return fail(DRB_ERR_INVALID_ARG, "invalid argument: handles is NULL");
  if (k < 1 || k > (1 << 20))
    return fail(DRB_ERR_INVALID_ARG, "invalid argument: k out of range");
  if (layout != DRB_COL_MAJOR && layout != DRB_ROW_MAJOR)
    return fail(DRB_ERR_INVALID_ARG, "invalid argument: layout");
  if (flags & ~DRB_FLAG_BF16_X_F32)
    return fail(DRB_ERR_INVALID_ARG, "invalid argument: flags");
  B.count = count;
  B.k = k;
  B.layout = layout;
  for (int i = 0; i < count; i++) {
    Csr *A = handles[i];
    if (!A)
      return fail(DRB_ERR_INVALID_ARG, "invalid argument: handles[%d] is NULL",
                  i);
    if (i == 0) {
      B.device = A->device;
      B.storage = A->storage;
    } else if (A->device != B.device || A->storage != B.storage) {
      return fail(DRB_ERR_INVALID_ARG,
                  "invalid argument: handles[%d] differs in device or storage "
                  "type from handles[0]",
                  i);
    }
    if (A->cbytes != 4 || A->rbytes != 4)
      return fail(DRB_ERR_UNSUPPORTED,
                  "batch needs 32-bit column indices and rowptr (handles[%d])",
                  i);
    if (A->m >= INT32_MAX)
      return fail(DRB_ERR_UNSUPPORTED, "batch needs m < 2^31 (handles[%d])",
                  i);
    B.mats.push_back(A);
  }
  if ((flags & DRB_FLAG_BF16_X_F32) && B.storage != DRB_BF16)
    return fail(DRB_ERR_INVALID_ARG,
                "invalid argument: BF16_X_F32 needs BF16 storage");
  B.x_f32 = (flags & DRB_FLAG_BF16_X_F32) != 0;
  B.vbytes = dtype_bytes(B.storage);
  B.xbytes = B.storage == DRB_BF16 ? (B.x_f32 ? 4 : 2) : B.vbytes;
  B.abytes = B.storage == DRB_F64 ? 8 : 4;
  // With one right-hand side both layouts are the same vector.
  B.xy_row_major = layout == DRB_ROW_MAJOR || k == 1;
  const int vmax = 16 / B.xbytes, vmin = B.xbytes == 2 ? 2 : 1;
  // Row-major X is gathered in place when k splits into VEC-wide slices;
  // otherwise (and always for column-major X with k > 1) it is packed with
  // row stride ldx = k rounded up to VEC.
  int vdirect = 0;
  if (B.xy_row_major)
    for (int v = vmax; v >= vmin; v >>= 1)
      if (k % v == 0) {
        vdirect = v;
        break;
      }
  if (vdirect) {
    B.pack = false;
    B.vec = vdirect;
    B.ldx = (int)k;
  } else {
    B.pack = true;
    int v = vmin;
    while (v < vmax && v < k)
      v <<= 1;
    B.vec = v;
    B.ldx = (int)((k + v - 1) / v * v);
  }
  B.KP = std::min(32, B.ldx / B.vec);
  B.S = 32 / B.KP;
  B.KB = B.KP * B.vec;
  B.nkb = (B.ldx + B.KB - 1) / B.KB;
  B.rmax = std::min(kRmax, std::max(1, kYBudget / ((B.KB + 1) * B.abytes)));
  B.kernel = pick_kernel(B.storage, B.x_f32, B.vec);
  if (!B.kernel)
    return fail(DRB_ERR_UNSUPPORTED,
                "no batch kernel for this type and vector width");
  DRB_TRY(B.dmats.alloc(sizeof(BMat) * count));
  B.hmats.resize(count);
  // pack tiles: 32 rows x 2^lcw columns (one per warp)
  B.pack_lcw = 0;
  while ((1 << B.pack_lcw) < std::min(B.ldx, 32))
    B.pack_lcw++;
  B.pack_ctiles = (B.ldx + (1 << B.pack_lcw) - 1) >> B.pack_lcw;
  int64_t tiles = 0, xpack_elems = 0;
  for (int i = 0; i < count; i++) {
    const Csr &A = *B.mats[i];
    BMat &bm = B.hmats[i];
    bm.rowptr = static_cast<const int32_t *>(A.rowptr.p);
    bm.colind = static_cast<const int32_t *>(A.colind.p);
    bm.vals = A.vals.p;
    bm.x = nullptr;
    bm.y = nullptr;
    bm.m = A.m;
    bm.n = A.n;
    bm.pad = 0;
    if (B.pack) {
      PackEnt pe;
      pe.src = nullptr;
      pe.dst = nullptr;
      pe.n = A.n;
      pe.tile0 = tiles;
      B.hpack.push_back(pe);
      tiles += ((A.n + 31) >> 5) * B.pack_ctiles;
      xpack_elems += (A.n * B.ldx + 15) / 16 * 16; // 16-element aligned
    }
  }
  if (tiles > INT32_MAX)
    return fail(DRB_ERR_UNSUPPORTED, "batch X too large to pack");
  B.pack_tiles = tiles;
  if (B.pack && tiles > 0) {
    B.pack_fn = pick_pack(B.xbytes, B.layout == DRB_COL_MAJOR && !B.xy_row_major, B.pack_lcw);
    B.pack_smem = (size_t)kPackWarps * 32 * ((1 << B.pack_lcw) + 1) * B.xbytes;
    int occ = 0, sms = 0;
    DRB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, B.pack_fn, kPackWarps * 32,
                                                               B.pack_smem));
    DRB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, B.device));
    const int64_t need = (tiles + kPackWarps - 1) / kPackWarps;
    B.pack_grid = (unsigned)std::max<int64_t>(
        1, std::min<int64_t>(need, (int64_t)std::max(1, occ) * sms));
  }
  if (B.pack) {
    DRB_TRY(B.xpack.alloc((size_t)std::max<int64_t>(1, xpack_elems) *
                          B.xbytes));
    DRB_TRY(B.dpack.alloc(sizeof(PackEnt) * count));
    int64_t off = 0;
    for (int i = 0; i < count; i++) {
      B.hpack[i].dst =
          static_cast<unsigned char *>(B.xpack.p) + off * B.xbytes;
      B.hmats[i].x = B.hpack[i].dst;
      off += (B.mats[i]->n * B.ldx + 15) / 16 * 16;
    }
  }
  // default variant: staging capacity 128, G near the mean row length / 8
  DRB_TRY(build_items(B, kCaps[1]));
  int G = 1;
  while ((B.KP & (B.KP - 1)) == 0 && G * 2 <= B.S && G * 2 * 8 <= B.avg_row)
    G *= 2;
  return set_variant(B, encode_variant(1, G));
}

drb_status bind(Batch &B, const void *const *x, void *const *y,
                cudaStream_t s) {
  if (!x || !y)
    return fail(DRB_ERR_INVALID_ARG, "invalid argument: x or y is NULL");
  const size_t align = (size_t)B.vec * B.xbytes;
  for (int i = 0; i < B.count; i++) {
    const Csr &A = *B.mats[i];
    if ((A.m > 0 && !y[i]) || (A.m > 0 && A.n > 0 && !x[i]))
      return fail(DRB_ERR_INVALID_ARG,
                  "invalid argument: x[%d] or y[%d] is NULL", i, i);
    if (B.pack) {
      B.hpack[i].src = x[i];
    } else {
      if (reinterpret_cast<uintptr_t>(x[i]) % align != 0)
        return fail(DRB_ERR_INVALID_ARG,
                    "invalid argument: row-major x[%d] must be %zu-byte "
                    "aligned",
                    i, align);
      B.hmats[i].x = x[i];
    }
    B.hmats[i].y = y[i];
  }
  DRB_CUDA_TRY(cudaMemcpyAsync(B.dmats.p, B.hmats.data(),
                               sizeof(BMat) * B.count, cudaMemcpyHostToDevice,
                               s));
  if (B.pack)
    DRB_CUDA_TRY(cudaMemcpyAsync(B.dpack.p, B.hpack.data(),
                                 sizeof(PackEnt) * B.count,
                                 cudaMemcpyHostToDevice, s));
  B.bound = true;
  return DRB_OK;
}

drb_status autotune(Batch &B, cudaStream_t s, int *chosen) {
  if (!B.bound)
    return fail(DRB_ERR_INVALID_ARG,
                "invalid argument: autotune needs x/y bound (drb_batch_bind)");
  cudaEvent_t e0, e1;
  DRB_CUDA_TRY(cudaEventCreate(&e0));
  DRB_CUDA_TRY(cudaEventCreate(&e1));
  // Two rounds over the variants, each variant's best kept: a single pass
  // let one noisy timing pick a variant that then ran up to a third slower.
  float best = 0;
  int bestv = B.variant;
  bool first = true;
  drb_status st = DRB_OK;
  for (int round = 0; round < 2 && st == DRB_OK; round++)
  for (int ci = 0; ci < kNumCaps && st == DRB_OK; ci++) {
    const int gmax = (B.KP & (B.KP - 1)) ? 1 : std::min(B.S, 8);
    for (int G = 1; G <= gmax && st == DRB_OK; G *= 2) {
      st = set_variant(B, encode_variant(ci, G));
      if (st == DRB_ERR_UNSUPPORTED) { // too much shared memory for this k
        clear_error();
        st = DRB_OK;
        continue;
      }
      if (st == DRB_OK)
        st = enqueue(B, s, true); // warm-up
      if (st != DRB_OK)
        break;
      cudaEventRecord(e0, s);
      for (int r = 0; r < 3 && st == DRB_OK; r++)
        st = enqueue(B, s, true);
      cudaEventRecord(e1, s);
      if (st != DRB_OK)
        break;
      if (cudaEventSynchronize(e1) != cudaSuccess) {
        st = fail(DRB_ERR_CUDA, "batch autotune: %s",
                  cudaGetErrorString(cudaGetLastError()));
        break;
      }
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      if (first || ms < best) {
        best = ms;
        bestv = B.variant;
        first = false;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  DRB_TRY(st);
  DRB_TRY(set_variant(B, bestv));
  if (B.use_graph)
    DRB_TRY(capture(B));
  if (chosen)
    *chosen = bestv;
  return DRB_OK;
}

} // namespace
} // namespace drb

namespace drb {

void BatchDeleter::operator()(Batch *p) const { delete p; }

drb_status multi_rhs_batch_launch(Csr &A, const void *x, void *y, int64_t k,
                                  drb_layout layout, cudaStream_t s, bool *used) {
  *used = false;
  if (A.cbytes != 4 || A.rbytes != 4 || A.nnz == 0 || A.m >= ((int64_t)1 << 31) ||
      (layout == DRB_ROW_MAJOR && reinterpret_cast<uintptr_t>(x) % 16 != 0))
    return DRB_OK;
  if (!A.mrhs || A.mrhs_k != k || A.mrhs_layout != (int)layout) {
    A.mrhs.reset();
    std::unique_ptr<Batch, BatchDeleter> B(new Batch());
    Csr *one = &A;
    DRB_TRY(make_batch(*B, 1, &one, k, layout, A.flags & DRB_FLAG_BF16_X_F32));
    DRB_CUDA_TRY(cudaStreamSynchronize(s)); // the work list is built on the host
    DRB_TRY(capture(*B));
    if (A.flags & DRB_FLAG_AUTOTUNE) {
      // times the variants writing y = A X (x is only read), then keeps one
      DRB_TRY(bind(*B, &x, &y, s));
      DRB_TRY(autotune(*B, s, nullptr));
    }
    A.mrhs = std::move(B);
    A.mrhs_k = k;
    A.mrhs_layout = (int)layout;
  }
  DRB_TRY(bind(*A.mrhs, &x, &y, s));
  DRB_TRY(launch(*A.mrhs, s));
  *used = true;
  return DRB_OK;
}

} // namespace drb

using namespace drb;

struct drb_batch_plan : public Batch {};

namespace {
// The handles as the library's matrix type (NULL stays NULL).
std::vector<Csr *> as_mats(int32_t count, const drb_csr_t *handles) {
  std::vector<Csr *> v;
  if (handles && count > 0)
    v.assign(handles, handles + count);
  return v;
}
} // namespace

extern "C" {

drb_status drb_batch_create(drb_batch_t *out, int32_t count,
                            const drb_csr_t *handles, int64_t k,
                            drb_layout layout, uint32_t flags, void *stream) {
  clear_error();
  if (!out)
    return fail(DRB_ERR_INVALID_ARG, "invalid argument: out is NULL");
  *out = nullptr;
  const std::vector<Csr *> mats = as_mats(count, handles);
  Csr *const *hs = handles ? mats.data() : nullptr;
  if (count < 1 || !handles || !handles[0]) {
    Batch probe;
    return make_batch(probe, count, hs, k, layout, flags);
  }
  DeviceGuard g(handles[0]->device);
  auto P = std::make_unique<drb_batch_plan>();
  DRB_TRY(make_batch(*P, count, hs, k, layout, flags));
  DRB_CUDA_TRY(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
  DRB_TRY(capture(*P));
  *out = P.release();
  return DRB_OK;
}

drb_status drb_batch_bind(drb_batch_t B, const void *const *x, void *const *y,
                          void *stream) {
  clear_error();
  if (!B)
    return fail(DRB_ERR_INVALID_ARG, "invalid argument: batch is NULL");
  DeviceGuard g(B->device);
  return bind(*B, x, y, static_cast<cudaStream_t>(stream));
}

drb_status drb_batch_gemv(drb_batch_t B, void *stream) {
  clear_error();
  if (!B)
    return fail(DRB_ERR_INVALID_ARG, "invalid argument: batch is NULL");
  DeviceGuard g(B->device);
  return launch(*B, static_cast<cudaStream_t>(stream));
}

drb_status drb_batch_variant(drb_batch_t B, int *variant) {
  clear_error();
  if (!B || !variant)
    return fail(DRB_ERR_INVALID_ARG, "invalid argument: NULL argument");
  *variant = B->variant;
  return DRB_OK;
}

drb_status drb_batch_set_variant(drb_batch_t B, int variant) {
  clear_error();
  if (!B)
    return fail(DRB_ERR_INVALID_ARG, "invalid argument: batch is NULL");
  DeviceGuard g(B->device);
  DRB_TRY(set_variant(*B, variant));
  if (B->use_graph)
    DRB_TRY(capture(*B));
  return DRB_OK;
}

drb_status drb_batch_autotune(drb_batch_t B, int *variant, void *stream) {
  clear_error();
  if (!B)
    return fail(DRB_ERR_INVALID_ARG, "invalid argument: batch is NULL");
  DeviceGuard g(B->device);
  return autotune(*B, static_cast<cudaStream_t>(stream), variant);
}

drb_status drb_batch_destroy(drb_batch_t B) {
  clear_error();
  if (!B)
    return DRB_OK;
  DeviceGuard g(B->device);
  delete B;
  return DRB_OK;
}

drb_status drb_batched_gemv(int32_t count, const drb_csr_t *handles,
                            const void *const *x, void *const *y, int64_t k,
                            drb_layout layout, uint32_t flags, void *stream) {
  clear_error();
  Batch probe;
  const std::vector<Csr *> mats = as_mats(count, handles);
  Csr *const *hs = handles ? mats.data() : nullptr;
  if (count < 1 || !handles || !handles[0])
    return make_batch(probe, count, hs, k, layout, flags);
  DeviceGuard g(handles[0]->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  probe.use_graph = false;
  DRB_TRY(make_batch(probe, count, hs, k, layout, flags));
  DRB_TRY(bind(probe, x, y, s));
  DRB_TRY(launch(probe, s));
  DRB_CUDA_TRY(cudaStreamSynchronize(s));
  return DRB_OK;
}

} // extern "C"
