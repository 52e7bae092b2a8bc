// dense_tc.cu -- batched dense multi-RHS product on the tensor cores:
// Y_i = A_i X_i for row-major BF16 A_i (m_i x n_i) and BF16 X_i (n_i x k),
// FP32 accumulation in tensor memory, FP32 Y_i, all matrices in one launch.
//
// No reference counterpart: the reference's dense products are
// dr::sp::gemv / local_gemm (include/dr/sp/algorithms/matrix/local_gemm.hpp:
// 18-62: a naive M x K x N loop with atomics or oneMKL gemm); this is the
// multi-RHS dense form of dr::mp::gemv for a batch of matrices.
//
// One CTA computes one 128-row tile of one matrix over the whole K range
// (tiles of all matrices in one grid, longest K first).  Six warps:
//   warp 0    : TMA producer -- for each 64-wide K step, the 128 x 64 tile
//               of A and the N x 64 tile of X (K-major, 128-byte swizzle)
//               into a STAGES-deep ring, completion counted on an mbarrier;
//   warp 1    : allocates N columns of tensor memory and, from one lane,
//               issues four tcgen05.mma (M = 128, N, K = 16, BF16 x BF16 ->
//               FP32) per stage; tcgen05.commit releases the stage and, after
//               the last, signals the epilogue;
//   warps 2-5 : epilogue -- tcgen05.ld of the accumulator (warp w reads TMEM
//               lanes 32*(w%4) .. +31, i.e. rows of the tile), then stores to
//               Y coalesced (column-major: 32 consecutive rows per store).
// A loads are streamed once (HBM-bound: 32 RHS make 32 FLOP per A byte, far
// below the tensor-core roofline), so the design goal is a full TMA ring per
// SM.  Every load fills the issuing CTA's own shared memory only.
//
// Every mbarrier wait gives up after one second of %globaltimer (a plan can
// shorten the limit): the CTA then records DRB_ERR_TIMEOUT in the launch's
// error word and leaves its loops; the producer and MMA lanes test the word
// before each stage and while they wait, so the other CTAs stop early.
// Before a CTA exits, its producer waits (bounded) until every bulk copy it
// issued has landed, and tensor memory is always freed.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "drb_internal.cuh"
#include "tma.cuh"

namespace drb {
namespace {

constexpr int kTileM = 128;     // rows per tile (UMMA M)
constexpr int kTileK = 64;      // K per TMA box: one 128-byte swizzle span
constexpr int kThreads = 192;   // producer, MMA, four epilogue warps
constexpr int kABytes = kTileM * kTileK * 2; // one A box

// Ring variants: {stages, boxes per stage}.
constexpr int kNumVariants = 5;
constexpr int kVarStages[kNumVariants] = {4, 5, 8, 2, 4};
constexpr int kVarBoxes[kNumVariants] = {1, 1, 1, 2, 2};
constexpr int kDefaultVariant = 1; // fastest on the 64-matrix, k = 32 batch

struct DMat {
  const CUtensorMap *tma; // A map
  const CUtensorMap *tmx; // X map (K-major: rows = right-hand sides)
  float *y;
  int64_t m;
  int64_t n;
};

struct DArgs {
  const DMat *mats;
  const int2 *tiles; // {matrix, first row}
  int k;             // right-hand sides
  int N;             // k rounded up to 16 (UMMA N)
  int tmem_cols;     // power of two >= max(32, N)
  int row_major;
  int *err;
  uint64_t wait_ns; // limit of every mbarrier wait
  int stall_tile;   // failure-detection hook: this CTA issues no loads (-1: none)
};

// ---- tcgen05 / TMA PTX wrappers --------------------------------------------

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map,
                                            int x, int y, uint64_t *bar) {
  asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::"
               "complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
                   tma::smem_u32(dst)),
               "l"(map), "r"(x), "r"(y), "r"(tma::smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void prefetch_map(const CUtensorMap *map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(map) : "memory");
}

// Shared-memory matrix descriptor of a K-major tile with 128-byte swizzle:
// rows of 128 bytes, 8-row groups 1024 bytes apart (SBO), LBO 16 bytes,
// descriptor version 1, layout type 2 (SWIZZLE_128B).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) |
         ((uint64_t)(1024 >> 4) << 32) | ((uint64_t)1 << 46) |
         ((uint64_t)2 << 61);
}

// Instruction descriptor: kind::f16 with BF16 A and B, FP32 D, both
// K-major, M = 128, N = n.
__device__ __forceinline__ uint32_t idesc_bf16(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(kTileM >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc,
                                          uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile("{\n\t.reg .pred p;\n\t"
               "setp.ne.b32 p, %4, 0;\n\t"
               "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(
                   tmem_d),
               "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
               : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::"
               "cluster.b64 [%0];" ::"r"(tma::smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// 32 lanes x 32 columns of 32-bit accumulators: thread i of the warp gets
// lane (taddr.lane + i), columns taddr.col .. +31.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, "
      "[%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]),
        "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]),
        "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
        "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]),
        "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ bool aborted(const int *err, volatile int *flag) {
  return *flag != 0 || *(volatile const int *)err != 0;
}

// Pipeline wait of the producer and MMA lanes: true when the phase
// completed.  False when the CTA must stop: this CTA's flag or the launch's
// error word was set meanwhile (by the other lane or another CTA), or the
// limit ran out (then recorded here as DRB_ERR_TIMEOUT).
__device__ __forceinline__ bool pipe_wait(uint64_t *bar, uint32_t parity, const DArgs &a,
                                          volatile int *flag) {
  const int r = tma::mbar_wait_or_stop(bar, parity, a.wait_ns, flag,
                                       (const volatile int *)a.err);
  if (r == 2) {
    *flag = 1;
    atomicExch(a.err, DRB_ERR_TIMEOUT);
  }
  return r == 0;
}

template <int kStages, int kBoxes>
__global__ void __launch_bounds__(kThreads, 1) dense_tc(const DArgs a) {
  extern __shared__ unsigned char raw_smem[];
  // 1024-byte aligned stage ring (128-byte swizzle atoms), then barriers;
  // a stage holds kBoxes consecutive 64-wide K boxes of A and of X
  unsigned char *base = reinterpret_cast<unsigned char *>(
      (reinterpret_cast<uintptr_t>(raw_smem) + 1023) & ~(uintptr_t)1023);
  const int bbytes = a.N * kTileK * 2;                 // one X box
  constexpr int kStageA = kBoxes * kABytes;
  const int stage_b = kBoxes * bbytes;
  unsigned char *sa = base;                            // kStages x kStageA
  unsigned char *sb = base + kStages * kStageA;        // kStages x stage_b
  uint64_t *full = reinterpret_cast<uint64_t *>(sb + kStages * stage_b);
  uint64_t *empty = full + kStages;
  uint64_t *done = empty + kStages;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int2 tile = a.tiles[blockIdx.x];
  const DMat mt = a.mats[tile.x];
  const int nk = (int)((mt.n + kBoxes * kTileK - 1) / (kBoxes * kTileK));

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; s++) {
      tma::mbar_init(&full[s], 1);
      tma::mbar_init(&empty[s], 1);
    }
    tma::mbar_init(done, 1);
    *abort_flag = 0;
    tma::fence_mbar_init();
    prefetch_map(mt.tma);
    prefetch_map(mt.tmx);
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 "
                 "[%0], %1;" ::"r"(tma::smem_u32(tmem_slot)),
                 "r"(a.tmem_cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;"
                 ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      const uint32_t tx = (uint32_t)(kStageA + stage_b);
      int issued = 0; // stages whose loads were issued
      if ((int)blockIdx.x != a.stall_tile) {
        for (int s = 0; s < nk; s++) {
          const int slot = s % kStages;
          const uint32_t ph = (uint32_t)((s / kStages) & 1);
          if (aborted(a.err, abort_flag))
            break;
          if (!pipe_wait(&empty[slot], ph ^ 1, a, abort_flag))
            break;
          tma::mbar_arrive_expect_tx(&full[slot], tx);
#pragma unroll
          for (int b = 0; b < kBoxes; b++) {
            const int kx = (s * kBoxes + b) * kTileK;
            tma_load_2d(sa + slot * kStageA + b * kABytes, mt.tma, kx, tile.y,
                        &full[slot]);
            tma_load_2d(sb + slot * stage_b + b * bbytes, mt.tmx, kx, 0,
                        &full[slot]);
          }
          issued = s + 1;
        }
      }
      // No bulk copy may still be writing this CTA's shared memory when it
      // exits: wait (bounded) for the last phase armed on every slot.  After
      // a normal run the MMA lane has consumed them all and these return at
      // once; after an abort they cover the stages it never reached.
      for (int s = issued > kStages ? issued - kStages : 0; s < issued; s++)
        if (!tma::mbar_wait(&full[s % kStages], (uint32_t)((s / kStages) & 1))) {
          *abort_flag = 1;
          atomicExch(a.err, DRB_ERR_TIMEOUT);
        }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc = idesc_bf16(a.N);
      for (int s = 0; s < nk; s++) {
        const int slot = s % kStages;
        const uint32_t ph = (uint32_t)((s / kStages) & 1);
        if (aborted(a.err, abort_flag))
          break;
        if (!pipe_wait(&full[slot], ph, a, abort_flag))
          break;
        tc_fence_after();
#pragma unroll
        for (int b = 0; b < kBoxes; b++) {
          const uint64_t ad =
              sw128_desc(tma::smem_u32(sa + slot * kStageA + b * kABytes));
          const uint64_t bd =
              sw128_desc(tma::smem_u32(sb + slot * stage_b + b * bbytes));
#pragma unroll
          for (int kk = 0; kk < kTileK / 16; kk++) // K = 16 (32 bytes) each
            umma_bf16(tmem, ad + 2 * kk, bd + 2 * kk, idesc,
                      (s > 0 || b > 0 || kk > 0) ? 1u : 0u);
        }
        umma_commit(&empty[slot]);
      }
      umma_commit(done); // arrives when every MMA above has completed
    }
  } else {
    // epilogue: warp w owns TMEM lanes 32*(w%4) .. +31 = tile rows
    const int q = warp & 3;
    // the MMA lane always commits `done` (also after an abort), so this wait
    // keeps the fixed one-second limit whatever the plan's pipeline limit
    const bool ok = tma::mbar_wait(done, 0);
    if (!ok) {
      *abort_flag = 1;
      atomicExch(a.err, DRB_ERR_TIMEOUT);
    }
    tc_fence_after();
    if (ok && !aborted(a.err, abort_flag)) {
      const int64_t r = (int64_t)tile.y + q * 32 + lane;
      for (int c0 = 0; c0 < a.N; c0 += 32) {
        uint32_t v[32];
        tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)c0, v);
        if (r < mt.m) {
#pragma unroll
          for (int j = 0; j < 32; j++) {
            const int c = c0 + j;
            if (c < a.k) {
              if (a.row_major)
                mt.y[r * a.k + c] = __uint_as_float(v[j]);
              else
                mt.y[r + (int64_t)c * mt.m] = __uint_as_float(v[j]);
            }
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    // every MMA has completed before the accumulator is freed (immediate
    // unless the epilogue gave up on `done`)
    if (lane == 0 && !tma::mbar_wait(done, 0))
      atomicExch(a.err, DRB_ERR_TIMEOUT);
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(
                     tmem),
                 "r"(a.tmem_cols)
                 : "memory");
  }
}

// Xp[j*ldp + c] = X(c, j) for c < n: the right-hand sides of every matrix
// as K-major rows, in one launch (blockIdx.y = matrix; a few blocks per
// matrix loop over its k right-hand sides).
struct RhsPack {
  const uint16_t *x;
  uint16_t *xp;
  int64_t n, ldp;
};

__global__ void pack_rhs_bf16(const RhsPack *__restrict__ packs, int k,
                              int row_major) {
  const RhsPack p = packs[blockIdx.y];
  for (int j = 0; j < k; j++)
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < p.n;
         c += (int64_t)gridDim.x * blockDim.x)
      p.xp[j * p.ldp + c] = row_major ? p.x[c * k + j] : p.x[c + j * p.n];
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault,
                                &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

template <class... Args>
drb_status fail(drb_status st, const char *fmt, Args... args) {
  set_error(fmt, args...);
  return st;
}

// 2-D BF16 tensor map: dims {inner, outer}, row pitch in bytes, box {64, rows}.
drb_status make_map(CUtensorMap *map, const void *ptr, uint64_t inner,
                    uint64_t outer, uint64_t pitch, uint32_t box_rows) {
  auto fn = encode_fn();
  if (!fn)
    return fail(DRB_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
  const cuuint64_t dims[2] = {inner, outer};
  const cuuint64_t strides[1] = {pitch};
  const cuuint32_t box[2] = {(cuuint32_t)kTileK, box_rows};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2,
                        const_cast<void *>(ptr), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_128B,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    return fail(DRB_ERR_INVALID_ARG,
                "invalid argument: tensor map rejected (error %d; A and x need "
                "16-byte aligned rows)",
                (int)r);
  return DRB_OK;
}

} // namespace

using DenseKernel = void (*)(const DArgs);

DenseKernel dense_kernel(int v) {
  switch (v) {
  case 0: return dense_tc<kVarStages[0], kVarBoxes[0]>;
  case 1: return dense_tc<kVarStages[1], kVarBoxes[1]>;
  case 2: return dense_tc<kVarStages[2], kVarBoxes[2]>;
  case 3: return dense_tc<kVarStages[3], kVarBoxes[3]>;
  default: return dense_tc<kVarStages[4], kVarBoxes[4]>;
  }
}

size_t dense_smem(int v, int N) {
  return 1024 +
         (size_t)kVarStages[v] * kVarBoxes[v] * (kABytes + (size_t)N * kTileK * 2) +
         (2 * kVarStages[v] + 1) * 8 + 16;
}

struct DenseBatch {
  int device = 0;
  int variant = 0;
  int count = 0;
  int64_t k = 1;
  int N = 16, tmem_cols = 32;
  bool row_major = false;
  int ntiles = 0;
  size_t smem = 0;
  int npacks = 0;
  int64_t max_n = 0;
  std::vector<std::pair<float *, size_t>> zero; // outputs of n == 0 matrices
  uint64_t wait_ns = tma::kWaitNs;
  int stall_tile = -1;
  DevBuf maps, mats, tiles, xp, packs, err;
};

namespace {

drb_status set_dense_variant(DenseBatch &P, int v) {
  if (v < 0 || v >= kNumVariants)
    return fail(DRB_ERR_INVALID_ARG, "invalid argument: dense variant %d", v);
  int optin = 0;
  DRB_CUDA_TRY(cudaDeviceGetAttribute(
      &optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, P.device));
  const size_t sm = dense_smem(v, P.N);
  if (sm > (size_t)optin)
    return fail(DRB_ERR_UNSUPPORTED, "dense variant %d needs %zu bytes of shared "
                "memory for k = %lld", v, sm, (long long)P.k);
  DRB_CUDA_TRY(cudaFuncSetAttribute(
      dense_kernel(v), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  P.variant = v;
  P.smem = sm;
  return DRB_OK;
}

drb_status make_dense_batch(DenseBatch &P, int32_t count, const int64_t *m,
                            const int64_t *n, const void *const *A,
                            const int64_t *lda, const void *const *x,
                            void *const *y, int64_t k, drb_layout layout) {
  if (count < 1 || !m || !n || !A || !lda || !x || !y)
    return fail(DRB_ERR_INVALID_ARG, "invalid argument: NULL array or count");
  if (count > 65535)
    return fail(DRB_ERR_UNSUPPORTED, "dense batch takes at most 65535 matrices");
  if (k < 1 || k > 256)
    return fail(DRB_ERR_UNSUPPORTED, "dense batch takes 1 <= k <= 256");
  if (layout != DRB_COL_MAJOR && layout != DRB_ROW_MAJOR)
    return fail(DRB_ERR_INVALID_ARG, "invalid argument: layout");
  int dev = 0;
  DRB_CUDA_TRY(cudaGetDevice(&dev));
  int major = 0, minor = 0;
  DRB_CUDA_TRY(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
  DRB_CUDA_TRY(cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev));
  if (major != 10 || minor != 0)
    return fail(DRB_ERR_NO_DEVICE, "tensor-core path needs sm_100 (got sm_%d%d)",
                major, minor);
  P.device = dev;
  P.count = count;
  P.k = k;
  P.N = (int)std::max<int64_t>(16, (k + 15) / 16 * 16);
  P.tmem_cols = 32;
  while (P.tmem_cols < P.N)
    P.tmem_cols *= 2;
  P.row_major = layout == DRB_ROW_MAJOR;
  std::vector<std::pair<int64_t, int2>> order; // (K, tile)
  int64_t xp_elems = 0;
  std::vector<int64_t> ldp(count, 0);
  for (int i = 0; i < count; i++) {
    if (m[i] < 0 || n[i] < 0 || m[i] >= INT32_MAX || n[i] >= INT32_MAX)
      return fail(DRB_ERR_INVALID_ARG, "invalid argument: m[%d] or n[%d]", i, i);
    if (m[i] > 0 && !y[i])
      return fail(DRB_ERR_INVALID_ARG, "invalid argument: y[%d] is NULL", i);
    if (m[i] == 0)
      continue;
    if (n[i] == 0) {
      P.zero.push_back({static_cast<float *>(y[i]), (size_t)m[i] * k});
      continue;
    }
    if (!A[i] || !x[i])
      return fail(DRB_ERR_INVALID_ARG, "invalid argument: A[%d] or x[%d] is NULL",
                  i, i);
    if (lda[i] < n[i] || lda[i] % 8 != 0 ||
        reinterpret_cast<uintptr_t>(A[i]) % 16 != 0)
      return fail(DRB_ERR_UNSUPPORTED,
                  "dense batch needs lda[%d] >= n, a multiple of 8, and A 16-byte "
                  "aligned",
                  i);
    ldp[i] = (n[i] + 63) / 64 * 64;
    xp_elems += ldp[i] * k;
    for (int64_t r0 = 0; r0 < m[i]; r0 += kTileM)
      order.push_back({n[i], make_int2(i, (int)r0)});
  }
  std::stable_sort(order.begin(), order.end(),
                   [](const auto &p, const auto &q) { return p.first > q.first; });
  P.ntiles = (int)order.size();
  DRB_TRY(P.err.alloc(sizeof(int)));
  DRB_CUDA_TRY(cudaMemset(P.err.p, 0, sizeof(int)));
  if (P.ntiles == 0)
    return DRB_OK;
  DRB_TRY(P.xp.alloc((size_t)xp_elems * 2));
  std::vector<CUtensorMap> maps(2 * (size_t)count);
  std::vector<RhsPack> hp;
  std::vector<DMat> dm(count);
  DRB_TRY(P.maps.alloc(sizeof(CUtensorMap) * maps.size()));
  int64_t off = 0;
  for (int i = 0; i < count; i++) {
    dm[i] = DMat{nullptr, nullptr, static_cast<float *>(y[i]), m[i], n[i]};
    if (ldp[i] == 0)
      continue;
    uint16_t *xpi = P.xp.as<uint16_t>() + off;
    off += ldp[i] * k;
    hp.push_back({static_cast<const uint16_t *>(x[i]), xpi, n[i], ldp[i]});
    P.max_n = std::max(P.max_n, n[i]);
    DRB_TRY(make_map(&maps[2 * i], A[i], (uint64_t)n[i], (uint64_t)m[i],
                     (uint64_t)lda[i] * 2, kTileM));
    DRB_TRY(make_map(&maps[2 * i + 1], xpi, (uint64_t)n[i], (uint64_t)k,
                     (uint64_t)ldp[i] * 2, (uint32_t)P.N));
    dm[i].tma = P.maps.as<CUtensorMap>() + 2 * i;
    dm[i].tmx = P.maps.as<CUtensorMap>() + 2 * i + 1;
  }
  P.npacks = (int)hp.size();
  DRB_TRY(P.packs.alloc(sizeof(RhsPack) * hp.size()));
  DRB_CUDA_TRY(cudaMemcpy(P.packs.p, hp.data(), sizeof(RhsPack) * hp.size(),
                          cudaMemcpyHostToDevice));
  DRB_TRY(P.mats.alloc(sizeof(DMat) * count));
  DRB_TRY(P.tiles.alloc(sizeof(int2) * P.ntiles));
  std::vector<int2> tl(P.ntiles);
  for (int t = 0; t < P.ntiles; t++)
    tl[t] = order[t].second;
  DRB_CUDA_TRY(cudaMemcpy(P.maps.p, maps.data(), sizeof(CUtensorMap) * maps.size(),
                          cudaMemcpyHostToDevice));
  DRB_CUDA_TRY(cudaMemcpy(P.mats.p, dm.data(), sizeof(DMat) * count,
                          cudaMemcpyHostToDevice));
  DRB_CUDA_TRY(cudaMemcpy(P.tiles.p, tl.data(), sizeof(int2) * P.ntiles,
                          cudaMemcpyHostToDevice));
  return set_dense_variant(P, kDefaultVariant);
}

drb_status dense_batch_launch(DenseBatch &P, cudaStream_t s) {
  for (auto &z : P.zero)
    DRB_CUDA_TRY(cudaMemsetAsync(z.first, 0, z.second * sizeof(float), s));
  if (P.ntiles == 0)
    return DRB_OK;
  {
    const dim3 grid((unsigned)std::min<int64_t>((P.max_n + 255) / 256, 8),
                    (unsigned)P.npacks);
    pack_rhs_bf16<<<grid, 256, 0, s>>>(P.packs.as<RhsPack>(), (int)P.k,
                                       P.row_major ? 1 : 0);
    DRB_CUDA_TRY(cudaGetLastError());
  }
  DArgs a;
  a.mats = P.mats.as<DMat>();
  a.tiles = P.tiles.as<int2>();
  a.k = (int)P.k;
  a.N = P.N;
  a.tmem_cols = P.tmem_cols;
  a.row_major = P.row_major ? 1 : 0;
  a.err = P.err.as<int>();
  a.wait_ns = P.wait_ns;
  a.stall_tile = P.stall_tile;
  dense_kernel(P.variant)<<<P.ntiles, kThreads, P.smem, s>>>(a);
  DRB_CUDA_TRY(cudaGetLastError());
  note_launch(2);
  return DRB_OK;
}

} // namespace
} // namespace drb

using namespace drb;

struct drb_dense_batch_plan : public DenseBatch {};

extern "C" {

drb_status drb_dense_batch_create(drb_dense_batch_t *out, int32_t count,
                                  const int64_t *m, const int64_t *n,
                                  const void *const *A, const int64_t *lda,
                                  const void *const *x, void *const *y,
                                  int64_t k, drb_layout layout, drb_dtype dtype,
                                  void *stream) {
  clear_error();
  if (!out)
    return fail(DRB_ERR_INVALID_ARG, "invalid argument: out is NULL");
  *out = nullptr;
  if (dtype != DRB_BF16)
    return fail(DRB_ERR_UNSUPPORTED,
                "dense batch runs BF16 on the tensor cores (use drb_dense_gemv "
                "for F32/F64)");
  int cnt = 0;
  if (cudaGetDeviceCount(&cnt) != cudaSuccess || cnt == 0)
    return fail(DRB_ERR_NO_DEVICE, "no CUDA device available");
  auto P = std::make_unique<drb_dense_batch_plan>();
  DRB_TRY(make_dense_batch(*P, count, m, n, A, lda, x, y, k, layout));
  DRB_CUDA_TRY(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
  *out = P.release();
  return DRB_OK;
}

drb_status drb_dense_batch_gemv(drb_dense_batch_t P, void *stream) {
  clear_error();
  if (!P)
    return fail(DRB_ERR_INVALID_ARG, "invalid argument: plan is NULL");
  DeviceGuard g(P->device);
  return dense_batch_launch(*P, static_cast<cudaStream_t>(stream));
}

drb_status drb_dense_batch_set_variant(drb_dense_batch_t P, int variant) {
  clear_error();
  if (!P)
    return fail(DRB_ERR_INVALID_ARG, "invalid argument: plan is NULL");
  DeviceGuard g(P->device);
  return set_dense_variant(*P, variant);
}

drb_status drb_dense_batch_set_wait(drb_dense_batch_t P, uint64_t wait_ns,
                                    int32_t stall_tile) {
  clear_error();
  if (!P)
    return fail(DRB_ERR_INVALID_ARG, "invalid argument: plan is NULL");
  if (stall_tile < -1)
    return fail(DRB_ERR_INVALID_ARG, "invalid argument: stall_tile %d", (int)stall_tile);
  P->wait_ns = wait_ns ? wait_ns : tma::kWaitNs;
  P->stall_tile = stall_tile;
  return DRB_OK;
}

drb_status drb_dense_batch_check(drb_dense_batch_t P, void *stream) {
  clear_error();
  if (!P)
    return fail(DRB_ERR_INVALID_ARG, "invalid argument: plan is NULL");
  DeviceGuard g(P->device);
  DRB_CUDA_TRY(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
  int e = 0;
  DRB_CUDA_TRY(cudaMemcpy(&e, P->err.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (e != 0) {
    DRB_CUDA_TRY(cudaMemset(P->err.p, 0, sizeof(int)));
    return fail(DRB_ERR_TIMEOUT,
                "dense batch: a pipeline wait expired (error word cleared)");
  }
  return DRB_OK;
}

drb_status drb_dense_batch_destroy(drb_dense_batch_t P) {
  clear_error();
  if (!P)
    return DRB_OK;
  DeviceGuard g(P->device);
  delete P;
  return DRB_OK;
}

} // extern "C"
