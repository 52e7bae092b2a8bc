// drb_internal.cuh -- shared declarations of the drb CUDA library.
//
// Data layout in HBM (one handle = one CSR matrix, all segments on one GPU):
//   rowptr  [m+1]   int32 when nnz < 2^31, else int64
//   colind  [nnz]   int32 when n < 2^31 (unless DRB_FLAG_KEEP_INDEX64)
//   values  [nnz]   f32 | f64 | bf16
// colind/values are padded to a multiple of kPadElems with zeros so that the
// 16-byte vector loads of a row-block tile may read past the last nonzero.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "drb.h"

namespace drb {

// ---- errors ----------------------------------------------------------------
void set_error(const char *fmt, ...);
void clear_error();

#define DRB_CUDA_TRY(...)                                                     \
  do {                                                                         \
    cudaError_t e_ = (__VA_ARGS__);                                                 \
    if (e_ != cudaSuccess) {                                                   \
      ::drb::set_error("%s failed: %s (%s:%d)", #__VA_ARGS__, cudaGetErrorString(e_), \
                       __FILE__, __LINE__);                                    \
      return e_ == cudaErrorMemoryAllocation ? DRB_ERR_OOM : DRB_ERR_CUDA;     \
    }                                                                          \
  } while (0)

#define DRB_TRY(...)                                                          \
  do {                                                                         \
    drb_status s_ = (__VA_ARGS__);                                                  \
    if (s_ != DRB_OK)                                                          \
      return s_;                                                               \
  } while (0)

// Every kernel launch goes through note_launch() so the process can report
// how many library kernels ran.
// While a thread captures a CUDA graph it sets g_count_pause: launches
// recorded into a graph are counted when the graph is launched.
extern std::atomic<uint64_t> g_launch_count;
extern thread_local int g_count_pause;
inline void note_launch(uint64_t n = 1) {
  if (!g_count_pause)
    g_launch_count.fetch_add(n);
}

// Makes `dev` current for the scope of an entry point, restoring the
// caller's device afterwards.
struct DeviceGuard {
  int prev = -1;
  bool switched = false;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) == cudaSuccess && prev != dev)
      switched = cudaSetDevice(dev) == cudaSuccess;
  }
  ~DeviceGuard() {
    if (switched)
      cudaSetDevice(prev);
  }
};

// Stream-ordered per-call scratch from a library-private pool that keeps its
// memory mapped (util.cu); release with scratch_free on the same stream.
drb_status scratch_alloc(void **p, size_t bytes, cudaStream_t s);
void scratch_free(void *p, cudaStream_t s);

// ---- device buffers ----------------------------------------------------------
struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  ~DevBuf() { release(); }
  drb_status alloc(size_t nbytes);
  drb_status ensure(size_t nbytes); // grow (contents not kept)
  void release();
  template <class T> T *as() const { return static_cast<T *>(p); }
};

constexpr int64_t kPadElems = 64;

// ---- execution plan --------------------------------------------------------
// A CTA work item ("row block").  {a, b}:
//   b >  0 : rows [a, b), whose aligned nnz span fits one tile;
//   b == -1: the single long row a (span > tile), one CTA loops over it;
//   b <= -2: chunk (-b - 2) of a row too long for one CTA (see Chunk).
struct Chunk {
  int64_t p0, p1;   // nnz range of this chunk
  int32_t row;      // the row it belongs to
  int32_t first;    // first chunk index of that row
  int32_t count;    // number of chunks of that row
  int32_t counter;  // index of the row's completion counter
};

struct Plan {
  int tile = 0;        // nnz capacity of a tile (aligned span)
  int rows_max = 0;    // max rows in one tile
  int long_max = 0;    // rows longer than this are chunked
  int group = 0;       // elements per 16-byte vector group (G)
  int64_t nblocks = 0; // CTA work items
  int64_t nchunks = 0;
  int64_t nsplit = 0;  // rows that are chunked
  DevBuf blocks;       // int2[nblocks]
  DevBuf chunks;       // Chunk[nchunks]
  DevBuf partials;     // double[nchunks * kmax] (grown on demand)
  DevBuf counters;     // int[nsplit], zero between launches
  int64_t partial_k = 0;
  DevBuf red;          // double[nblocks] + int ticket: residual reduction
};

// Work item of the persistent SpMV (32 bytes).  Every item covers at most
// `tile` elements of colind/values counted from the 16-byte aligned start
// (p0 rounded down to the vector group):
//   nrows > 0 : whole rows [r0, r0 + nrows), nnz [p0, p0 + len);
//   nrows == 0: one chunk of row r0, nnz [p0, p0 + len); chunk indexes the
//               Chunk table (partials + ticket finish, as in Plan).
struct Item {
  int64_t p0;
  int32_t len;
  int32_t r0;
  int32_t nrows;
  int32_t chunk;
  int32_t pad0, pad1;
};
static_assert(sizeof(Item) == 32, "Item is 32 bytes");

struct PipePlan {
  int tile = 0, rows = 0, group = 0;
  bool skew = false; // skewed product layout in the row reduction
  bool two_slot = false; // the pipelined kernel (spmv_warp_pipe) for plain products
  int64_t nitems = 0, nchunks = 0, nsplit = 0;
  DevBuf items;    // Item[nitems]
  DevBuf chunks;   // Chunk[nchunks]
  DevBuf splits;   // int4 {row, first chunk, chunks, 0} per split row, in chunk order
  std::vector<int64_t> split_first; // host copy of each split row's first chunk
  DevBuf partials; // value type [nchunks]
  DevBuf counters; // unsigned work counter of the persistent kernel (zeroed per launch)
  DevBuf err;      // int: device-side error word (DRB_ERR_TIMEOUT)
  DevBuf red;      // double[grid] + int ticket: fused residual
  // The same items ordered by row and cut into row segments (built on the
  // first host-pointer gemv): segment s is seg_items[seg_i0[s], seg_i0[s+1])
  // and covers rows [seg_r0[s], seg_r0[s+1]).
  DevBuf seg_items;
  std::vector<int64_t> seg_i0, seg_r0;
  std::vector<int64_t> seg_c0;      // first chunk of each segment (+ end)
  std::vector<int> seg_blk;         // column-split plans: the x block each segment waits for
  int64_t fin_c0 = 0, fin_c1 = -1;  // chunks the plain launch finishes (-1: all)
  uint64_t gen = 0; // bumped by every (re)build
};

drb_status build_pipe_plan(PipePlan &plan, int64_t m, const void *rowptr_host,
                           int rbytes, int group, int tile, int rows);
// Elements per 16-byte vector group of a plan over values of vbytes and
// column indices of cbytes.
int plan_group(int vbytes, int cbytes);

// rowptr buffers carry this many extra zeroed elements past rowptr[m] so a
// 16-byte-rounded bulk copy of a rowptr slice stays inside the allocation.
constexpr int64_t kRowptrPad = 8;

// Sliced-ELL copy of a matrix with short, regular rows (sell.cu): slices of
// 32 rows, slice s padded to its longest row and stored k-major at
// off[s] + 32*k + lane.  `on` routes the single-right-hand-side entry points
// (gemv, fused residual, conjugate gradients) to it.
struct Sell {
  bool built = false, on = false;
  int64_t nslices = 0, padded = 0;
  int maxw = 0;
  DevBuf vals, cols, off;            // V[padded], int32[padded], int64[nslices+1]
  std::vector<int64_t> off_h;        // host copy of off
  std::vector<int64_t> seg_s0;       // slice cuts of the host-pointer gemv
};

constexpr int kVariantSell = 2048; // drb_csr_variant code of the sliced-ELL kernel

struct CgPlan; // conjugate-gradient workspace (cg.cu)
struct CgPlanDeleter {
  void operator()(CgPlan *p) const;
};
struct Batch; // batched SpMM plan (batch.cu)
struct BatchDeleter {
  void operator()(Batch *p) const;
};

struct Csr {
  int device = 0;
  int64_t m = 0, n = 0, nnz = 0;
  int64_t max_row = 0; // nonzeros in the longest row
  drb_dtype value_type = DRB_F32; // caller's element type
  drb_dtype storage = DRB_F32;    // device element type
  int cbytes = 4, rbytes = 4;     // stored index widths
  int nseg = 1;
  drb_partition part = DRB_PART_ROW;
  uint32_t flags = 0;
  DevBuf rowptr, colind, vals;
  Plan plan;      // row blocks: multi-RHS kernel
  PipePlan pipe;  // work items: the persistent single-RHS kernel
  Sell sell;      // sliced-ELL copy for short regular rows (when eligible)
  std::vector<int64_t> seg_row0, seg_row1, seg_nz0, seg_nz1;
  // adjoint plan: A^T as a CSR matrix of shape n x m (colptr, rowidx, values
  // in column order, its own row-block plan) and perm[nnz] (CSC position ->
  // CSR position, perm_bytes wide) used to refresh the transposed values.
  bool has_adjoint = false;
  std::unique_ptr<Csr> tr;
  DevBuf perm;
  int perm_bytes = 4;
  // scratch for multi-RHS layout changes and host staging; the second stream
  // and events overlap y's copy back with the remaining row segments
  DevBuf xs, ys, xh_dev, yh_dev;
  cudaStream_t copy_stream = nullptr;
  std::vector<cudaEvent_t> seg_done;
  // conjugate-gradient workspace and its captured iteration graph
  std::unique_ptr<CgPlan, CgPlanDeleter> cg;
  // k > 1 products: a batch of this one handle, for one (k, layout)
  std::unique_ptr<Batch, BatchDeleter> mrhs;
  int64_t mrhs_k = 0;
  int mrhs_layout = -1;
  // host copy of rowptr (int64), filled on first drb_csr_get_entries
  std::vector<int64_t> rowptr_h;
  // column-blocked copy for the single-RHS gemv when x does not stay in L2
  // (colsplit.cu): a virtual CSR whose row b*(m+1) + r holds row r's nonzeros
  // of columns [cbounds[b], cbounds[b+1]), its block-major partial sums and the
  // block count (0: no split)
  std::unique_ptr<Csr> csplit;
  DevBuf csplit_y;
  int csplit_nblk = 0;
  std::vector<int64_t> cbounds;
  ~Csr();
};

// ---- launchers (defined in the .cu files) ------------------------------------
// y = A X for k > 1 through a cached batch of this one handle (batch.cu);
// *used = false, without launching, when the handle or the call does not
// qualify (64-bit indices, no nonzeros, misaligned row-major X).
drb_status multi_rhs_batch_launch(Csr &A, const void *x, void *y, int64_t k,
                                  drb_layout layout, cudaStream_t s, bool *used);
drb_status build_plan(Plan &plan, int64_t m, const void *rowptr_host,
                      int rbytes, int group, int tile, int rows_max,
                      int long_max);

drb_status spmv_launch(Csr &A, const void *x, void *y, int64_t k,
                       drb_layout layout, cudaStream_t s);
drb_status spmv_t_launch(Csr &A, const void *ybar, void *xbar, cudaStream_t s);
drb_status spmv_pipe_launch(Csr &A, const void *x, void *y, cudaStream_t s);
drb_status residual_pipe_launch(Csr &A, const void *x, const void *b, void *y,
                                double *out, cudaStream_t s);
// y = A x and *out = sum_i y_i w_i (w indexed by row); returns at once when
// *stop != 0 (stop may be null).  F32/F64 storage.
drb_status rowdot_pipe_launch(Csr &A, const void *x, const void *w, void *y,
                              double *out, const int *stop, cudaStream_t s);
// Allocates (zeroed) the per-CTA partials and ticket of the fused reductions;
// called before a graph capture so that no allocation happens inside it.
drb_status fused_scratch(Csr &A);
drb_status pipe_check(Csr &A, cudaStream_t s);
// Builds A.sell from the host rowptr when the rows are short and regular
// (longest <= 64, padding <= 20%, memory to spare); otherwise leaves it off.
drb_status sell_build(Csr &A, const void *rowptr_host, int rbytes, cudaStream_t s);
void sell_release(Csr &A);
drb_status sell_pack_values(Csr &A, cudaStream_t s); // after the CSR values change
namespace warpk {
struct WarpResid;
}
// The sliced-ELL kernel over slices [s0, s1), with the row-block kernel's
// fused row reduction contract when ra is given.
drb_status sell_launch(Csr &A, const void *x, void *y, const warpk::WarpResid *ra,
                       int64_t s0, int64_t s1, cudaStream_t s);
drb_status autotune_pipe(Csr &A, cudaStream_t s, int *chosen);
// Column split (colsplit.cu): build A.csplit when x is too large for L2 (or
// as DRB_COLSPLIT asks), refresh its values after A's change, run the
// single-RHS gemv over it, and time its kernel variants.
drb_status colsplit_build(Csr &A, cudaStream_t s);
drb_status colsplit_refresh_values(Csr &A, cudaStream_t s);
drb_status colsplit_launch(Csr &A, const void *x, void *y, cudaStream_t s);
// ||A x - b||^2 on the split copy: the same launch, the residual folded into
// the combine pass (a fixed grouping: repeatable bit for bit).
drb_status colsplit_residual(Csr &A, const void *x, const void *b, void *y, double *out,
                             cudaStream_t s);
drb_status colsplit_tune(Csr &A, cudaStream_t s);
// The host-pointer gemv of a column-split handle: x goes up block by block and
// each block's items run as soon as its slice has arrived; the last block runs
// in row segments whose rows copy back while later ones compute.  y is
// bit-identical to colsplit_launch's.
drb_status colsplit_gemv_host(Csr &A, const void *x_host, void *y_host, size_t xb,
                              size_t yb, cudaStream_t s);
drb_status abar_launch(Csr &A, const void *ybar, const void *x, void *abar,
                       cudaStream_t s);
drb_status residual_launch(Csr &A, const void *x, const void *b, void *y,
                           double *out, cudaStream_t s);
drb_status adjoint_build(Csr &A, cudaStream_t s);
drb_status adjoint_refresh_values(Csr &A, cudaStream_t s);
drb_status dense_launch(int64_t m, int64_t n, const void *A, int64_t lda,
                        const void *x, void *y, int64_t k, drb_layout layout,
                        drb_dtype dt, cudaStream_t s);
drb_status dot_launch(int64_t n, const void *a, const void *b, drb_dtype dt,
                      double *out, cudaStream_t s);
drb_status dot_noalloc_launch(int64_t n, const void *a, const void *b,
                              drb_dtype dt, double *out, cudaStream_t s);
int64_t dot_noalloc_max_n();
drb_status convert_launch(const void *in, int in_bytes, void *out,
                          int out_bytes, int64_t count, bool to_bf16,
                          cudaStream_t s);
drb_status transpose_launch(const void *in, void *out, int64_t rows,
                            int64_t cols, int elem_bytes, cudaStream_t s);

inline int dtype_bytes(drb_dtype t) {
  return (t == DRB_F64 || t == DRB_INT64) ? 8 : (t == DRB_BF16 ? 2 : 4);
}

// ---- vectors (reduce.cu) and conjugate gradients (cg.cu) ----------------------
bool elementwise_dtype(drb_dtype t); // F32, F64, INT32, INT64
drb_status reduce_launch(int64_t n, const void *x, drb_dtype dt, drb_reduce_op op,
                         const void *init, void *out, cudaStream_t s);
drb_status iota_launch(int64_t n, void *x, drb_dtype dt, int64_t start, cudaStream_t s);
drb_status fill_launch(int64_t n, void *x, drb_dtype dt, const void *value, cudaStream_t s);
drb_status cg_solve(Csr &A, const void *b, void *x, int64_t max_iters, double rtol,
                    drb_cg_info *info, cudaStream_t s);

} // namespace drb

// The opaque handle type of drb.h is the library's Csr.
struct drb_csr_matrix : public drb::Csr {};

// ---- PTX helpers ---------------------------------------------------------------
namespace drb::ptx {

// L2 policies: streamed matrix data is evicted first, the gathered vector x
// is kept (evict_last) so it stays L2-resident across the whole launch.
__device__ __forceinline__ uint64_t policy_evict_first() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t policy_evict_normal() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t policy_evict_last() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}

// 16-byte streaming load through the non-coherent path, not allocated in L1.
__device__ __forceinline__ uint4 ld_stream16(const void *ptr, uint64_t pol) {
  uint4 r;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.u32 "
               "{%0,%1,%2,%3}, [%4], %5;"
               : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
               : "l"(ptr), "l"(pol));
  return r;
}

// Store with an L2 eviction policy (results written once, e.g. y).
__device__ __forceinline__ void st_hint(float *ptr, float v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(ptr), "f"(v), "l"(pol)
               : "memory");
}
__device__ __forceinline__ void st_hint(double *ptr, double v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(ptr), "d"(v), "l"(pol)
               : "memory");
}

__device__ __forceinline__ float ld_keep(const float *ptr, uint64_t pol) {
  float r;
  asm("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;"
               : "=f"(r)
               : "l"(ptr), "l"(pol));
  return r;
}
__device__ __forceinline__ double ld_keep(const double *ptr, uint64_t pol) {
  double r;
  asm("ld.global.nc.L2::cache_hint.f64 %0, [%1], %2;"
               : "=d"(r)
               : "l"(ptr), "l"(pol));
  return r;
}
__device__ __forceinline__ float ld_keep(const __nv_bfloat16 *ptr,
                                         uint64_t pol) {
  unsigned short r;
  asm("ld.global.nc.L2::cache_hint.u16 %0, [%1], %2;"
               : "=h"(r)
               : "l"(ptr), "l"(pol));
  return __uint_as_float(((unsigned)r) << 16);
}

} // namespace drb::ptx
