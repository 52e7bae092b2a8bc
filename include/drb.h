/*
 * drb.h -- C ABI of the B200-native gemv hot path of Distributed Ranges.
 *
 * One process owns one B200.  A CSR matrix is uploaded once into a handle
 * (device-resident row-block segments plus the execution plan) and multiplied
 * many times, as dr::mp::distributed_sparse_matrix is constructed once and
 * passed to dr::mp::gemv repeatedly.  Every entry point is extern "C", takes
 * plain pointers and sizes, never throws, and returns a drb_status.  After a
 * non-zero status, drb_last_error() returns a message for the calling thread.
 *
 * Reference interfaces replaced (paths relative to the reference project):
 *   drb_csr_create / drb_csr_destroy
 *       distributed_sparse_matrix(csr_matrix_view, root, distribution)
 *       include/dr/mp/containers/distributed_sparse_matrix.hpp:131-134, with
 *       csr_row_distribution::init (matrix_formats/csr_row_distribution.hpp:
 *       205-318) or csr_eq_distribution::init (csr_eq_distribution.hpp:
 *       220-333) and the destructors (:33-42 / :33-41).
 *   drb_csr_shape / drb_csr_num_segments / drb_csr_segment /
 *   drb_csr_get_entries
 *       shape(), nnz(), segments() and the segment iterator's get()
 *       (distributed_sparse_matrix.hpp:141-149; csr_row_segment.hpp:140-208).
 *   drb_read_matrix_market
 *       dr::read_csr (include/dr/detail/matrix_io.hpp:120-256).
 *   drb_csr_gemv / drb_csr_gemv_host
 *       dr::mp::gemv(root, res, A, broadcasted_vector | broadcasted_slim_matrix)
 *       include/dr/mp/algorithms/matrix/gemv.hpp:16-39 ->
 *       local_gemv_and_collect (distributed_sparse_matrix.hpp:153-158,
 *       csr_row_distribution.hpp:137-153, csr_eq_distribution.hpp:134-153).
 *
 *   drb_reduce / drb_iota / drb_fill
 *       dr::mp::reduce / iota / fill over a distributed_vector
 *       (include/dr/mp/algorithms/reduce.hpp:58-181, iota.hpp:20-34,
 *       fill.hpp:21-30).
 *
 * Entry points with no reference counterpart (new API shaped after gemv):
 *   drb_dense_gemv, drb_dot, drb_csr_residual_norm2, drb_csr_gemv_backward,
 *   drb_csr_update_values, drb_batch_*, drb_batched_gemv, drb_dense_batch_*,
 *   drb_csr_cg.
 *
 * Layouts.  Multi-RHS blocks follow broadcasted_slim_matrix: column-major,
 * x[c + j*n], y[r + j*m] (gemv.hpp:29-39, csr_row_distribution.hpp:129-130).
 * DRB_ROW_MAJOR (x[c*k + j], y[r*k + j]) is also accepted.
 *
 * Threads and streams.  Distinct handles may be used concurrently on distinct
 * streams; one handle must not be used by two threads at once.  All compute
 * entry points are asynchronous on the given stream (a cudaStream_t passed as
 * void*; NULL = the legacy default stream) except the *_host variants, which
 * synchronise the stream before returning.
 */
#ifndef DRB_H
#define DRB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int drb_status;
#define DRB_OK 0
#define DRB_ERR_INVALID_ARG 1 /* null pointer, negative size, bad enum      */
#define DRB_ERR_BAD_CSR 2     /* rowptr not monotone / column out of range  */
#define DRB_ERR_OOM 3         /* device or pinned host allocation failed    */
#define DRB_ERR_CUDA 4        /* a CUDA runtime call failed                 */
#define DRB_ERR_TIMEOUT 5     /* a bounded device-side wait expired         */
#define DRB_ERR_UNSUPPORTED 6 /* valid request this build does not handle   */
#define DRB_ERR_NO_DEVICE 7   /* no CUDA device / wrong architecture        */
#define DRB_ERR_IO 8          /* file missing, unreadable or not parsable   */

/* Element types.  DRB_INT32 / DRB_INT64 are accepted only by the vector
 * entry points (drb_reduce, drb_iota, drb_fill). */
typedef enum {
  DRB_F32 = 0,
  DRB_F64 = 1,
  DRB_BF16 = 2,
  DRB_INT32 = 3,
  DRB_INT64 = 4
} drb_dtype;
typedef enum { DRB_I32 = 0, DRB_I64 = 1 } drb_itype;
typedef enum { DRB_COL_MAJOR = 0, DRB_ROW_MAJOR = 1 } drb_layout;
/* How the rows are split into segments (the reference's MatrixDistrT):
 * DRB_PART_ROW = csr_row_distribution (rank r owns rows [r*ceil(m/P), ...)),
 * DRB_PART_EQ  = csr_eq_distribution (rank r owns nnz [r*ceil(nnz/P), ...);
 *                a row that straddles two segments is summed from both). */
typedef enum { DRB_PART_ROW = 0, DRB_PART_EQ = 1 } drb_partition;

/* drb_csr_create flags */
#define DRB_FLAG_DEVICE_INPUT 0x1u   /* rowptr/colind/values are device ptrs */
#define DRB_FLAG_KEEP_INDEX64 0x2u   /* keep 64-bit indices on the device    */
#define DRB_FLAG_SKIP_VALIDATE 0x4u  /* skip the host-side CSR validation    */
#define DRB_FLAG_ADJOINT 0x8u        /* build the CSC plan for gemv_backward */
#define DRB_FLAG_COMPENSATED 0x10u   /* two-sum compensated FP32 row sums    */
#define DRB_FLAG_AUTOTUNE 0x20u      /* run drb_csr_autotune at create       */
#define DRB_FLAG_BF16_X_F32 0x40u    /* BF16 storage: x stays f32 (not bf16)  */

typedef struct drb_csr_matrix *drb_csr_t;

/* ---- lifecycle ------------------------------------------------------------ */

/* Upload an m x n CSR matrix (rowptr[m+1], colind[nnz], values[nnz]; the
 * csr_matrix_view triple, csr_matrix_view.hpp:125-220) and build its plan.
 * value_type is the caller's element type (F32 or F64); storage is the device
 * element type: equal to value_type, or DRB_BF16 for F32 input (values are
 * rounded to bfloat16, gemv then takes bf16 x and writes f32 y).  nsegments
 * is the number of logical segments (the reference's MPI rank count; >= 1);
 * all segments live on the current device.  Index width: 64-bit input
 * indices are narrowed to 32 bits on the device when they fit, unless
 * DRB_FLAG_KEEP_INDEX64.  The stream orders the uploads; the call returns
 * after they complete. */
drb_status drb_csr_create(drb_csr_t *out, int64_t m, int64_t n, int64_t nnz,
                          const void *rowptr, const void *colind,
                          const void *values, drb_itype index_type,
                          drb_dtype value_type, drb_dtype storage,
                          int nsegments, drb_partition partition,
                          uint32_t flags, void *stream);

drb_status drb_csr_destroy(drb_csr_t A);

drb_status drb_csr_shape(drb_csr_t A, int64_t *m, int64_t *n, int64_t *nnz);

/* Device storage actually used: value bytes, column-index bytes, rowptr
 * bytes per element (for algorithmic-byte accounting). */
drb_status drb_csr_storage(drb_csr_t A, int *value_bytes, int *col_bytes,
                           int *rowptr_bytes);

drb_status drb_csr_num_segments(drb_csr_t A, int *nsegments);

/* Row and nnz range of segment `seg` (csr_row: rows [r*ceil(m/P), ...) and
 * their nnz; csr_eq: nnz [r*ceil(nnz/P), ...) and the rows they touch). */
drb_status drb_csr_segment(drb_csr_t A, int seg, int64_t *row_begin,
                           int64_t *row_end, int64_t *nnz_begin,
                           int64_t *nnz_end);

/* Copy `count` entries starting at global nnz offset `offset` to host arrays
 * (row, column, value as double); any output pointer may be NULL.  This is
 * the global iterator's dereference (distributed_sparse_matrix.hpp:103-107). */
drb_status drb_csr_get_entries(drb_csr_t A, int64_t offset, int64_t count,
                               int64_t *rows, int64_t *cols, double *values);

/* ---- the hot call ------------------------------------------------------- */

/* y = A * x for k right-hand sides, device pointers.  Element types: x and y
 * have the storage type, except BF16 storage: x bf16 (f32 with
 * DRB_FLAG_BF16_X_F32), y f32, row sums two-sum compensated in f32 per
 * block of four products (a bf16 x bf16 product being exact in f32 and a
 * bf16 x f32 one rounding once; the block sums add at most 3u of their
 * magnitudes, as drb_batch_*).  k > 1 runs
 * the batched SpMM kernel on a batch of this one handle, built on the first
 * call with a given (k, layout) -- that call synchronises `stream`, and the
 * handle then keeps a row-major copy of X (n * k elements, rows padded to 16
 * bytes) -- or, for 64-bit indices or a row-major x not 16-byte aligned, a
 * row-block kernel (F32/F64 only).  y is overwritten (the reference
 * zero-fills its partial result first). */
drb_status drb_csr_gemv(drb_csr_t A, const void *x, void *y, int64_t k,
                        drb_layout layout, void *stream);

/* Same product with HOST x and y (any host memory; pinned is fastest): the
 * call copies x to the device, multiplies, copies y back and synchronises,
 * as gemv(root, res, A, x) returns res on the host.  For k = 1 the copies
 * overlap the product (y comes back in row segments behind the compute, and
 * a column-split handle also uploads x block by block ahead of it); y has
 * the bits of drb_csr_gemv. */
drb_status drb_csr_gemv_host(drb_csr_t A, const void *x_host, void *y_host,
                             int64_t k, drb_layout layout, void *stream);

/* Kernel variant of the single right-hand-side product: item span (128, 256
 * or 512 nonzeros) | 2 for the two-slot pipelined kernel (the next item's
 * gathers in flight while the current item's rows are summed; 128 or 256,
 * skewed) | 1 when the skewed (bank-conflict-free) product layout is
 * used, or 2048 for the sliced-ELL copy (slices of 32 rows padded to their
 * longest row, lane = row), which drb_csr_create takes by default when the
 * longest row has <= 64 nonzeros, padding adds <= 20% and twice the copy's
 * size is free (the copy costs padded * (value + 4) bytes; the CSR arrays
 * stay for the other paths).  drb_csr_autotune times the row-block variants
 * and, when the matrix qualifies, the sliced copy on this matrix's sparsity
 * pattern, keeps the fastest (also for the adjoint's transposed matrix) and
 * returns it; it synchronises `stream`.  Results are identical across
 * variants up to the summation order inside a row.  For a column-split handle
 * (drb_csr_column_blocks) the variant is that of the block-major copy's plan,
 * which gemv runs (autotuned on its own). */
drb_status drb_csr_variant(drb_csr_t A, int *variant);
drb_status drb_csr_autotune(drb_csr_t A, int *variant, void *stream);

/* Column blocks of the single right-hand-side product (no counterpart in the
 * reference; a layout choice inside the handle).  A randomly gathered x stays
 * in B200's L2 only up to about 48 MB, so drb_csr_create regroups the
 * nonzeros of an F32/F64 handle whose x is larger than 48 MiB (and that
 * reuses x at least twice, nnz >= 2n) into *nblocks column blocks (x slices
 * of at most 48 MiB; *block_width is the first block's width: 45% of the
 * columns when there are two, so that the host-pointer call's first block
 * finishes as x's last slice lands; the others share the remaining columns
 * equally), kept as a second copy of the values
 * and column indices on the device (block-major: every row's nonzeros of
 * block 0, then of block 1, ...), with nblocks partial sums per row of
 * scratch, when that fits with 1 GB to spare.  drb_csr_gemv (k = 1) then runs
 * one launch over the copy -- its warps move through the blocks in order, so
 * one x slice at a time is hot in L2 -- and a short pass that adds each row's
 * block sums in block order.  drb_csr_gemv_host pipelines the same work over
 * the blocks: x goes up slice by slice, each block runs once its slice has
 * arrived, and the last block runs in row segments whose rows copy back
 * while the later segments compute.  Both are deterministic and give the same
 * bits.  The adjoint's transposed matrix is split the same way.  The
 * environment variables DRB_COLSPLIT=<n> (n blocks; 0 or 1: none) and
 * DRB_COLSPLIT_FIRST=<f> (a first block of f*n columns, 0 < f < 1; any other
 * value: equal widths), read when a handle is created, override the choice.  A handle on its sliced-ELL copy (short
 * regular rows, whose gathers are local) is not split.  *nblocks = 1 (and
 * *block_width = n) when the handle is not split. */
drb_status drb_csr_column_blocks(drb_csr_t A, int *nblocks, int64_t *block_width);

/* Synchronise `stream` and report device-side failures of earlier launches
 * on this handle: DRB_ERR_TIMEOUT when a bounded in-kernel wait expired (the
 * kernel then skipped the rest of its work; the error word is cleared). */
drb_status drb_csr_check(drb_csr_t A, void *stream);

/* Fused residual: out[0] = || A*x - b ||_2^2 accumulated in f64 (device
 * double*), y = A*x also written when y != NULL.  k = 1. */
drb_status drb_csr_residual_norm2(drb_csr_t A, const void *x, const void *b,
                                  void *y, double *out, void *stream);

/* ---- adjoint (needs DRB_FLAG_ADJOINT at create) ------------------------- */

/* For L(y) with y = A x and upstream gradient ybar (length m):
 *   xbar = A^T ybar (length n), atomics-free over the CSC plan;
 *   abar[p] = ybar[row(p)] * x[col(p)] for every stored entry p (CSR order).
 * Either output may be NULL to skip it.  Types as drb_csr_gemv (k = 1). */
drb_status drb_csr_gemv_backward(drb_csr_t A, const void *ybar, const void *x,
                                 void *xbar, void *abar, void *stream);

/* Replace the stored values (device pointer, CSR order, storage type) and
 * refresh the CSC copy used by gemv_backward. */
drb_status drb_csr_update_values(drb_csr_t A, const void *values,
                                 void *stream);

/* ---- batched execution ---------------------------------------------------
 * Y_i = A_i X_i for many handles in ONE persistent kernel launch, replayed
 * from a CUDA graph.  The reference multiplies one matrix per gemv call
 * (include/dr/mp/algorithms/matrix/gemv.hpp:29-39 with a
 * broadcasted_slim_matrix of k columns); a batch is that call for `count`
 * matrices at once.  X_i is n_i x k and Y_i is m_i x k, both in `layout`
 * (DRB_COL_MAJOR is the reference's slim-matrix layout, x[c + j*n]).
 * Element types as drb_csr_gemv: the storage type, or for BF16 storage bf16
 * X (f32 with DRB_FLAG_BF16_X_F32) and f32 Y; BF16 sums are two-sum
 * compensated f32, per block of four products (a fused multiply-add chain per
 * block): a row's error stays within about 5 f32 roundings of sum |a x|.
 * Handles must share the device and the storage type, have 32-bit rowptr and
 * column indices (nnz < 2^31 each), and must outlive the batch. */
typedef struct drb_batch_plan *drb_batch_t;

/* Build the batch's work list and capture its graph.  flags: 0 or
 * DRB_FLAG_BF16_X_F32.  The call synchronises `stream`. */
drb_status drb_batch_create(drb_batch_t *out, int32_t count,
                            const drb_csr_t *handles, int64_t k,
                            drb_layout layout, uint32_t flags, void *stream);

/* Bind the device pointers x[i], y[i] (arrays of `count` pointers, read
 * during the call).  The pointer table is updated in stream order, so later
 * launches on `stream` see it; rebinding needs no new graph.  Row-major X
 * must be aligned to the kernel's vector width (16 bytes always suffices). */
drb_status drb_batch_bind(drb_batch_t B, const void *const *x, void *const *y,
                          void *stream);

/* Launch the captured graph on `stream` (asynchronous).  A batch is not
 * reentrant: do not overlap two launches of the same batch. */
drb_status drb_batch_gemv(drb_batch_t B, void *stream);

/* Kernel variant: (c << 4) | G, with staging capacity 128 << c nonzeros per
 * work unit (c = 0, 1, 2) and G slots summing one row (1, 2, 4, 8).  The
 * default is c = 1 with G from the mean row length.  Results depend on G
 * only (the order of each row's sum), not on c, for rows of at most 128
 * nonzeros.  drb_batch_set_variant re-captures the graph;
 * drb_batch_autotune times every variant with the bound x and y (which it
 * overwrites with the product), keeps the fastest, re-captures the graph and
 * synchronises `stream`. */
drb_status drb_batch_variant(drb_batch_t B, int *variant);
drb_status drb_batch_set_variant(drb_batch_t B, int variant);
drb_status drb_batch_autotune(drb_batch_t B, int *variant, void *stream);

drb_status drb_batch_destroy(drb_batch_t B);

/* One-shot form: create, bind, launch (no graph), synchronise, destroy. */
drb_status drb_batched_gemv(int32_t count, const drb_csr_t *handles,
                            const void *const *x, void *const *y, int64_t k,
                            drb_layout layout, uint32_t flags, void *stream);

/* ---- dense and reductions ------------------------------------------------ */

/* y = A x for a row-major m x n matrix (leading dimension lda >= n), k RHS in
 * `layout`.  F32 or F64 (accumulated in the element type).  Device ptrs. */
drb_status drb_dense_gemv(int64_t m, int64_t n, const void *A, int64_t lda,
                          const void *x, void *y, int64_t k, drb_layout layout,
                          drb_dtype dtype, void *stream);

/* Batched dense multi-RHS product on the tensor cores: Y_i = A_i X_i for
 * `count` row-major BF16 matrices A_i (m[i] x n[i], leading dimension lda[i]:
 * a multiple of 8, A_i 16-byte aligned) and BF16 X_i (n[i] x k, 1 <= k <=
 * 256) in `layout`; Y_i (m[i] x k, `layout`) is FP32, accumulated in FP32
 * (tcgen05.mma into tensor memory).  dtype must be DRB_BF16.  The plan binds
 * the pointers and is launched any number of times; all matrices run in one
 * kernel (plus one small kernel that lays every X out K-major).  No
 * reference counterpart: it is gemv's multi-RHS form for a batch of dense
 * matrices (the reference's dense product is local_gemm,
 * include/dr/sp/algorithms/matrix/local_gemm.hpp:18-62). */
typedef struct drb_dense_batch_plan *drb_dense_batch_t;
drb_status drb_dense_batch_create(drb_dense_batch_t *out, int32_t count,
                                  const int64_t *m, const int64_t *n,
                                  const void *const *A, const int64_t *lda,
                                  const void *const *x, void *const *y,
                                  int64_t k, drb_layout layout,
                                  drb_dtype dtype, void *stream);
drb_status drb_dense_batch_gemv(drb_dense_batch_t P, void *stream);
/* TMA ring variant {stages, 64-wide K boxes per stage}: 0 = {4, 1},
 * 1 = {5, 1} (the default), 2 = {8, 1}, 3 = {2, 2}, 4 = {4, 2}.  Results do
 * not depend on the variant. */
drb_status drb_dense_batch_set_variant(drb_dense_batch_t P, int variant);
/* Synchronise `stream`; DRB_ERR_TIMEOUT when a bounded in-kernel wait of an
 * earlier launch expired (the error word is cleared). */
drb_status drb_dense_batch_check(drb_dense_batch_t P, void *stream);
/* Failure detection (no counterpart in the reference).  Later launches of
 * the plan limit every in-kernel wait to wait_ns nanoseconds (0 = the default,
 * one second), and with stall_tile >= 0 the CTA of that output tile issues no
 * loads, so its waits run out: the launch then stops early, leaves the
 * unfinished tiles of Y unwritten and drb_dense_batch_check returns
 * DRB_ERR_TIMEOUT; the plan stays usable.  stall_tile = -1 restores normal
 * launches. */
drb_status drb_dense_batch_set_wait(drb_dense_batch_t P, uint64_t wait_ns,
                                    int32_t stall_tile);
drb_status drb_dense_batch_destroy(drb_dense_batch_t P);

/* out[0] = sum_i a[i]*b[i] (a == b gives the squared norm), f64 accumulation
 * with a deterministic order; out is a device double*.  F32 or F64. */
drb_status drb_dot(int64_t n, const void *a, const void *b, drb_dtype dtype,
                   double *out, void *stream);

/* drb_dot without any allocation.  No counterpart in the reference: it exists
 * for callers that must not allocate device memory during the call -- code
 * running under a fixed memory budget, inside a caller's own allocator or
 * memory-pool callback, or on a stream whose allocations the caller has to
 * account for.  drb_dot takes its per-call scratch (one partial per CTA and a
 * completion ticket) from cudaMallocAsync; this variant takes it from a static
 * device array of 512 KiB that the library reserves on every GPU that loads
 * it, until process exit.  Limit: n <= 2^29 (536,870,912) elements; larger n
 * returns DRB_ERR_INVALID_ARG (use drb_dot).  The first call on each device
 * looks up the array's device address (cudaGetSymbolAddress) with that
 * device current, so make that first call before any stream capture.  The
 * address is kept per CUDA context: after the device's context is destroyed
 * and created again (cudaDeviceReset), the next call looks it up again, and
 * that call too belongs outside a capture.  Every
 * call shares the one array: calls that overlap on the GPU (different
 * streams, or different host threads) race and may return wrong sums, so
 * serialise them.  Same result contract as drb_dot (f64, deterministic for a
 * given n), though its partial sums are grouped differently. */
drb_status drb_dot_noalloc(int64_t n, const void *a, const void *b,
                           drb_dtype dtype, double *out, void *stream);

/* ---- vectors: mp::reduce, iota, fill ----------------------------------------
 * drb_reduce replaces dr::mp::reduce(root, r, init, op) / reduce(r, init, op)
 * / reduce(r) over a distributed_vector's segments
 * (include/dr/mp/algorithms/reduce.hpp:58-181): every segment is on this GPU,
 * so it is one launch over x[0, n).  op is std::plus, or std::min / std::max
 * (the reference tests' lambdas, test/gtest/common/reduce.cpp).  init: a host
 * pointer to one element of `dtype`, applied last as op(init, reduce(x)) as
 * reduce.hpp:110-120 does; NULL = no init.  n == 0 gives init, or zero without
 * one (reduce.hpp:63-65, 116-118).  out: a DEVICE pointer to one element of
 * `dtype`, written asynchronously on `stream`.  Integer sums wrap (the
 * sequential loop's result, bit for bit); float sums accumulate in f64 and
 * round once to dtype before init is added; min/max use std::min/std::max's
 * comparison.  Deterministic for a given n and x % 16. */
typedef enum {
  DRB_REDUCE_SUM = 0,
  DRB_REDUCE_MIN = 1,
  DRB_REDUCE_MAX = 2
} drb_reduce_op;
drb_status drb_reduce(int64_t n, const void *x, drb_dtype dtype,
                      drb_reduce_op op, const void *init, void *out,
                      void *stream);
/* x[i] = start + i (dr::mp::iota, include/dr/mp/algorithms/iota.hpp:20-34), and
 * x[i] = *value (dr::mp::fill, fill.hpp:21-30; value is a host pointer to one
 * element of dtype).  x is a device pointer; asynchronous on `stream`. */
drb_status drb_iota(int64_t n, void *x, drb_dtype dtype, int64_t start,
                    void *stream);
drb_status drb_fill(int64_t n, void *x, drb_dtype dtype, const void *value,
                    void *stream);

/* ---- device-resident conjugate gradients --------------------------------------
 * No counterpart in the reference: the loop its pieces allow (gemv + reduce +
 * element-wise updates) run entirely on the GPU.  Solves A x = b for a
 * symmetric positive definite A (m == n, F32 or F64 storage; x and b are
 * device vectors of that type; x holds the initial guess on entry) with
 * unpreconditioned CG (Hestenes-Stiefel):
 *   r = b - A x;  p = r;  rr = r.r
 *   repeat: q = A p;  alpha = rr / p.q;  x += alpha p;  r -= alpha q;
 *           rr' = r.r;  stop if rr' <= rtol^2 b.b;  p = r + (rr'/rr) p
 * The SpMV carries the p.q reduction in its epilogue; the x/r update carries
 * r.r.  Scalars stay in device memory (f64); the loop is replayed from a
 * CUDA graph in blocks of 8 iterations with one small device-to-host read
 * per block, and iterations after convergence return at once.  Stops on
 * convergence, at max_iters updates, or on breakdown (p.q <= 0 or not finite:
 * A is not SPD; x is left as it was before that iteration).  The call
 * synchronises `stream`. */
typedef struct {
  int64_t iterations;   /* updates applied to x                    */
  double residual_norm; /* ||r|| of the recurrence at exit          */
  double b_norm;        /* ||b||                                    */
  int converged;        /* ||r|| <= rtol ||b||                      */
  int breakdown;        /* p.Ap <= 0 or not finite                  */
} drb_cg_info;
drb_status drb_csr_cg(drb_csr_t A, const void *b, void *x, int64_t max_iters,
                      double rtol, drb_cg_info *info, void *stream);

/* ---- ingest ----------------------------------------------------------------
 * drb_read_matrix_market replaces dr::read_csr<T, I>(path, one_indexed)
 * (include/dr/detail/matrix_io.hpp:120-256): a coordinate Matrix Market file
 * (field real, integer or pattern -- pattern entries get value 1; symmetry
 * general or symmetric -- off-diagonal entries of a symmetric file are stored
 * at (i, j) and (j, i)) into host CSR arrays with rows sorted by column
 * (entries with equal columns keep their file order).  Errors, with the
 * reference's messages: DRB_ERR_IO (cannot open, not a coordinate Matrix
 * Market file, malformed line), DRB_ERR_UNSUPPORTED (skew-symmetric,
 * hermitian, ...), DRB_ERR_BAD_CSR (entry out of bounds, more entries than
 * the size line declares; the first one in file order is reported).  Blank
 * lines are skipped.  The arrays are allocated by the library: release them
 * with drb_csr_host_free.  Pass the result to drb_csr_create (DRB_I64,
 * DRB_F64) to upload it. */
typedef struct {
  int64_t m, n, nnz;
  int64_t *rowptr; /* m + 1 */
  int64_t *colind; /* nnz */
  double *values;  /* nnz */
} drb_csr_host;
drb_status drb_read_matrix_market(const char *path, int one_indexed,
                                  drb_csr_host *out);
void drb_csr_host_free(drb_csr_host *h);

/* ---- device memory (the reference's allocator and sycl_copy) --------------
 * Replaces dr::mp::__detail::allocator (include/dr/mp/allocator.hpp:14-33,
 * sycl::malloc_device under mp::init(queue, usm::alloc::device)) and
 * __detail::sycl_copy (include/dr/mp/sycl_support.hpp:51-53), so host code
 * above this ABI needs no CUDA headers.  kind: 0 host->device, 1 device->host,
 * 2 device->device.  drb_memcpy is asynchronous on `stream` (host memory must
 * stay valid until the stream is synchronised). */
drb_status drb_malloc(void **ptr, size_t bytes);
drb_status drb_free(void *ptr);
drb_status drb_memcpy(void *dst, const void *src, size_t bytes, int kind,
                      void *stream);
drb_status drb_memset(void *dst, int value, size_t bytes, void *stream);
drb_status drb_stream_synchronize(void *stream);

/* ---- misc ----------------------------------------------------------------- */

const char *drb_last_error(void);
const char *drb_version(void);
/* Number of kernels this library has launched in the calling process. */
uint64_t drb_launch_count(void);

#ifdef __cplusplus
}
#endif

#endif /* DRB_H */
