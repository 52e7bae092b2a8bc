/*
 * oracle.h -- CPU restatement of Distributed Ranges' gemv hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load it.  Nothing in the product (distributed-ranges_b200/) links or calls
 * it, and the product never falls back to it.
 *
 * Every function restates one piece of the reference's algorithm and cites
 * the reference file:line it follows (paths are relative to the reference
 * project root).  Value-type codes: 0 = float, 1 = double.  Index-type codes:
 * 0 = int32, 1 = int64, 2 = uint64 (the reference tests' `unsigned long`).
 *
 * Accumulation modes for the gemv restatements:
 *   ORC_ACC_T      accumulate in the value type T (the reference's own
 *                  semantics: `T sum`, `res[...] += ...` in T);
 *   ORC_ACC_F64    accumulate in double, output double;
 *   ORC_ACC_LD     accumulate in x87 long double, output double (a near-exact
 *                  FP64 oracle for error statistics).
 */
#ifndef DRB_ORACLE_H
#define DRB_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_F32 = 0, ORC_F64 = 1 };
enum { ORC_I32 = 0, ORC_I64 = 1, ORC_U64 = 2 };
enum { ORC_ACC_T = 0, ORC_ACC_F64 = 1, ORC_ACC_LD = 2 };

/* ---- generators (include/dr/detail/generate_csr.hpp) ------------------- */

/* nnz that generate_random_csr produces: size_t(density * m * n)
 * (generate_csr.hpp:48). */
int64_t orc_random_csr_nnz(int64_t m, int64_t n, double density);

/* Restates dr::generate_random_csr<T, I>(shape, density, seed)
 * (generate_csr.hpp:40-103): mt19937(seed), row then column draws from
 * uniform_int_distribution<I>, a uniform_real_distribution<T>(0,1) value for
 * each new (row, col) pair, entries sorted by (row, col), then the CSR fill.
 * Output buffers: rowptr[m+1], colind[nnz], vals[nnz] of the given types. */
int orc_gen_random_csr(int vtype, int itype, int64_t m, int64_t n,
                       double density, uint32_t seed, void *rowptr,
                       void *colind, void *vals);

/* nnz of generate_band_csr (generate_csr.hpp:111-113). */
int64_t orc_band_csr_nnz(int64_t size, int64_t up, int64_t down);

/* Restates dr::generate_band_csr<T, I>(size, up, down)
 * (generate_csr.hpp:108-153): all values 1, columns i-down..i+up. */
int orc_gen_band_csr(int vtype, int itype, int64_t size, int64_t up,
                     int64_t down, void *rowptr, void *colind, void *vals);

/* ---- gemv (csr_row / csr_eq CPU branches) ------------------------------ */

/* y = A*x over `nseg` row-block segments, restating
 * csr_row_distribution::local_gemv's CPU branch
 * (include/dr/mp/containers/matrix_formats/csr_row_distribution.hpp:116-133)
 * per segment plus gather_gemv_vector's reassembly (:159-204).
 * x is n*k column-major (x[c + j*n]); y is m*k column-major (y[r + j*m]).
 * With acc = ORC_ACC_T, y has the value type; otherwise y is double. */
int orc_csr_gemv_row(int vtype, int itype, int acc, int64_t m, int64_t n,
                     const void *rowptr, const void *colind, const void *vals,
                     const void *x, int64_t k, void *y, int nseg);

/* Same product over `nseg` equal-nnz segments, restating
 * csr_eq_distribution::local_gemv's CPU branch
 * (include/dr/mp/containers/matrix_formats/csr_eq_distribution.hpp:112-130),
 * the row ranges of init (:253-272) and the gather that adds each segment's
 * first (possibly split) row and copies the rest (:185-205). */
int orc_csr_gemv_eq(int vtype, int itype, int acc, int64_t m, int64_t n,
                    const void *rowptr, const void *colind, const void *vals,
                    const void *x, int64_t k, void *y, int nseg);

/* CPU baseline: the csr_row CPU loop run by `nthreads` std::threads, each
 * owning the reference's row block ceil(m/P) (one thread stands in for one
 * MPI rank).  Accumulates in T.  Returns elapsed seconds of the local phase in
 * *t_local and of the gather (copy into y) in *t_gather. */
int orc_csr_gemv_row_threads(int vtype, int itype, int64_t m, int64_t n,
                             const void *rowptr, const void *colind,
                             const void *vals, const void *x, int64_t k,
                             void *y, int nthreads, double *t_local,
                             double *t_gather);

/* Per-row error denominators: d[r + j*m] = sum_p |a_p * x[col_p + j*n]|
 * (double).  Used for relative-error gates under cancellation. */
int orc_csr_absdot(int vtype, int itype, int64_t m, int64_t n,
                   const void *rowptr, const void *colind, const void *vals,
                   const void *x, int64_t k, double *d);

/* ---- dense gemv (no reference symbol; row-dot restatement) ------------- */

/* y[r + j*m] = sum_c A[r*lda + c] * x[c + j*n], accumulated per `acc`. */
int orc_dense_gemv(int vtype, int acc, int64_t m, int64_t n, const void *A,
                   int64_t lda, const void *x, int64_t k, void *y);

/* ---- adjoint ----------------------------------------------------------- */

/* Explicit CSR -> CSC transpose on the host (stable: rows ascending within
 * a column).  Outputs colptr[n+1], rowidx[nnz], vals_t[nnz] in the input
 * types. */
int orc_csr_transpose(int vtype, int itype, int64_t m, int64_t n,
                      const void *rowptr, const void *colind, const void *vals,
                      void *colptr, void *rowidx, void *vals_t);

/* abar[p] = ybar[row(p)] * x[col(p)] on the sparsity pattern (double). */
int orc_csr_abar(int vtype, int itype, int64_t m, const void *rowptr,
                 const void *colind, const void *ybar, const void *x,
                 double *abar);

/* ---- reductions (include/dr/mp/algorithms/reduce.hpp:9-20 std_reduce) -- */

/* sum_i a[i]*b[i] accumulated in long double, returned as double. */
double orc_dot(int vtype, int64_t n, const void *a, const void *b);

/* ---- parity statistics (the checker at full sizes) ----------------------- */

/* Element-type codes of the checkers: ORC_F32, ORC_F64, or ORC_BF16 (bfloat16
 * bits, widened exactly to float). */
enum { ORC_BF16 = 3 };

/* Per-row error of a result y against the csr_row loop
 * (csr_row_distribution.hpp:116-133), for every row r and right-hand side j:
 *   ref = sum_p a_p * x[col_p + j*n]     accumulated in long double,
 *   d   = sum_p |a_p * x[col_p + j*n]|   (long double),
 *   err = |y[r + j*m] - ref| / d          (|y - ref| when d == 0).
 * vtype / xtype: element types of the values and of x (F32 | F64 | BF16);
 * itype: of rowptr and colind (I32 | I64); ytype: of y (F32 | F64).  x is
 * n*k column-major, y m*k column-major (k = 1: plain vectors).  Rows are split
 * over `nthreads` threads.  Statistics per bin of row length (rows of length
 * L with edges[b] <= L < edges[b+1], b < nbins): bmax[b], bsum[b] (sum of
 * err, for the mean), bcount[b] (row x rhs pairs); *worst = the largest err
 * over all rows and *worst_row its row.  NaN in y counts as an infinite err.
 * Returns 0, or 1 on an unsupported type code. */
int orc_csr_check(int vtype, int xtype, int itype, int ytype, int64_t m,
                  int64_t n, const void *rowptr, const void *colind,
                  const void *vals, const void *x, int64_t k, const void *y,
                  int nthreads, const int64_t *edges, int nbins, double *bmax,
                  double *bsum, int64_t *bcount, double *worst,
                  int64_t *worst_row);

/* The same statistics for a dense row-major A (m x n, leading dimension lda,
 * element type atype = F32 | F64 | BF16), x n*k and y m*k column-major:
 * ref_r = sum_c A[r*lda + c] * x[c + j*n] in long double, d = sum |.|.
 * One bin (all rows): *max, *sum, *count. */
int orc_dense_check(int atype, int xtype, int ytype, int64_t m, int64_t n,
                    const void *A, int64_t lda, const void *x, int64_t k,
                    const void *y, int nthreads, double *max, double *sum,
                    int64_t *count);

/* ---- bf16 helpers -------------------------------------------------------- */

/* Round-to-nearest-even float -> bfloat16 bits (NaN kept quiet). */
void orc_f32_to_bf16(int64_t n, const float *in, uint16_t *out);
void orc_bf16_to_f32(int64_t n, const uint16_t *in, float *out);

/* ---- Matrix Market ingest (include/dr/detail/matrix_io.hpp) ------------ */

/* Restates dr::read_csr<double, I>(path, one_indexed)
 * (matrix_io.hpp:120-256): header "%%MatrixMarket matrix coordinate <field>
 * <general|symmetric>" (field "pattern" gives value 1), '%' comment lines,
 * the "m n nnz" line, then one entry per line, 1-based when one_indexed;
 * off-diagonal entries of a symmetric file are also stored mirrored; rows are
 * sorted by column (stable here; the reference's std::sort leaves equal
 * columns in an unspecified order); blank lines are skipped (the reference
 * does not handle them).  Arrays are malloc'd (free with orc_free).
 * Returns 0, or 1 cannot open, 2 not a coordinate Matrix Market file,
 * 3 unsupported symmetry, 4 entry out of bounds, 5 more entries than the
 * size line declares, 6 malformed line; `err` receives a message. */
int orc_read_matrix_market(const char *path, int one_indexed, int64_t *m,
                           int64_t *n, int64_t *nnz, int64_t **rowptr,
                           int64_t **colind, double **values, char *err,
                           int errlen);
void orc_free(void *p);

/* ---- conjugate gradients (no reference symbol) ------------------------- */

/* Unpreconditioned CG (Hestenes-Stiefel), all in double, built from the
 * reference's own pieces: the product q = A p is the csr_row CPU loop
 * (csr_row_distribution.hpp:116-133, accumulated in double) and each dot is
 * the sequential std::reduce of zip | transform(mul) (examples/mp/
 * dot_product_benchmark.cpp:71-79, dot_product_sequential):
 *   r = b - A x; p = r; rr = r.r
 *   repeat: q = A p; alpha = rr / p.q; (stop as breakdown if p.q <= 0 or
 *           alpha not finite) x += alpha p; r -= alpha q; rr' = r.r;
 *           stop if rr' <= rtol^2 b.b, or after max_iters updates;
 *           p = r + (rr'/rr) p
 * x holds the initial guess and receives the result.  status: 1 converged,
 * 2 breakdown, 3 max_iters.  hist (may be NULL, max_iters + 1 entries):
 * ||r|| after 0, 1, ... updates. */
int orc_cg(int vtype, int itype, int64_t n, const void *rowptr,
           const void *colind, const void *vals, const double *b, double *x,
           int64_t max_iters, double rtol, int64_t *iters, double *rnorm,
           double *bnorm, int *status, double *hist);

#ifdef __cplusplus
}
#endif

#endif /* DRB_ORACLE_H */
