/*
 * drb_gen.h -- seeded synthetic CSR workloads (host side, multithreaded).
 *
 * The reference generates its test and benchmark matrices on the host with
 * dr::generate_random_csr / dr::generate_band_csr
 * (include/dr/detail/generate_csr.hpp:40-153).  Those two are mirrored exactly
 * in include/drb/generate.hpp.  The functions here produce the larger
 * synthetic shapes this project benchmarks (power-law row lengths, fixed row
 * lengths, the 2-D 5-point Laplacian).  Every random quantity comes from a
 * counter-based generator keyed by (seed, stream, row), so the output does not
 * depend on the number of threads.
 *
 * Index arrays: rowptr is int64[m+1]; colind is int32 or int64 (itype).
 * Columns within a row are distinct and ascending.
 */
#ifndef DRB_GEN_H
#define DRB_GEN_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Value distributions */
#define DRB_GEN_UNIFORM_PM1 0   /* U(-1, 1)                               */
#define DRB_GEN_NORMAL 1        /* N(0, 1)                                */
#define DRB_GEN_NORMAL_ROWSCALE 2 /* N(0,1) * 10^U(-3,3), one scale per row */
#define DRB_GEN_ONES 3          /* 1                                      */

/* Exponent alpha of a Zipf law truncated to [lo, hi] whose mean is `mean`
 * (bisection).  Returns NaN when the mean is outside (lo, hi). */
double drb_gen_zipf_alpha_for_mean(int64_t lo, int64_t hi, double mean);

/* Mean of the Zipf law P(L = k) ~ k^-alpha truncated to [lo, hi]. */
double drb_gen_zipf_mean(int64_t lo, int64_t hi, double alpha);

/* Row lengths drawn from the truncated Zipf law (inverse-CDF table), capped at
 * n; writes rowptr[m+1] (prefix sums) and returns nnz (or -1 on error). */
int64_t drb_gen_rowptr_zipf(int64_t m, int64_t n, double alpha, int64_t lo,
                            int64_t hi, uint64_t seed, int64_t *rowptr,
                            int nthreads);

/* Row lengths drawn uniformly from [lo, hi] (capped at n); returns nnz. */
int64_t drb_gen_rowptr_uniform(int64_t m, int64_t n, int64_t lo, int64_t hi,
                               uint64_t seed, int64_t *rowptr, int nthreads);

/* Every row has exactly `len` entries (len <= n); returns nnz. */
int64_t drb_gen_rowptr_fixed(int64_t m, int64_t n, int64_t len,
                             int64_t *rowptr);

/* Fill colind (distinct, ascending, uniform over [0, n)) and values for the
 * rows described by rowptr.  itype: 0 = int32, 1 = int64.  vtype: 0 = f32,
 * 1 = f64.  dist: DRB_GEN_*.  Returns 0 on success. */
int drb_gen_fill_uniform(int64_t m, int64_t n, const int64_t *rowptr,
                         uint64_t seed, int itype, void *colind, int vtype,
                         void *values, int dist, int nthreads);

/* 5-point Laplacian of a g x g grid with Dirichlet boundary (out-of-grid
 * neighbours dropped): diagonal 4, neighbours -1, rows in row-major grid
 * order, columns ascending.  m = g*g rows.  Sizes first: returns nnz
 * (= 5*g*g - 4*g); buffers may be NULL to only count. */
int64_t drb_gen_laplacian2d(int64_t g, int64_t *rowptr, int itype,
                            void *colind, int vtype, void *values);

/* Dense vector / matrix entries: out[i] for i in [0, count), drawn from dist
 * with the counter-based generator keyed by (seed, i). */
int drb_gen_values(int64_t count, uint64_t seed, int vtype, void *out,
                   int dist, int nthreads);

#ifdef __cplusplus
}
#endif

#endif /* DRB_GEN_H */
