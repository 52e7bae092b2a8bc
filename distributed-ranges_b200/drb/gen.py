"""Seeded synthetic CSR workloads (include/drb_gen.h), returned as numpy
arrays ready for distributed_sparse_matrix / csr_matrix_view."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi as capi

UNIFORM_PM1, NORMAL, NORMAL_ROWSCALE, ONES = 0, 1, 2, 3


def _p(a):
    return C.c_void_p(a.ctypes.data)


def zipf_alpha_for_mean(lo: int, hi: int, mean: float) -> float:
    return float(capi.lib.drb_gen_zipf_alpha_for_mean(lo, hi, mean))


def zipf_mean(lo: int, hi: int, alpha: float) -> float:
    return float(capi.lib.drb_gen_zipf_mean(lo, hi, alpha))


def _fill(m, n, rowptr64, seed, index_dtype, value_dtype, dist, nthreads):
    nnz = int(rowptr64[m])
    it = 0 if np.dtype(index_dtype) == np.int32 else 1
    vt = 0 if np.dtype(value_dtype) == np.float32 else 1
    colind = np.empty(max(nnz, 1), dtype=index_dtype)[:nnz]
    vals = np.empty(max(nnz, 1), dtype=value_dtype)[:nnz]
    rc = capi.lib.drb_gen_fill_uniform(m, n, _p(rowptr64), seed, it,
                                      C.c_void_p(colind.ctypes.data), vt,
                                      C.c_void_p(vals.ctypes.data), dist, nthreads)
    if rc != 0:
        raise ValueError("drb_gen_fill_uniform failed")
    rowptr = rowptr64 if it == 1 else rowptr64.astype(np.int32)
    return rowptr, colind, vals


def powerlaw_csr(m: int, n: int, *, alpha: float, lo: int = 1, hi: int = 16384,
                 seed: int = 0, index_dtype=np.int32, value_dtype=np.float32,
                 dist: int = UNIFORM_PM1, nthreads: int = 0):
    """Row lengths ~ truncated Zipf(alpha) on [lo, hi], uniform distinct sorted
    columns, values from `dist`.  Returns (rowptr, colind, values)."""
    rp = np.empty(m + 1, np.int64)
    nnz = capi.lib.drb_gen_rowptr_zipf(m, n, alpha, lo, hi, seed, _p(rp), nthreads)
    if nnz < 0:
        raise ValueError("drb_gen_rowptr_zipf failed")
    return _fill(m, n, rp, seed, index_dtype, value_dtype, dist, nthreads)


def uniform_rows_csr(m: int, n: int, *, lo: int, hi: int, seed: int = 0,
                     index_dtype=np.int32, value_dtype=np.float32,
                     dist: int = UNIFORM_PM1, nthreads: int = 0):
    """Row lengths ~ U[lo, hi] (integers)."""
    rp = np.empty(m + 1, np.int64)
    nnz = capi.lib.drb_gen_rowptr_uniform(m, n, lo, hi, seed, _p(rp), nthreads)
    if nnz < 0:
        raise ValueError("drb_gen_rowptr_uniform failed")
    return _fill(m, n, rp, seed, index_dtype, value_dtype, dist, nthreads)


def fixed_rows_csr(m: int, n: int, *, length: int, seed: int = 0,
                   index_dtype=np.int32, value_dtype=np.float32,
                   dist: int = UNIFORM_PM1, nthreads: int = 0):
    """Exactly `length` distinct sorted uniform columns per row."""
    rp = np.empty(m + 1, np.int64)
    if capi.lib.drb_gen_rowptr_fixed(m, n, length, _p(rp)) < 0:
        raise ValueError("drb_gen_rowptr_fixed failed")
    return _fill(m, n, rp, seed, index_dtype, value_dtype, dist, nthreads)


def laplacian2d_csr(g: int, *, index_dtype=np.int32, value_dtype=np.float64):
    """5-point Laplacian of a g x g grid (Dirichlet): m = g*g rows."""
    it = 0 if np.dtype(index_dtype) == np.int32 else 1
    vt = 0 if np.dtype(value_dtype) == np.float32 else 1
    nnz = capi.lib.drb_gen_laplacian2d(g, None, it, None, vt, None)
    rp = np.empty(g * g + 1, np.int64)
    ci = np.empty(nnz, index_dtype)
    v = np.empty(nnz, value_dtype)
    capi.lib.drb_gen_laplacian2d(g, _p(rp), it, _p(ci), vt, _p(v))
    return (rp if it == 1 else rp.astype(np.int32)), ci, v


def values(count: int, *, seed: int = 0, dtype=np.float32, dist: int = UNIFORM_PM1,
           nthreads: int = 0) -> np.ndarray:
    out = np.empty(max(count, 1), dtype)[:count]
    vt = 0 if np.dtype(dtype) == np.float32 else 1
    if capi.lib.drb_gen_values(count, seed, vt, C.c_void_p(out.ctypes.data), dist,
                               nthreads) != 0:
        raise ValueError("drb_gen_values failed")
    return out
