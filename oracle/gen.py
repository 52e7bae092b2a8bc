"""The seeded workload generator (include/drb_gen.h) as linked into
oracle/liboracle.so.

TEST INFRASTRUCTURE ONLY.  The same source file builds the product's
drb.gen; this copy lets bench.py's reference arm and the tests build the
bench matrices without loading the CUDA library.  tests/test_oracle_golden.py
checks that both produce the same bytes.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import lib

UNIFORM_PM1, NORMAL, NORMAL_ROWSCALE, ONES = 0, 1, 2, 3

_v, _i64, _i, _u64, _d = C.c_void_p, C.c_int64, C.c_int, C.c_uint64, C.c_double
for _n, _r, _a in (
        ("drb_gen_zipf_alpha_for_mean", _d, [_i64, _i64, _d]),
        ("drb_gen_zipf_mean", _d, [_i64, _i64, _d]),
        ("drb_gen_rowptr_zipf", _i64, [_i64, _i64, _d, _i64, _i64, _u64, _v, _i]),
        ("drb_gen_rowptr_uniform", _i64, [_i64, _i64, _i64, _i64, _u64, _v, _i]),
        ("drb_gen_rowptr_fixed", _i64, [_i64, _i64, _i64, _v]),
        ("drb_gen_fill_uniform", _i, [_i64, _i64, _v, _u64, _i, _v, _i, _v, _i, _i]),
        ("drb_gen_values", _i, [_i64, _u64, _i, _v, _i, _i])):
    _f = getattr(lib, _n)
    _f.restype = _r
    _f.argtypes = _a


def _p(a):
    return C.c_void_p(a.ctypes.data)


def zipf_alpha_for_mean(lo: int, hi: int, mean: float) -> float:
    return float(lib.drb_gen_zipf_alpha_for_mean(lo, hi, mean))


def zipf_mean(lo: int, hi: int, alpha: float) -> float:
    return float(lib.drb_gen_zipf_mean(lo, hi, alpha))


def _fill(m, n, rowptr64, seed, index_dtype, value_dtype, dist, nthreads):
    nnz = int(rowptr64[m])
    it = 0 if np.dtype(index_dtype) == np.int32 else 1
    vt = 0 if np.dtype(value_dtype) == np.float32 else 1
    colind = np.empty(max(nnz, 1), dtype=index_dtype)[:nnz]
    vals = np.empty(max(nnz, 1), dtype=value_dtype)[:nnz]
    if lib.drb_gen_fill_uniform(m, n, _p(rowptr64), seed, it, _p(colind), vt, _p(vals),
                                dist, nthreads) != 0:
        raise ValueError("drb_gen_fill_uniform failed")
    rowptr = rowptr64 if it == 1 else rowptr64.astype(np.int32)
    return rowptr, colind, vals


def powerlaw_csr(m: int, n: int, *, alpha: float, lo: int = 1, hi: int = 16384,
                 seed: int = 0, index_dtype=np.int32, value_dtype=np.float32,
                 dist: int = UNIFORM_PM1, nthreads: int = 0):
    """Row lengths ~ truncated Zipf(alpha) on [lo, hi], uniform distinct sorted
    columns, values from `dist`: (rowptr, colind, values)."""
    rp = np.empty(m + 1, np.int64)
    if lib.drb_gen_rowptr_zipf(m, n, alpha, lo, hi, seed, _p(rp), nthreads) < 0:
        raise ValueError("drb_gen_rowptr_zipf failed")
    return _fill(m, n, rp, seed, index_dtype, value_dtype, dist, nthreads)


def uniform_rows_csr(m: int, n: int, *, lo: int, hi: int, seed: int = 0,
                     index_dtype=np.int32, value_dtype=np.float32,
                     dist: int = UNIFORM_PM1, nthreads: int = 0):
    """Row lengths ~ U[lo, hi]."""
    rp = np.empty(m + 1, np.int64)
    if lib.drb_gen_rowptr_uniform(m, n, lo, hi, seed, _p(rp), nthreads) < 0:
        raise ValueError("drb_gen_rowptr_uniform failed")
    return _fill(m, n, rp, seed, index_dtype, value_dtype, dist, nthreads)


def values(count: int, *, seed: int = 0, dtype=np.float32, dist: int = UNIFORM_PM1,
           nthreads: int = 0) -> np.ndarray:
    out = np.empty(max(count, 1), dtype)[:count]
    vt = 0 if np.dtype(dtype) == np.float32 else 1
    if lib.drb_gen_values(count, seed, vt, _p(out), dist, nthreads) != 0:
        raise ValueError("drb_gen_values failed")
    return out
