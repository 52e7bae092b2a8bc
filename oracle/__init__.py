"""Python access to the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, always as the checker or the timed CPU
baseline, never as the product path.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_GEN = os.path.join(HERE, "_ref", "ref_gen")
REF_MMREAD = os.path.join(HERE, "_ref", "ref_mmread")

F32, F64 = 0, 1
BF16 = 3  # bfloat16 bits held in uint16 arrays (the checkers only)
I32, I64, U64 = 0, 1, 2
ACC_T, ACC_F64, ACC_LD = 0, 1, 2

if not os.path.exists(LIB_PATH):
    raise ImportError(f"oracle not built ({LIB_PATH}); run make -C oracle")

lib = C.CDLL(LIB_PATH)
_v, _i64, _i = C.c_void_p, C.c_int64, C.c_int
_SIGS = {
    "orc_random_csr_nnz": (_i64, [_i64, _i64, C.c_double]),
    "orc_gen_random_csr": (_i, [_i, _i, _i64, _i64, C.c_double, C.c_uint32, _v, _v, _v]),
    "orc_band_csr_nnz": (_i64, [_i64, _i64, _i64]),
    "orc_gen_band_csr": (_i, [_i, _i, _i64, _i64, _i64, _v, _v, _v]),
    "orc_csr_gemv_row": (_i, [_i, _i, _i, _i64, _i64, _v, _v, _v, _v, _i64, _v, _i]),
    "orc_csr_gemv_eq": (_i, [_i, _i, _i, _i64, _i64, _v, _v, _v, _v, _i64, _v, _i]),
    "orc_csr_gemv_row_threads": (_i, [_i, _i, _i64, _i64, _v, _v, _v, _v, _i64, _v, _i,
                                      C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "orc_csr_absdot": (_i, [_i, _i, _i64, _i64, _v, _v, _v, _v, _i64, _v]),
    "orc_dense_gemv": (_i, [_i, _i, _i64, _i64, _v, _i64, _v, _i64, _v]),
    "orc_csr_transpose": (_i, [_i, _i, _i64, _i64, _v, _v, _v, _v, _v, _v]),
    "orc_csr_abar": (_i, [_i, _i, _i64, _v, _v, _v, _v, _v]),
    "orc_dot": (C.c_double, [_i, _i64, _v, _v]),
    "orc_csr_check": (_i, [_i, _i, _i, _i, _i64, _i64, _v, _v, _v, _v, _i64, _v, _i, _v, _i,
                           _v, _v, _v, C.POINTER(C.c_double), C.POINTER(_i64)]),
    "orc_dense_check": (_i, [_i, _i, _i, _i64, _i64, _v, _i64, _v, _i64, _v, _i,
                             C.POINTER(C.c_double), C.POINTER(C.c_double),
                             C.POINTER(_i64)]),
    "orc_f32_to_bf16": (None, [_i64, _v, _v]),
    "orc_bf16_to_f32": (None, [_i64, _v, _v]),
    "orc_read_matrix_market": (_i, [C.c_char_p, _i, C.POINTER(_i64), C.POINTER(_i64),
                                    C.POINTER(_i64), C.POINTER(C.c_void_p),
                                    C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                    C.c_char_p, _i]),
    "orc_free": (None, [_v]),
    "orc_cg": (_i, [_i, _i, _i64, _v, _v, _v, _v, _v, _i64, C.c_double,
                    C.POINTER(_i64), C.POINTER(C.c_double), C.POINTER(C.c_double),
                    C.POINTER(_i), _v]),
}
for _n, (_r, _a) in _SIGS.items():
    _f = getattr(lib, _n)
    _f.restype = _r
    _f.argtypes = _a


def _p(a):
    return C.c_void_p(a.ctypes.data) if a is not None else C.c_void_p(0)


def vcode(dtype) -> int:
    return {np.dtype(np.float32): F32, np.dtype(np.float64): F64}[np.dtype(dtype)]


def icode(dtype) -> int:
    return {np.dtype(np.int32): I32, np.dtype(np.int64): I64,
            np.dtype(np.uint64): U64}[np.dtype(dtype)]


def random_csr(m, n, density, seed=0, value_dtype=np.float32, index_dtype=np.uint64):
    """dr::generate_random_csr<T, I>(shape, density, seed), restated."""
    nnz = lib.orc_random_csr_nnz(m, n, density)
    rp = np.empty(m + 1, index_dtype)
    ci = np.empty(max(nnz, 1), index_dtype)[:nnz]
    v = np.empty(max(nnz, 1), value_dtype)[:nnz]
    rc = lib.orc_gen_random_csr(vcode(value_dtype), icode(index_dtype), m, n, density,
                                seed, _p(rp), _p(ci), _p(v))
    assert rc == 0
    return rp, ci, v


def band_csr(size, up=3, down=3, value_dtype=np.float32, index_dtype=np.uint64):
    """dr::generate_band_csr<T, I>(size, up, down), restated."""
    nnz = lib.orc_band_csr_nnz(size, up, down)
    rp = np.empty(size + 1, index_dtype)
    ci = np.empty(nnz, index_dtype)
    v = np.empty(nnz, value_dtype)
    rc = lib.orc_gen_band_csr(vcode(value_dtype), icode(index_dtype), size, up, down,
                              _p(rp), _p(ci), _p(v))
    assert rc == 0
    return rp, ci, v


def _gemv(fn, rp, ci, v, x, m, n, k, acc, nseg):
    x = np.ascontiguousarray(x, dtype=v.dtype)
    out_dtype = v.dtype if acc == ACC_T else np.float64
    y = np.empty(max(m * k, 1), out_dtype)[: m * k]
    rc = fn(vcode(v.dtype), icode(ci.dtype), acc, m, n, _p(rp), _p(ci), _p(v), _p(x), k,
            _p(y), nseg)
    assert rc == 0, "oracle gemv failed"
    return y


def gemv_row(rp, ci, v, x, m, n, k=1, acc=ACC_T, nseg=1):
    """csr_row_distribution CPU loop + gather; x, y column-major."""
    return _gemv(lib.orc_csr_gemv_row, rp, ci, v, x, m, n, k, acc, nseg)


def gemv_eq(rp, ci, v, x, m, n, k=1, acc=ACC_T, nseg=1):
    """csr_eq_distribution CPU loop + split-row gather; x, y column-major."""
    return _gemv(lib.orc_csr_gemv_eq, rp, ci, v, x, m, n, k, acc, nseg)


def gemv_row_threads(rp, ci, v, x, m, n, k=1, nthreads=1):
    x = np.ascontiguousarray(x, dtype=v.dtype)
    y = np.empty(max(m * k, 1), v.dtype)[: m * k]
    tl, tg = C.c_double(), C.c_double()
    rc = lib.orc_csr_gemv_row_threads(vcode(v.dtype), icode(ci.dtype), m, n, _p(rp),
                                      _p(ci), _p(v), _p(x), k, _p(y), nthreads,
                                      C.byref(tl), C.byref(tg))
    assert rc == 0
    return y, tl.value, tg.value


def absdot(rp, ci, v, x, m, n, k=1):
    x = np.ascontiguousarray(x, dtype=v.dtype)
    d = np.empty(max(m * k, 1), np.float64)[: m * k]
    assert lib.orc_csr_absdot(vcode(v.dtype), icode(ci.dtype), m, n, _p(rp), _p(ci), _p(v),
                              _p(x), k, _p(d)) == 0
    return d


def dense_gemv(A, x, k=1, acc=ACC_F64):
    m, n = A.shape
    A = np.ascontiguousarray(A)
    x = np.ascontiguousarray(x, dtype=A.dtype)
    y = np.empty(m * k, A.dtype if acc == ACC_T else np.float64)
    assert lib.orc_dense_gemv(vcode(A.dtype), acc, m, n, _p(A), n, _p(x), k, _p(y)) == 0
    return y


def transpose(rp, ci, v, m, n):
    nnz = int(rp[m])
    cp = np.empty(n + 1, ci.dtype)
    ri = np.empty(max(nnz, 1), ci.dtype)[:nnz]
    vt = np.empty(max(nnz, 1), v.dtype)[:nnz]
    assert lib.orc_csr_transpose(vcode(v.dtype), icode(ci.dtype), m, n, _p(rp), _p(ci),
                                 _p(v), _p(cp), _p(ri), _p(vt)) == 0
    return cp, ri, vt


def abar(rp, ci, ybar, x, m):
    nnz = int(rp[m])
    ybar = np.ascontiguousarray(ybar)
    x = np.ascontiguousarray(x, dtype=ybar.dtype)
    out = np.empty(max(nnz, 1), np.float64)[:nnz]
    assert lib.orc_csr_abar(vcode(ybar.dtype), icode(ci.dtype), m, _p(rp), _p(ci),
                            _p(ybar), _p(x), _p(out)) == 0
    return out


def dot(a, b):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b, dtype=a.dtype)
    return float(lib.orc_dot(vcode(a.dtype), a.size, _p(a), _p(b)))


# row-length bins of the parity statistics: [1], [2, 4], [5, 16], [17, 64],
# [65, 256], [257, 1024], [1025, ...)
ROW_BINS = (1, 2, 5, 17, 65, 257, 1025, 1 << 62)


def _ecode(a) -> int:
    return {np.dtype(np.float32): F32, np.dtype(np.float64): F64,
            np.dtype(np.uint16): BF16}[np.dtype(a.dtype)]


def _nthreads(n):
    return int(n) if n else (os.cpu_count() or 1)


def csr_check(rp, ci, v, x, m, n, y, k=1, nthreads=0, edges=ROW_BINS):
    """Per-row error of y against the csr_row loop accumulated in long double
    (orc_csr_check): err = |y - ref| / sum|a x| per row and right-hand side.
    v, x: float32 / float64 / uint16 (bf16 bits) arrays; x n*k and y m*k
    column-major.  Returns {"max", "mean", "count", "worst_row", "bins":
    {"lo-hi": {"rows", "max", "mean"}}} (bins of row length)."""
    assert ci.dtype == rp.dtype and ci.dtype in (np.int32, np.int64)
    y = np.ascontiguousarray(y)
    x = np.ascontiguousarray(x)
    nb = len(edges) - 1
    e = np.asarray(edges, np.int64)
    bmax, bsum = np.zeros(nb), np.zeros(nb)
    bcnt = np.zeros(nb, np.int64)
    worst, wrow = C.c_double(), _i64()
    rc = lib.orc_csr_check(_ecode(v), _ecode(x), icode(ci.dtype), _ecode(y), m, n, _p(rp),
                           _p(ci), _p(v), _p(x), k, _p(y), _nthreads(nthreads), _p(e), nb,
                           _p(bmax), _p(bsum), _p(bcnt), C.byref(worst), C.byref(wrow))
    assert rc == 0, "orc_csr_check failed"
    total = int(bcnt.sum())
    bins = {}
    for b in range(nb):
        if bcnt[b]:
            hi = "max" if e[b + 1] >= (1 << 60) else str(int(e[b + 1]) - 1)
            bins[f"{int(e[b])}-{hi}"] = {"rows": int(bcnt[b]), "max": float(bmax[b]),
                                         "mean": float(bsum[b] / bcnt[b])}
    return {"max": float(worst.value), "mean": float(bsum.sum() / total) if total else 0.0,
            "count": total, "worst_row": int(wrow.value), "bins": bins}


def dense_check(A, x, y, k=1, n=None, nthreads=0):
    """Per-row error of y against a long-double row-dot product: A row-major
    (m x lda; the first n columns are the matrix), x n*k and y m*k
    column-major; float32 / float64 / uint16 (bf16 bits) arrays.  Returns
    {"max", "mean", "count"}."""
    A = np.ascontiguousarray(A)
    m, lda = A.shape
    n = lda if n is None else n
    x = np.ascontiguousarray(x)
    y = np.ascontiguousarray(y)
    mx, sm, cnt = C.c_double(), C.c_double(), _i64()
    rc = lib.orc_dense_check(_ecode(A), _ecode(x), _ecode(y), m, n, _p(A), lda, _p(x), k,
                             _p(y), _nthreads(nthreads), C.byref(mx), C.byref(sm),
                             C.byref(cnt))
    assert rc == 0, "orc_dense_check failed"
    return {"max": float(mx.value), "mean": float(sm.value / max(cnt.value, 1)),
            "count": int(cnt.value)}


def f32_to_bf16_bits(a):
    a = np.ascontiguousarray(a, np.float32)
    out = np.empty(a.size, np.uint16)
    lib.orc_f32_to_bf16(a.size, _p(a), _p(out))
    return out


def bf16_bits_to_f32(b):
    b = np.ascontiguousarray(b, np.uint16)
    out = np.empty(b.size, np.float32)
    lib.orc_bf16_to_f32(b.size, _p(b), _p(out))
    return out


def fp_equal(a, b, eps=None) -> bool:
    """The reference tests' fp_equal (test/gtest/include/common-tests.hpp:
    82-111): |a-b| < max(min_normal, eps*(|a|+|b|)), eps = 128 * machine eps
    of the element type; identical values always pass."""
    a = np.asarray(a)
    b = np.asarray(b)
    if a.shape != b.shape:
        return False
    ft = np.result_type(a.dtype, b.dtype)
    if eps is None:
        eps = 128 * np.finfo(ft).eps
    tiny = np.finfo(ft).tiny
    diff = np.abs(a.astype(np.float64) - b.astype(np.float64))
    norm = np.minimum(np.abs(a.astype(np.float64)) + np.abs(b.astype(np.float64)),
                      np.finfo(np.float32).max)
    ok = (a == b) | (diff < np.maximum(tiny, eps * norm))
    return bool(np.all(ok))


def read_ref_bin(path):
    """Read a CSR written by oracle/_ref/ref_gen (or a fixture in that
    layout): int64 m, n, nnz; rowptr; colind; values."""
    raw = open(path, "rb").read()
    m, n, nnz = np.frombuffer(raw[:24], np.int64)
    return int(m), int(n), int(nnz), raw[24:]


class MatrixMarketError(RuntimeError):
    def __init__(self, code, msg):
        self.code = code
        super().__init__(msg)


def read_matrix_market(path, one_indexed=True):
    """Restated dr::read_csr<double, long>: (m, n, rowptr, colind, values)
    as int64 / int64 / float64 arrays; raises MatrixMarketError(code, msg)."""
    m, n, nnz = _i64(), _i64(), _i64()
    rp, ci, v = C.c_void_p(), C.c_void_p(), C.c_void_p()
    err = C.create_string_buffer(512)
    rc = lib.orc_read_matrix_market(str(path).encode(), int(one_indexed), C.byref(m),
                                    C.byref(n), C.byref(nnz), C.byref(rp), C.byref(ci),
                                    C.byref(v), err, 512)
    if rc != 0:
        raise MatrixMarketError(rc, err.value.decode())
    try:
        k = nnz.value
        rowptr = np.ctypeslib.as_array(C.cast(rp, C.POINTER(_i64)), (m.value + 1,)).copy()
        colind = (np.ctypeslib.as_array(C.cast(ci, C.POINTER(_i64)), (k,)).copy()
                  if k else np.zeros(0, np.int64))
        values = (np.ctypeslib.as_array(C.cast(v, C.POINTER(C.c_double)), (k,)).copy()
                  if k else np.zeros(0, np.float64))
    finally:
        for q in (rp, ci, v):
            lib.orc_free(q)
    return m.value, n.value, rowptr, colind, values


def cg(rp, ci, v, b, x0, max_iters, rtol, history=False):
    """The CG restatement (orc_cg): returns (x, iterations, ||r||, ||b||,
    status[, history]) with status 1 converged, 2 breakdown, 3 max_iters."""
    n = len(rp) - 1
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.array(x0, dtype=np.float64, copy=True)
    it, rn, bn, st = C.c_int64(), C.c_double(), C.c_double(), C.c_int()
    hist = np.zeros(max_iters + 1) if history else None
    assert lib.orc_cg(vcode(v.dtype), icode(ci.dtype), n, _p(rp), _p(ci), _p(v), _p(b),
                      _p(x), max_iters, rtol, C.byref(it), C.byref(rn), C.byref(bn),
                      C.byref(st), _p(hist)) == 0
    out = (x, it.value, rn.value, bn.value, st.value)
    return out + (hist[: it.value + 1],) if history else out


def reduce_seq(x, init=None, op="plus"):
    """std::reduce(first, last[, init], op) as the reference's tests compute
    it (test/gtest/common/reduce.cpp): op(init, fold(x)); integer sums wrap
    in the element type; float sums are accumulated sequentially in double
    here (the test tolerance covers the order)."""
    x = np.asarray(x)
    if op == "plus":
        if np.issubdtype(x.dtype, np.integer):
            t = x.sum(dtype=x.dtype) if len(x) else x.dtype.type(0)
            return t if init is None else x.dtype.type(t + x.dtype.type(init))
        t = float(np.sum(x.astype(np.float64))) if len(x) else 0.0
        t = x.dtype.type(t)
        return t if init is None else x.dtype.type(x.dtype.type(init) + t)
    f = {"min": lambda a, c: c if c < a else a, "max": lambda a, c: c if a < c else a}[op]
    if len(x) == 0:
        return x.dtype.type(0) if init is None else x.dtype.type(init)
    t = x.min() if op == "min" else x.max()
    return t if init is None else f(x.dtype.type(init), t)
