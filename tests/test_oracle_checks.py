"""The oracle's per-row parity checkers (orc_csr_check, orc_dense_check),
which bench.py uses to check every timed result at full size.  On the CPU:
an exact long-double result scores ~0; a result with one planted mistake
scores exactly that mistake's relative size, at the planted row and in its
row-length bin; the denominator is sum |a x| (so cancellation cannot hide or
inflate an error); bf16 inputs are read as their exact f32 values; k
right-hand sides are column-major."""
import numpy as np
import pytest

import oracle
import oracle.gen as og


def matrix(seed=3, m=3000, n=4000, dtype=np.float32):
    a = og.zipf_alpha_for_mean(1, 300, 12.0)
    rp, ci, v = og.powerlaw_csr(m, n, alpha=a, hi=300, seed=seed,
                                value_dtype=dtype)
    x = og.values(n, seed=seed + 1, dtype=dtype)
    return rp, ci, v, x, m, n


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_exact_result_scores_zero_and_planted_error_is_found(dtype):
    rp, ci, v, x, m, n = matrix(dtype=dtype)
    y = oracle.gemv_row(rp, ci, v, x, m, n, 1, oracle.ACC_LD)  # long double -> f64
    res = oracle.csr_check(rp, ci, v, x, m, n, y.astype(dtype))
    eps = np.finfo(dtype).eps
    assert res["max"] <= eps and res["count"] == m
    d = oracle.absdot(rp, ci, v, x, m, n)
    lens = np.diff(rp.astype(np.int64))
    r = int(np.argmax(lens))  # the longest row: the last bin
    bad = y.copy()
    bad[r] += 1e-3 * d[r]
    got = oracle.csr_check(rp, ci, v, x, m, n, bad.astype(np.float64))
    assert got["worst_row"] == r
    assert abs(got["max"] - 1e-3) <= 1e-9
    L = int(lens[r])
    hit = [k for k, b in got["bins"].items() if b["max"] > 1e-4]
    lo, hi = hit[0].split("-")
    assert hit and int(lo) <= L and (hi == "max" or L <= int(hi))
    assert sum(b["rows"] for b in got["bins"].values()) == m


def test_denominator_is_sum_of_abs_products():
    # one row a = (1, -1), x = (1, 1 + 2^-20): y = -2^-20, sum|ax| ~ 2
    rp = np.array([0, 2], np.int32)
    ci = np.array([0, 1], np.int32)
    v = np.array([1.0, -1.0])
    x = np.array([1.0, 1.0 + 2.0 ** -20])
    res = oracle.csr_check(rp, ci, v, x, 1, 2, np.array([0.0]))
    assert abs(res["max"] - 2.0 ** -20 / (2.0 + 2.0 ** -20)) <= 1e-15


def test_empty_rows_and_nan():
    rp = np.array([0, 0, 1, 1], np.int32)
    ci = np.array([2], np.int32)
    v = np.array([3.0], np.float32)
    x = np.array([0.0, 0.0, 2.0], np.float32)
    assert oracle.csr_check(rp, ci, v, x, 3, 3, np.array([0, 6, 0], np.float32))["max"] == 0
    # an empty row must come out exactly 0: any value is an absolute error
    assert oracle.csr_check(rp, ci, v, x, 3, 3, np.array([0.5, 6, 0], np.float32))["max"] == 0.5
    nan = oracle.csr_check(rp, ci, v, x, 3, 3, np.array([0, np.nan, 0], np.float32))
    assert nan["max"] == np.inf and nan["worst_row"] == 1


def test_bf16_inputs_and_multiple_rhs():
    rp, ci, v, x, m, n = matrix(seed=7, m=500, n=600)
    k = 3
    X = og.values(n * k, seed=9)
    vb, xb = oracle.f32_to_bf16_bits(v), oracle.f32_to_bf16_bits(X)
    vr, xr = oracle.bf16_bits_to_f32(vb), oracle.bf16_bits_to_f32(xb)
    y = oracle.gemv_row(rp, ci, vr.astype(np.float64), xr.astype(np.float64), m, n, k,
                        oracle.ACC_LD)
    # against the rounded inputs the exact sums score ~0 ...
    assert oracle.csr_check(rp, ci, vb, xb, m, n, y, k=k)["max"] <= 1e-15
    # ... and against the original inputs they carry the rounding, within 2u + u^2
    e2e = oracle.csr_check(rp, ci, v, X, m, n, y, k=k)
    u = 2.0 ** -8
    assert 1e-4 < e2e["max"] <= 2 * u + u * u and e2e["count"] == m * k
    # a mistake in the last right-hand side is seen there
    bad = y.copy()
    bad[2 * m + 17] += 0.5 * abs(bad[2 * m + 17]) + 1.0
    assert oracle.csr_check(rp, ci, vb, xb, m, n, bad, k=k)["worst_row"] == 17


def test_dense_check():
    rng = np.random.default_rng(4)
    m, n, lda, k = 37, 50, 56, 4
    A = rng.standard_normal((m, lda)).astype(np.float32)
    X = rng.standard_normal(n * k).astype(np.float32)
    y = oracle.dense_gemv(np.ascontiguousarray(A[:, :n]), X, k, oracle.ACC_LD)
    assert oracle.dense_check(A, X, y, k=k, n=n)["max"] <= 1e-15
    bad = y.copy()
    bad[m + 5] *= 1.01
    den = np.abs(A[5, :n]).astype(np.float64) @ np.abs(X[n:2 * n]).astype(np.float64)
    got = oracle.dense_check(A, X, bad, k=k, n=n)
    assert abs(got["max"] - abs(0.01 * y[m + 5]) / den) <= 1e-12
    assert got["count"] == m * k
