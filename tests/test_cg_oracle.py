"""CPU: the oracle's conjugate-gradient restatement (orc_cg) and its
sequential reduce.  CG has no counterpart in the reference, so the oracle is
checked against an independent implementation (scipy.sparse.linalg.cg, same
stopping rule ||r|| <= rtol ||b||) and against its own invariants; the
reduce helper is pinned by the reference's own reduce test cases
(test/gtest/common/reduce.cpp, test/gtest/mp/reduce.cpp: a 10-element
distributed_vector<int> filled by iota(100), init 3)."""
import numpy as np
import pytest

import drb
import oracle


def lap(g):
    return drb.gen.laplacian2d_csr(g, index_dtype=np.int32, value_dtype=np.float64)


def test_reduce_seq_reference_cases():
    v = np.arange(100, 110, dtype=np.int32)      # Ops1<T> ops(10): iota(dist_vec, 100)
    assert oracle.reduce_seq(v, 0, "plus") == 1045   # ReduceMP.RootRange
    assert oracle.reduce_seq(v[1:-1], 0, "plus") == 836  # RootIterators
    assert oracle.reduce_seq(v, 3, "max") == 109     # Reduce.Range (max lambda)
    assert oracle.reduce_seq(v, 3, "plus") == 1048   # Reduce.Max / RangeDefaultOp
    assert oracle.reduce_seq(v) == 1045              # RangeDefaultInit
    assert oracle.reduce_seq(v + 1, 1, "min") == 1   # ReduceMP.TransformReduce
    assert oracle.reduce_seq(v[:0], 3, "plus") == 3  # empty range gives init
    big = np.full(4, 2**30 + 7, np.int32)            # wraps like the sequential loop
    with np.errstate(over="ignore"):
        assert oracle.reduce_seq(big) == np.int32(np.int64(4 * (2**30 + 7)) - 2**32)


@pytest.mark.parametrize("g", [16, 40])
def test_cg_oracle_matches_scipy(g):
    sla = pytest.importorskip("scipy.sparse.linalg")
    sp = pytest.importorskip("scipy.sparse")
    rp, ci, v = lap(g)
    n = g * g
    b = np.random.default_rng(g).standard_normal(n)
    x, it, rn, bn, st, hist = oracle.cg(rp, ci, v, b, np.zeros(n), 5000, 1e-10, history=True)
    assert st == 1 and it > 0
    A = sp.csr_matrix((v, ci, rp), shape=(n, n))
    count = [0]

    def cb(_):
        count[0] += 1
    xs, info = sla.cg(A, b, rtol=1e-10, atol=0.0, maxiter=5000, callback=cb)
    assert info == 0
    assert abs(count[0] - it) <= 2
    assert np.linalg.norm(x - xs) <= 1e-8 * np.linalg.norm(xs)
    # the recurrence residual tracks the true one and meets the tolerance
    true_r = np.linalg.norm(b - A @ x)
    assert true_r <= 2e-10 * bn
    assert rn <= 1e-10 * bn
    assert abs(hist[-1] - rn) <= 1e-14 * bn
    assert np.isclose(bn, np.linalg.norm(b))


def test_cg_oracle_stops():
    rp, ci, v = lap(12)
    n = 144
    b = np.random.default_rng(1).standard_normal(n)
    *_, st = oracle.cg(rp, ci, v, b, np.zeros(n), 3, 1e-12)
    assert st == 3
    x, it, rn, bn, st = oracle.cg(rp, ci, v, np.zeros(n), np.zeros(n), 10, 1e-8)
    assert (it, st, rn) == (0, 1, 0.0)
    x, it, _, _, st = oracle.cg(rp, ci, -v, b, np.zeros(n), 10, 1e-8)  # negative definite
    assert (it, st) == (0, 2) and not x.any()
