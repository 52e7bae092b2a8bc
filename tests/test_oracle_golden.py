"""CPU: the oracle is pinned to the reference.

* its restated generators reproduce, bit for bit, the matrices that the
  reference's own include/dr/detail/generate_csr.hpp produced (fixtures made
  by tests/golden/make_golden.py through oracle/_ref/ref_gen);
* its restated csr_row / csr_eq CPU loops reproduce the reference tests'
  expected results (test/gtest/mp/gemv.cpp) under fp_equal, and exactly where
  the summation order is the same.
"""
import glob
import os

import numpy as np
import pytest

import oracle

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return dict(np.load(os.path.join(GOLD, name + ".npz")))


@pytest.mark.parametrize("shape", [(100, 100), (1000, 10), (10, 1000)])
def test_random_csr_matches_reference_generator(shape):
    f = load(f"mp_gemv_{shape[0]}x{shape[1]}")
    rp, ci, v = oracle.random_csr(shape[0], shape[1], float(np.float32(0.1)), 0,
                                  np.float32, np.uint64)
    assert np.array_equal(rp, f["rowptr"])
    assert np.array_equal(ci, f["colind"])
    assert np.array_equal(v.view(np.uint32), f["values"].view(np.uint32))


@pytest.mark.parametrize("it,dtype", [("i32", np.int32), ("i64", np.int64)])
def test_random_csr_index_types(it, dtype):
    f = load(f"random_f64_{it}_200x150_seed7")
    rp, ci, v = oracle.random_csr(200, 150, float(np.float32(0.1)), 7, np.float64, dtype)
    assert np.array_equal(rp, f["rowptr"]) and np.array_equal(ci, f["colind"])
    assert np.array_equal(v.view(np.uint64), f["values"].view(np.uint64))


def test_very_sparse_generator():
    f = load("sp_very_sparse_100x100")
    rp, ci, v = oracle.random_csr(100, 100, float(np.float32(0.001)), 0)
    assert int(rp[-1]) == 10
    assert np.array_equal(rp, f["rowptr"]) and np.array_equal(ci, f["colind"])


@pytest.mark.parametrize("name,size,up,down,vt,it", [
    ("band_f64_1000_20_20", 1000, 20, 20, np.float64, np.int64),
    ("band_f64_257_3_3", 257, 3, 3, np.float64, np.int64),
    ("band_f32_100_3_3", 100, 3, 3, np.float32, np.uint64),
])
def test_band_matches_reference_generator(name, size, up, down, vt, it):
    f = load(name)
    rp, ci, v = oracle.band_csr(size, up, down, vt, it)
    assert np.array_equal(rp, f["rowptr"]) and np.array_equal(ci, f["colind"])
    assert np.array_equal(v, f["values"])


@pytest.mark.parametrize("name", ["mp_gemv_100x100", "mp_gemv_1000x10", "mp_gemv_10x1000",
                                  "sp_very_sparse_100x100", "band_f32_100_3_3",
                                  "sp_empty_100x100", "sp_zero_vector_100x100"])
@pytest.mark.parametrize("nseg", [1, 2, 3, 4])
def test_oracle_gemv_row_reproduces_reference_test(name, nseg):
    f = load(name)
    m, n = int(f["m"]), int(f["n"])
    y = oracle.gemv_row(f["rowptr"], f["colind"], f["values"], f["x"], m, n, 1,
                        oracle.ACC_T, nseg)
    # csr_row keeps each row's nnz order: identical bits to the test's c_ref
    assert np.array_equal(y, f["expected"])
    assert oracle.fp_equal(f["expected"], y)


@pytest.mark.parametrize("name", ["mp_gemv_100x100", "mp_gemv_1000x10", "mp_gemv_10x1000",
                                  "sp_very_sparse_100x100", "sp_empty_100x100"])
@pytest.mark.parametrize("nseg", [1, 2, 3, 4])
def test_oracle_gemv_eq_reproduces_reference_test(name, nseg):
    f = load(name)
    m, n = int(f["m"]), int(f["n"])
    y = oracle.gemv_eq(f["rowptr"], f["colind"], f["values"], f["x"], m, n, 1,
                       oracle.ACC_T, nseg)
    assert oracle.fp_equal(f["expected"], y)


@pytest.mark.parametrize("name", ["mp_gemv_100x100", "mp_gemv_1000x10", "mp_gemv_10x1000"])
@pytest.mark.parametrize("eq", [False, True])
def test_oracle_gemm_width20(name, eq):
    f = load(name)
    m, n = int(f["m"]), int(f["n"])
    fn = oracle.gemv_eq if eq else oracle.gemv_row
    y = fn(f["rowptr"], f["colind"], f["values"], f["x_w20"], m, n, 20, oracle.ACC_T, 3)
    assert oracle.fp_equal(f["expected_w20"], y)
    if not eq:
        assert np.array_equal(y, f["expected_w20"])


@pytest.mark.parametrize("name", ["band_f64_1000_20_20", "band_f64_257_3_3"])
def test_oracle_band_exact(name):
    # examples/mp/sparse_matrix.cpp:84-102 compares with `!=`
    f = load(name)
    m, n = int(f["m"]), int(f["n"])
    for fn in (oracle.gemv_row, oracle.gemv_eq):
        y = fn(f["rowptr"], f["colind"], f["values"], f["x"], m, n, 1, oracle.ACC_T, 4)
        assert np.array_equal(y, f["expected"])


def test_planted_mistake_is_caught():
    # A wrong oracle must fail the check: perturb one stored value on the CPU.
    f = load("mp_gemv_100x100")
    v = f["values"].copy()
    v[17] += np.float32(1e-3)
    y = oracle.gemv_row(f["rowptr"], f["colind"], v, f["x"], 100, 100)
    assert not oracle.fp_equal(f["expected"], y)


def test_oracle_transpose_and_abar_against_dense():
    rp, ci, v = oracle.random_csr(60, 45, 0.2, 3, np.float64, np.int64)
    D = np.zeros((60, 45))
    for i in range(60):
        for p in range(rp[i], rp[i + 1]):
            D[i, ci[p]] = v[p]
    cp, ri, vt = oracle.transpose(rp, ci, v, 60, 45)
    yb = np.random.default_rng(0).standard_normal(60)
    xb = oracle.gemv_row(cp, ri, vt, yb, 45, 60, 1, oracle.ACC_LD)
    assert np.allclose(xb, D.T @ yb, rtol=1e-13, atol=1e-13)
    x = np.random.default_rng(1).standard_normal(45)
    ab = oracle.abar(rp, ci, yb, x, 60)
    rows = np.repeat(np.arange(60), np.diff(rp))
    assert np.allclose(ab, yb[rows] * x[ci])


def test_oracle_dense_dot_absdot():
    rng = np.random.default_rng(5)
    A = rng.standard_normal((37, 53))
    x = rng.standard_normal((53, 3))
    y = oracle.dense_gemv(A, x.T.ravel(), 3)
    assert np.allclose(y.reshape(3, 37).T, A @ x, rtol=1e-12)
    a = rng.standard_normal(1001)
    assert abs(oracle.dot(a, a) - float(a @ a)) < 1e-10
    rp, ci, v = oracle.random_csr(50, 50, 0.1, 1, np.float64, np.int64)
    xx = rng.standard_normal(50)
    d = oracle.absdot(rp, ci, v, xx, 50, 50)
    rows = np.repeat(np.arange(50), np.diff(rp))
    ref = np.zeros(50)
    np.add.at(ref, rows, np.abs(v * xx[ci]))
    assert np.allclose(d, ref)


def test_bf16_rounding_rne():
    vals = np.array([1.0, 1.00390625, 1.01171875, -3.14159, 1e-40, np.inf], np.float32)
    bits = oracle.f32_to_bf16_bits(vals)
    back = oracle.bf16_bits_to_f32(bits)
    assert back[0] == 1.0
    assert back[1] == 1.0            # halfway 1 + 2^-8 rounds to even (1.0)
    assert back[2] == np.float32(1.015625)  # halfway rounds up to even mantissa
    assert np.isinf(back[5])
    assert abs(back[3] - vals[3]) <= abs(vals[3]) * 2 ** -8


def test_all_fixtures_have_sources():
    files = glob.glob(os.path.join(GOLD, "*.npz"))
    assert len(files) >= 10
    for p in files:
        assert "source" in np.load(p).files


@pytest.mark.parametrize("kind", ["powerlaw", "uniform_rows", "values"])
def test_oracle_generator_copy_matches_product_generator(kind):
    """The bench's reference arm builds its inputs with oracle.gen (the
    package's generate.cpp linked into the oracle library): the same bytes
    as drb.gen for the same seeds, whatever the thread count."""
    import drb
    import oracle.gen as og
    if kind == "powerlaw":
        a = og.zipf_alpha_for_mean(1, 512, 20.0)
        assert a == drb.gen.zipf_alpha_for_mean(1, 512, 20.0)
        got = og.powerlaw_csr(3000, 5000, alpha=a, hi=512, seed=11, nthreads=3)
        ref = drb.gen.powerlaw_csr(3000, 5000, alpha=a, hi=512, seed=11, nthreads=1)
    elif kind == "uniform_rows":
        got = og.uniform_rows_csr(2000, 2000, lo=8, hi=64, seed=12, value_dtype=np.float64)
        ref = drb.gen.uniform_rows_csr(2000, 2000, lo=8, hi=64, seed=12,
                                       value_dtype=np.float64)
    else:
        got = (og.values(100_003, seed=13, dist=og.NORMAL_ROWSCALE),)
        ref = (drb.gen.values(100_003, seed=13, dist=drb.gen.NORMAL_ROWSCALE),)
    for g, r in zip(got, ref):
        assert g.dtype == r.dtype and g.tobytes() == r.tobytes()
