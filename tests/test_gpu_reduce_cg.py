"""GPU parity for mp::reduce / iota / fill over a distributed_vector (the
reference's own reduce test cases, then large random vectors against the
oracle's sequential reduce) and for the device-resident conjugate-gradient
loop against the oracle's CG restatement."""
import operator

import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mp():
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from drb import mp as _mp
    return _mp


# ---- the reference's reduce tests (test/gtest/common/reduce.cpp,
#      test/gtest/mp/reduce.cpp): Ops1<distributed_vector<int>> ops(10),
#      iota(dist_vec, 100), compared with std::reduce on the local copy ----
@pytest.fixture
def ops1(mp):
    dv = mp.distributed_vector(10, dtype=torch.int32, nsegments=3)
    mp.iota(dv, 100)
    return dv, np.arange(100, 110, dtype=np.int32)


def test_reduce_root_range(mp, ops1):
    dv, vec = ops1
    assert mp.reduce(0, dv, 0, operator.add) == oracle.reduce_seq(vec, 0, "plus") == 1045


def test_reduce_root_iterators(mp, ops1):
    dv, vec = ops1
    r = mp.reduce(0, dv.begin() + 1, dv.end() - 1, 0, operator.add)
    assert r == oracle.reduce_seq(vec[1:-1], 0, "plus") == 836


def test_reduce_range_max(mp, ops1):
    dv, vec = ops1
    assert mp.reduce(dv, 3, max) == oracle.reduce_seq(vec, 3, "max") == 109


@pytest.mark.parametrize("form", ["op", "default_op", "iter", "iter_default_op"])
def test_reduce_plus_with_init(mp, ops1, form):
    dv, vec = ops1
    r = {"op": lambda: mp.reduce(dv, 3, operator.add),
         "default_op": lambda: mp.reduce(dv, 3),
         "iter": lambda: mp.reduce(dv.begin(), dv.end(), 3, operator.add),
         "iter_default_op": lambda: mp.reduce(dv.begin(), dv.end(), 3)}[form]()
    assert r == oracle.reduce_seq(vec, 3, "plus") == 1048


def test_reduce_default_init(mp, ops1):
    dv, vec = ops1
    assert mp.reduce(dv) == mp.reduce(dv.begin(), dv.end()) == oracle.reduce_seq(vec) == 1045


def test_transform_reduce_min_case(mp, ops1):
    # ReduceMP.TransformReduce: transform(dist_vec, +1) then reduce(root, ., 1, min)
    dv, vec = ops1
    t = mp.distributed_vector(10, dtype=torch.int32)
    t.tensor.copy_(dv.tensor + 1)
    assert mp.reduce(0, t, 1, min) == oracle.reduce_seq(vec + 1, 1, "min") == 1


def test_segments_follow_block_rule(mp):
    dv = mp.distributed_vector(10, dtype=torch.int64, nsegments=4)
    segs = dv.segments()
    assert [(s.begin, s.end) for s in segs] == [(0, 3), (3, 6), (6, 9), (9, 10)]
    mp.iota(dv, -5)
    assert sum(mp.reduce(s) for s in segs) == mp.reduce(dv) == sum(range(-5, 5))


# ---- large vectors: every dtype and op, aligned and unaligned starts ----------
DTYPES = [np.int32, np.int64, np.float32, np.float64]


def _data(dtype, n, seed):
    rng = np.random.default_rng(seed)
    if np.issubdtype(dtype, np.integer):
        info = np.iinfo(dtype)
        return rng.integers(info.min // 2, info.max // 2, n, dtype=dtype)
    return rng.standard_normal(n).astype(dtype)


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("op", ["plus", "min", "max"])
@pytest.mark.parametrize("n,off", [(0, 0), (1, 0), (7, 1), (4097, 3), (10_000_019, 1)])
def test_reduce_random(mp, dtype, op, n, off):
    h = _data(dtype, n + off, seed=n + off)
    t = torch.from_numpy(h).cuda()[off:]
    pyop = {"plus": operator.add, "min": min, "max": max}[op]
    init = dtype(5)
    got = mp.reduce(t, init, pyop)
    got_noinit = mp.reduce(t, None, pyop) if n else None
    want = oracle.reduce_seq(h[off:], init, op)
    if np.issubdtype(dtype, np.integer) or op != "plus":
        assert got == want                       # integer sums wrap bit for bit
        if n:
            assert got_noinit == oracle.reduce_seq(h[off:], None, op)
    else:
        scale = float(np.abs(h[off:].astype(np.float64)).sum()) + 5.0
        eps = np.finfo(dtype).eps
        assert abs(float(got) - float(want)) <= 2 * eps * scale + eps * abs(float(want))
    if n:
        again = mp.reduce(t, init, pyop)
        assert np.asarray(again, dtype).tobytes() == np.asarray(got, dtype).tobytes()


def test_reduce_async_out_and_stream(mp):
    h = np.arange(1, 1001, dtype=np.int64)
    t = torch.from_numpy(h).cuda()
    out = torch.zeros(1, dtype=torch.int64, device="cuda")
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        res = mp.reduce(t, 0, operator.add, out=out, stream=s)
    s.synchronize()
    assert res is out and int(out.item()) == 500500


@pytest.mark.parametrize("dtype", [torch.int32, torch.int64, torch.float32, torch.float64])
def test_iota_fill(mp, dtype):
    n = 1_000_003
    dv = mp.distributed_vector(n, dtype=dtype, nsegments=5)
    start = 2**40 if dtype in (torch.int64, torch.float64) else -7
    mp.iota(dv, start)
    want = (np.arange(n, dtype=np.int64) + start).astype(dv.numpy().dtype)
    assert np.array_equal(dv.numpy(), want)
    mp.fill(dv.begin() + 10, dv.end() - 10, 3)
    got = dv.numpy()
    assert np.array_equal(got[:10], want[:10]) and np.array_equal(got[-10:], want[-10:])
    assert (got[10:-10] == 3).all()
    v2 = mp.distributed_vector(33, value=-2, dtype=dtype)
    assert (v2.numpy() == -2).all() and v2[32] == -2
    mp.iota(v2.begin() + 3, v2.end(), 40)
    assert v2.numpy().tolist()[:5] == [-2, -2, -2, 40, 41] and v2[32] == 69


def test_reduce_rejects_other_ops(mp):
    dv = mp.distributed_vector(4, value=1.0)
    with pytest.raises(ValueError):
        mp.reduce(dv, 0.0, operator.mul)


# ---- conjugate gradients ----------------------------------------------------------
def lap(g, dtype=np.float64):
    import drb
    return drb.gen.laplacian2d_csr(g, index_dtype=np.int32, value_dtype=dtype)


def cg_gpu(mp, rp, ci, v, b, x0, max_iters, rtol, **kw):
    n = len(rp) - 1
    a = mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp, ci, (n, n)), 0, **kw)
    bt = torch.from_numpy(np.ascontiguousarray(b, v.dtype)).cuda()
    xt = torch.from_numpy(np.array(x0, v.dtype)).cuda()
    info = mp.conjugate_gradient(a, bt, xt, max_iters=max_iters, rtol=rtol)
    return a, xt, bt, info


def true_rel_residual(rp, ci, v, b, x):
    n = len(rp) - 1
    ax = oracle.gemv_row(rp, ci, v.astype(np.float64), np.asarray(x, np.float64), n, n, 1,
                         oracle.ACC_LD)
    return np.linalg.norm(b - ax) / np.linalg.norm(b)


@pytest.mark.parametrize("g", [32, 100])
def test_cg_f64_laplacian_matches_oracle(mp, g):
    rp, ci, v = lap(g)
    n = g * g
    b = np.random.default_rng(g).standard_normal(n)
    a, xt, _, info = cg_gpu(mp, rp, ci, v, b, np.zeros(n), 5000, 1e-10)
    x_o, it_o, rn_o, bn_o, st_o = oracle.cg(rp, ci, v, b, np.zeros(n), 5000, 1e-10)
    assert st_o == 1 and info["converged"] and not info["breakdown"]
    assert abs(info["iterations"] - it_o) <= 2
    x = xt.cpu().numpy()
    assert np.linalg.norm(x - x_o) <= 1e-8 * np.linalg.norm(x_o)
    assert info["residual_norm"] <= 1e-10 * info["b_norm"]
    assert abs(info["b_norm"] - bn_o) <= 1e-12 * bn_o
    assert true_rel_residual(rp, ci, v, b, x) <= 2e-10


def test_cg_f32_laplacian_converges(mp):
    rp, ci, v = lap(64, np.float32)
    n = 64 * 64
    b = np.random.default_rng(3).standard_normal(n).astype(np.float32)
    _, xt, _, info = cg_gpu(mp, rp, ci, v, b, np.zeros(n), 3000, 1e-5)
    assert info["converged"]
    x_o, it_o, *_ = oracle.cg(rp, ci, v, b.astype(np.float64), np.zeros(n), 3000, 1e-5)
    assert abs(info["iterations"] - it_o) <= max(3, it_o // 20)
    # the recurrence residual meets rtol; the true residual of an f32 solve
    # drifts from it by O(eps_f32 * cond(A)) (cond ~ 1.7e3 here)
    assert info["residual_norm"] <= 1e-5 * info["b_norm"]
    assert true_rel_residual(rp, ci, v, b.astype(np.float64), xt.cpu().numpy()) <= 3e-4


@pytest.mark.parametrize("k", [1, 5, 8, 9, 17])
def test_cg_fixed_iterations_follow_oracle(mp, k):
    """max_iters = k: exactly k updates, and x after k updates equals the
    oracle's x after k updates (same recurrence; only the summation order of
    the SpMV rows and dots differs)."""
    rp, ci, v = lap(48)
    n = 48 * 48
    rng = np.random.default_rng(k)
    b, x0 = rng.standard_normal(n), rng.standard_normal(n)
    _, xt, _, info = cg_gpu(mp, rp, ci, v, b, x0, k, 1e-14)
    x_o, it_o, rn_o, _, st_o = oracle.cg(rp, ci, v, b, x0, k, 1e-14)
    assert (info["iterations"], it_o, st_o) == (k, k, 3)
    assert not info["converged"] and not info["breakdown"]
    x = xt.cpu().numpy()
    assert np.linalg.norm(x - x_o) <= 1e-12 * np.linalg.norm(x_o)
    assert abs(info["residual_norm"] - rn_o) <= 1e-9 * rn_o


def test_cg_edge_cases(mp):
    rp, ci, v = lap(20)
    n = 400
    rng = np.random.default_rng(9)
    xs = rng.standard_normal(n)
    b = oracle.gemv_row(rp, ci, v, xs, n, n, 1, oracle.ACC_LD)
    # zero right-hand side from x0 = 0: converged before any update
    _, xt, _, info = cg_gpu(mp, rp, ci, v, np.zeros(n), np.zeros(n), 100, 1e-8)
    assert (info["iterations"], info["converged"]) == (0, True)
    assert not xt.cpu().numpy().any()
    # max_iters = 0: no update at all
    _, xt, _, info = cg_gpu(mp, rp, ci, v, b, np.zeros(n), 0, 1e-8)
    assert info["iterations"] == 0 and not info["converged"]
    # negative definite: breakdown at the first p.Ap, x left untouched
    x0 = rng.standard_normal(n)
    _, xt, _, info = cg_gpu(mp, rp, ci, -v, b, x0, 100, 1e-8)
    assert info["breakdown"] and info["iterations"] == 0
    assert np.array_equal(xt.cpu().numpy(), x0)


def spd_with_long_rows(n, seed):
    """Symmetric, strictly diagonally dominant (so SPD) matrix whose first
    rows/columns are dense enough (about 59 000 and 5 000 nonzeros) that the SpMV
    chunks them: S = B + B^T + diag(rowsum|B + B^T| + 1)."""
    sp = pytest.importorskip("scipy.sparse")
    rng = np.random.default_rng(seed)
    nnz = 6 * n
    r = rng.integers(0, n, nnz)
    c = rng.integers(0, n, nnz)
    r = np.concatenate([r, np.zeros(70_000, np.int64), np.full(5000, n // 2)])
    c = np.concatenate([c, rng.integers(0, n, 70_000), rng.integers(0, n, 5000)])
    B = sp.csr_matrix((rng.uniform(-1, 1, len(r)), (r, c)), shape=(n, n))
    S = (B + B.T).tocsr()
    d = np.asarray(abs(S).sum(axis=1)).ravel() + 1.0
    S = (S + sp.diags(d)).tocsr()
    S.sort_indices()
    return S.indptr.astype(np.int32), S.indices.astype(np.int32), S.data


def test_cg_spd_chunked_rows_and_graph_reuse(mp):
    n = 200_000
    rp, ci, v = spd_with_long_rows(n, 4)
    assert np.diff(rp).max() > 4096     # chunked by the SpMV plan
    b = np.random.default_rng(5).standard_normal(n)
    a, xt, bt, info = cg_gpu(mp, rp, ci, v, b, np.zeros(n), 500, 1e-10)
    x_o, it_o, *_ = oracle.cg(rp, ci, v, b, np.zeros(n), 500, 1e-10)
    # One eigenvalue near 6e4 (the dense row) against a cluster in [1, ~14]:
    # finite-precision CG revisits the outlier after losing orthogonality,
    # so the iteration count depends on rounding order (65 here, 69 for the
    # oracle's sequential sums).  Gate on the true residual, and on x within
    # cond(A) * rtol.
    assert info["converged"] and abs(info["iterations"] - it_o) <= max(2, it_o // 10)
    x1 = xt.cpu().numpy()
    assert true_rel_residual(rp, ci, v, b, x1) <= 2e-10
    assert np.linalg.norm(x1 - x_o) <= 1e-6 * np.linalg.norm(x_o)
    # the same solve again (captured graph replayed): bit-identical
    xt.zero_()
    info2 = mp.conjugate_gradient(a, bt, xt, max_iters=500, rtol=1e-10)
    assert info2 == info and np.array_equal(xt.cpu().numpy(), x1)
    # a new x buffer and a rebuilt SpMV plan (autotune) force a fresh capture
    a.autotune()
    x2 = torch.zeros(n, dtype=torch.float64, device="cuda")
    info3 = mp.conjugate_gradient(a, bt, x2, max_iters=500, rtol=1e-10)
    assert info3["converged"]
    assert true_rel_residual(rp, ci, v, b, x2.cpu().numpy()) <= 2e-10


def test_cg_counts_its_launches(mp):
    from drb import _capi as capi
    rp, ci, v = lap(16)
    n = 256
    b = np.random.default_rng(2).standard_normal(n)
    a, xt, bt, _ = cg_gpu(mp, rp, ci, v, b, np.zeros(n), 3, 1e-14)
    torch.cuda.synchronize()
    c0 = capi.launch_count()
    xt.zero_()
    mp.conjugate_gradient(a, bt, xt, max_iters=3, rtol=1e-14)
    # init SpMV + cg_init, then replays of 8 iterations x 3 kernels: the
    # host runs one replay ahead, so 3 updates take two replays
    assert capi.launch_count() - c0 == 2 + 2 * 24


def test_cg_rejects_bad_input(mp):
    from drb._capi import DrbError, DRB_ERR_INVALID_ARG, DRB_ERR_UNSUPPORTED
    rp, ci, v = lap(8)
    a = mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp, ci, (64, 64)), 0)
    bt = torch.ones(64, dtype=torch.float64, device="cuda")
    with pytest.raises(DrbError) as e:
        mp.conjugate_gradient(a, bt, torch.zeros_like(bt), max_iters=-1)
    assert e.value.status == DRB_ERR_INVALID_ARG
    rect = mp.distributed_sparse_matrix(mp.csr_matrix_view(
        np.ones(2), np.array([0, 1, 2], np.int32), np.array([0, 2], np.int32), (2, 3)), 0)
    with pytest.raises(DrbError) as e:
        mp.conjugate_gradient(rect, bt[:2], torch.zeros(3, dtype=torch.float64, device="cuda"))
    assert e.value.status == DRB_ERR_INVALID_ARG
    v32 = v.astype(np.float32)
    abf = mp.distributed_sparse_matrix(mp.csr_matrix_view(v32, rp, ci, (64, 64)), 0,
                                       storage=torch.bfloat16)
    with pytest.raises(DrbError) as e:
        mp.conjugate_gradient(abf, bt.float(), torch.zeros(64, device="cuda"))
    assert e.value.status == DRB_ERR_UNSUPPORTED
