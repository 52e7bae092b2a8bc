"""GPU parity: the sm_100a kernels against the reference's own test cases
(golden fixtures) and the CPU oracle, through the C ABI."""
import ctypes as C
import os

import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return dict(np.load(os.path.join(GOLD, name + ".npz")))


@pytest.fixture(scope="module")
def mp():
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from drb import mp as _mp
    return _mp


def view(mp, f):
    return mp.csr_matrix_view(f["values"], f["rowptr"], f["colind"],
                              (int(f["m"]), int(f["n"])))


def rel_err(y, y_ref, denom):
    d = np.maximum(np.asarray(denom, np.float64), np.finfo(np.float64).tiny)
    return float(np.max(np.abs(np.asarray(y, np.float64) - y_ref) / d)) if len(d) else 0.0


# ---- the reference tests' own cases (test/gtest/mp/gemv.cpp, sp/gemv.cpp) ----
KAT = ["mp_gemv_100x100", "mp_gemv_1000x10", "mp_gemv_10x1000", "sp_very_sparse_100x100",
       "sp_empty_100x100", "sp_zero_vector_100x100", "band_f32_100_3_3"]


@pytest.mark.parametrize("name", KAT)
@pytest.mark.parametrize("distr", ["row", "eq"])
@pytest.mark.parametrize("nseg", [1, 3])
def test_reference_gemv_cases(mp, name, distr, nseg):
    f = load(name)
    pol = mp.csr_row_distribution if distr == "row" else mp.csr_eq_distribution
    a = mp.distributed_sparse_matrix(view(mp, f), 0, distr=pol, nsegments=nseg)
    m, n = a.shape()
    b = mp.broadcasted_vector()
    b.broadcast_data(n, 0, f["x"], mp.default_comm())
    c = [0.0] * m
    mp.gemv(c, a, b)                      # no-root overload, gemv.hpp:41-55
    assert oracle.fp_equal(f["expected"], np.array(c, np.float32))
    c2 = np.zeros(m, np.float32)
    mp.gemv(0, c2, a, b)                  # root overload, gemv.hpp:16-27
    assert np.array_equal(np.array(c, np.float32), c2)


@pytest.mark.parametrize("name", ["mp_gemv_100x100", "mp_gemv_1000x10", "mp_gemv_10x1000"])
@pytest.mark.parametrize("distr", ["row", "eq"])
def test_reference_gemm_width20(mp, name, distr):
    f = load(name)
    pol = mp.csr_row_distribution if distr == "row" else mp.csr_eq_distribution
    a = mp.distributed_sparse_matrix(view(mp, f), 0, distr=pol, nsegments=2)
    m, n = a.shape()
    b = mp.broadcasted_slim_matrix()
    b.broadcast_data(n, 20, 0, f["x_w20"], mp.default_comm())
    c = np.zeros(m * 20, np.float32)
    mp.gemv(0, c, a, b)                   # gemv.hpp:29-39
    assert oracle.fp_equal(f["expected_w20"], c)


@pytest.mark.parametrize("name", ["band_f64_1000_20_20", "band_f64_257_3_3"])
def test_band_f64_exact(mp, name):
    # examples/mp/sparse_matrix.cpp:84-102: res[i] != ref[i] is a mismatch
    f = load(name)
    for pol in (mp.csr_eq_distribution, mp.csr_row_distribution):
        a = mp.distributed_sparse_matrix(view(mp, f), 0, distr=pol, nsegments=4)
        b = mp.broadcasted_vector()
        b.broadcast_data(a.shape()[1], 0, f["x"])
        res = np.zeros(a.shape()[0], np.float64)
        mp.gemv(0, res, a, b)
        assert np.array_equal(res, f["expected"])


def test_entries_iteration_matches_source(mp):
    # IterRow/IterEq (test/gtest/mp/sparse_matrix.cpp): entry-wise equality
    f = load("mp_gemv_100x100")
    for pol in (mp.csr_row_distribution, mp.csr_eq_distribution):
        a = mp.distributed_sparse_matrix(view(mp, f), 0, distr=pol, nsegments=3)
        got = list(a)
        src = list(mp.csr_matrix_view(f["values"], f["rowptr"], f["colind"], (100, 100)))
        assert len(got) == len(src) == a.size()
        for (i1, v1), (i2, v2) in zip(got, src):
            assert i1 == i2 and np.float32(v1) == v2
        total = sum(len(s) for s in a.segments())
        assert total == a.size()
        assert a[5] == got[5]


def test_segments_follow_reference_rules(mp):
    f = load("mp_gemv_1000x10")
    rp = f["rowptr"].astype(np.int64)
    m, nnz = 1000, int(rp[-1])
    for P in (1, 2, 3, 7):
        a = mp.distributed_sparse_matrix(view(mp, f), 0, distr=mp.csr_row_distribution,
                                         nsegments=P)
        seg = -(-m // P)
        for r, s in enumerate(a.segments()):
            r0, r1 = min(m, r * seg), min(m, (r + 1) * seg)
            assert (s.row_begin, s.row_end) == (r0, r1)
            assert (s.nnz_begin, s.nnz_end) == (rp[r0], rp[r1])
        a = mp.distributed_sparse_matrix(view(mp, f), 0, distr=mp.csr_eq_distribution,
                                         nsegments=P)
        seg = -(-nnz // P)
        for r, s in enumerate(a.segments()):
            z0, z1 = min(nnz, r * seg), min(nnz, (r + 1) * seg)
            assert (s.nnz_begin, s.nnz_end) == (z0, z1)
            if z0 < z1:
                assert s.row_begin == np.searchsorted(rp[:m], z0, side="right") - 1
                assert s.row_end == np.searchsorted(rp[:m], z1 - 1, side="right")


# ---- parity against the FP64 oracle at the benchmark shapes ---------------------
def gpu_gemv(mp, rp, ci, v, m, n, x, k=1, layout=0, **kw):
    a = mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp, ci, (m, n)), 0, **kw)
    xt = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    yt = torch.empty(m * k, dtype=xt.dtype, device="cuda")
    a.gemv_device(xt, yt, k, layout)
    torch.cuda.synchronize()
    a.check()  # no device-side wait timed out
    return a, yt.cpu().numpy()


def test_fixed16_fp32_vs_fp64_oracle(mp):
    # 131072 x 131072, exactly 16 distinct sorted uniform columns per row
    import drb
    m = 131072
    rp, ci, v = drb.gen.fixed_rows_csr(m, m, length=16, seed=20261204)
    x = drb.gen.values(m, seed=77)
    _, y = gpu_gemv(mp, rp, ci, v, m, m, x)
    y64 = oracle.gemv_row(rp, ci, v, x, m, m, 1, oracle.ACC_LD)
    d = oracle.absdot(rp, ci, v, x, m, m)
    assert rel_err(y, y64, d) <= 1e-5
    y32 = oracle.gemv_row(rp, ci, v, x, m, m)   # the reference's own fp32 loop
    assert rel_err(y, y32.astype(np.float64), d) <= 1e-5


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_powerlaw_long_rows(mp, dtype):
    import drb
    m = 300_000
    a_ = drb.gen.zipf_alpha_for_mean(1, 16384, 20.0)
    rp, ci, v = drb.gen.powerlaw_csr(m, m, alpha=a_, hi=16384, seed=5, value_dtype=dtype)
    assert np.diff(rp).max() > 2048     # long rows are exercised
    x = drb.gen.values(m, seed=6, dtype=dtype)
    _, y = gpu_gemv(mp, rp, ci, v, m, m, x)
    y64 = oracle.gemv_row(rp, ci, v, x, m, m, 1, oracle.ACC_LD)
    d = oracle.absdot(rp, ci, v, x, m, m)
    tol = 1e-5 if dtype == np.float32 else 1e-12
    assert rel_err(y, y64, d) <= tol


def chunky_matrix(dtype, idx=np.int32):
    """Rows of every kind: empty, short, tile-boundary, long, and two rows
    longer than one CTA's chunk limit (chunked with a ticketed finish)."""
    rng = np.random.default_rng(3)
    n = 400_000
    lens = np.concatenate([
        rng.integers(0, 40, 5000), [2047, 2048, 2049, 0, 0, 1], [70_000, 0, 300_001],
        rng.integers(0, 5, 3000), [65536, 65537], rng.integers(100, 3000, 200)])
    m = len(lens)
    rp = np.zeros(m + 1, np.int64)
    rp[1:] = np.cumsum(lens)
    ci = np.empty(rp[-1], idx)
    for r in range(m):
        L = lens[r]
        if L:
            ci[rp[r]:rp[r + 1]] = np.sort(rng.choice(n, L, replace=False))
    v = rng.uniform(-1, 1, rp[-1]).astype(dtype)
    return rp.astype(idx), ci, v, m, n


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_chunked_rows_deterministic(mp, dtype):
    rp, ci, v, m, n = chunky_matrix(dtype)
    x = np.random.default_rng(4).uniform(-1, 1, n).astype(dtype)
    a, y1 = gpu_gemv(mp, rp, ci, v, m, n, x)
    xt = torch.from_numpy(x).cuda()
    yt = torch.empty(m, dtype=xt.dtype, device="cuda")
    for _ in range(3):  # counters must be re-armed between launches
        a.gemv_device(xt, yt)
    torch.cuda.synchronize()
    assert np.array_equal(y1.view(np.uint8), yt.cpu().numpy().view(np.uint8))
    y64 = oracle.gemv_row(rp, ci, v, x, m, n, 1, oracle.ACC_LD)
    d = oracle.absdot(rp, ci, v, x, m, n)
    assert rel_err(y1, y64, d) <= (1e-5 if dtype == np.float32 else 1e-12)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_autotune_variants_agree(mp, dtype):
    """Every kernel variant (item span x product layout) and the autotuned
    choice give results within tolerance of the FP64 oracle."""
    rp, ci, v, m, n = chunky_matrix(dtype)
    x = np.random.default_rng(12).uniform(-1, 1, n).astype(dtype)
    y64 = oracle.gemv_row(rp, ci, v, x, m, n, 1, oracle.ACC_LD)
    d = oracle.absdot(rp, ci, v, x, m, n)
    tol = 1e-5 if dtype == np.float32 else 1e-12
    a = mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp, ci, (m, n)), 0,
                                     adjoint=True, autotune=True)
    assert a.variant() in (128, 129, 131, 256, 257, 259, 512, 513)
    xt = torch.from_numpy(x).cuda()
    yt = torch.empty(m, dtype=xt.dtype, device="cuda")
    a.gemv_device(xt, yt)
    a.check()
    assert rel_err(yt.cpu().numpy(), y64, d) <= tol
    chosen = a.autotune()
    assert chosen == a.variant()
    a.gemv_device(xt, yt)
    assert rel_err(yt.cpu().numpy(), y64, d) <= tol


@pytest.mark.parametrize("variant", ["128,0", "128,1", "256,0", "256,1", "512,0", "512,1",
                                     "128,1,1", "256,1,1"])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_each_variant_parity(mp, variant, dtype, monkeypatch):
    """Every item span and layout, and the two-slot pipelined kernel ("t,1,1"),
    within the gate of the oracle, with the fused residual on the same plan
    (the residual keeps the one-slot kernel)."""
    monkeypatch.setenv("DRB_SPMV_VARIANT", variant)
    rp, ci, v, m, n = chunky_matrix(dtype)
    x = np.random.default_rng(13).uniform(-1, 1, n).astype(dtype)
    a, y = gpu_gemv(mp, rp, ci, v, m, n, x)
    parts = [int(s) for s in variant.split(",")] + [0]
    t, sk, two = parts[0], parts[1], parts[2]
    assert a.variant() == (t | sk | (2 if two else 0))
    y64 = oracle.gemv_row(rp, ci, v, x, m, n, 1, oracle.ACC_LD)
    tol = 1e-5 if dtype == np.float32 else 1e-12
    assert rel_err(y, y64, oracle.absdot(rp, ci, v, x, m, n)) <= tol
    # the fused residual on the same variant
    b = np.random.default_rng(14).uniform(-1, 1, m).astype(dtype)
    bt = torch.from_numpy(b).cuda()
    yt = torch.empty(m, dtype=bt.dtype, device="cuda")
    r2 = float(mp.residual_norm2(a, torch.from_numpy(x).cuda(), bt, yt))
    ref = float(np.sum((y64 - b.astype(np.float64)) ** 2))
    assert abs(r2 - ref) <= 1e-4 * ref
    if two:  # the pipelined kernel gives the same bits as the one-slot kernel
        monkeypatch.setenv("DRB_SPMV_VARIANT", f"{t},1")
        _, y1 = gpu_gemv(mp, rp, ci, v, m, n, x)
        assert np.array_equal(y.view(np.uint8), y1.view(np.uint8))


@pytest.mark.parametrize("keep64", [False, True])
def test_int64_indices(mp, keep64):
    rp, ci, v, m, n = chunky_matrix(np.float64, np.int64)
    x = np.random.default_rng(8).standard_normal(n)
    a, y = gpu_gemv(mp, rp, ci, v, m, n, x, keep_index64=keep64)
    vb, cb, rb = a.storage_bytes()
    assert (vb, cb) == (8, 8 if keep64 else 4)
    y64 = oracle.gemv_row(rp, ci, v, x, m, n, 1, oracle.ACC_LD)
    assert rel_err(y, y64, oracle.absdot(rp, ci, v, x, m, n)) <= 1e-12


@pytest.mark.parametrize("k", [2, 3, 8, 16, 33])
@pytest.mark.parametrize("layout", [0, 1])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_multi_rhs(mp, k, layout, dtype):
    rp, ci, v, m, n = chunky_matrix(dtype)
    rng = np.random.default_rng(k)
    X = rng.uniform(-1, 1, (n, k)).astype(dtype)           # X[c, j]
    xin = X.T.ravel() if layout == 0 else X.ravel()
    _, y = gpu_gemv(mp, rp, ci, v, m, n, xin, k, layout)
    Y = y.reshape(k, m).T if layout == 0 else y.reshape(m, k)
    y64 = oracle.gemv_row(rp, ci, v, X.T.ravel(), m, n, k, oracle.ACC_LD).reshape(k, m).T
    d = oracle.absdot(rp, ci, v, X.T.ravel(), m, n, k).reshape(k, m).T
    tol = 1e-5 if dtype == np.float32 else 1e-12
    assert rel_err(Y.ravel(), y64.ravel(), d.ravel()) <= tol


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_multi_rhs_large_column_major_y(mp, dtype):
    """A column-major Y larger than 64 MB (1,048,584 rows x 16, m a multiple of
    a 32-byte sector's rows) has its items cut on sector boundaries; the cut
    changes no row's sum, so Y has the bits of the row-major call (whose items
    are not cut so) and agrees with the oracle."""
    import drb
    m = n = 1_048_584
    k = 16
    rp, ci, v = drb.gen.uniform_rows_csr(m, n, lo=0, hi=24, seed=31, value_dtype=dtype)
    rng = np.random.default_rng(32)
    X = rng.uniform(-1, 1, (n, k)).astype(dtype)           # X[c, j]
    a = mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp, ci, (m, n)), 0)
    xc = torch.from_numpy(np.ascontiguousarray(X.T).ravel()).cuda()
    xr = torch.from_numpy(X.ravel()).cuda()
    yc = torch.empty(m * k, dtype=xc.dtype, device="cuda")
    yr = torch.empty_like(yc)
    a.gemv_device(xc, yc, k, 0)
    a.gemv_device(xr, yr, k, 1)
    torch.cuda.synchronize()
    a.check()
    Yc = yc.cpu().numpy().reshape(k, m).T
    Yr = yr.cpu().numpy().reshape(m, k)
    assert np.array_equal(Yc, Yr)
    y64 = oracle.gemv_row(rp, ci, v, X.T.ravel(), m, n, k, oracle.ACC_LD)
    d = oracle.absdot(rp, ci, v, X.T.ravel(), m, n, k)
    tol = 1e-5 if dtype == np.float32 else 1e-12
    assert rel_err(Yc.T.ravel(), y64, d) <= tol


@pytest.mark.parametrize("layout", [0, 1])
def test_multi_rhs_fallback_and_repeat(mp, layout):
    """k > 1 runs on a batch of the one handle; 64-bit indices (kept) and a
    row-major x off a 16-byte boundary take the row-block kernel instead.
    Both agree with the oracle, and repeated calls (the cached batch, and a
    new k that rebuilds it) give the same bits."""
    rp, ci, v, m, n = chunky_matrix(np.float64, np.int64)
    k = 5
    rng = np.random.default_rng(9)
    X = rng.uniform(-1, 1, (n, k))
    xin = X.T.ravel() if layout == 0 else X.ravel()
    y64 = oracle.gemv_row(rp, ci, v, X.T.ravel(), m, n, k, oracle.ACC_LD).reshape(k, m).T
    d = oracle.absdot(rp, ci, v, X.T.ravel(), m, n, k).reshape(k, m).T
    outs = []
    for keep64 in (False, True):
        a, y = gpu_gemv(mp, rp, ci, v, m, n, xin, k, layout, keep_index64=keep64)
        Y = y.reshape(k, m).T if layout == 0 else y.reshape(m, k)
        assert rel_err(Y.ravel(), y64.ravel(), d.ravel()) <= 1e-12
        outs.append(y)
        if not keep64:
            xt = torch.from_numpy(xin).cuda()
            y2 = torch.empty(m * k, dtype=torch.float64, device="cuda")
            a.gemv_device(xt, y2, k, layout)
            a.gemv_device(torch.zeros(n * 3, dtype=torch.float64, device="cuda"),
                          torch.empty(m * 3, dtype=torch.float64, device="cuda"), 3, layout)
            a.gemv_device(xt, y2, k, layout)
            assert np.array_equal(y2.cpu().numpy(), y)
    if layout == 1:
        # a row-major x at an 8-byte offset: the row-block kernel
        a = mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp, ci, (m, n)), 0)
        buf = torch.from_numpy(np.concatenate([[0.0], xin])).cuda()
        y3 = torch.empty(m * k, dtype=torch.float64, device="cuda")
        a.gemv_device(buf[1:], y3, k, layout)
        Y = y3.cpu().numpy().reshape(m, k)
        assert rel_err(Y.ravel(), y64.ravel(), d.ravel()) <= 1e-12


def test_multi_rhs_bf16(mp):
    """BF16 storage with k > 1 (the batched kernel's plain f32 sums): within
    f32 accumulation error of the FP64 product of the bf16-rounded inputs."""
    import drb
    m = 20_000
    rp, ci, v = drb.gen.uniform_rows_csr(m, m, lo=1, hi=90, seed=4)
    k = 6
    X = np.random.default_rng(5).uniform(-1, 1, (m, k)).astype(np.float32)
    xb = torch.from_numpy(X.T.ravel().copy()).to(torch.bfloat16)
    a = mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp, ci, (m, m)), 0,
                                     storage=torch.bfloat16)
    y = torch.empty(m * k, dtype=torch.float32, device="cuda")
    a.gemv_device(xb.cuda(), y, k, 0)
    vr = torch.from_numpy(v).to(torch.bfloat16).double().numpy()
    xr = xb.double().numpy()
    ref = oracle.gemv_row(rp, ci, vr, xr, m, m, k, oracle.ACC_LD)
    d = oracle.absdot(rp, ci, vr, xr, m, m, k)
    assert rel_err(y.cpu().numpy(), ref, d) <= 1e-5


def test_host_gemv_matches_device(mp):
    import drb
    m = 50_000
    rp, ci, v = drb.gen.uniform_rows_csr(m, m, lo=8, hi=64, seed=2)
    x = drb.gen.values(m, seed=3)
    a, y_dev = gpu_gemv(mp, rp, ci, v, m, m, x)
    xh = torch.from_numpy(x).pin_memory()
    yh = torch.empty(m, dtype=torch.float32).pin_memory()
    a.gemv_host(xh.numpy(), yh.numpy())
    assert np.array_equal(yh.numpy(), y_dev)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("pinned", [True, False])
def test_host_gemv_row_segments(mp, dtype, pinned):
    """Above 4M nonzeros the host-pointer gemv runs in row segments and
    copies each segment's rows of y back while the later ones compute; the
    segments cut only between rows, so chunked long rows (70 000 and 300 001
    nonzeros, placed mid-matrix) stay whole.  The result is bit-identical to
    the device-pointer gemv, on the first call and on a repeat."""
    rng = np.random.default_rng(31)
    m, n = 240_000, 500_000
    lens = rng.integers(0, 40, m)
    lens[[1000, 120_000, 120_001, m - 1]] = [300_001, 70_000, 0, 5000]
    rp = np.zeros(m + 1, np.int32)
    rp[1:] = np.cumsum(lens)
    assert rp[-1] > (1 << 22)
    rows = np.repeat(np.arange(m), lens)
    cols = rng.integers(0, n, rp[-1])
    ci = cols[np.lexsort((cols, rows))].astype(np.int32)
    v = rng.uniform(-1, 1, rp[-1]).astype(dtype)
    x = rng.uniform(-1, 1, n).astype(dtype)
    a, y_dev = gpu_gemv(mp, rp, ci, v, m, n, x)
    if pinned:
        xh = torch.from_numpy(x).pin_memory().numpy()
        yh = torch.empty(m, dtype=torch.from_numpy(x).dtype).pin_memory().numpy()
    else:
        xh, yh = x.copy(), np.empty(m, dtype)
    for _ in range(2):
        yh[:] = np.nan
        a.gemv_host(xh, yh)
        assert np.array_equal(yh.view(np.uint8), y_dev.view(np.uint8))
    y64 = oracle.gemv_row(rp, ci, v, x, m, n, 1, oracle.ACC_LD)
    d = oracle.absdot(rp, ci, v, x, m, n)
    assert rel_err(yh, y64, d) <= (1e-5 if dtype == np.float32 else 1e-12)


@pytest.mark.parametrize("m,n", [(1, 1), (2, 3), (31, 33), (32, 32), (33, 31), (1, 5000)])
def test_ragged_small_shapes(mp, m, n):
    rp, ci, v = oracle.random_csr(m, n, 0.5 if m * n > 1 else 0.0, 1, np.float64, np.int64)
    if m * n == 1:
        rp, ci, v = np.array([0, 1], np.int64), np.array([0], np.int64), np.array([2.5])
    x = np.random.default_rng(0).standard_normal(n)
    _, y = gpu_gemv(mp, rp, ci, v, m, n, x)
    y64 = oracle.gemv_row(rp, ci, v, x, m, n, 1, oracle.ACC_LD)
    assert rel_err(y, y64, oracle.absdot(rp, ci, v, x, m, n)) <= 1e-12


def test_bad_csr_rejected(mp):
    from drb._capi import DrbError, DRB_ERR_BAD_CSR
    rp = np.array([0, 2, 1, 3], np.int32)
    ci = np.array([0, 1, 2], np.int32)
    v = np.ones(3, np.float32)
    with pytest.raises(DrbError) as e:
        mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp, ci, (3, 3)), 0)
    assert e.value.status == DRB_ERR_BAD_CSR
    rp = np.array([0, 1, 2, 3], np.int32)
    ci = np.array([0, 3, 1], np.int32)      # column 3 of a 3-column matrix
    with pytest.raises(DrbError) as e:
        mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp, ci, (3, 3)), 0)
    assert e.value.status == DRB_ERR_BAD_CSR


def test_gemv_size_mismatch_raises(mp):
    f = load("mp_gemv_100x100")
    a = mp.distributed_sparse_matrix(view(mp, f), 0)
    b = mp.broadcasted_vector()
    b.broadcast_data(100, 0, f["x"])
    with pytest.raises(ValueError):
        mp.gemv(0, [0.0] * 99, a, b)
    with pytest.raises(ValueError):
        mp.gemv(1, [0.0] * 100, a, b)


# ---- dense gemv, dot, fused residual ------------------------------------------
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("m,n,k,pad", [(257, 1024, 1, 0), (300, 777, 1, 3), (129, 512, 3, 0),
                                       (64, 96, 8, 4), (65, 100, 9, 0), (5, 1, 1, 0),
                                       # several 8 KB column slabs per row, wide and tall
                                       (33, 5000, 1, 0), (7, 100_000, 2, 4),
                                       (3, 1 << 20, 1, 0), (1000, 8192, 8, 0),
                                       (1001, 4100, 5, 0), (20_000, 64, 1, 0)])
@pytest.mark.parametrize("layout", [0, 1])
def test_dense_gemv(mp, dtype, m, n, k, pad, layout):
    g = torch.Generator().manual_seed(m * 7 + n)
    A_full = torch.randn(m, n + pad, generator=g, dtype=torch.float64)
    X = torch.randn(n, k, generator=g, dtype=torch.float64)
    A = A_full.to(dtype).cuda()[:, :n]
    xin = (X.t().contiguous() if layout == 0 else X.contiguous()).to(dtype).cuda()
    y = torch.empty(m * k, dtype=dtype, device="cuda")
    mp.dense_gemv(A, xin, y, k, layout)
    torch.cuda.synchronize()
    Y = y.cpu().view(k, m).t() if layout == 0 else y.cpu().view(m, k)
    ref = oracle.dense_gemv(A.cpu().double().contiguous().numpy(),
                            X.to(dtype).double().t().contiguous().numpy().ravel(), k,
                            oracle.ACC_LD).reshape(k, m).T
    denom = (A.cpu().double().abs() @ X.to(dtype).double().abs()).numpy()
    tol = 1e-5 if dtype == torch.float32 else 1e-12
    assert rel_err(Y.double().numpy().ravel(), ref.ravel(), denom.ravel()) <= tol


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("n", [0, 1, 7, 1000, 1 << 20, (1 << 20) + 3, 5_000_011])
def test_dot(mp, dtype, n):
    g = torch.Generator().manual_seed(n)
    a = torch.randn(n, generator=g, dtype=torch.float64).to(dtype)
    b = torch.randn(n, generator=g, dtype=torch.float64).to(dtype)
    out = mp.dot(a.cuda(), b.cuda())
    out2 = mp.dot(a.cuda(), b.cuda())
    ref = oracle.dot(a.numpy(), b.numpy())
    got = float(out.item())
    assert got == float(out2.item())        # deterministic
    assert abs(got - ref) <= 1e-12 * max(1.0, float((a.double().abs() * b.double().abs()).sum()))
    if n:
        ad = a.cuda()
        nrm = float(mp.dot(ad, ad).item())   # a is b: one stream read
        assert abs(nrm - oracle.dot(a.numpy(), a.numpy())) <= 1e-12 * nrm


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_residual_norm2(mp, dtype):
    rp, ci, v, m, n = chunky_matrix(dtype)
    rng = np.random.default_rng(1)
    x = rng.uniform(-1, 1, n).astype(dtype)
    b = rng.uniform(-1, 1, m).astype(dtype)
    a = mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp, ci, (m, n)), 0)
    y = torch.empty(m, dtype=torch.from_numpy(x).dtype, device="cuda")
    out = mp.residual_norm2(a, torch.from_numpy(x).cuda(), torch.from_numpy(b).cuda(), y)
    out2 = mp.residual_norm2(a, torch.from_numpy(x).cuda(), torch.from_numpy(b).cuda())
    y_gpu = y.cpu().numpy().astype(np.float64)
    ref = float(((y_gpu - b.astype(np.float64)) ** 2).sum())
    assert abs(out.item() - ref) <= 1e-10 * ref
    assert out.item() == out2.item()
    y64 = oracle.gemv_row(rp, ci, v, x, m, n, 1, oracle.ACC_LD)
    assert rel_err(y_gpu, y64, oracle.absdot(rp, ci, v, x, m, n)) <= (
        1e-5 if dtype == np.float32 else 1e-12)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_residual_norm2_repeatable_with_dynamic_schedule(mp, dtype):
    """Warps take work items dynamically, so which warp runs an item changes
    from launch to launch; each item's rows reduce into the item's own slot and
    the slots are summed in a fixed order, so ||Ax - b||^2 repeats bit for bit."""
    import drb
    m = n = 300_000
    rp, ci, v = drb.gen.powerlaw_csr(m, n, alpha=1.76, hi=8192, seed=11)
    v = v.astype(dtype)
    rng = np.random.default_rng(3)
    x = torch.from_numpy(rng.uniform(-1, 1, n).astype(dtype)).cuda()
    b = torch.from_numpy(rng.uniform(-1, 1, m).astype(dtype)).cuda()
    a = mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp, ci, (m, n)), 0)
    y = torch.empty(m, dtype=x.dtype, device="cuda")
    outs = [mp.residual_norm2(a, x, b, y).item() for _ in range(6)]
    assert len(set(outs)) == 1
    ref = float(((y.double() - b.double()) ** 2).sum())
    assert abs(outs[0] - ref) <= 1e-10 * ref


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("index", [np.int32, np.int64])
def test_gather_probe_runs_and_checks_storage(mp, dtype, index):
    """The measurement-only gather probe reads a handle's columns (and values)
    and x without writing anything visible; BF16 storage is refused."""
    from drb import _capi as capi
    rp, ci, v, m, n = chunky_matrix(dtype)
    a = mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp.astype(index), ci.astype(index),
                                                        (m, n)), 0)
    x = torch.from_numpy(np.random.default_rng(2).uniform(-1, 1, n).astype(dtype)).cuda()
    y0 = torch.empty(m, dtype=x.dtype, device="cuda")
    a.gemv_device(x, y0)
    x0 = x.clone()
    import drb_probe
    drb_probe.gather_probe(a, x)
    drb_probe.gather_probe(a, x, with_values=False)
    y1 = torch.empty_like(y0)
    a.gemv_device(x, y1)
    assert torch.equal(x, x0) and torch.equal(y0, y1)
    a.check()
    vb = v.astype(np.float32)
    b16 = mp.distributed_sparse_matrix(mp.csr_matrix_view(vb, rp, ci, (m, n)), 0,
                                       storage=torch.bfloat16)
    rc = drb_probe.lib.drb_csr_gather_probe(b16.handle, C.c_void_p(x.data_ptr()), 1, None)
    assert rc == capi.DRB_ERR_UNSUPPORTED


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("index", [np.int32, np.int64])
def test_gather_rows_probe_runs_and_checks_shapes(mp, dtype, index):
    """The row form of the probe gathers whole X rows (k = 16, and a padded
    row stride) without writing anything visible; row widths that are not a
    power-of-two number of 16-byte vectors, a short stride, a misaligned X and
    BF16 storage are refused."""
    from drb import _capi as capi
    import drb_probe
    rp, ci, v, m, n = chunky_matrix(dtype)
    a = mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp.astype(index), ci.astype(index),
                                                        (m, n)), 0)
    X = torch.from_numpy(np.random.default_rng(3).uniform(-1, 1, n * 24).astype(dtype)).cuda()
    X0 = X.clone()
    drb_probe.gather_rows_probe(a, X, 16)
    drb_probe.gather_rows_probe(a, X, 16, with_values=False)
    drb_probe.gather_rows_probe(a, X, 8, ldx=24)
    torch.cuda.synchronize()
    assert torch.equal(X, X0)
    a.check()
    lib = drb_probe.lib

    def rc(ptr, ldx, k, h=a.handle):
        return lib.drb_csr_gather_rows_probe(h, C.c_void_p(ptr), ldx, k, 1, None)
    assert rc(X.data_ptr(), 24, 3) == capi.DRB_ERR_UNSUPPORTED  # 3 elements: not 16-byte vectors
    assert rc(X.data_ptr(), 24, 24) == capi.DRB_ERR_UNSUPPORTED  # 6 or 12 vectors per row
    assert rc(X.data_ptr(), 8, 16) == capi.DRB_ERR_UNSUPPORTED  # ldx < k
    assert rc(X.data_ptr() + 4, 16, 16) == capi.DRB_ERR_INVALID_ARG  # misaligned X
    vb = v.astype(np.float32)
    b16 = mp.distributed_sparse_matrix(mp.csr_matrix_view(vb, rp, ci, (m, n)), 0,
                                       storage=torch.bfloat16)
    assert rc(X.data_ptr(), 16, 16, b16.handle) == capi.DRB_ERR_UNSUPPORTED


# ---- adjoint ------------------------------------------------------------------------
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("kind", ["chunky", "laplacian"])
def test_adjoint_against_transposed_oracle(mp, dtype, kind):
    """Row-block kernels (irregular rows), and the sliced-ELL copies of A and
    A^T (a Laplacian with random values: short regular rows both ways)."""
    if kind == "chunky":
        rp, ci, v, m, n = chunky_matrix(dtype)
    else:
        import drb
        rp, ci, v = drb.gen.laplacian2d_csr(300, value_dtype=dtype)
        m = n = 300 * 300
        v = np.random.default_rng(5).uniform(-1, 1, len(v)).astype(dtype)
    rng = np.random.default_rng(2)
    x = rng.uniform(-1, 1, n).astype(dtype)
    yb = rng.uniform(-1, 1, m).astype(dtype)
    a = mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp, ci, (m, n)), 0, adjoint=True)
    assert (a.variant() == 2048) == (kind == "laplacian")
    tdt = torch.from_numpy(x).dtype
    xbar = torch.empty(n, dtype=tdt, device="cuda")
    abar = torch.empty(len(v), dtype=tdt, device="cuda")
    mp.gemv_backward(a, torch.from_numpy(yb).cuda(), torch.from_numpy(x).cuda(), xbar, abar)
    torch.cuda.synchronize()
    cp, ri, vt = oracle.transpose(rp, ci, v, m, n)
    xb_ref = oracle.gemv_row(cp, ri, vt, yb, n, m, 1, oracle.ACC_LD)
    d = oracle.absdot(cp, ri, vt, yb, n, m)
    tol = 1e-5 if dtype == np.float32 else 1e-12
    assert rel_err(xbar.cpu().numpy(), xb_ref, d) <= tol
    ab_ref = oracle.abar(rp, ci, yb, x, m)
    assert np.allclose(abar.cpu().numpy(), ab_ref, rtol=1e-6 if dtype == np.float32 else 1e-15,
                       atol=0)
    # values updated in CSR order must reach the transposed copy
    v2 = (v * 2).astype(dtype)
    a.update_values(torch.from_numpy(v2).cuda())
    mp.gemv_backward(a, torch.from_numpy(yb).cuda(), None, xbar, None)
    torch.cuda.synchronize()
    assert rel_err(xbar.cpu().numpy(), 2 * xb_ref, 2 * d) <= tol


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("m", [1, 31, 33, 1031])
def test_abar_short_rows_edges(mp, dtype, m):
    """Rows of 0..64 nonzeros (many empty, m not a multiple of the 32-row
    groups): abar = ybar_i * x_j is one rounded product per entry, so it
    matches numpy's bit for bit."""
    rng = np.random.default_rng(m)
    n = 700
    lens = rng.integers(0, 65, m)
    lens[rng.random(m) < 0.3] = 0
    lens[0] = 64
    rp = np.zeros(m + 1, np.int64)
    rp[1:] = np.cumsum(lens)
    ci = np.concatenate([np.sort(rng.choice(n, k, replace=False)) for k in lens]
                        + [np.zeros(0, np.int64)]).astype(np.int32)
    v = rng.uniform(-1, 1, len(ci)).astype(dtype)
    x = rng.uniform(-1, 1, n).astype(dtype)
    yb = rng.uniform(-1, 1, m).astype(dtype)
    a = mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp, ci, (m, n)), 0, adjoint=True)
    tdt = torch.from_numpy(x).dtype
    abar = torch.full((len(v),), 7.0, dtype=tdt, device="cuda")
    mp.gemv_backward(a, torch.from_numpy(yb).cuda(), torch.from_numpy(x).cuda(), None, abar)
    rows = np.repeat(np.arange(m), lens)
    assert np.array_equal(abar.cpu().numpy(), yb[rows] * x[ci])


@pytest.mark.parametrize("variant", ["128,1", "256,0", "512,1", "128,1,1"])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_abar_items_edges(mp, dtype, variant, monkeypatch):
    """A longest row above 64 nonzeros sends abar to the forward product's
    work items (one item ahead, rows from stamps and a warp max-scan): empty
    rows, runs of 0-2 nonzero rows (64-row items), rows split into chunks of
    every item span, and an output not 16-byte aligned (scalar stores); one
    rounded product per entry, so numpy's bits."""
    monkeypatch.setenv("DRB_SPMV_VARIANT", variant)
    rng = np.random.default_rng(11)
    n = 5000
    lens = np.concatenate([rng.integers(0, 3, 3000), [0, 0, 1, 2000, 0, 70, 129, 257, 513, 0],
                           rng.integers(0, 200, 300), rng.integers(0, 2, 1000), [64, 65, 0]])
    m = len(lens)
    rp = np.zeros(m + 1, np.int64)
    rp[1:] = np.cumsum(lens)
    ci = np.concatenate([np.sort(rng.choice(n, k, replace=False)) for k in lens]).astype(np.int32)
    v = rng.uniform(-1, 1, len(ci)).astype(dtype)
    x = rng.uniform(-1, 1, n).astype(dtype)
    yb = rng.uniform(-1, 1, m).astype(dtype)
    a = mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp, ci, (m, n)), 0, adjoint=True)
    assert a.variant() & ~3 == int(variant.split(",")[0])
    tdt = torch.from_numpy(x).dtype
    ref = yb[np.repeat(np.arange(m), lens)] * x[ci]
    xt, ybt = torch.from_numpy(x).cuda(), torch.from_numpy(yb).cuda()
    for shift in (0, 1):  # 1: abar one element past a 16-byte boundary
        buf = torch.full((len(v) + 1,), 7.0, dtype=tdt, device="cuda")
        abar = buf[shift:shift + len(v)]
        for _ in range(2):
            mp.gemv_backward(a, ybt, xt, None, abar)
        a.check()
        assert np.array_equal(abar.cpu().numpy(), ref)
        assert buf[len(v) if shift == 0 else 0].item() == 7.0  # nothing outside abar written
    a.destroy()


def test_adjoint_finite_differences_laplacian(mp):
    """Central differences (h = 1e-6, fp64) of L = 0.5 ||A x - b||^2 through
    the forward gemv.  The loss difference is formed row by row as
    0.5 (y+ - y-)(y+ + y- - 2b), which equals L(+) - L(-) but does not lose
    digits to the cancellation of two large sums; rows the perturbation does
    not reach contribute exactly 0."""
    import drb
    g = 48
    rp, ci, v = drb.gen.laplacian2d_csr(g, value_dtype=np.float64)
    m = g * g
    rng = np.random.default_rng(9)
    x = rng.standard_normal(m)
    b = rng.standard_normal(m)
    a = mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp, ci, (m, m)), 0, adjoint=True)
    xt, bt = torch.from_numpy(x).cuda(), torch.from_numpy(b).cuda()
    y = torch.empty(m, dtype=torch.float64, device="cuda")
    a.gemv_device(xt, y)
    r = y - bt
    xbar = torch.empty(m, dtype=torch.float64, device="cuda")
    abar = torch.empty(len(v), dtype=torch.float64, device="cuda")
    mp.gemv_backward(a, r, xt, xbar, abar)

    def fwd(xx):
        yy = torch.empty(m, dtype=torch.float64, device="cuda")
        a.gemv_device(xx, yy)
        return yy

    def dloss(yp, ym):
        return float((0.5 * (yp - ym) * (yp + ym - 2 * bt)).sum().item())

    h = 1e-6
    for i in rng.choice(m, 64, replace=False):
        e = torch.zeros(m, dtype=torch.float64, device="cuda")
        e[i] = h
        fd = dloss(fwd(xt + e), fwd(xt - e)) / (2 * h)
        assert abs(fd - xbar[i].item()) <= 1e-6 * max(1.0, abs(fd))
    vt = torch.from_numpy(v.copy()).cuda()
    for p in rng.choice(len(v), 32, replace=False):
        vp, vm = vt.clone(), vt.clone()
        vp[p] += h
        vm[p] -= h
        a.update_values(vp)
        yp = fwd(xt)
        a.update_values(vm)
        ym = fwd(xt)
        fd = dloss(yp, ym) / (2 * h)
        assert abs(fd - abar[p].item()) <= 1e-6 * max(1.0, abs(fd))
    a.update_values(vt)


def test_launch_count_increases(mp):
    from drb import _capi
    f = load("mp_gemv_100x100")
    a = mp.distributed_sparse_matrix(view(mp, f), 0)
    b = mp.broadcasted_vector()
    b.broadcast_data(100, 0, f["x"])
    c0 = _capi.launch_count()
    mp.gemv(0, np.zeros(100, np.float32), a, b)
    assert _capi.launch_count() == c0 + 1


# ---- sliced-ELL copy for short, regular rows ---------------------------------------
def stencil_like(m, n, seed, dtype):
    """Rows of 3-5 nonzeros (mostly 5) with a few empty rows, columns near the
    diagonal plus one far band, as a 2-D stencil has."""
    rng = np.random.default_rng(seed)
    lens = rng.choice([3, 4, 5], size=m, p=[0.05, 0.15, 0.8])
    lens[[7 % m, m // 2, m - 1]] = 0
    rp = np.zeros(m + 1, np.int64)
    rp[1:] = np.cumsum(lens)
    rows = np.repeat(np.arange(m), lens)
    k = np.arange(rp[-1]) - np.repeat(rp[:-1], lens)
    off = np.array([-300, -1, 0, 1, 300])[k]
    ci = np.clip(rows + off, 0, n - 1).astype(np.int32)
    v = rng.uniform(-1, 1, rp[-1]).astype(dtype)
    return rp.astype(np.int32), ci, v


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("m", [1000, 100_003, 1_000_000])
def test_sell_short_rows_match_oracle_and_row_blocks(mp, dtype, m, monkeypatch):
    rp, ci, v = stencil_like(m, m, m, dtype)
    x = np.random.default_rng(1).uniform(-1, 1, m).astype(dtype)
    a, y = gpu_gemv(mp, rp, ci, v, m, m, x)
    assert a.variant() == 2048                      # the sliced-ELL kernel runs
    y64 = oracle.gemv_row(rp, ci, v, x, m, m, 1, oracle.ACC_LD)
    d = oracle.absdot(rp, ci, v, x, m, m)
    tol = 1e-5 if dtype == np.float32 else 1e-12
    assert rel_err(y, y64, d) <= tol
    assert (y[[7 % m, m // 2, m - 1]] == 0).all()  # empty rows
    monkeypatch.setenv("DRB_SPMV_VARIANT", "256,1")  # the row-block kernel
    b, y2 = gpu_gemv(mp, rp, ci, v, m, m, x)
    assert b.variant() == 257
    assert rel_err(y, y2.astype(np.float64), d) <= 2 * tol


def test_sell_not_taken_for_irregular_rows(mp):
    rp, ci, v, m, n = chunky_matrix(np.float32)
    a = mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp, ci, (m, n)), 0)
    assert a.variant() != 2048


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_sell_fused_residual_and_value_update(mp, dtype):
    m = 200_001
    rp, ci, v = stencil_like(m, m, 9, dtype)
    rng = np.random.default_rng(10)
    x = rng.uniform(-1, 1, m).astype(dtype)
    b = rng.uniform(-1, 1, m).astype(dtype)
    a = mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp, ci, (m, m)), 0)
    assert a.variant() == 2048
    xt, bt = torch.from_numpy(x).cuda(), torch.from_numpy(b).cuda()
    yt = torch.empty_like(xt)
    r2 = float(mp.residual_norm2(a, xt, bt, yt).item())
    y64 = oracle.gemv_row(rp, ci, v, x, m, m, 1, oracle.ACC_LD)
    want = float(np.sum((y64 - b.astype(np.float64)) ** 2))
    assert abs(r2 - want) <= (1e-4 if dtype == np.float32 else 1e-10) * want
    # new values reach the sliced copy
    v2 = (v * -2.5).astype(dtype)
    a.update_values(torch.from_numpy(v2).cuda())
    a.gemv_device(xt, yt)
    y2 = oracle.gemv_row(rp, ci, v2, x, m, m, 1, oracle.ACC_LD)
    d = oracle.absdot(rp, ci, v2, x, m, m)
    assert rel_err(yt.cpu().numpy(), y2, d) <= (1e-5 if dtype == np.float32 else 1e-12)


def test_sell_host_gemv_segments_bit_identical(mp):
    import drb
    rp, ci, v = drb.gen.laplacian2d_csr(2048, value_dtype=np.float64)
    m = len(rp) - 1
    assert rp[-1] > (1 << 22)                       # the segmented host path
    x = np.random.default_rng(11).standard_normal(m)
    a, y_dev = gpu_gemv(mp, rp.astype(np.int32), ci, v, m, m, x)
    assert a.variant() == 2048
    xh = torch.from_numpy(x).pin_memory().numpy()
    yh = torch.empty(m, dtype=torch.float64).pin_memory().numpy()
    for _ in range(2):
        yh[:] = np.nan
        a.gemv_host(xh, yh)
        assert np.array_equal(yh.view(np.uint8), y_dev.view(np.uint8))


def test_sell_autotune_keeps_a_valid_choice(mp):
    m = 300_000
    rp, ci, v = stencil_like(m, m, 12, np.float64)
    x = np.random.default_rng(13).standard_normal(m)
    a, y = gpu_gemv(mp, rp, ci, v, m, m, x)
    chosen = a.autotune()
    assert chosen == a.variant() and chosen in (256, 257, 512, 513, 2048)
    xt = torch.from_numpy(x).cuda()
    yt = torch.empty_like(xt)
    a.gemv_device(xt, yt)
    y64 = oracle.gemv_row(rp, ci, v, x, m, m, 1, oracle.ACC_LD)
    assert rel_err(yt.cpu().numpy(), y64, oracle.absdot(rp, ci, v, x, m, m)) <= 1e-12
