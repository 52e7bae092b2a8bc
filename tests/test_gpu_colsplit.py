"""The column-blocked single-RHS plan (csrc/colsplit.cu) against the oracle.

drb_csr_create regroups a handle's nonzeros by column block when x is too
large to stay in L2 (above 48 MiB); DRB_COLSPLIT=<n>, read at creation,
forces n blocks on the small matrices used here.  Each case checks the
split product against the oracle's long-double csr_row loop (FP32 within
1e-5, FP64 within 1e-12 of sum |a x| per row), determinism, the host-pointer
call (bit-identical to the device call), a value update, and the adjoint
whose transposed matrix is split as well."""
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


def rel_err(y, y_ref, denom):
    d = np.maximum(np.asarray(denom, np.float64), np.finfo(np.float64).tiny)
    return float(np.max(np.abs(np.asarray(y, np.float64) - y_ref) / d)) if len(d) else 0.0


def mixed_rows(dtype, unsorted, seed=3):
    """Empty, short, long and chunked rows (longer than one 512-nonzero item,
    and one of 70,001 nonzeros), columns uniform over 300,000; with
    `unsorted` each row's columns are shuffled."""
    rng = np.random.default_rng(seed)
    n = 300_000
    lens = np.concatenate([rng.integers(0, 40, 4000), [0, 1, 2047, 2049, 0],
                           [70_001], rng.integers(0, 6, 2000), rng.integers(100, 2000, 100)])
    m = len(lens)
    rp = np.zeros(m + 1, np.int64)
    rp[1:] = np.cumsum(lens)
    ci = np.empty(rp[-1], np.int32)
    for r in range(m):
        if lens[r]:
            c = rng.choice(n, lens[r], replace=False)
            ci[rp[r]:rp[r + 1]] = c if unsorted else np.sort(c)
    v = rng.uniform(-1, 1, rp[-1]).astype(dtype)
    return rp.astype(np.int32), ci, v, m, n


def check(y, rp, ci, v, x, m, n, tol):
    y64 = oracle.gemv_row(rp, ci, v, x, m, n, 1, oracle.ACC_LD)
    assert rel_err(y, y64, oracle.absdot(rp, ci, v, x, m, n)) <= tol


@pytest.mark.parametrize("unsorted", [False, True])
@pytest.mark.parametrize("nblk", [2, 3, 8])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_split_gemv_parity(mp, dtype, nblk, unsorted, monkeypatch):
    monkeypatch.setenv("DRB_COLSPLIT", str(nblk))
    rp, ci, v, m, n = mixed_rows(dtype, unsorted)
    tol = 1e-5 if dtype == np.float32 else 1e-12
    a = mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp, ci, (m, n)), 0)
    nb, bw = a.column_blocks()
    # two blocks: a first block of 45% of the columns; more: equal widths
    assert nb == nblk and bw == (int(0.45 * n) if nblk == 2 else -(-n // nblk))
    x = np.random.default_rng(7).uniform(-1, 1, n).astype(dtype)
    xt = torch.from_numpy(x).cuda()
    yt = torch.full((m,), float("nan"), dtype=xt.dtype, device="cuda")
    a.gemv_device(xt, yt)
    a.check()
    y1 = yt.cpu().numpy()
    check(y1, rp, ci, v, x, m, n, tol)
    for _ in range(2):  # repeat launches: same bits
        a.gemv_device(xt, yt)
    assert np.array_equal(yt.cpu().numpy().view(np.uint8), y1.view(np.uint8))
    yh = np.empty(m, dtype)
    a.gemv_host(x, yh)  # host pointers: the same blocks, the same bits
    assert np.array_equal(yh.view(np.uint8), y1.view(np.uint8))
    # new values reach the blocks' copy
    v2 = (np.random.default_rng(8).uniform(-1, 1, len(v))).astype(dtype)
    a.update_values(torch.from_numpy(v2).cuda())
    a.gemv_device(xt, yt)
    check(yt.cpu().numpy(), rp, ci, v2, x, m, n, tol)
    a.destroy()


@pytest.mark.parametrize("nblk,first,segs,growth", [
    (2, "0.3", "6", "1.5"), (2, "0.45", "1", "1.5"), (3, "", "8", "0.7"),
    (2, "0.7", "3", "2.0"), (8, "0.05", "5", "1.2")])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_split_host_pipeline(mp, dtype, nblk, first, segs, growth, monkeypatch):
    """The host-pointer gemv of a split handle uploads x block by block, runs
    each block once its slice has arrived and the last block in row segments
    whose rows copy back behind the later ones: the device call's bits, for an
    uneven first block (DRB_COLSPLIT_FIRST) and any segment count and growth,
    with pinned and pageable host buffers, call after call.  (An empty
    DRB_COLSPLIT_FIRST asks for equal widths.)"""
    monkeypatch.setenv("DRB_COLSPLIT", str(nblk))
    monkeypatch.setenv("DRB_COLSPLIT_FIRST", first)
    monkeypatch.setenv("DRB_HOST_SEGMENTS", segs)
    monkeypatch.setenv("DRB_HOST_SPLIT_GROWTH", growth)
    rp, ci, v, m, n = mixed_rows(dtype, True, seed=41)
    a = mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp, ci, (m, n)), 0)
    nb, bw = a.column_blocks()
    assert nb == nblk
    assert bw == (int(float(first) * n) if first else -(-n // nblk))
    x = np.random.default_rng(42).uniform(-1, 1, n).astype(dtype)
    xt = torch.from_numpy(x).cuda()
    yt = torch.empty(m, dtype=xt.dtype, device="cuda")
    a.gemv_device(xt, yt)
    yd = yt.cpu().numpy()
    check(yd, rp, ci, v, x, m, n, 1e-5 if dtype == np.float32 else 1e-12)
    xp = torch.from_numpy(x).pin_memory()
    yp = torch.full((m,), float("nan"), dtype=xp.dtype).pin_memory()
    for _ in range(2):
        a.gemv_host(xp.numpy(), yp.numpy())
        assert np.array_equal(yp.numpy().view(np.uint8), yd.view(np.uint8))
    yh = np.full(m, np.nan, dtype)
    a.gemv_host(x, yh)
    assert np.array_equal(yh.view(np.uint8), yd.view(np.uint8))
    a.destroy()


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_split_matches_unsplit_within_tolerance(mp, dtype, monkeypatch):
    """The same handle without a split (DRB_COLSPLIT=0): both within the gate
    of the oracle, and the unsplit one reports one block."""
    rp, ci, v, m, n = mixed_rows(dtype, False, seed=11)
    x = np.random.default_rng(12).uniform(-1, 1, n).astype(dtype)
    tol = 1e-5 if dtype == np.float32 else 1e-12
    out = {}
    for nb in ("0", "4"):
        monkeypatch.setenv("DRB_COLSPLIT", nb)
        a = mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp, ci, (m, n)), 0,
                                         autotune=True)
        assert a.column_blocks()[0] == (1 if nb == "0" else 4)
        xt = torch.from_numpy(x).cuda()
        yt = torch.empty(m, dtype=xt.dtype, device="cuda")
        a.gemv_device(xt, yt)
        out[nb] = yt.cpu().numpy()
        check(out[nb], rp, ci, v, x, m, n, tol)
        a.destroy()


@pytest.mark.parametrize("nblk", [2, 3, 8])
def test_split_compensated_fp32(mp, nblk, monkeypatch):
    """A compensated FP32 handle keeps compensated sums within each column
    block; the combine adds the nblk block sums plainly, at most (nblk - 1)
    roundings of sum |a x| more: within the 1e-6 gate of the compensated
    product, and the host path gives the same bits."""
    monkeypatch.setenv("DRB_COLSPLIT", str(nblk))
    rp, ci, v, m, n = mixed_rows(np.float32, True, seed=61)
    a = mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp, ci, (m, n)), 0,
                                     compensated=True)
    assert a.column_blocks()[0] == nblk
    x = np.random.default_rng(62).uniform(-1, 1, n).astype(np.float32)
    xt = torch.from_numpy(x).cuda()
    y = torch.empty(m, device="cuda")
    a.gemv_device(xt, y)
    check(y.cpu().numpy(), rp, ci, v, x, m, n, 1e-6)
    yh = np.empty(m, np.float32)
    a.gemv_host(x, yh)
    assert np.array_equal(yh, y.cpu().numpy())
    a.destroy()


@pytest.mark.parametrize("nblk", [2, 3])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_split_residual(mp, dtype, nblk, monkeypatch):
    """||A x - b||^2 on a split handle: the split launch with the residual
    folded into the combine pass.  y has the gemv's bits (the same combine),
    the norm is the double sum of its terms (within summation order), the
    same bits call after call, and without a y buffer; y against the oracle."""
    monkeypatch.setenv("DRB_COLSPLIT", str(nblk))
    rp, ci, v, m, n = mixed_rows(dtype, False, seed=51)
    a = mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp, ci, (m, n)), 0)
    assert a.column_blocks()[0] == nblk
    rng = np.random.default_rng(52)
    x = rng.uniform(-1, 1, n).astype(dtype)
    b = rng.uniform(-1, 1, m).astype(dtype)
    xt, bt = torch.from_numpy(x).cuda(), torch.from_numpy(b).cuda()
    y = torch.full((m,), float("nan"), dtype=xt.dtype, device="cuda")
    outs = [mp.residual_norm2(a, xt, bt, y).item() for _ in range(3)]
    outs.append(mp.residual_norm2(a, xt, bt).item())
    assert len(set(outs)) == 1
    yg = torch.empty_like(y)
    a.gemv_device(xt, yg)
    assert torch.equal(y, yg)
    ref = float(((y.double() - bt.double()) ** 2).sum())
    assert abs(outs[0] - ref) <= 1e-10 * ref
    check(y.cpu().numpy(), rp, ci, v, x, m, n, 1e-5 if dtype == np.float32 else 1e-12)
    a.destroy()


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_split_adjoint(mp, dtype, monkeypatch):
    """x-bar = A^T y-bar on the split transposed matrix, against the oracle's
    csr_row loop on the explicit transpose; a-bar unchanged by the split."""
    monkeypatch.setenv("DRB_COLSPLIT", "3")
    rp, ci, v, m, n = mixed_rows(dtype, False, seed=21)
    a = mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp, ci, (m, n)), 0, adjoint=True)
    yb = np.random.default_rng(22).uniform(-1, 1, m).astype(dtype)
    x = np.random.default_rng(23).uniform(-1, 1, n).astype(dtype)
    xbar = torch.empty(n, dtype=torch.from_numpy(x).dtype, device="cuda")
    abar = torch.empty(len(v), dtype=xbar.dtype, device="cuda")
    mp.gemv_backward(a, torch.from_numpy(yb).cuda(), torch.from_numpy(x).cuda(), xbar, abar)
    a.check()
    cp, ri, vt = oracle.transpose(rp, ci, v, m, n)
    tol = 1e-5 if dtype == np.float32 else 1e-12
    check(xbar.cpu().numpy(), cp, ri, vt, yb, n, m, tol)
    ab_ref = oracle.abar(rp, ci, yb, x, m)
    assert np.allclose(abar.cpu().numpy(), ab_ref, rtol=1e-6 if dtype == np.float32 else 1e-15,
                       atol=0)
    a.destroy()


def test_stencil_stays_on_sliced_ell(mp, monkeypatch):
    """A 5-point Laplacian (short regular rows, local gathers) keeps its
    sliced-ELL copy and is not split, even when a split is asked for."""
    import drb
    monkeypatch.setenv("DRB_COLSPLIT", "3")
    rp, ci, v = drb.gen.laplacian2d_csr(256, value_dtype=np.float64)
    rp = rp.astype(np.int32)
    m = len(rp) - 1
    a = mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp, ci, (m, m)), 0)
    assert a.variant() == 2048 and a.column_blocks() == (1, m)
    x = np.random.default_rng(31).uniform(-1, 1, m)
    y = torch.empty(m, dtype=torch.float64, device="cuda")
    a.gemv_device(torch.from_numpy(x).cuda(), y)
    check(y.cpu().numpy(), rp, ci, v, x, m, m, 1e-12)
    a.destroy()
