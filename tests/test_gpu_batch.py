"""GPU parity of the batched SpMM (drb_batch_*, drb_batched_gemv): every
matrix of a batch against the oracle's column-major multi-RHS gemv
(fp64-accumulated), through the C ABI.

Errors are relative to sum_j |a_ij x_j| per output element.  Gates: f32
1e-5, f64 1e-12, bf16 storage 1e-5 against the oracle on the bf16-rounded
inputs (a bf16 x bf16 product is exact in f32; only the f32 sums round)."""
import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu

COL, ROW = 0, 1


@pytest.fixture(scope="module")
def mp():
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from drb import mp as _mp
    return _mp


def long_row_csr(m, n, long_row, long_len, seed, dtype=np.float32):
    """Rows of 0..30 nonzeros and one row of long_len nonzeros."""
    rng = np.random.default_rng(seed)
    lens = rng.integers(0, 31, size=m)
    lens[long_row] = long_len
    rp = np.zeros(m + 1, np.int32)
    rp[1:] = np.cumsum(lens)
    ci = np.concatenate([np.sort(rng.choice(n, size=int(L), replace=False))
                         for L in lens]).astype(np.int32)
    v = rng.uniform(-1, 1, size=int(rp[-1])).astype(dtype)
    return rp, ci, v


def empty_csr(m, dtype=np.float32):
    return np.zeros(m + 1, np.int32), np.zeros(0, np.int32), np.zeros(0, dtype)


def mixed_batch(dtype=np.float32):
    """(m, n, rowptr, colind, values) for a batch of uneven shapes: tiny,
    empty rows, an all-empty matrix, wide, tall, and a row longer than every
    staging capacity."""
    import drb
    out = []
    for (m, n, lo, hi, seed) in [(1000, 1200, 8, 64, 1), (3, 5, 0, 3, 2), (1, 1, 1, 1, 3),
                                 (2000, 50, 0, 50, 4), (500, 20000, 0, 10, 5),
                                 (777, 777, 8, 64, 6)]:
        rp, ci, v = drb.gen.uniform_rows_csr(m, n, lo=lo, hi=hi, seed=seed,
                                             value_dtype=dtype)
        out.append((m, n, rp, ci, v))
    rp, ci, v = long_row_csr(40, 20000, 7, 5000, 7, dtype)
    out.append((40, 20000, rp, ci, v))
    rp, ci, v = empty_csr(64, dtype)
    out.append((64, 64, rp, ci, v))
    return out


def to_layout(a_cm, rows, k, layout):
    """Column-major rows x k block -> the requested layout (flat)."""
    if layout == COL:
        return np.ascontiguousarray(a_cm)
    return np.ascontiguousarray(a_cm.reshape(k, rows).T).reshape(-1)


def from_layout(a, rows, k, layout):
    if layout == COL:
        return np.asarray(a)
    return np.asarray(a).reshape(rows, k).T.reshape(-1)


def bf16_round(a):
    return oracle.bf16_bits_to_f32(oracle.f32_to_bf16_bits(a))


def run_batch(mp, mats_np, k, layout, *, storage=None, x_dtype=None, seed=100,
              autotune=False, one_shot=False):
    import drb
    vdt = mats_np[0][4].dtype
    mats, xs, ys, xs_np = [], [], [], []
    for i, (m, n, rp, ci, v) in enumerate(mats_np):
        a = mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp, ci, (m, n)), 0,
                                         storage=storage, x_dtype=x_dtype)
        mats.append(a)
        x_cm = drb.gen.values(n * k, seed=seed + i, dtype=vdt)
        xs_np.append(x_cm)
        xs.append(torch.from_numpy(to_layout(x_cm, n, k, layout)).cuda().to(a.x_dtype))
        ydt = torch.float64 if vdt == np.float64 else torch.float32
        ys.append(torch.full((m * k,), float("nan"), dtype=ydt, device="cuda"))
    tuned = None
    if one_shot:
        mp.batched_gemv(mats, xs, ys, k, layout)
    else:
        b = mp.batch(mats, k, layout)
        b.bind(xs, ys)
        if autotune:
            tuned = b.autotune()
        b.gemv()
        torch.cuda.synchronize()
        b.destroy()
    return mats, xs_np, [y.cpu().numpy() for y in ys], tuned


def check_against_oracle(mats_np, xs_np, ys, k, layout, tol, round_bf16=None):
    for (m, n, rp, ci, v), x, y in zip(mats_np, xs_np, ys):
        vv, xx = v, x
        if round_bf16 is not None:
            vv = bf16_round(v)
            xx = bf16_round(x) if round_bf16 == "x" else x
        vv = vv.astype(np.float64)
        xx = xx.astype(np.float64)
        ref = oracle.gemv_row(rp, ci, vv, xx, m, n, k, oracle.ACC_LD)
        d = np.maximum(oracle.absdot(rp, ci, vv, xx, m, n, k), np.finfo(np.float64).tiny)
        got = from_layout(y, m, k, layout).astype(np.float64)
        assert not np.isnan(got).any(), f"unwritten outputs (m={m}, n={n})"
        if m * k:
            err = float(np.max(np.abs(got - ref) / d))
            assert err <= tol, (m, n, k, err)


@pytest.mark.parametrize("layout", [COL, ROW])
@pytest.mark.parametrize("k", [1, 3, 12, 16, 40])
def test_batch_f32(mp, k, layout):
    mats_np = mixed_batch()
    _, xs, ys, _ = run_batch(mp, mats_np, k, layout)
    check_against_oracle(mats_np, xs, ys, k, layout, 1e-5)


@pytest.mark.parametrize("layout", [COL, ROW])
def test_batch_f32_wide_k(mp, layout):
    """k = 200: right-hand sides in two blocks of 128 over the staged items."""
    mats_np = mixed_batch()[:4]
    _, xs, ys, _ = run_batch(mp, mats_np, 200, layout)
    check_against_oracle(mats_np, xs, ys, 200, layout, 1e-5)


@pytest.mark.parametrize("k", [1, 16])
def test_batch_f64(mp, k):
    mats_np = mixed_batch(np.float64)
    _, xs, ys, _ = run_batch(mp, mats_np, k, COL)
    check_against_oracle(mats_np, xs, ys, k, COL, 1e-12)


@pytest.mark.parametrize("layout", [COL, ROW])
@pytest.mark.parametrize("k", [1, 16, 33])
def test_batch_bf16(mp, k, layout):
    mats_np = mixed_batch()
    _, xs, ys, _ = run_batch(mp, mats_np, k, layout, storage=torch.bfloat16)
    check_against_oracle(mats_np, xs, ys, k, layout, 1e-5, round_bf16="x")


def test_batch_bf16_f32_x(mp):
    mats_np = mixed_batch()
    _, xs, ys, _ = run_batch(mp, mats_np, 16, COL, storage=torch.bfloat16,
                             x_dtype=torch.float32)
    check_against_oracle(mats_np, xs, ys, 16, COL, 1e-5, round_bf16="v")


@pytest.mark.parametrize("x_dtype", [None, torch.float32])
def test_batch_bf16_sums_are_compensated(mp, x_dtype):
    """BF16 storage sums two-sum compensated per block of four products (a
    fused multiply-add chain per block, a two-sum into the row's sum): against
    the long-double oracle on the bf16-rounded inputs the kernel read, a row's
    error stays within 5u = 3.0e-7 of sum|a x| however long the row (the
    batch holds one of 5000 nonzeros, where plain f32 sums drift by about
    sqrt(5000) roundings)."""
    mats_np = mixed_batch()
    _, xs, ys, _ = run_batch(mp, mats_np, 16, COL, storage=torch.bfloat16, x_dtype=x_dtype)
    check_against_oracle(mats_np, xs, ys, 16, COL, 5 * 2.0 ** -24,
                         round_bf16="x" if x_dtype is None else "v")


def test_batch_deterministic_rebind_and_launch_count(mp):
    """Two graph launches give identical bits; rebinding new x/y needs no new
    graph; each launch runs the pack and SpMM kernels (column-major)."""
    import drb
    from drb import _capi as capi
    mats_np = mixed_batch()
    k = 16
    mats = [mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp, ci, (m, n)), 0)
            for (m, n, rp, ci, v) in mats_np]
    b = mp.batch(mats, k, COL)
    xs1 = [torch.from_numpy(drb.gen.values(n * k, seed=200 + i)).cuda()
           for i, (m, n, *_r) in enumerate(mats_np)]
    xs2 = [torch.from_numpy(drb.gen.values(n * k, seed=300 + i)).cuda()
           for i, (m, n, *_r) in enumerate(mats_np)]
    ya = [torch.empty(m * k, device="cuda") for (m, *_r) in mats_np]
    yb = [torch.empty(m * k, device="cuda") for (m, *_r) in mats_np]
    yc = [torch.empty(m * k, device="cuda") for (m, *_r) in mats_np]
    b.bind(xs1, ya)
    c0 = capi.launch_count()
    b.gemv()
    assert capi.launch_count() - c0 == 2
    b.bind(xs1, yb)
    b.gemv()
    b.bind(xs2, yc)
    b.gemv()
    torch.cuda.synchronize()
    for p, q in zip(ya, yb):
        assert torch.equal(p, q)
    check_against_oracle(mats_np, [x.cpu().numpy() for x in xs2],
                         [y.cpu().numpy() for y in yc], k, COL, 1e-5)
    b.destroy()


def test_batch_variants_agree(mp):
    """Every variant is correct.  Variants with the same G (slots per row)
    give identical bits whatever their staging capacity, since these rows
    have at most 64 nonzeros; the one-shot call equals the default graph;
    autotune returns one of the variants."""
    import drb
    mats_np = []
    for i in range(12):
        m = 3000 + 997 * i
        rp, ci, v = drb.gen.uniform_rows_csr(m, m, lo=8, hi=64, seed=40 + i)
        mats_np.append((m, m, rp, ci, v))
    k = 16
    mats = [mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp, ci, (m, n)), 0)
            for (m, n, rp, ci, v) in mats_np]
    xs_np = [drb.gen.values(n * k, seed=500 + i) for i, (m, n, *_r) in enumerate(mats_np)]
    xs = [torch.from_numpy(x).cuda() for x in xs_np]
    ys = [torch.empty(m * k, device="cuda") for (m, *_r) in mats_np]
    b = mp.batch(mats, k, COL)
    b.bind(xs, ys)
    default = b.variant()
    out = {}
    for c in range(3):
        for G in (1, 2, 4, 8):
            b.set_variant((c << 4) | G)
            assert b.variant() == (c << 4) | G
            b.gemv()
            torch.cuda.synchronize()
            out[(c, G)] = [y.cpu().numpy() for y in ys]
            check_against_oracle(mats_np, xs_np, out[(c, G)], k, COL, 1e-5)
    for G in (1, 2, 4, 8):
        for c in (1, 2):
            for p, q in zip(out[(0, G)], out[(c, G)]):
                assert np.array_equal(p, q), (c, G)
    ys1 = [torch.empty(m * k, device="cuda") for (m, *_r) in mats_np]
    mp.batched_gemv(mats, xs, ys1, k, COL)
    for p, q in zip(out[(default >> 4, default & 15)], ys1):
        assert np.array_equal(p, q.cpu().numpy())
    v = b.autotune()
    assert (v >> 4) in (0, 1, 2) and (v & 15) in (1, 2, 4, 8)
    b.destroy()


def test_batch_rejects_mixed_and_misaligned(mp):
    import drb
    from drb import _capi as capi
    rp, ci, v = drb.gen.uniform_rows_csr(100, 100, lo=1, hi=9, seed=9)
    a32 = mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp, ci, (100, 100)), 0)
    a64 = mp.distributed_sparse_matrix(
        mp.csr_matrix_view(v.astype(np.float64), rp, ci, (100, 100)), 0)
    with pytest.raises(capi.DrbError) as e:
        mp.batch([a32, a64], 16)
    assert e.value.status == capi.DRB_ERR_INVALID_ARG
    b = mp.batch([a32], 16, ROW)
    x = torch.zeros(100 * 16 + 1, device="cuda")[1:]  # 4-byte offset: not 16-byte aligned
    y = torch.zeros(100 * 16, device="cuda")
    with pytest.raises(capi.DrbError) as e:
        b.bind([x], [y])
    assert e.value.status == capi.DRB_ERR_INVALID_ARG
    with pytest.raises(capi.DrbError) as e:
        b.gemv()  # nothing bound
    assert e.value.status == capi.DRB_ERR_INVALID_ARG
    b.destroy()
