"""GPU parity of the batched dense BF16 product on the tensor cores
(drb_dense_batch_*): Y_i = A_i X_i with FP32 accumulation, against the
oracle's FP64 dense gemv on the same bf16 values.

A bf16 x bf16 product is exact in fp32, so the only error is the fp32
accumulation of n terms: gated at 1e-4 relative to sum_j |a_ij x_j| per
output element (typical errors are ~sqrt(n) 2^-24).  The padding columns of
every A (lda > n) hold NaN, so a read outside the matrix shows up as NaN."""
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


def make(m, n, k, layout, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    lda = (n + 7) // 8 * 8 + (8 if n % 3 == 0 else 0)
    A = torch.randn(m, lda, device="cuda", generator=g).to(torch.bfloat16)
    if lda > n:
        A[:, n:] = float("nan")
    x_cm = torch.randn(n * k, device="cuda", generator=g).to(torch.bfloat16)
    x = x_cm if layout == COL else x_cm.view(k, n).t().contiguous().view(-1)
    y = torch.full((m * k,), float("nan"), device="cuda")
    return A, x, x_cm, y


def reference(A, x_cm, n, k):
    a = A[:, :n].float().cpu().numpy().astype(np.float64)
    xv = x_cm.float().cpu().numpy().astype(np.float64)
    ref = oracle.dense_gemv(a, xv, k, oracle.ACC_F64)
    den = oracle.dense_gemv(np.abs(a), np.abs(xv), k, oracle.ACC_F64)
    return ref, np.maximum(den, np.finfo(np.float64).tiny)


def check(y, A, x_cm, m, n, k, layout, tol=1e-4):
    got = y.cpu().numpy().astype(np.float64)
    if layout == ROW:
        got = got.reshape(m, k).T.reshape(-1)
    assert not np.isnan(got).any(), "unwritten output or a read past n"
    ref, den = reference(A, x_cm, n, k)
    err = float(np.max(np.abs(got - ref) / den)) if m * k else 0.0
    assert err <= tol, (m, n, k, err)
    return err


def test_dense_tc_one_tile(mp):
    """One 128 x 64 tile: one TMA stage, four MMAs."""
    A, x, x_cm, y = make(128, 64, 32, COL, 1)
    P = mp.dense_batch([A], [x], [y], 32, COL, ns=[64])
    P.gemv()
    P.check()
    check(y, A, x_cm, 128, 64, 32, COL)
    P.destroy()


@pytest.mark.parametrize("layout", [COL, ROW])
@pytest.mark.parametrize("k", [32, 1, 20, 64])
def test_dense_tc_ragged_batch(mp, k, layout):
    """Shapes that are not multiples of the 128 x 64 tile, tall and wide,
    several K stages and ring wrap-around, in one launch."""
    shapes = [(300, 257), (129, 64), (1, 1000), (1000, 1), (513, 777), (64, 4100), (256, 256)]
    As, xs, xcs, ys = [], [], [], []
    for i, (m, n) in enumerate(shapes):
        A, x, x_cm, y = make(m, n, k, layout, 10 + i)
        As.append(A), xs.append(x), xcs.append(x_cm), ys.append(y)
    P = mp.dense_batch(As, xs, ys, k, layout, ns=[n for _, n in shapes])
    for _ in range(2):
        P.gemv()
    P.check()
    for (m, n), A, x_cm, y in zip(shapes, As, xcs, ys):
        check(y, A, x_cm, m, n, k, layout)
    P.destroy()


def test_dense_tc_deterministic_and_launches(mp):
    from drb import _capi as capi
    A, x, x_cm, y = make(700, 3000, 32, COL, 5)
    P = mp.dense_batch([A], [x], [y], 32, COL, ns=[3000])
    c0 = capi.launch_count()
    P.gemv()
    assert capi.launch_count() - c0 == 2  # X layout kernel + the tensor-core kernel
    y1 = y.clone()
    P.gemv()
    P.check()
    assert torch.equal(y, y1)
    check(y, A, x_cm, 700, 3000, 32, COL)
    P.destroy()


def test_dense_tc_wait_timeout_is_reported_and_the_plan_recovers(mp):
    """Failure detection without a fault: the CTA of one tile issues no loads
    (drb_dense_batch_set_wait), so its pipeline wait runs out after 2 ms; the
    kernel records DRB_ERR_TIMEOUT, the other CTAs stop at their next wait
    after draining the copies they issued, and drb_dense_batch_check reports
    it.  The next launch with normal waits gives oracle-correct results."""
    from drb import _capi as capi
    shapes = [(1000, 3000), (300, 257), (513, 777)]
    As, xs, xcs, ys = [], [], [], []
    for i, (m, n) in enumerate(shapes):
        A, x, x_cm, y = make(m, n, 32, COL, 40 + i)
        As.append(A), xs.append(x), xcs.append(x_cm), ys.append(y)
    P = mp.dense_batch(As, xs, ys, 32, COL, ns=[n for _, n in shapes])
    P.gemv()
    P.check()
    for tile in (0, 5):
        P.set_wait(2_000_000, tile)
        P.gemv()
        with pytest.raises(capi.DrbError) as e:
            P.check()
        assert e.value.status == capi.DRB_ERR_TIMEOUT
        P.check()  # the error word was cleared
    P.set_wait()
    for y in ys:
        y.fill_(float("nan"))
    P.gemv()
    P.check()
    for (m, n), A, x_cm, y in zip(shapes, As, xcs, ys):
        check(y, A, x_cm, m, n, 32, COL)
    P.destroy()


def test_dense_tc_rejects(mp):
    from drb import _capi as capi
    A = torch.zeros(64, 100, device="cuda", dtype=torch.bfloat16)  # lda 100: not % 8
    x = torch.zeros(100 * 32, device="cuda", dtype=torch.bfloat16)
    y = torch.zeros(64 * 32, device="cuda")
    with pytest.raises(capi.DrbError) as e:
        mp.dense_batch([A], [x], [y], 32, COL)
    assert e.value.status == capi.DRB_ERR_UNSUPPORTED
    A = torch.zeros(64, 104, device="cuda", dtype=torch.bfloat16)
    with pytest.raises(capi.DrbError) as e:
        mp.dense_batch([A], [x], [y], 300, COL, ns=[100])
    assert e.value.status == capi.DRB_ERR_UNSUPPORTED
