"""GPU: BF16 storage with compensated FP32 accumulation, and compensated FP32.

Errors are relative to the per-row denominator sum_j |a_ij x_j| (plain
relative error is unbounded under cancellation).  Two FP64 references:
  * the oracle on the bf16-ROUNDED inputs: isolates the accumulation error
    (a bf16 x bf16 product is exact in fp32; compensated sums add only the
    final rounding);
  * the oracle on the ORIGINAL fp32 inputs: the end-to-end error, dominated by
    rounding values and x to bf16 (at most about 2^-8 relative per product).
"""
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


def rel(y, ref, d):
    d = np.maximum(d, np.finfo(np.float64).tiny)
    r = np.abs(np.asarray(y, np.float64) - ref) / d
    return float(r.max()), float(r.mean())


def bf16_round(a):
    return oracle.bf16_bits_to_f32(oracle.f32_to_bf16_bits(a))


def powerlaw_rowscale(m, seed):
    import drb
    alpha = drb.gen.zipf_alpha_for_mean(1, 65536, 32.0)
    return drb.gen.powerlaw_csr(m, m, alpha=alpha, hi=65536, seed=seed,
                                dist=drb.gen.NORMAL_ROWSCALE)


U_BF16 = 2.0 ** -8  # unit roundoff of bfloat16 (8-bit significand)


@pytest.mark.parametrize("x_f32", [False, True])
@pytest.mark.parametrize("autotune", [False, True])
def test_bf16_storage_error(mp, autotune, x_f32):
    """bf16 values with bf16 x: each product carries at most 2u + u^2 relative
    error from rounding its two inputs, so a single-product row can be off by
    ~7.8e-3; the norm-wise and mean errors are gated at 4e-3.  bf16 values
    with f32 x: at most u = 3.9e-3 per product, gated row by row at 4e-3."""
    import drb
    m = 300_000
    rp, ci, v = powerlaw_rowscale(m, 41)
    x = drb.gen.values(m, seed=42)
    a = mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp, ci, (m, m)), 0,
                                     storage=torch.bfloat16, autotune=autotune,
                                     x_dtype=torch.float32 if x_f32 else None)
    assert a.storage_bytes()[0] == 2
    xb = torch.from_numpy(x).cuda().to(a.x_dtype)
    y = torch.empty(m, dtype=torch.float32, device="cuda")
    a.gemv_device(xb, y)
    torch.cuda.synchronize()
    a.check()
    y = y.cpu().numpy()
    vr = bf16_round(v).astype(np.float64)
    xr = (x if x_f32 else bf16_round(x)).astype(np.float64)
    y_acc = oracle.gemv_row(rp, ci, vr, xr, m, m, 1, oracle.ACC_LD)
    e_acc, _ = rel(y, y_acc, oracle.absdot(rp, ci, vr, xr, m, m))
    assert e_acc <= 1e-6, e_acc          # compensated fp32 accumulation
    y64 = oracle.gemv_row(rp, ci, v.astype(np.float64), x.astype(np.float64), m, m, 1,
                          oracle.ACC_LD)
    d = oracle.absdot(rp, ci, v, x, m, m)
    e_max, e_mean = rel(y, y64, d)
    normwise = float(np.linalg.norm(y.astype(np.float64) - y64) / np.linalg.norm(d))
    if x_f32:
        assert e_max <= 4e-3, e_max
    else:
        assert e_max <= 2 * U_BF16 + U_BF16 ** 2, e_max
        assert normwise <= 4e-3, normwise
    assert e_mean <= 4e-3, e_mean
    # the mirror's gemv takes fp32 x and converts it to the storage type
    b = mp.broadcasted_vector()
    b.broadcast_data(m, 0, x)
    res = np.zeros(m, np.float32)
    mp.gemv(0, res, a, b)
    assert np.array_equal(res, y)


def test_bf16_host_path(mp):
    import drb
    m = 50_000
    rp, ci, v = powerlaw_rowscale(m, 43)
    x = drb.gen.values(m, seed=44)
    a = mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp, ci, (m, m)), 0,
                                     storage=torch.bfloat16)
    xb = torch.from_numpy(x).to(torch.bfloat16)
    yd = torch.empty(m, dtype=torch.float32, device="cuda")
    a.gemv_device(xb.cuda(), yd)
    xh = xb.pin_memory()
    yh = torch.empty(m, dtype=torch.float32).pin_memory()
    a.gemv_host(xh.view(torch.int16).numpy(), yh.numpy())
    assert np.array_equal(yh.numpy(), yd.cpu().numpy())


def test_compensated_fp32(mp):
    import drb
    m = 300_000
    rp, ci, v = powerlaw_rowscale(m, 45)
    x = drb.gen.values(m, seed=46)
    y64 = oracle.gemv_row(rp, ci, v, x, m, m, 1, oracle.ACC_LD)
    d = oracle.absdot(rp, ci, v, x, m, m)
    xt = torch.from_numpy(x).cuda()
    out = {}
    for comp in (False, True):
        a = mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp, ci, (m, m)), 0,
                                         compensated=comp)
        y = torch.empty(m, dtype=torch.float32, device="cuda")
        a.gemv_device(xt, y)
        torch.cuda.synchronize()
        out[comp] = rel(y.cpu().numpy(), y64, d)[0]
    assert out[False] <= 1e-5
    assert out[True] <= 1e-6, out
