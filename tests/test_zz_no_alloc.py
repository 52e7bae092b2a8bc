"""drb_dot_noalloc: the dot product for callers that must not allocate.

Some callers may not allocate device memory during a call (a fixed memory
budget, code running inside their own allocator or pool callback, streams
whose allocations they must account for).  drb_dot takes its scratch from
cudaMallocAsync; drb_dot_noalloc takes it from a static device array of the
library, which holds vectors of up to 2^29 elements (one f64 partial per
8192-element block, 65,536 of them).  These tests call both entry points
through the C ABI and require the same sums as each other and as the oracle's
long-double dot, within the tolerance the other dot tests use, on calls in a
row: the static array keeps the previous call's contents, so later calls
check that nothing stale leaks in, including after a call that used every
slot and one with fewer blocks than the call before.

This file is named to be collected last, so a run that stops at the first
failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from drb import _capi as capi

MAX_N = 1 << 29
BLOCK = 8192  # elements per CTA (per scratch slot)


def _p(t):
    return C.c_void_p(t.data_ptr())


def test_noalloc_rejects_n_beyond_its_scratch():
    # the size check comes before any device use, so this runs without a GPU
    out = C.c_double()
    rc = capi.lib.drb_dot_noalloc(MAX_N + 1, C.c_void_p(16), C.c_void_p(16), capi.DRB_F32,
                                  C.byref(out), None)
    assert rc == capi.DRB_ERR_INVALID_ARG
    msg = capi.last_error()
    assert "maximum" in msg and str(MAX_N) in msg


def _both(a, b, dcode, stream):
    """(drb_dot, drb_dot_noalloc) of a and b (1-D device tensors, any offset)."""
    import torch
    n = a.numel()
    ref = torch.empty(1, dtype=torch.float64, device="cuda")
    got = torch.empty(1, dtype=torch.float64, device="cuda")
    capi.check(capi.lib.drb_dot(n, _p(a), _p(b), dcode, _p(ref), stream))
    capi.check(capi.lib.drb_dot_noalloc(n, _p(a), _p(b), dcode, _p(got), stream))
    torch.cuda.synchronize()
    return ref.item(), got.item()


def _check(a, b, dcode, stream, label):
    ref, got = _both(a, b, dcode, stream)
    ah, bh = a.cpu().numpy(), b.cpu().numpy()
    exact = oracle.dot(ah, bh)
    scale = max(1.0, float(np.abs(ah.astype(np.float64)) @ np.abs(bh.astype(np.float64))))
    assert abs(got - ref) <= 1e-12 * scale, (label, got, ref)
    assert abs(got - exact) <= 1e-12 * scale, (label, got, exact)


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["float32", "float64"])
@pytest.mark.parametrize("n", [1, 1000, 3_000_001, BLOCK * 37 - 1, BLOCK * 37,
                               BLOCK * 37 + 1])
def test_noalloc_matches_dot_on_two_calls(dtype, n):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    tdt = getattr(torch, dtype)
    dcode = capi.DRB_F32 if dtype == "float32" else capi.DRB_F64
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    g = torch.Generator().manual_seed(n)
    for call in range(2):
        a = torch.randn(n, generator=g, dtype=torch.float64).to(tdt).cuda()
        b = torch.randn(n, generator=g, dtype=torch.float64).to(tdt).cuda()
        _check(a, b, dcode, stream, f"call {call}")


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_noalloc_unaligned_vectors(dtype):
    """Vectors that start off a 16-byte boundary take the kernel's scalar
    loads; the sums still match."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    tdt = getattr(torch, dtype)
    dcode = capi.DRB_F32 if dtype == "float32" else capi.DRB_F64
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    g = torch.Generator().manual_seed(5)
    base_a = torch.randn(BLOCK * 9 + 7, generator=g, dtype=torch.float64).to(tdt).cuda()
    base_b = torch.randn(BLOCK * 9 + 7, generator=g, dtype=torch.float64).to(tdt).cuda()
    for off_a, off_b in ((1, 1), (1, 0), (0, 3)):
        n = BLOCK * 9 + 7 - max(off_a, off_b)
        _check(base_a[off_a:off_a + n], base_b[off_b:off_b + n], dcode, stream,
               f"offsets {off_a},{off_b}")


@pytest.mark.gpu
def test_noalloc_full_scratch_then_smaller_calls():
    """n = 2^29 fills all 65,536 partial slots; the calls after it use fewer
    blocks, so stale partials and a stale ticket would show up in their sums."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    if torch.cuda.mem_get_info()[0] < (6 << 30):
        pytest.skip("needs 6 GB of free device memory")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    g = torch.Generator(device="cuda").manual_seed(29)
    a = torch.empty(MAX_N, device="cuda").uniform_(-1, 1, generator=g)
    b = torch.empty(MAX_N, device="cuda").uniform_(-1, 1, generator=g)
    _check(a, b, capi.DRB_F32, stream, "n = 2^29")
    for n in (BLOCK * 3 + 1, 1000, MAX_N // 2 + 5):
        _check(a[:n], b[:n], capi.DRB_F32, stream, f"n = {n} after a larger call")
    del a, b
    torch.cuda.empty_cache()
