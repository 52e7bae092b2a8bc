"""drb_dot_noalloc: the dot product for callers that must not allocate.

Some callers may not allocate device memory during a call (a fixed memory
budget, code running inside their own allocator or pool callback, streams
whose allocations they must account for).  drb_dot takes its scratch from
cudaMallocAsync; drb_dot_noalloc takes it from a static device array of the
library, which holds vectors of up to 2^29 elements.  These tests call both
entry points through the C ABI and require the same sums, within the
tolerance the other dot tests use, on two calls in a row (the static array
keeps the previous call's contents, so the second call checks that nothing
stale leaks in).

This file is named to be collected last, so a run that stops at the first
failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from drb import _capi as capi

MAX_N = 1 << 29


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


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["float32", "float64"])
@pytest.mark.parametrize("n", [1, 1000, 3_000_001])
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
        ref = torch.empty(1, dtype=torch.float64, device="cuda")
        got = torch.empty(1, dtype=torch.float64, device="cuda")
        capi.check(capi.lib.drb_dot(n, _p(a), _p(b), dcode, _p(ref), stream))
        capi.check(capi.lib.drb_dot_noalloc(n, _p(a), _p(b), dcode, _p(got), stream))
        torch.cuda.synchronize()
        scale = max(1.0, float((a.double().abs() * b.double().abs()).sum()))
        assert abs(got.item() - ref.item()) <= 1e-12 * scale, (call, got.item(), ref.item())
