"""CPU: the C-ABI library loads, exports every declared entry point, rejects
bad arguments before touching a GPU, and its host-side generators are
deterministic and match their stated distributions."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import drb
from drb import _capi as capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(drb_[a-z0-9_]+)\s*\(", src)))


@pytest.mark.parametrize("header", ["drb.h", "drb_gen.h"])
def test_library_exports_every_declared_symbol(header):
    names = declared(header)
    assert len(names) >= 8
    for name in names:
        assert hasattr(capi.lib, name), f"{name} declared in {header} but not exported"


def test_python_binding_covers_header():
    bound = {n for n, _, _ in capi.DRB_SYMBOLS + capi.GEN_SYMBOLS}
    assert set(declared("drb.h")) <= bound
    assert set(declared("drb_gen.h")) <= bound


def test_version_and_counter():
    assert b"sm_100a" in capi.lib.drb_version()
    assert capi.launch_count() >= 0


def _create(**kw):
    args = dict(m=4, n=4, nnz=0, rowptr=np.zeros(5, np.int32), colind=None, values=None,
                it=capi.DRB_I32, vt=capi.DRB_F32, st=capi.DRB_F32, nseg=1,
                part=capi.DRB_PART_ROW, flags=0)
    args.update(kw)
    h = C.c_void_p()
    p = lambda a: None if a is None else C.c_void_p(a.ctypes.data)
    rc = capi.lib.drb_csr_create(C.byref(h), args["m"], args["n"], args["nnz"],
                                 p(args["rowptr"]), p(args["colind"]), p(args["values"]),
                                 args["it"], args["vt"], args["st"], args["nseg"],
                                 args["part"], args["flags"], None)
    return rc, h


@pytest.mark.parametrize("kw", [
    dict(m=-1), dict(nnz=-3), dict(rowptr=None), dict(nnz=2),
    dict(it=7), dict(vt=capi.DRB_BF16), dict(vt=capi.DRB_F64, st=capi.DRB_BF16),
    dict(nseg=0), dict(part=5),
])
def test_invalid_arguments_rejected_without_gpu(kw):
    rc, h = _create(**kw)
    assert rc == capi.DRB_ERR_INVALID_ARG, (rc, capi.last_error())
    assert capi.last_error().startswith("invalid argument")
    assert not h.value


def test_null_out_pointer():
    rc = capi.lib.drb_csr_create(None, 1, 1, 0, None, None, None, 0, 0, 0, 1, 0, 0, None)
    assert rc == capi.DRB_ERR_INVALID_ARG


def test_no_device_reported_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    rc, h = _create()
    assert rc == capi.DRB_ERR_NO_DEVICE
    assert "CUDA" in capi.last_error() or "device" in capi.last_error()


def test_gemv_rejects_null_handle():
    assert capi.lib.drb_csr_gemv(None, None, None, 1, 0, None) == capi.DRB_ERR_INVALID_ARG
    assert capi.lib.drb_csr_gemv_backward(None, None, None, None, None, None) == \
        capi.DRB_ERR_INVALID_ARG
    assert capi.lib.drb_dense_gemv(4, 4, None, 2, None, None, 1, 0, 0, None) == \
        capi.DRB_ERR_INVALID_ARG


def test_batch_rejects_bad_arguments_without_gpu():
    lib = capi.lib
    out = C.c_void_p()
    hs = (C.c_void_p * 2)(None, None)
    assert lib.drb_batch_create(None, 1, hs, 16, 0, 0, None) == capi.DRB_ERR_INVALID_ARG
    assert lib.drb_batch_create(C.byref(out), 0, hs, 16, 0, 0, None) == \
        capi.DRB_ERR_INVALID_ARG
    assert lib.drb_batch_create(C.byref(out), 2, None, 16, 0, 0, None) == \
        capi.DRB_ERR_INVALID_ARG
    assert lib.drb_batch_create(C.byref(out), 2, hs, 16, 0, 0, None) == \
        capi.DRB_ERR_INVALID_ARG
    assert "handles" in capi.last_error()
    assert not out.value
    assert lib.drb_batch_gemv(None, None) == capi.DRB_ERR_INVALID_ARG
    assert lib.drb_batch_bind(None, None, None, None) == capi.DRB_ERR_INVALID_ARG
    assert lib.drb_batch_autotune(None, None, None) == capi.DRB_ERR_INVALID_ARG
    assert lib.drb_batch_destroy(None) == capi.DRB_OK
    assert lib.drb_batched_gemv(0, hs, None, None, 16, 0, 0, None) == \
        capi.DRB_ERR_INVALID_ARG


def test_zipf_alpha_solver():
    a = drb.gen.zipf_alpha_for_mean(1, 16384, 20.0)
    assert abs(a - 1.7613) < 1e-3
    assert abs(drb.gen.zipf_mean(1, 16384, a) - 20.0) < 1e-9
    assert abs(drb.gen.zipf_mean(1, 16384, 1.5) - 98.02) < 0.01
    assert abs(drb.gen.zipf_alpha_for_mean(1, 65536, 32.0) - 1.7448) < 1e-3


def _check_csr(rp, ci, m, n):
    assert rp[0] == 0 and np.all(np.diff(rp) >= 0)
    for r in range(m):
        row = ci[rp[r]:rp[r + 1]]
        assert np.all(np.diff(row) > 0) and (len(row) == 0 or (row[0] >= 0 and row[-1] < n))


def test_powerlaw_generator_stats_and_determinism():
    m = 200_000
    a = drb.gen.zipf_alpha_for_mean(1, 16384, 20.0)
    rp1, ci1, v1 = drb.gen.powerlaw_csr(m, m, alpha=a, hi=16384, seed=11, nthreads=1)
    rp2, ci2, v2 = drb.gen.powerlaw_csr(m, m, alpha=a, hi=16384, seed=11, nthreads=7)
    assert np.array_equal(rp1, rp2) and np.array_equal(ci1, ci2) and np.array_equal(v1, v2)
    mean = rp1[-1] / m
    assert 17.0 < mean < 23.0, mean
    assert np.abs(v1).max() <= 1.0
    _check_csr(rp1[:2001], ci1, 2000, m)
    rp3, _, _ = drb.gen.powerlaw_csr(m, m, alpha=a, hi=16384, seed=12)
    assert not np.array_equal(rp1, rp3)


def test_fixed_and_uniform_rows():
    rp, ci, v = drb.gen.fixed_rows_csr(1000, 5000, length=16, seed=3)
    assert np.all(np.diff(rp) == 16)
    _check_csr(rp, ci, 1000, 5000)
    rp, ci, v = drb.gen.uniform_rows_csr(1000, 3000, lo=8, hi=64, seed=4)
    d = np.diff(rp)
    assert d.min() >= 8 and d.max() <= 64
    _check_csr(rp, ci, 1000, 3000)
    rp, ci, v = drb.gen.fixed_rows_csr(10, 16, length=16, seed=3)  # full rows
    assert np.array_equal(ci[:16], np.arange(16))


def test_laplacian():
    rp, ci, v = drb.gen.laplacian2d_csr(64)
    assert rp[-1] == 5 * 64 * 64 - 4 * 64
    import scipy.sparse as sp
    A = sp.csr_matrix((v, ci, rp), shape=(64 * 64, 64 * 64)).toarray()
    assert np.allclose(A, A.T)
    assert np.allclose(A.sum(axis=1)[64 + 1], 0.0)  # interior row sums to 0
    _check_csr(rp, ci, 64 * 64, 64 * 64)


def test_values_distributions():
    u = drb.gen.values(100_000, seed=1, dist=drb.gen.UNIFORM_PM1)
    assert -1 <= u.min() and u.max() <= 1 and abs(u.mean()) < 0.02
    g = drb.gen.values(100_000, seed=1, dtype=np.float64, dist=drb.gen.NORMAL)
    assert abs(g.std() - 1) < 0.02
    assert np.array_equal(drb.gen.values(5000, seed=9, nthreads=1),
                          drb.gen.values(5000, seed=9, nthreads=5))


def test_vector_and_cg_entry_points_reject_bad_arguments_without_gpu():
    lib = capi.lib
    out = C.c_void_p(1)
    assert lib.drb_reduce(-1, None, capi.DRB_F32, 0, None, out, None) == capi.DRB_ERR_INVALID_ARG
    assert lib.drb_reduce(4, None, capi.DRB_F32, 0, None, out, None) == capi.DRB_ERR_INVALID_ARG
    assert lib.drb_reduce(0, None, capi.DRB_F32, 0, None, None, None) == capi.DRB_ERR_INVALID_ARG
    assert lib.drb_reduce(0, None, capi.DRB_BF16, 0, None, out, None) == capi.DRB_ERR_INVALID_ARG
    assert lib.drb_reduce(0, None, capi.DRB_INT32, 7, None, out, None) == capi.DRB_ERR_INVALID_ARG
    assert "op" in capi.last_error()
    assert lib.drb_iota(3, None, capi.DRB_INT64, 0, None) == capi.DRB_ERR_INVALID_ARG
    assert lib.drb_fill(3, out, capi.DRB_INT64, None, None) == capi.DRB_ERR_INVALID_ARG
    assert lib.drb_fill(0, None, 9, out, None) == capi.DRB_ERR_INVALID_ARG
    info = capi.CgInfo()
    assert lib.drb_csr_cg(None, None, None, 10, 1e-6, C.byref(info), None) == \
        capi.DRB_ERR_INVALID_ARG
