"""Matrix Market ingest (drb_read_matrix_market / mp.read_csr) against the
reference's own reader: the golden fixtures in tests/golden/mtx_*.npz hold
what dr::read_csr<double, long> (include/dr/detail/matrix_io.hpp, compiled
from the reference source) returned for tests/golden/mtx/*.mtx -- its CSR
arrays, or its exception message.  The oracle's restatement is held to the
same fixtures, and the library is also compared with the oracle on inputs
the reference cannot take (CRLF, blank lines) and on multi-megabyte files
that the library parses in several threads."""
import os

import numpy as np
import pytest

import oracle
from drb import _capi as capi
from drb import mp

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = sorted(f[4:-4] for f in os.listdir(GOLD) if f.startswith("mtx_") and f.endswith(".npz"))
STATUS = {"could not be parsed": capi.DRB_ERR_IO,
          "unsupported matrix type": capi.DRB_ERR_UNSUPPORTED,
          "out of bounds": capi.DRB_ERR_BAD_CSR,
          "more nonzeros than reported": capi.DRB_ERR_BAD_CSR}


def mtx(name):
    return os.path.join(GOLD, "mtx", name + ".mtx")


def lib_read(path):
    v = mp.read_csr(path)
    m, n = v.shape()
    return m, n, v.rowptr_data(), v.colind_data(), v.values_data()


def test_fixture_set_is_complete():
    assert len(CASES) >= 14
    assert any(c.startswith("err_") for c in CASES)


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("reader", ["library", "oracle"])
def test_reader_matches_reference(case, reader):
    g = dict(np.load(os.path.join(GOLD, f"mtx_{case}.npz")))
    read = lib_read if reader == "library" else oracle.read_matrix_market
    if "error" in g:
        msg = str(g["error"])
        exc = capi.DrbError if reader == "library" else oracle.MatrixMarketError
        with pytest.raises(exc) as e:
            read(mtx(case))
        assert msg in str(e.value), (msg, str(e.value))
        if reader == "library":
            want = next(s for k, s in STATUS.items() if k in msg)
            assert e.value.status == want
        return
    m, n, rp, ci, v = read(mtx(case))
    assert (m, n) == (int(g["m"]), int(g["n"]))
    assert np.array_equal(rp, g["rowptr"])
    assert np.array_equal(ci, g["colind"])
    assert np.array_equal(v, g["values"])


def test_missing_file():
    with pytest.raises(capi.DrbError) as e:
        mp.read_csr("/nonexistent/file.mtx")
    assert e.value.status == capi.DRB_ERR_IO
    assert "cannot open" in str(e.value)


def test_zero_indexed_and_dtypes(tmp_path):
    p = tmp_path / "z.mtx"
    p.write_text("%%MatrixMarket matrix coordinate real general\n3 3 3\n0 0 1\n2 1 2\n1 2 3\n")
    v = mp.read_csr(p, one_indexed=False, dtype=np.float32, index_dtype=np.int32)
    assert v.values_data().dtype == np.float32 and v.rowptr_data().dtype == np.int32
    m, n, rp, ci, vv = oracle.read_matrix_market(p, one_indexed=False)
    assert np.array_equal(v.rowptr_data(), rp) and np.array_equal(v.colind_data(), ci)
    assert np.array_equal(v.values_data(), vv.astype(np.float32))


def test_crlf_and_blank_lines(tmp_path):
    """Inputs the reference has no case for: both readers skip blank lines
    and accept CRLF line ends."""
    p = tmp_path / "crlf.mtx"
    p.write_bytes(b"%%MatrixMarket matrix coordinate real symmetric\r\n% c\r\n"
                  b"3 3 3\r\n2 1 -1.5\r\n\r\n1 1 2\r\n3 3 4\r\n\r\n\r\n")
    a = lib_read(p)
    b = oracle.read_matrix_market(p)
    assert a[:2] == b[:2] == (3, 3)
    for x, y in zip(a[2:], b[2:]):
        assert np.array_equal(x, y)
    assert a[2].tolist() == [0, 2, 3, 4]


def write_random_mtx(path, m, n, count, symmetric, pattern, seed, extra=""):
    rng = np.random.default_rng(seed)
    i = rng.integers(1, m + 1, size=count)
    j = rng.integers(1, n + 1, size=count)
    if symmetric:
        i, j = np.maximum(i, j), np.minimum(i, j)
    v = rng.standard_normal(count)
    field = "pattern" if pattern else "real"
    sym = "symmetric" if symmetric else "general"
    with open(path, "w") as f:
        f.write(f"%%MatrixMarket matrix coordinate {field} {sym}\n% random\n{m} {n} {count}\n")
        if pattern:
            f.write("\n".join(f"{a} {b}" for a, b in zip(i, j)))
        else:
            f.write("\n".join(f"{a} {b} {c:.17g}" for a, b, c in zip(i, j, v)))
        f.write("\n" + extra)


@pytest.mark.parametrize("symmetric,pattern", [(False, False), (True, False), (False, True)])
def test_large_file_threads_match_oracle(tmp_path, symmetric, pattern):
    """About 4-8 MB: the library splits the entry lines over threads; with
    random duplicates the stable column sort keeps file order, as the
    oracle does."""
    p = tmp_path / "big.mtx"
    m = n = 20000
    write_random_mtx(p, m, n, 300_000, symmetric, pattern, seed=5)
    a = lib_read(p)
    b = oracle.read_matrix_market(p)
    assert a[:2] == b[:2]
    for x, y in zip(a[2:], b[2:]):
        assert np.array_equal(x, y)
    assert int(a[2][-1]) >= 300_000


def test_first_error_in_file_order(tmp_path):
    """Errors late in a multi-chunk file: the one a sequential read meets
    first is reported (bounds before count at the same entry)."""
    p = tmp_path / "late_oob.mtx"
    write_random_mtx(p, 1000, 1000, 200_000, False, False, seed=6, extra="1001 1 1.0\n")
    # the size line declares 200000 entries: the 200001st is out of bounds
    with pytest.raises(capi.DrbError) as e:
        mp.read_csr(p)
    with pytest.raises(oracle.MatrixMarketError) as o:
        oracle.read_matrix_market(p)
    assert "out of bounds" in str(e.value) and "out of bounds" in str(o.value)
    q = tmp_path / "late_extra.mtx"
    write_random_mtx(q, 1000, 1000, 200_000, False, False, seed=7,
                     extra="5 5 1.0\n1001 1 1.0\n")
    with pytest.raises(capi.DrbError) as e:
        mp.read_csr(q)
    with pytest.raises(oracle.MatrixMarketError) as o:
        oracle.read_matrix_market(q)
    assert "more nonzeros" in str(e.value) and "more nonzeros" in str(o.value)


@pytest.mark.gpu
def test_read_upload_gemv(tmp_path):
    """The full ingest path: file -> read_csr -> device handle -> gemv."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    p = tmp_path / "sym.mtx"
    write_random_mtx(p, 5000, 5000, 40_000, True, False, seed=8)
    view = mp.read_csr(p)
    m, n = view.shape()
    a = mp.distributed_sparse_matrix(view, 0)
    x = np.random.default_rng(9).standard_normal(n)
    b = mp.broadcasted_vector()
    b.broadcast_data(n, 0, x)
    res = np.zeros(m)
    mp.gemv(0, res, a, b)
    ref = oracle.gemv_row(view.rowptr_data(), view.colind_data(), view.values_data(), x,
                          m, n, 1, oracle.ACC_LD)
    d = oracle.absdot(view.rowptr_data(), view.colind_data(), np.abs(view.values_data()),
                      np.abs(x), m, n)
    assert float(np.max(np.abs(res - ref) / np.maximum(d, 1e-300))) <= 1e-12
    a.destroy()
