"""The C++ host mirror (include/drb/mp.hpp via include/drb/dr_mp.hpp).

CPU: its generate_random_csr reproduces the reference generator's matrices
(the golden fixtures made from the reference's generate_csr.hpp), and its
read_csr returns what the reference's own Matrix Market reader returned.
GPU: the reference's gemv test cases, written with the dr::mp names, pass."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CPP = os.path.join(ROOT, "tests", "cpp")
EXE = os.path.join(CPP, "_build", "test_mp_gemv")


@pytest.fixture(scope="module")
def exe():
    subprocess.run(["make", "-C", CPP], check=True, capture_output=True)
    return EXE


@pytest.mark.parametrize("m,n", [(100, 100), (1000, 10), (10, 1000)])
def test_cpp_generator_matches_reference(exe, tmp_path, m, n):
    out = tmp_path / "g.bin"
    subprocess.run([exe, "dump-random", str(m), str(n), "0", str(out)], check=True)
    raw = out.read_bytes()
    mm, nn, nnz = np.frombuffer(raw[:24], np.int64)
    o = 24
    rp = np.frombuffer(raw[o:o + 8 * (m + 1)], np.uint64)
    o += 8 * (m + 1)
    ci = np.frombuffer(raw[o:o + 8 * nnz], np.uint64)
    o += 8 * nnz
    v = np.frombuffer(raw[o:o + 4 * nnz], np.float32)
    f = np.load(os.path.join(ROOT, "tests", "golden", f"mp_gemv_{m}x{n}.npz"))
    assert np.array_equal(rp, f["rowptr"]) and np.array_equal(ci, f["colind"])
    assert np.array_equal(v, f["values"])


MTX = sorted(f[4:-4] for f in os.listdir(os.path.join(ROOT, "tests", "golden"))
             if f.startswith("mtx_") and f.endswith(".npz"))


@pytest.mark.parametrize("case", MTX)
def test_cpp_read_csr_matches_reference(exe, tmp_path, case):
    """dr::read_csr<double, long> through the mirror against what the
    reference's own reader returned for the same file."""
    gold = dict(np.load(os.path.join(ROOT, "tests", "golden", f"mtx_{case}.npz")))
    out = tmp_path / "m.bin"
    r = subprocess.run([exe, "dump-mtx", os.path.join(ROOT, "tests", "golden", "mtx",
                                                      case + ".mtx"), str(out)],
                       capture_output=True, text=True)
    if "error" in gold:
        assert r.returncode == 3 and str(gold["error"]) in r.stderr
        return
    assert r.returncode == 0, r.stderr
    raw = out.read_bytes()
    m, n, nnz = (int(v) for v in np.frombuffer(raw[:24], np.int64))
    o = 24
    rp = np.frombuffer(raw[o:o + 8 * (m + 1)], np.int64)
    o += 8 * (m + 1)
    ci = np.frombuffer(raw[o:o + 8 * nnz], np.int64)
    o += 8 * nnz
    v = np.frombuffer(raw[o:o + 8 * nnz], np.float64)
    assert (m, n) == (int(gold["m"]), int(gold["n"]))
    assert np.array_equal(rp, gold["rowptr"]) and np.array_equal(ci, gold["colind"])
    assert np.array_equal(v, gold["values"])


@pytest.mark.gpu
def test_cpp_reference_gemv_cases(exe):
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "OK: 0 failure(s)" in r.stdout
    assert r.stdout.count("PASS") >= 50
    for case in ("ReduceMP.RootRange", "ReduceMP.RootIterators", "Reduce.Range",
                 "Reduce.IteratorsDefaultInit", "ReduceMP.TransformReduce",
                 "FillIterators", "VectorSegments", "ConjugateGradient1D"):
        assert f"PASS {case}\n" in r.stdout, case
