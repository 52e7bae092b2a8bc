"""Generate the golden fixtures in tests/golden/ from the REFERENCE's own code.

The matrices come from oracle/_ref/ref_gen, which is the reference's
include/dr/detail/generate_csr.hpp compiled from the reference tree by
oracle/Makefile (`make -C oracle ref`).  The expected outputs follow the
reference tests' own rule for the expected result:

  * test/gtest/mp/gemv.cpp:6-25   testMatrixGemv: x = 1, c_ref[i] += v over
    the matrix entries in order (float);
  * test/gtest/mp/gemv.cpp:27-52  testMatrixGemm: width 20, base_b[i] = i
    (column-major), c_ref[i + j*m] += v * base_b[k + j*n] (float);
  * test/gtest/sp/gemv.cpp        EmptyGemv (nnz = 0), ZeroVector (dense 100x100
    with values i+j times x = 0), VerySparseMatrix (density 0.001);
  * examples/mp/sparse_matrix.cpp:84-102  double/long matrix, x[i] = i,
    ref[m] += n*val compared exactly (a band matrix stands in for the Matrix
    Market file, which the reference does not ship).

The Matrix Market fixtures (tests/golden/mtx/*.mtx, written below) are read
by oracle/_ref/ref_mmread, the reference's own dr::read_csr<double, long>
(include/dr/detail/matrix_io.hpp) compiled from its source; its CSR arrays
or its exception message are stored in mtx_<case>.npz.

Run in the build container (the reference tree is needed only here):
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF_GEN = os.path.join(ROOT, "oracle", "_ref", "ref_gen")
REF_MMREAD = os.path.join(ROOT, "oracle", "_ref", "ref_mmread")
MTX_DIR = os.path.join(HERE, "mtx")

# Matrix Market inputs: valid files in every field/symmetry the reader takes,
# and the malformed ones it must reject.  (No blank lines: the reference's
# reader has no case for them.)
MTX_CASES = {
    "general_real": """%%MatrixMarket matrix coordinate real general
% entries out of order, an empty row, exponents and a leading '+'
%
5 4 7
3 2 1.5e-3
1 4 -2.0
1 1 3.25
5 4 7
3 1 -0.5
1 2 1e2
5 1 +4
""",
    "symmetric_real": """%%MatrixMarket matrix coordinate real symmetric
4 4 6
1 1 2.0
2 1 -1.0
2 2 2.0
4 1 0.25
3 3 2.0
4 3 -1.0
""",
    "pattern_general": """%%MatrixMarket matrix coordinate pattern general
3 5 5
2 5
1 1
3 2
2 1
1 5
""",
    "integer_symmetric": """%%MatrixMarket matrix coordinate integer symmetric
% integer field
3 3 4
1 1 7
3 1 -2
2 2 5
3 2 9
""",
    "pattern_symmetric": """%%MatrixMarket matrix coordinate pattern symmetric
4 4 4
1 1
3 1
4 2
4 4
""",
    "zero_entries": """%%MatrixMarket matrix coordinate real general
3 3 0
""",
    "duplicates_equal": """%%MatrixMarket matrix coordinate real general
2 2 4
2 2 1.5
1 2 3.0
2 2 1.5
1 1 -1.0
""",
    "fewer_than_declared": """%%MatrixMarket matrix coordinate real general
3 3 5
1 1 1.0
3 3 3.0
2 2 2.0
""",
    "tall": """%%MatrixMarket matrix coordinate real general
6 2 5
6 2 1.0
1 1 2.0
4 1 3.0
4 2 4.0
2 2 5.0
""",
    "err_array": """%%MatrixMarket matrix array real general
2 2
1.0
2.0
3.0
4.0
""",
    "err_skew": """%%MatrixMarket matrix coordinate real skew-symmetric
2 2 1
2 1 1.0
""",
    "err_out_of_bounds": """%%MatrixMarket matrix coordinate real general
3 3 2
1 1 1.0
4 1 1.0
""",
    "err_too_many": """%%MatrixMarket matrix coordinate real general
3 3 2
1 1 1.0
2 2 1.0
3 3 1.0
""",
    "err_not_mm": """hello
1 1 1
""",
}


def run_mmread(path):
    out = os.path.join(HERE, "_tmp_mm.bin")
    r = subprocess.run([REF_MMREAD, path, out], capture_output=True, text=True)
    if r.returncode == 3:
        return None, r.stderr.strip()
    if r.returncode != 0:
        raise RuntimeError(f"ref_mmread failed on {path}: {r.returncode} {r.stderr}")
    raw = open(out, "rb").read()
    os.remove(out)
    m, n, nnz = (int(v) for v in np.frombuffer(raw[:24], np.int64))
    o = 24
    rp = np.frombuffer(raw[o:o + 8 * (m + 1)], np.int64).copy()
    o += 8 * (m + 1)
    ci = np.frombuffer(raw[o:o + 8 * nnz], np.int64).copy()
    o += 8 * nnz
    v = np.frombuffer(raw[o:o + 8 * nnz], np.float64).copy()
    return (m, n, rp, ci, v), None
F32_0P1 = float(np.float32(0.1))     # the tests pass 0.1f
F32_0P001 = float(np.float32(0.001))  # VerySparseMatrix passes 0.001f

_VT = {"f32": np.float32, "f64": np.float64}
_IT = {"u64": np.uint64, "i64": np.int64, "i32": np.int32}


def run_ref(args, vt, it):
    out = os.path.join(HERE, "_tmp.bin")
    subprocess.run([REF_GEN] + args + [out], check=True)
    raw = open(out, "rb").read()
    os.remove(out)
    m, n, nnz = (int(v) for v in np.frombuffer(raw[:24], np.int64))
    ib = np.dtype(_IT[it]).itemsize
    vb = np.dtype(_VT[vt]).itemsize
    o = 24
    rp = np.frombuffer(raw[o:o + ib * (m + 1)], _IT[it]).copy()
    o += ib * (m + 1)
    ci = np.frombuffer(raw[o:o + ib * nnz], _IT[it]).copy()
    o += ib * nnz
    v = np.frombuffer(raw[o:o + vb * nnz], _VT[vt]).copy()
    return m, n, rp, ci, v


def expected_gemm(m, n, rp, ci, v, x, width, T):
    """c_ref[i + j*m] += v * x[k + j*n] over entries in order, in type T."""
    y = [T(0)] * (m * width)
    for i in range(m):
        for p in range(int(rp[i]), int(rp[i + 1])):
            k = int(ci[p])
            for j in range(width):
                y[i + j * m] = T(y[i + j * m] + T(v[p] * x[k + j * n]))
    return np.array(y, dtype=T)


def expected_rowsum(m, rp, v, T):
    y = [T(0)] * m
    for i in range(m):
        for p in range(int(rp[i]), int(rp[i + 1])):
            y[i] = T(y[i] + v[p])
    return np.array(y, dtype=T)


def save(name, **arrays):
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
    print("wrote", name)


def main():
    if not os.path.exists(REF_GEN):
        sys.exit(f"{REF_GEN} missing: run `make -C oracle ref` first")
    # --- test/gtest/mp/gemv.cpp: Gemv{Row,Eq}{,NotSquare,NotSquareDifferentAxis}
    for (m, n) in [(100, 100), (1000, 10), (10, 1000)]:
        mm, nn, rp, ci, v = run_ref(["random", "f32", "u64", str(m), str(n),
                                     repr(F32_0P1), "0"], "f32", "u64")
        x1 = np.ones(n, np.float32)
        xw = np.arange(n * 20, dtype=np.float32)  # base_b[i] = i, width 20
        save(f"mp_gemv_{m}x{n}", m=mm, n=nn, rowptr=rp, colind=ci, values=v,
             x=x1, expected=expected_rowsum(mm, rp, v, np.float32),
             x_w20=xw, expected_w20=expected_gemm(mm, nn, rp, ci, v, xw, 20, np.float32),
             source=np.array("generate_random_csr<float,unsigned long>(shape, 0.1f, 0)"))
    # --- test/gtest/sp/gemv.cpp: VerySparseMatrix (density 0.001f)
    mm, nn, rp, ci, v = run_ref(["random", "f32", "u64", "100", "100",
                                 repr(F32_0P001), "0"], "f32", "u64")
    save("sp_very_sparse_100x100", m=mm, n=nn, rowptr=rp, colind=ci, values=v,
         x=np.ones(100, np.float32), expected=expected_rowsum(mm, rp, v, np.float32),
         source=np.array("generate_random_csr<float,unsigned long>({100,100}, 0.001f, 0)"))
    # --- test/gtest/sp/gemv.cpp: EmptyGemv (coo of size 0 -> all-zero rowptr)
    save("sp_empty_100x100", m=100, n=100, rowptr=np.zeros(101, np.int32),
         colind=np.zeros(0, np.int32), values=np.zeros(0, np.float32),
         x=np.ones(100, np.float32), expected=np.zeros(100, np.float32),
         source=np.array("convert_to_csr(empty coo_matrix<float,int>, {100,100})"))
    # --- test/gtest/sp/gemv.cpp: ZeroVector (dense values i+j, x = 0)
    m = n = 100
    rp = (np.arange(m + 1) * n).astype(np.int32)
    ci = np.tile(np.arange(n, dtype=np.int32), m)
    v = (np.arange(m)[:, None] + np.arange(n)[None, :]).astype(np.float32).ravel()
    save("sp_zero_vector_100x100", m=m, n=n, rowptr=rp, colind=ci, values=v,
         x=np.zeros(n, np.float32), expected=np.zeros(m, np.float32),
         source=np.array("convert_to_csr(dense {i+j}, {100,100}) * zeros"))
    # --- examples/mp/sparse_matrix.cpp check (double/long, x[i] = i, exact)
    for (size, up, down) in [(1000, 20, 20), (257, 3, 3)]:
        mm, nn, rp, ci, v = run_ref(["band", "f64", "i64", str(size), str(up), str(down)],
                                    "f64", "i64")
        x = np.arange(nn, dtype=np.float64)
        save(f"band_f64_{size}_{up}_{down}", m=mm, n=nn, rowptr=rp, colind=ci, values=v,
             x=x, expected=expected_gemm(mm, nn, rp, ci, v, x, 1, np.float64),
             source=np.array(f"generate_band_csr<double,long>({size},{up},{down})"))
    # --- the default band (float, unsigned long, 3/3) used by dr::sp tests
    mm, nn, rp, ci, v = run_ref(["band", "f32", "u64", "100", "3", "3"], "f32", "u64")
    save("band_f32_100_3_3", m=mm, n=nn, rowptr=rp, colind=ci, values=v,
         x=np.ones(nn, np.float32), expected=expected_rowsum(mm, rp, v, np.float32),
         source=np.array("generate_band_csr<float,unsigned long>(100)"))
    # --- Matrix Market ingest: the reference's read_csr<double, long>
    if not os.path.exists(REF_MMREAD):
        sys.exit(f"{REF_MMREAD} missing: run `make -C oracle ref` first")
    os.makedirs(MTX_DIR, exist_ok=True)
    for name, text in MTX_CASES.items():
        path = os.path.join(MTX_DIR, name + ".mtx")
        with open(path, "w") as f:
            f.write(text)
        res, err = run_mmread(path)
        if res is None:
            # the message without the path prefix
            save("mtx_" + name, error=np.array(err.replace(path, "").strip()),
                 source=np.array("dr::read_csr<double,long> exception"))
        else:
            m, n, rp, ci, v = res
            save("mtx_" + name, m=m, n=n, rowptr=rp, colind=ci, values=v,
                 source=np.array("dr::read_csr<double,long>"))
    # --- the other index types of the generator (same seed): int32 and long
    for it in ("i32", "i64"):
        mm, nn, rp, ci, v = run_ref(["random", "f64", it, "200", "150", repr(F32_0P1), "7"],
                                    "f64", it)
        save(f"random_f64_{it}_200x150_seed7", m=mm, n=nn, rowptr=rp, colind=ci,
             values=v, source=np.array(f"generate_random_csr<double,{it}>({{200,150}}, 0.1f, 7)"))


if __name__ == "__main__":
    main()
