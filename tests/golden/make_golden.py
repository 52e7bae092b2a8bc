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
    # --- the other index types of the generator (same seed): int32 and long
    for it in ("i32", "i64"):
        mm, nn, rp, ci, v = run_ref(["random", "f64", it, "200", "150", repr(F32_0P1), "7"],
                                    "f64", it)
        save(f"random_f64_{it}_200x150_seed7", m=mm, n=nn, rowptr=rp, colind=ci,
             values=v, source=np.array(f"generate_random_csr<double,{it}>({{200,150}}, 0.1f, 7)"))


if __name__ == "__main__":
    main()
