"""The streaming-gather probe (lib/libdrb_probe.so, drb_probe/drb_probe.h):
measurement only, loaded by the bench and its test, not part of drb."""
from __future__ import annotations

import ctypes as C
import os

from drb import _capi as capi

LIB_PATH = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "lib",
                        "libdrb_probe.so")
if not os.path.exists(LIB_PATH):
    raise ImportError(f"{LIB_PATH} not built; run make in distributed-ranges_b200")
lib = C.CDLL(LIB_PATH)
lib.drb_csr_gather_probe.restype = C.c_int
lib.drb_csr_gather_probe.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
lib.drb_csr_gather_rows_probe.restype = C.c_int
lib.drb_csr_gather_rows_probe.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, C.c_int,
                                          C.c_void_p]


def gather_probe(a, x, with_values: bool = True, stream=None) -> None:
    """Stream A's column indices (and values) and gather x at each: the reads
    of y = A x without rows or y.  Computes nothing visible."""
    s = stream if stream is not None else _current_stream()
    capi.check(lib.drb_csr_gather_probe(a.handle, C.c_void_p(x.data_ptr()),
                                        int(bool(with_values)), s))


def gather_rows_probe(a, X, k: int, ldx: int | None = None, with_values: bool = True,
                      stream=None) -> None:
    """Stream A's column indices (and values) and gather the k-element row of
    the row-major X (ldx elements per row, default k) at each: the reads of
    Y = A X without rows or Y.  Computes nothing visible."""
    s = stream if stream is not None else _current_stream()
    capi.check(lib.drb_csr_gather_rows_probe(a.handle, C.c_void_p(X.data_ptr()),
                                             int(ldx if ldx is not None else k), int(k),
                                             int(bool(with_values)), s))


def _current_stream():
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)
