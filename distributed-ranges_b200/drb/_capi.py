"""ctypes binding of the C ABI in include/drb.h and include/drb_gen.h.

The shared library is built in-tree (``distributed-ranges_b200/lib/libdrb.so``
by ``make -C distributed-ranges_b200``).  There is no fallback: if the library
is missing, importing this module raises ImportError, and every compute call
goes to the CUDA kernels in that library.
"""
from __future__ import annotations

import ctypes as C
import os

_PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(_PKG_ROOT, "lib", "libdrb.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"drb: CUDA library not built ({LIB_PATH} missing); run "
        f"`make -C {_PKG_ROOT}` or __graft_entry__.build()")

lib = C.CDLL(LIB_PATH)

# ---- enums (drb.h) -----------------------------------------------------------
DRB_OK = 0
DRB_ERR_INVALID_ARG = 1
DRB_ERR_BAD_CSR = 2
DRB_ERR_OOM = 3
DRB_ERR_CUDA = 4
DRB_ERR_TIMEOUT = 5
DRB_ERR_UNSUPPORTED = 6
DRB_ERR_NO_DEVICE = 7
DRB_ERR_IO = 8

DRB_F32, DRB_F64, DRB_BF16, DRB_INT32, DRB_INT64 = 0, 1, 2, 3, 4
DRB_REDUCE_SUM, DRB_REDUCE_MIN, DRB_REDUCE_MAX = 0, 1, 2
DRB_I32, DRB_I64 = 0, 1
DRB_COL_MAJOR, DRB_ROW_MAJOR = 0, 1
DRB_PART_ROW, DRB_PART_EQ = 0, 1

DRB_FLAG_DEVICE_INPUT = 0x1
DRB_FLAG_KEEP_INDEX64 = 0x2
DRB_FLAG_SKIP_VALIDATE = 0x4
DRB_FLAG_ADJOINT = 0x8
DRB_FLAG_COMPENSATED = 0x10
DRB_FLAG_AUTOTUNE = 0x20
DRB_FLAG_BF16_X_F32 = 0x40

STATUS_NAMES = {
    0: "DRB_OK", 1: "DRB_ERR_INVALID_ARG", 2: "DRB_ERR_BAD_CSR",
    3: "DRB_ERR_OOM", 4: "DRB_ERR_CUDA", 5: "DRB_ERR_TIMEOUT",
    6: "DRB_ERR_UNSUPPORTED", 7: "DRB_ERR_NO_DEVICE", 8: "DRB_ERR_IO",
}


class CsrHost(C.Structure):
    """drb_csr_host: host CSR arrays allocated by the library."""
    _fields_ = [("m", C.c_int64), ("n", C.c_int64), ("nnz", C.c_int64),
                ("rowptr", C.POINTER(C.c_int64)), ("colind", C.POINTER(C.c_int64)),
                ("values", C.POINTER(C.c_double))]


class CgInfo(C.Structure):
    """drb_cg_info: how a drb_csr_cg solve ended."""
    _fields_ = [("iterations", C.c_int64), ("residual_norm", C.c_double),
                ("b_norm", C.c_double), ("converged", C.c_int), ("breakdown", C.c_int)]


class DrbError(RuntimeError):
    """A non-zero drb_status, with drb_last_error()'s message."""

    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")


_vp = C.c_void_p
_i64 = C.c_int64
_i32 = C.c_int
_u32 = C.c_uint32
_st = C.c_int

# exported symbols of include/drb.h: (name, restype, argtypes)
DRB_SYMBOLS = [
    ("drb_csr_create", _st, [C.POINTER(_vp), _i64, _i64, _i64, _vp, _vp, _vp,
                             _i32, _i32, _i32, _i32, _i32, _u32, _vp]),
    ("drb_csr_destroy", _st, [_vp]),
    ("drb_csr_shape", _st, [_vp, C.POINTER(_i64), C.POINTER(_i64), C.POINTER(_i64)]),
    ("drb_csr_storage", _st, [_vp, C.POINTER(_i32), C.POINTER(_i32), C.POINTER(_i32)]),
    ("drb_csr_num_segments", _st, [_vp, C.POINTER(_i32)]),
    ("drb_csr_segment", _st, [_vp, _i32, C.POINTER(_i64), C.POINTER(_i64),
                              C.POINTER(_i64), C.POINTER(_i64)]),
    ("drb_csr_get_entries", _st, [_vp, _i64, _i64, _vp, _vp, _vp]),
    ("drb_csr_gemv", _st, [_vp, _vp, _vp, _i64, _i32, _vp]),
    ("drb_csr_gemv_host", _st, [_vp, _vp, _vp, _i64, _i32, _vp]),
    ("drb_csr_check", _st, [_vp, _vp]),
    ("drb_csr_variant", _st, [_vp, C.POINTER(_i32)]),
    ("drb_csr_autotune", _st, [_vp, C.POINTER(_i32), _vp]),
    ("drb_csr_column_blocks", _st, [_vp, C.POINTER(_i32), C.POINTER(_i64)]),
    ("drb_csr_residual_norm2", _st, [_vp, _vp, _vp, _vp, _vp, _vp]),
    ("drb_csr_gemv_backward", _st, [_vp, _vp, _vp, _vp, _vp, _vp]),
    ("drb_csr_update_values", _st, [_vp, _vp, _vp]),
    ("drb_batch_create", _st, [C.POINTER(_vp), _i32, C.POINTER(_vp), _i64, _i32,
                               _u32, _vp]),
    ("drb_batch_bind", _st, [_vp, C.POINTER(_vp), C.POINTER(_vp), _vp]),
    ("drb_batch_gemv", _st, [_vp, _vp]),
    ("drb_batch_variant", _st, [_vp, C.POINTER(_i32)]),
    ("drb_batch_set_variant", _st, [_vp, _i32]),
    ("drb_batch_autotune", _st, [_vp, C.POINTER(_i32), _vp]),
    ("drb_batch_destroy", _st, [_vp]),
    ("drb_batched_gemv", _st, [_i32, C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp),
                               _i64, _i32, _u32, _vp]),
    ("drb_dense_gemv", _st, [_i64, _i64, _vp, _i64, _vp, _vp, _i64, _i32, _i32, _vp]),
    ("drb_dense_batch_create", _st, [C.POINTER(_vp), _i32, C.POINTER(_i64), C.POINTER(_i64),
                                     C.POINTER(_vp), C.POINTER(_i64), C.POINTER(_vp),
                                     C.POINTER(_vp), _i64, _i32, _i32, _vp]),
    ("drb_dense_batch_gemv", _st, [_vp, _vp]),
    ("drb_dense_batch_set_variant", _st, [_vp, _i32]),
    ("drb_dense_batch_check", _st, [_vp, _vp]),
    ("drb_dense_batch_set_wait", _st, [_vp, C.c_uint64, _i32]),
    ("drb_dense_batch_destroy", _st, [_vp]),
    ("drb_dot", _st, [_i64, _vp, _vp, _i32, _vp, _vp]),
    ("drb_dot_noalloc", _st, [_i64, _vp, _vp, _i32, _vp, _vp]),
    ("drb_reduce", _st, [_i64, _vp, _i32, _i32, _vp, _vp, _vp]),
    ("drb_iota", _st, [_i64, _vp, _i32, _i64, _vp]),
    ("drb_fill", _st, [_i64, _vp, _i32, _vp, _vp]),
    ("drb_csr_cg", _st, [_vp, _vp, _vp, _i64, C.c_double, C.POINTER(CgInfo), _vp]),
    ("drb_read_matrix_market", _st, [C.c_char_p, _i32, C.POINTER(CsrHost)]),
    ("drb_csr_host_free", None, [C.POINTER(CsrHost)]),
    ("drb_malloc", _st, [C.POINTER(_vp), C.c_size_t]),
    ("drb_free", _st, [_vp]),
    ("drb_memcpy", _st, [_vp, _vp, C.c_size_t, _i32, _vp]),
    ("drb_memset", _st, [_vp, _i32, C.c_size_t, _vp]),
    ("drb_stream_synchronize", _st, [_vp]),
    ("drb_last_error", C.c_char_p, []),
    ("drb_version", C.c_char_p, []),
    ("drb_launch_count", C.c_uint64, []),
]

# exported symbols of include/drb_gen.h
GEN_SYMBOLS = [
    ("drb_gen_zipf_alpha_for_mean", C.c_double, [_i64, _i64, C.c_double]),
    ("drb_gen_zipf_mean", C.c_double, [_i64, _i64, C.c_double]),
    ("drb_gen_rowptr_zipf", _i64, [_i64, _i64, C.c_double, _i64, _i64, C.c_uint64, _vp, _i32]),
    ("drb_gen_rowptr_uniform", _i64, [_i64, _i64, _i64, _i64, C.c_uint64, _vp, _i32]),
    ("drb_gen_rowptr_fixed", _i64, [_i64, _i64, _i64, _vp]),
    ("drb_gen_fill_uniform", _i32, [_i64, _i64, _vp, C.c_uint64, _i32, _vp, _i32, _vp, _i32, _i32]),
    ("drb_gen_laplacian2d", _i64, [_i64, _vp, _i32, _vp, _i32, _vp]),
    ("drb_gen_values", _i32, [_i64, C.c_uint64, _i32, _vp, _i32, _i32]),
]

for _name, _res, _args in DRB_SYMBOLS + GEN_SYMBOLS:
    _f = getattr(lib, _name)
    _f.restype = _res
    _f.argtypes = _args


def last_error() -> str:
    return (lib.drb_last_error() or b"").decode()


def check(status: int) -> None:
    if status != DRB_OK:
        raise DrbError(status, last_error())


def launch_count() -> int:
    return int(lib.drb_launch_count())
