"""Python mirror of the reference's ``dr::mp`` gemv interface over the C ABI.

Names, argument meaning and error behaviour follow the reference
(include/dr/mp/algorithms/matrix/gemv.hpp,
include/dr/mp/containers/distributed_sparse_matrix.hpp,
include/dr/mp/containers/broadcasted_vector.hpp,
include/dr/mp/containers/broadcasted_slim_matrix.hpp,
include/dr/views/csr_matrix_view.hpp) so a test written against the
reference reads the same here.  One process owns one GPU: the "ranks" of the
reference become logical segments of one device-resident matrix, rank 0 is the
only root, and ``gemv`` runs the sm_100a kernels of libdrb.so.  Device memory
and streams are torch's (torch.cuda tensors, the current stream).
"""
from __future__ import annotations

import ctypes as C
from typing import Iterator, Sequence

import numpy as np
import torch

from . import _capi as capi
from ._capi import check

__all__ = [
    "csr_matrix_view", "distribution", "csr_row_distribution",
    "csr_eq_distribution", "distributed_sparse_matrix", "broadcasted_vector",
    "broadcasted_slim_matrix", "gemv", "gemv_backward", "dense_gemv", "dot",
    "residual_norm2", "default_comm", "init", "finalize", "batch", "batched_gemv",
    "dense_batch", "read_csr", "distributed_vector", "iota", "fill", "reduce",
    "conjugate_gradient",
]

_TORCH_DT = {torch.float32: capi.DRB_F32, torch.float64: capi.DRB_F64,
             torch.bfloat16: capi.DRB_BF16}
_NP_DT = {np.dtype(np.float32): capi.DRB_F32, np.dtype(np.float64): capi.DRB_F64}
_NP_IT = {np.dtype(np.int32): capi.DRB_I32, np.dtype(np.int64): capi.DRB_I64,
          np.dtype(np.uint64): capi.DRB_I64}
_STORAGE_TORCH = {capi.DRB_F32: torch.float32, capi.DRB_F64: torch.float64,
                  capi.DRB_BF16: torch.bfloat16}


def _stream(stream=None) -> C.c_void_p:
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def _ptr(t) -> C.c_void_p:
    if t is None:
        return C.c_void_p(0)
    if isinstance(t, torch.Tensor):
        return C.c_void_p(t.data_ptr())
    return C.c_void_p(t.ctypes.data)


class _Comm:
    """The single-process communicator: rank 0 of 1 (the reference's
    default_comm(), include/dr/mp/global.hpp)."""

    def rank(self) -> int:
        return 0

    def size(self) -> int:
        return 1


_COMM = _Comm()
_DIST_COMM = None


def default_comm():
    """Rank 0 of 1, or -- when torch.distributed is initialised with more
    than one rank (one process per GPU) -- the world group as a
    communicator (drb.dist.DistComm)."""
    global _DIST_COMM
    if torch.distributed.is_available() and torch.distributed.is_initialized() and \
            torch.distributed.get_world_size() > 1:
        if _DIST_COMM is None:
            from .dist import DistComm
            _DIST_COMM = DistComm()
        return _DIST_COMM
    return _COMM


class _DeviceBlock:
    """A rank's segment as a single-process device handle on its GPU (the
    local product of a multi-process matrix)."""

    def __init__(self, rowptr, colind, values, shape, **kw):
        self.a = distributed_sparse_matrix(csr_matrix_view(values, rowptr, colind, shape), 0,
                                           distr=csr_row_distribution, comm=_COMM, **kw)
        self.rows = shape[0]

    def gemv(self, x: torch.Tensor, k: int) -> torch.Tensor:
        y = torch.empty(self.rows * k, dtype=self.a.compute_dtype, device="cuda")
        self.a.gemv_device(x.to(device="cuda", dtype=self.a.x_dtype), y, k, capi.DRB_COL_MAJOR)
        return y


def init(device: int | None = None) -> None:
    """mp::init(): select the CUDA device (global.hpp:130-135, 191-197)."""
    if device is not None:
        torch.cuda.set_device(device)


def finalize() -> None:
    torch.cuda.synchronize()


class csr_matrix_view:
    """Non-owning host CSR triple (csr_matrix_view.hpp:125-220):
    values[nnz], rowptr[m+1], colind[nnz], shape (m, n)."""

    def __init__(self, values, rowptr, colind, shape, nnz=None, rank=0):
        self._values = np.ascontiguousarray(values)
        self._rowptr = np.ascontiguousarray(rowptr)
        self._colind = np.ascontiguousarray(colind)
        self._shape = (int(shape[0]), int(shape[1]))
        self._nnz = int(self._rowptr[self._shape[0]]) if nnz is None else int(nnz)
        self._rank = rank

    def shape(self):
        return self._shape

    def size(self) -> int:
        return self._nnz

    def rank(self) -> int:
        return self._rank

    def values_data(self):
        return self._values

    def rowptr_data(self):
        return self._rowptr

    def colind_data(self):
        return self._colind

    def __iter__(self):
        rp, ci, v = self._rowptr, self._colind, self._values
        for i in range(self._shape[0]):
            for p in range(int(rp[i]), int(rp[i + 1])):
                yield (i, int(ci[p])), v[p]


def read_csr(path, one_indexed: bool = True, dtype=np.float64, index_dtype=np.int64):
    """dr::read_csr<T, I>(path, one_indexed) (include/dr/detail/matrix_io.hpp:
    246-256): a coordinate Matrix Market file as a host csr_matrix_view
    (values ``dtype``, indices ``index_dtype``), parsed by the library
    (drb_read_matrix_market).  Raises DrbError (DRB_ERR_IO, _UNSUPPORTED or
    _BAD_CSR) with the reference's messages."""
    h = capi.CsrHost()
    check(capi.lib.drb_read_matrix_market(str(path).encode(), int(one_indexed),
                                          C.byref(h)))
    try:
        m, n, nnz = h.m, h.n, h.nnz
        rp = np.ctypeslib.as_array(h.rowptr, (m + 1,)).astype(index_dtype, copy=True)
        ci = (np.ctypeslib.as_array(h.colind, (nnz,)).astype(index_dtype, copy=True)
              if nnz else np.zeros(0, index_dtype))
        v = (np.ctypeslib.as_array(h.values, (nnz,)).astype(dtype, copy=True)
             if nnz else np.zeros(0, dtype))
    finally:
        capi.lib.drb_csr_host_free(C.byref(h))
    return csr_matrix_view(v, rp, ci, (m, n))


class distribution:
    """Distribution options (include/dr/mp/containers/distribution.hpp:11-44).
    distributed_sparse_matrix only stores it, as the reference does."""

    def __init__(self, halo=(0, 0), periodic=False, granularity=1):
        self.halo = halo
        self.periodic = periodic
        self.granularity = granularity


class csr_row_distribution:
    """Row-block policy: segment r owns rows [r*ceil(m/P), ...)
    (matrix_formats/csr_row_distribution.hpp)."""
    partition = capi.DRB_PART_ROW


class csr_eq_distribution:
    """Equal-nnz policy, the reference's default MatrixDistrT
    (matrix_formats/csr_eq_distribution.hpp)."""
    partition = capi.DRB_PART_EQ


class _Segment:
    """One row-block segment (the reference's csr_row_segment /
    csr_eq_segment): rank(), size(), is_local(), iteration over entries."""

    def __init__(self, mat: "distributed_sparse_matrix", idx: int, bounds=None):
        self._m = mat
        self._idx = idx
        if bounds is None:
            r0, r1, z0, z1 = (C.c_int64(), C.c_int64(), C.c_int64(), C.c_int64())
            check(capi.lib.drb_csr_segment(mat._h, idx, C.byref(r0), C.byref(r1),
                                           C.byref(z0), C.byref(z1)))
            bounds = (r0.value, r1.value, z0.value, z1.value)
        self.row_begin, self.row_end, self.nnz_begin, self.nnz_end = bounds

    def rank(self) -> int:
        return self._idx

    def size(self) -> int:
        return self.nnz_end - self.nnz_begin

    def __len__(self) -> int:
        return self.size()

    def is_local(self) -> bool:
        sh = self._m._sharded
        # one process: every segment lives on its GPU; several: rank r's
        return sh is None or sh.comm.rank() == self._idx

    def entries(self):
        return self._m._entries(self.nnz_begin, self.size())

    def __iter__(self):
        rows, cols, vals = self.entries()
        for i in range(len(rows)):
            yield (int(rows[i]), int(cols[i])), vals[i]


class distributed_sparse_matrix:
    """distributed_sparse_matrix<T, I, Backend, MatrixDistrT>
    (distributed_sparse_matrix.hpp:29-162) resident on one GPU.

    csr_view   host csr_matrix_view (or any object with the same accessors)
    root       the rank that holds csr_view (only 0 exists)
    dist       distribution (stored only)
    distr      csr_eq_distribution (default, as in the reference) or
               csr_row_distribution
    nsegments  number of logical segments (the reference's rank count)
    storage    torch.bfloat16 to store f32 values as bf16
    adjoint    build the CSC plan used by gemv_backward
    """

    def __init__(self, csr_view, root: int = 0, dist: distribution | None = None,
                 *, distr=csr_eq_distribution, nsegments: int = 1,
                 storage=None, adjoint: bool = False,
                 keep_index64: bool = False, autotune: bool = False,
                 compensated: bool = False, x_dtype=None, stream=None,
                 comm=None, local_block=None):
        self._h = C.c_void_p(0)
        self._sharded = None
        self.distribution = dist or distribution()
        comm = comm if comm is not None else default_comm()
        if comm.size() > 1:
            # one segment per rank (drb.dist): this rank's rows on its GPU
            from .dist import ShardedCsr
            opts = dict(adjoint=adjoint, keep_index64=keep_index64, autotune=autotune,
                        compensated=compensated)
            factory = local_block or (lambda rp, ci, v, shape: _DeviceBlock(rp, ci, v, shape,
                                                                            **opts))
            self._sharded = ShardedCsr(csr_view, root, distr.partition == capi.DRB_PART_EQ,
                                       comm, factory)
            sh = self._sharded
            self._shape = (sh.m, sh.n)
            self._nnz = sh.nnz
            self.value_dtype = self.storage_dtype = self.compute_dtype = sh.dtype
            self.x_dtype = sh.dtype
            self._ybuf = {}
            return
        if root != 0:
            raise ValueError(f"root {root} is not a rank: one process owns the GPU")
        values = np.ascontiguousarray(csr_view.values_data())
        rowptr = np.ascontiguousarray(csr_view.rowptr_data())
        colind = np.ascontiguousarray(csr_view.colind_data())
        m, n = csr_view.shape()
        nnz = int(csr_view.size())
        if values.dtype not in _NP_DT:
            raise TypeError(f"values dtype {values.dtype} (need float32/float64)")
        vt = _NP_DT[values.dtype]
        it = np.promote_types(rowptr.dtype, colind.dtype)
        if it not in _NP_IT:
            raise TypeError(f"index dtype {it} (need int32/int64)")
        if rowptr.dtype != it:
            rowptr = rowptr.astype(it)
        if colind.dtype != it:
            colind = colind.astype(it)
        st = vt if storage is None else _TORCH_DT[storage]
        flags = 0
        if adjoint:
            flags |= capi.DRB_FLAG_ADJOINT
        if keep_index64:
            flags |= capi.DRB_FLAG_KEEP_INDEX64
        if autotune:
            flags |= capi.DRB_FLAG_AUTOTUNE
        if compensated:
            flags |= capi.DRB_FLAG_COMPENSATED
        if st == capi.DRB_BF16 and x_dtype == torch.float32:
            flags |= capi.DRB_FLAG_BF16_X_F32
        h = C.c_void_p()
        check(capi.lib.drb_csr_create(
            C.byref(h), m, n, nnz, _ptr(rowptr), _ptr(colind), _ptr(values),
            _NP_IT[it], vt, st, int(nsegments), distr.partition, flags,
            _stream(stream)))
        self._h = h
        self._shape = (int(m), int(n))
        self._nnz = nnz
        self.value_dtype = _STORAGE_TORCH[vt]
        self.storage_dtype = _STORAGE_TORCH[st]
        self.compute_dtype = torch.float32 if st == capi.DRB_BF16 else self.storage_dtype
        # element type of x: the storage type, except bf16 values with f32 x
        self.x_dtype = (torch.float32 if flags & capi.DRB_FLAG_BF16_X_F32
                        else self.storage_dtype)
        self._ybuf: dict = {}

    # ---- reference accessors ----
    def shape(self):
        return self._shape

    def size(self) -> int:
        return self._nnz

    def nnz(self) -> int:
        return self._nnz

    def segments(self) -> list:
        if self._sharded is not None:
            return [_Segment(self, r, tuple(b)) for r, *b in self._sharded.segments()]
        nseg = C.c_int()
        check(capi.lib.drb_csr_num_segments(self._h, C.byref(nseg)))
        return [_Segment(self, i) for i in range(nseg.value)]

    def fence(self) -> None:
        if self._sharded is not None:
            torch.distributed.barrier(group=self._sharded.comm.group)
            return
        torch.cuda.current_stream().synchronize()

    def local(self):
        """This rank's segment as a local block (several ranks), else self."""
        return self._sharded.local if self._sharded is not None else self

    def storage_bytes(self):
        v, c, r = C.c_int(), C.c_int(), C.c_int()
        check(capi.lib.drb_csr_storage(self._h, C.byref(v), C.byref(c), C.byref(r)))
        return v.value, c.value, r.value

    def _entries(self, offset: int, count: int):
        if self._sharded is not None:
            if not hasattr(self, "_all"):
                self._all = self._sharded.all_entries()
            r, c, v = self._all
            return (r[offset:offset + count], c[offset:offset + count],
                    v[offset:offset + count].astype(np.float64))
        rows = np.empty(count, np.int64)
        cols = np.empty(count, np.int64)
        vals = np.empty(count, np.float64)
        check(capi.lib.drb_csr_get_entries(self._h, offset, count, _ptr(rows),
                                           _ptr(cols), _ptr(vals)))
        return rows, cols, vals

    def __iter__(self) -> Iterator:
        rows, cols, vals = self._entries(0, self._nnz)
        for i in range(self._nnz):
            yield (int(rows[i]), int(cols[i])), vals[i]

    def __getitem__(self, n: int):
        rows, cols, vals = self._entries(int(n), 1)
        return (int(rows[0]), int(cols[0])), vals[0]

    @property
    def handle(self) -> C.c_void_p:
        if self._sharded is not None:
            blk = self._sharded.local
            return blk.a.handle if isinstance(blk, _DeviceBlock) else C.c_void_p(0)
        return self._h

    # ---- the hot call ----
    def local_gemv_and_collect(self, root: int, res, x: torch.Tensor,
                               width: int, stream=None) -> None:
        """distributed_sparse_matrix.hpp:153-158: y = A x for `width` RHS
        (column-major), result written into `res` on root (on every rank
        when root is None)."""
        if self._sharded is not None:
            self._sharded.gemv(root, res, x, width)
            return
        m = self._shape[0]
        if isinstance(res, torch.Tensor) and res.is_cuda:
            y = res
        else:
            key = (width,)
            y = self._ybuf.get(key)
            if y is None:
                y = torch.empty(m * width, dtype=self.compute_dtype, device="cuda")
                self._ybuf[key] = y
        check(capi.lib.drb_csr_gemv(self._h, _ptr(x), _ptr(y), int(width),
                                    capi.DRB_COL_MAJOR, _stream(stream)))
        if y is res:
            return
        host = y.cpu().numpy()
        if isinstance(res, np.ndarray):
            res[...] = host.reshape(res.shape)
        elif isinstance(res, torch.Tensor):
            res.copy_(torch.from_numpy(host).view(res.shape))
        else:
            res[:] = host.tolist()

    def gemv_device(self, x: torch.Tensor, y: torch.Tensor, k: int = 1,
                    layout: int = capi.DRB_COL_MAJOR, stream=None) -> None:
        check(capi.lib.drb_csr_gemv(self._h, _ptr(x), _ptr(y), int(k), layout,
                                    _stream(stream)))

    def gemv_host(self, x_host, y_host, k: int = 1,
                  layout: int = capi.DRB_COL_MAJOR, stream=None) -> None:
        check(capi.lib.drb_csr_gemv_host(self._h, _ptr(x_host), _ptr(y_host),
                                         int(k), layout, _stream(stream)))

    def variant(self) -> int:
        """Single-RHS kernel variant: item span (128/256/512) | 1 if skewed, or
        2048 for the sliced-ELL copy (short, regular rows)."""
        v = C.c_int()
        check(capi.lib.drb_csr_variant(self._h, C.byref(v)))
        return v.value

    def column_blocks(self):
        """(blocks, first block's width) of the single-RHS product's column
        split (drb_csr_column_blocks): (1, n) when x stays in L2."""
        nb, bw = C.c_int(), C.c_int64()
        check(capi.lib.drb_csr_column_blocks(self._h, C.byref(nb), C.byref(bw)))
        return nb.value, bw.value

    def autotune(self, stream=None) -> int:
        """Time the kernel variants on this sparsity pattern, keep the best."""
        v = C.c_int()
        check(capi.lib.drb_csr_autotune(self._h, C.byref(v), _stream(stream)))
        return v.value

    def check(self, stream=None) -> None:
        """Synchronise and raise DrbError if an earlier launch timed out."""
        check(capi.lib.drb_csr_check(self._h, _stream(stream)))

    def update_values(self, values: torch.Tensor, stream=None) -> None:
        check(capi.lib.drb_csr_update_values(self._h, _ptr(values), _stream(stream)))

    def destroy(self) -> None:
        if self._h and self._h.value:
            capi.lib.drb_csr_destroy(self._h)
            self._h = C.c_void_p(0)

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.destroy()


class broadcasted_vector:
    """x replicated on every rank (broadcasted_vector.hpp:9-51); here the
    single copy lives on the GPU."""

    def __init__(self):
        self._data = None

    def broadcast_data(self, data_size: int, root: int, root_data,
                       comm=None, dtype=None) -> None:
        comm = comm if comm is not None else default_comm()
        if comm.size() > 1:
            from .dist import broadcast_tensor
            self._data = broadcast_tensor(comm, root, root_data, data_size, dtype)
            return
        if root != 0:
            raise ValueError(f"root {root} is not a rank")
        t = torch.as_tensor(np.asarray(root_data) if not isinstance(root_data, torch.Tensor) else root_data)
        if dtype is not None:
            t = t.to(dtype)
        t = t.reshape(-1)[:data_size].contiguous()
        if t.numel() != data_size:
            raise ValueError("root_data shorter than data_size")
        self._data = t.cuda()

    def destroy_data(self) -> None:
        self._data = None

    def broadcasted_data(self) -> torch.Tensor:
        return self._data

    def size(self) -> int:
        return 0 if self._data is None else self._data.numel()

    def __getitem__(self, i):
        return self._data[i]


def _slim_array(root_data, height: int, width: int) -> np.ndarray:
    """The T** overload (a list of `width` columns) or one flat
    column-major block, as a flat array of height*width elements."""
    if isinstance(root_data, (list, tuple)) and root_data and hasattr(root_data[0], "__len__") \
            and len(root_data) == width and not isinstance(root_data[0], (int, float)):
        return np.concatenate([np.asarray(c)[:height] for c in root_data])
    return np.asarray(root_data).reshape(-1)[: height * width]


class broadcasted_slim_matrix:
    """A height x width block replicated on every rank, column-major:
    element (i, j) at i + j*height (broadcasted_slim_matrix.hpp:9-80)."""

    def __init__(self):
        self._data = None
        self._width = 0
        self._height = 0

    def broadcast_data(self, height: int, width: int, root: int, root_data,
                       comm=None, dtype=None) -> None:
        comm = comm if comm is not None else default_comm()
        if comm.size() > 1:
            from .dist import broadcast_tensor
            arr = None
            if comm.rank() == root:
                arr = _slim_array(root_data, height, width)
            self._data = broadcast_tensor(comm, root, arr, height * width, dtype)
            self._width, self._height = width, height
            return
        if root != 0:
            raise ValueError(f"root {root} is not a rank")
        if isinstance(root_data, (list, tuple)) and root_data and hasattr(root_data[0], "__len__") \
                and len(root_data) == width and not isinstance(root_data[0], (int, float)):
            cols = [np.asarray(c)[:height] for c in root_data]  # T** overload
            arr = np.concatenate(cols)
        else:
            arr = np.asarray(root_data).reshape(-1)[: height * width]
        t = torch.as_tensor(arr)
        if dtype is not None:
            t = t.to(dtype)
        self._data = t.contiguous().cuda()
        self._width = width
        self._height = height

    def destroy_data(self) -> None:
        self._data = None

    def broadcasted_data(self) -> torch.Tensor:
        return self._data

    def width(self) -> int:
        return self._width

    def __getitem__(self, j):
        return self._data[j * self._height:(j + 1) * self._height]


def gemv(*args, stream=None) -> None:
    """dr::mp::gemv overloads (gemv.hpp:16-71):
        gemv(root, res, A, b)  -> result on root
        gemv(res, A, b)        -> result everywhere (one rank here)
    b is a broadcasted_vector or broadcasted_slim_matrix; res holds
    m (or m*width, column-major) elements."""
    if len(args) == 4:
        root, res, a, b = args
    elif len(args) == 3:
        res, a, b = args
        root = None
    else:
        raise TypeError("gemv(root, res, A, b) or gemv(res, A, b)")
    sharded = getattr(a, "_sharded", None) is not None
    if not sharded:
        if root is None:
            root = 0  # one rank: the root's result is everyone's
        if root != default_comm().rank():
            raise ValueError(f"root {root} is not a rank: one process owns the GPU")
    elif root is not None and not 0 <= root < a._sharded.comm.size():
        raise ValueError(f"root {root} is not a rank")
    m, n = a.shape()
    on_root = root is None or not sharded or a._sharded.comm.rank() == root
    if isinstance(b, broadcasted_slim_matrix):
        width = b.width()
        if on_root and m * width != len(res):
            raise ValueError(f"res has {len(res)} elements, expected {m * width}")
    else:
        width = 1
        if on_root and m != len(res):
            raise ValueError(f"res has {len(res)} elements, expected {m}")
        if b.size() != n:
            raise ValueError(f"x has {b.size()} elements, expected {n}")
    x = b.broadcasted_data()
    if x.dtype != a.x_dtype:
        x = x.to(a.x_dtype)
    a.local_gemv_and_collect(root, res, x, width, stream=stream)


def _ptr_array(ts) -> C.Array:
    return (C.c_void_p * len(ts))(*[_ptr(t).value for t in ts])


class batch:
    """Y_i = A_i X_i for many matrices in one persistent launch replayed from
    a CUDA graph (drb_batch_*).  X_i is n_i x k and Y_i is m_i x k in
    ``layout`` (column-major by default, the broadcasted_slim_matrix layout).
    The matrices must outlive the batch."""

    def __init__(self, mats: Sequence[distributed_sparse_matrix], k: int,
                 layout: int = capi.DRB_COL_MAJOR, stream=None):
        self._b = C.c_void_p(0)
        self._mats = list(mats)
        self.k = int(k)
        self.layout = layout
        hs = (C.c_void_p * len(self._mats))(*[m.handle.value for m in self._mats])
        flags = 0
        if self._mats and self._mats[0].x_dtype == torch.float32 and \
                self._mats[0].storage_bytes()[0] == 2:
            flags |= capi.DRB_FLAG_BF16_X_F32
        h = C.c_void_p(0)
        check(capi.lib.drb_batch_create(C.byref(h), len(self._mats), hs, self.k,
                                        layout, flags, _stream(stream)))
        self._b = h
        self._bound = None

    def bind(self, xs: Sequence[torch.Tensor], ys: Sequence[torch.Tensor],
             stream=None) -> None:
        if len(xs) != len(self._mats) or len(ys) != len(self._mats):
            raise ValueError("one x and one y per matrix")
        self._bound = (list(xs), list(ys))  # keep the tensors alive
        check(capi.lib.drb_batch_bind(self._b, _ptr_array(xs), _ptr_array(ys),
                                      _stream(stream)))

    def gemv(self, stream=None) -> None:
        check(capi.lib.drb_batch_gemv(self._b, _stream(stream)))

    def variant(self) -> int:
        v = C.c_int(0)
        check(capi.lib.drb_batch_variant(self._b, C.byref(v)))
        return v.value

    def set_variant(self, variant: int) -> None:
        check(capi.lib.drb_batch_set_variant(self._b, int(variant)))

    def autotune(self, stream=None) -> int:
        v = C.c_int(0)
        check(capi.lib.drb_batch_autotune(self._b, C.byref(v), _stream(stream)))
        return v.value

    def destroy(self) -> None:
        if self._b and self._b.value:
            capi.lib.drb_batch_destroy(self._b)
            self._b = C.c_void_p(0)

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def batched_gemv(mats: Sequence[distributed_sparse_matrix], xs, ys, k: int,
                 layout: int = capi.DRB_COL_MAJOR, stream=None) -> None:
    """One-shot batch: Y_i = A_i X_i for all i (synchronises the stream)."""
    hs = (C.c_void_p * len(mats))(*[m.handle.value for m in mats])
    flags = 0
    if mats and mats[0].x_dtype == torch.float32 and mats[0].storage_bytes()[0] == 2:
        flags |= capi.DRB_FLAG_BF16_X_F32
    check(capi.lib.drb_batched_gemv(len(mats), hs, _ptr_array(xs), _ptr_array(ys),
                                    int(k), layout, flags, _stream(stream)))


def gemv_backward(a: distributed_sparse_matrix, ybar: torch.Tensor,
                  x: torch.Tensor | None = None, xbar: torch.Tensor | None = None,
                  abar: torch.Tensor | None = None, stream=None) -> None:
    """Adjoint of y = A x: xbar = A^T ybar, abar[p] = ybar[row p] * x[col p]."""
    check(capi.lib.drb_csr_gemv_backward(a.handle, _ptr(ybar), _ptr(x), _ptr(xbar),
                                         _ptr(abar), _stream(stream)))


def residual_norm2(a: distributed_sparse_matrix, x: torch.Tensor, b: torch.Tensor,
                   y: torch.Tensor | None = None, stream=None) -> torch.Tensor:
    """|| A x - b ||^2 fused into the SpMV epilogue (f64 device scalar)."""
    out = torch.empty(1, dtype=torch.float64, device="cuda")
    check(capi.lib.drb_csr_residual_norm2(a.handle, _ptr(x), _ptr(b), _ptr(y),
                                          _ptr(out), _stream(stream)))
    return out


def dense_gemv(A: torch.Tensor, x: torch.Tensor, y: torch.Tensor, k: int = 1,
               layout: int = capi.DRB_COL_MAJOR, stream=None) -> None:
    """y = A x for a row-major (m, n) tensor A with k RHS."""
    m, n = A.shape
    lda = A.stride(0)
    check(capi.lib.drb_dense_gemv(m, n, _ptr(A), lda, _ptr(x), _ptr(y), int(k), layout,
                                  _TORCH_DT[A.dtype], _stream(stream)))


class dense_batch:
    """Y_i = A_i X_i for row-major BF16 matrices on the tensor cores
    (drb_dense_batch_*): A_i a 2-D bf16 tensor (rows may be padded: its
    stride(0) is the leading dimension, a multiple of 8), X_i n_i x k bf16 and
    Y_i m_i x k fp32, flat, in ``layout``.  The tensors must outlive the plan."""

    def __init__(self, As: Sequence[torch.Tensor], xs: Sequence[torch.Tensor],
                 ys: Sequence[torch.Tensor], k: int, layout: int = capi.DRB_COL_MAJOR,
                 ns: Sequence[int] | None = None, stream=None):
        cnt = len(As)
        if not (len(xs) == len(ys) == cnt):
            raise ValueError("one x and one y per matrix")
        self._keep = (list(As), list(xs), list(ys))
        m = (C.c_int64 * cnt)(*[a.shape[0] for a in As])
        n = (C.c_int64 * cnt)(*(ns if ns is not None else [a.shape[1] for a in As]))
        lda = (C.c_int64 * cnt)(*[a.stride(0) for a in As])
        h = C.c_void_p(0)
        self._p = C.c_void_p(0)
        check(capi.lib.drb_dense_batch_create(C.byref(h), cnt, m, n, _ptr_array(As), lda,
                                              _ptr_array(xs), _ptr_array(ys), int(k),
                                              layout, capi.DRB_BF16, _stream(stream)))
        self._p = h

    def gemv(self, stream=None) -> None:
        check(capi.lib.drb_dense_batch_gemv(self._p, _stream(stream)))

    def set_variant(self, variant: int) -> None:
        check(capi.lib.drb_dense_batch_set_variant(self._p, int(variant)))

    def check(self, stream=None) -> None:
        check(capi.lib.drb_dense_batch_check(self._p, _stream(stream)))

    def set_wait(self, wait_ns: int = 0, stall_tile: int = -1) -> None:
        """drb_dense_batch_set_wait: limit the in-kernel waits of later
        launches to wait_ns (0 = one second); stall_tile >= 0 makes that
        tile's CTA issue no loads (failure detection)."""
        check(capi.lib.drb_dense_batch_set_wait(self._p, int(wait_ns), int(stall_tile)))

    def destroy(self) -> None:
        if self._p and self._p.value:
            capi.lib.drb_dense_batch_destroy(self._p)
            self._p = C.c_void_p(0)

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def dot(a: torch.Tensor, b: torch.Tensor, out: torch.Tensor | None = None,
        stream=None) -> torch.Tensor:
    """sum(a*b) in f64 with a fixed order (a is b: squared norm)."""
    if out is None:
        out = torch.empty(1, dtype=torch.float64, device="cuda")
    check(capi.lib.drb_dot(a.numel(), _ptr(a), _ptr(b), _TORCH_DT[a.dtype], _ptr(out),
                           _stream(stream)))
    return out


# ---- distributed_vector, iota, fill, reduce --------------------------------------
_VEC_DT = {torch.float32: capi.DRB_F32, torch.float64: capi.DRB_F64,
           torch.int32: capi.DRB_INT32, torch.int64: capi.DRB_INT64}
_NP_OF = {capi.DRB_F32: np.float32, capi.DRB_F64: np.float64,
          capi.DRB_INT32: np.int32, capi.DRB_INT64: np.int64}
_OPS = {"plus": capi.DRB_REDUCE_SUM, "min": capi.DRB_REDUCE_MIN, "max": capi.DRB_REDUCE_MAX}


def _op_code(op) -> int:
    import operator
    if op is None or op is operator.add or op is sum:
        return capi.DRB_REDUCE_SUM
    if op is min:
        return capi.DRB_REDUCE_MIN
    if op is max:
        return capi.DRB_REDUCE_MAX
    if isinstance(op, str) and op in _OPS:
        return _OPS[op]
    raise ValueError("drb: reduce supports plus (operator.add), min and max; "
                     f"got {op!r}")


class _VecSegment:
    """One block of a distributed_vector: elements [begin, end) owned by
    `rank` (dv_segment, include/dr/mp/containers/segment.hpp:214-248)."""

    def __init__(self, vec: "distributed_vector", rank: int, begin: int, end: int):
        self._vec, self._rank, self.begin, self.end = vec, rank, begin, end

    def rank(self) -> int:
        return self._rank

    def size(self) -> int:
        return self.end - self.begin

    def __len__(self) -> int:
        return self.size()

    def is_local(self) -> bool:
        return True

    def data(self) -> torch.Tensor:
        return self._vec.tensor[self.begin:self.end]


class _Iter:
    """Random-access position in a distributed_vector (the reference's
    iterator: parent + offset, distributed_vector.hpp:159-230)."""

    def __init__(self, vec: "distributed_vector", off: int):
        self.vec, self.off = vec, off

    def __add__(self, d: int) -> "_Iter":
        return _Iter(self.vec, self.off + int(d))

    __radd__ = __add__

    def __sub__(self, d):
        if isinstance(d, _Iter):
            return self.off - d.off
        return _Iter(self.vec, self.off - int(d))

    def __eq__(self, o) -> bool:
        return isinstance(o, _Iter) and o.vec is self.vec and o.off == self.off


class distributed_vector:
    """dr::mp::distributed_vector<T> (include/dr/mp/containers/
    distributed_vector.hpp:150-340) on one GPU: the n elements live in one
    device tensor; segment r holds [r*ceil(n/P), min(n, (r+1)*ceil(n/P)))
    (segment_size, distributed_vector.hpp:310), P = nsegments.  dtype:
    torch.float32/float64/int32/int64."""

    def __init__(self, n: int, value=None, dtype=torch.float64, nsegments: int = 1,
                 dist: distribution | None = None):
        if n < 0 or nsegments < 1:
            raise ValueError("drb: n must be >= 0 and nsegments >= 1")
        if dtype not in _VEC_DT:
            raise ValueError(f"drb: distributed_vector dtype {dtype} not supported")
        self._n, self._P, self.dtype = int(n), int(nsegments), dtype
        self.tensor = torch.empty(max(self._n, 1), dtype=dtype, device="cuda")[: self._n]
        if value is not None:
            fill(self, value)

    @property
    def code(self) -> int:
        return _VEC_DT[self.dtype]

    def size(self) -> int:
        return self._n

    def __len__(self) -> int:
        return self._n

    def segment_size(self) -> int:
        return -(-self._n // self._P) if self._n else 0

    def segments(self) -> list:
        seg = self.segment_size()
        return [_VecSegment(self, r, min(self._n, r * seg), min(self._n, (r + 1) * seg))
                for r in range(self._P)]

    def begin(self) -> _Iter:
        return _Iter(self, 0)

    def end(self) -> _Iter:
        return _Iter(self, self._n)

    def __getitem__(self, i: int):
        return self.tensor[int(i)].item()

    def __setitem__(self, i: int, v) -> None:
        self.tensor[int(i)] = v

    def fence(self) -> None:
        torch.cuda.current_stream().synchronize()

    def numpy(self) -> np.ndarray:
        return self.tensor.cpu().numpy()


def _span(r, last=None):
    """(tensor slice, dtype code) of a vector, a segment, an iterator pair or
    a CUDA tensor."""
    if isinstance(r, _Iter):
        if not isinstance(last, _Iter) or last.vec is not r.vec or last.off < r.off:
            raise ValueError("drb: [first, last) must be iterators of one vector")
        return r.vec.tensor[r.off:last.off], r.vec.code
    if isinstance(r, distributed_vector):
        return r.tensor, r.code
    if isinstance(r, _VecSegment):
        return r.data(), r._vec.code
    if isinstance(r, torch.Tensor):
        if not r.is_cuda or r.dtype not in _VEC_DT or not r.is_contiguous():
            raise ValueError("drb: expected a contiguous CUDA tensor of f32/f64/i32/i64")
        return r, _VEC_DT[r.dtype]
    raise TypeError(f"drb: not a distributed range: {type(r).__name__}")


def _range_and_value(args, name):
    """(r, value) or (first, last, value), as the reference's overloads."""
    if len(args) == 2:
        return _span(args[0]), args[1]
    if len(args) == 3:
        return _span(args[0], args[1]), args[2]
    raise TypeError(f"drb: {name}(r, value) or {name}(first, last, value)")


def iota(*args, stream=None) -> None:
    """dr::mp::iota(r, value) and iota(first, last, value)
    (include/dr/mp/algorithms/iota.hpp:20-34): element i gets value + i."""
    (t, code), value = _range_and_value(args, "iota")
    check(capi.lib.drb_iota(t.numel(), _ptr(t), code, int(value), _stream(stream)))


def fill(*args, stream=None) -> None:
    """dr::mp::fill(r, value) and fill(first, last, value)
    (include/dr/mp/algorithms/fill.hpp:21-30)."""
    (t, code), value = _range_and_value(args, "fill")
    v = np.array([value], dtype=_NP_OF[code])
    check(capi.lib.drb_fill(t.numel(), _ptr(t), code, C.c_void_p(v.ctypes.data),
                            _stream(stream)))


def _reduce_span(t, code, init, op, out, stream):
    res = out if out is not None else torch.empty(1, dtype=t.dtype, device="cuda")
    if init is not None:
        iv = np.array([init], dtype=_NP_OF[code])
        ip = C.c_void_p(iv.ctypes.data)
    else:
        ip = C.c_void_p(0)
    check(capi.lib.drb_reduce(t.numel(), _ptr(t), code, _op_code(op), ip, _ptr(res),
                              _stream(stream)))
    return res if out is not None else res.item()


def reduce(*args, out: torch.Tensor | None = None, stream=None):
    """dr::mp::reduce (include/dr/mp/algorithms/reduce.hpp:127-181), every
    overload: reduce(r), reduce(r, init), reduce(r, init, op),
    reduce(root, r[, init[, op]]), and the same with an iterator pair
    (first, last) in place of r.  op: operator.add (default), min or max --
    the reference's std::plus and its tests' min/max lambdas.  init is
    applied last: op(init, reduce(r)).  Returns the value on the host (root
    0 is the only rank), or, with `out` (a 1-element CUDA tensor of the
    element type), writes it there asynchronously and returns `out`."""
    a = list(args)
    if a and isinstance(a[0], (int, np.integer)) and not isinstance(a[0], bool) and \
            len(a) > 1 and isinstance(a[1], (distributed_vector, _Iter, _VecSegment,
                                             torch.Tensor)):
        root = int(a.pop(0))
        if root != 0:
            raise ValueError("drb: root is not a rank")
    if not a:
        raise TypeError("drb: reduce needs a range")
    if isinstance(a[0], _Iter):
        t, code = _span(a[0], a[1] if len(a) > 1 else None)
        rest = a[2:]
    else:
        t, code = _span(a[0])
        rest = a[1:]
    init = rest[0] if len(rest) > 0 else None
    op = rest[1] if len(rest) > 1 else None
    return _reduce_span(t, code, init, op, out, stream)


def conjugate_gradient(a: distributed_sparse_matrix, b: torch.Tensor, x: torch.Tensor,
                       max_iters: int = 1000, rtol: float = 1e-8, stream=None) -> dict:
    """Solve a x = b (a symmetric positive definite, F32/F64 storage) by
    unpreconditioned CG entirely on the GPU (drb_csr_cg); x holds the initial
    guess and receives the solution.  Returns iterations, residual_norm,
    b_norm, converged, breakdown."""
    info = capi.CgInfo()
    check(capi.lib.drb_csr_cg(a.handle, _ptr(b), _ptr(x), int(max_iters), float(rtol),
                              C.byref(info), _stream(stream)))
    return {"iterations": int(info.iterations), "residual_norm": float(info.residual_norm),
            "b_norm": float(info.b_norm), "converged": bool(info.converged),
            "breakdown": bool(info.breakdown)}
