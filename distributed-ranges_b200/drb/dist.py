"""Multi-process distribution of a CSR matrix: one rank per GPU over
torch.distributed, mirroring the reference's MPI distributions.

csr_row_distribution (include/dr/mp/containers/matrix_formats/
csr_row_distribution.hpp): rank r owns rows [r*ceil(m/P), (r+1)*ceil(m/P))
and their nonzeros (init, :205-318).  csr_eq_distribution
(csr_eq_distribution.hpp): rank r owns nonzeros [r*ceil(nnz/P), ...) and the
rows they touch (found by upper_bound over rowptr, :253-272), so a row may be
split between ranks.  x is replicated on every rank (broadcasted_vector);
each rank multiplies its segment on its own GPU with the single-process
kernels, and the partial results are gathered and assembled as the
reference's gather_gemv_vector does: with a root, only the root receives
the ranks' blocks (the reference's MPI_Gather_c / MPI_Gatherv_c,
csr_row_distribution.hpp:159-168, csr_eq_distribution.hpp:175); without one
(the reference's gemv + broadcast) every rank does.  csr_row copies each
rank's rows into place (:159-204); csr_eq zero-fills the result, adds each
rank's first row (the one a previous rank may also hold) and copies the
rest, in rank order (csr_eq_distribution.hpp:159-216).  The assembly runs on
the receiving rank's device (the GPU under NCCL), vectorised over the
right-hand sides.

Set-up follows the reference's init: the root broadcasts the shape and the
per-rank segment table (the reference's val_information broadcast) and
sends every rank its slice of rowptr, column indices and values.  The
collectives are torch.distributed's: NCCL tensors on the GPU, or gloo
tensors on the host (the CPU tests).  The per-rank product is a pluggable
"local block" (an object with gemv(x, k) -> y): by default a device handle
of this library on the rank's GPU; CPU tests plug in the oracle.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist

_VCODE = {np.dtype(np.float32): 0, np.dtype(np.float64): 1}
_VDT = {0: (np.float32, torch.float32), 1: (np.float64, torch.float64)}


class DistComm:
    """A torch.distributed process group as the reference's communicator:
    rank(), size(), and where its tensors live (the current GPU for NCCL,
    the host otherwise)."""

    def __init__(self, group=None):
        self.group = group
        self.backend = dist.get_backend(group)

    def rank(self) -> int:
        return dist.get_rank(self.group)

    def size(self) -> int:
        return dist.get_world_size(self.group)

    def device(self) -> torch.device:
        if self.backend == "nccl":
            return torch.device("cuda", torch.cuda.current_device())
        return torch.device("cpu")

    def global_rank(self, r: int) -> int:
        return r if self.group is None else dist.get_global_rank(self.group, r)

    def bcast(self, t: torch.Tensor, root: int) -> torch.Tensor:
        dist.broadcast(t, src=self.global_rank(root), group=self.group)
        return t


def segment_table(rowptr, m: int, nnz: int, P: int, eq: bool) -> np.ndarray:
    """(P, 4) int64 rows [row0, row1) and nonzeros [nz0, nz1) of every
    rank's segment.  csr_row: ceil(m/P) rows per rank (the segment size of
    distributed_vector<I>(m), distributed_vector.hpp:310).  csr_eq:
    ceil(nnz/P) nonzeros per rank; the rows are [upper_bound(nz0) - 1,
    upper_bound(nz1 - 1)) over rowptr[0..m); an empty segment owns no rows."""
    rp = np.asarray(rowptr, dtype=np.int64)
    t = np.zeros((P, 4), np.int64)
    if not eq:
        seg = -(-m // P) if m else 0
        for r in range(P):
            r0, r1 = min(m, r * seg), min(m, (r + 1) * seg)
            t[r] = (r0, r1, rp[r0], rp[r1])
        return t
    seg = -(-nnz // P) if nnz else 0
    head = rp[:m]
    for r in range(P):
        z0, z1 = min(nnz, r * seg), min(nnz, (r + 1) * seg)
        if z0 >= z1:
            t[r] = (m, m, z0, z1)
            continue
        row0 = max(0, int(np.searchsorted(head, z0, side="right")) - 1)
        row1 = int(np.searchsorted(head, z1 - 1, side="right"))
        t[r] = (row0, row1, z0, z1)
    return t


class ShardedCsr:
    """One rank's segment of a CSR matrix distributed over a DistComm.

    view         the csr_matrix_view; only the root's is read
    root         the rank that holds the matrix
    eq           csr_eq_distribution (else csr_row_distribution)
    local_block  callable(rowptr, colind, values, (rows, n)) -> object with
                 gemv(x, k) -> y (x: n*k, y: rows*k, column-major tensors
                 on comm.device())
    """

    def __init__(self, view, root: int, eq: bool, comm: DistComm, local_block):
        self.comm, self.root, self.eq = comm, int(root), bool(eq)
        rank, P = comm.rank(), comm.size()
        if not 0 <= self.root < P:
            raise ValueError(f"root {root} is not a rank of {P}")
        dev = comm.device()
        meta = torch.zeros(5, dtype=torch.int64, device=dev)
        if rank == self.root:
            vals = np.ascontiguousarray(view.values_data())
            rp = np.ascontiguousarray(view.rowptr_data()).astype(np.int64)
            ci = np.ascontiguousarray(view.colind_data())
            m, n = view.shape()
            if vals.dtype not in _VCODE:
                raise TypeError(f"values dtype {vals.dtype} (need float32/float64)")
            # column indices travel as int32 whenever the columns fit
            wide = int(n >= 2**31 - 1)
            meta[:] = torch.tensor([m, n, int(rp[m]) if m else 0, _VCODE[vals.dtype], wide])
        comm.bcast(meta, self.root)
        m, n, nnz, vcode, wide = (int(v) for v in meta.cpu())
        self.m, self.n, self.nnz = m, n, nnz
        self.np_dtype, self.dtype = _VDT[vcode]
        ci_np, ci_t = (np.int64, torch.int64) if wide else (np.int32, torch.int32)
        table = torch.zeros((P, 4), dtype=torch.int64, device=dev)
        if rank == self.root:
            table[:] = torch.from_numpy(segment_table(rp, m, nnz, P, self.eq))
        comm.bcast(table, self.root)
        self.table = table.cpu().numpy()
        # the root sends every other rank its slice (rowptr rebased and, for
        # csr_eq, clipped to the rank's nonzero range)
        r0, r1, z0, z1 = (int(v) for v in self.table[rank])
        rows, cnt = r1 - r0, z1 - z0
        if rank == self.root:
            for r in range(P):
                a0, a1, b0, b1 = (int(v) for v in self.table[r])
                lrp = np.clip(rp[a0:a1 + 1], b0, b1) - b0 if a1 > a0 else np.zeros(1, np.int64)
                parts = (lrp.astype(np.int64), ci[b0:b1].astype(ci_np, copy=False),
                         vals[b0:b1])
                if r == rank:
                    lrp_l, lci, lv = parts
                    continue
                for arr in parts:
                    if arr.size:
                        dist.send(torch.from_numpy(np.ascontiguousarray(arr)).to(dev),
                                  dst=comm.global_rank(r), group=comm.group)
        else:
            lrp_t = torch.empty(max(rows, 0) + 1, dtype=torch.int64, device=dev)
            lci_t = torch.empty(cnt, dtype=ci_t, device=dev)
            lv_t = torch.empty(cnt, dtype=self.dtype, device=dev)
            for t in (lrp_t, lci_t, lv_t):
                if t.numel():
                    dist.recv(t, src=comm.global_rank(self.root), group=comm.group)
            if rows == 0:
                lrp_t.zero_()
            lrp_l, lci, lv = lrp_t.cpu().numpy(), lci_t.cpu().numpy(), lv_t.cpu().numpy()
        self.rows = rows
        it = np.int32 if max(n, cnt) < 2**31 - 1 else np.int64
        self.local_csr = (lrp_l.astype(it), lci.astype(it), lv)
        self.local = local_block(self.local_csr[0], self.local_csr[1], self.local_csr[2],
                                 (rows, n)) if rows > 0 else None

    # ---- segments -----------------------------------------------------------------
    def segments(self):
        """(rank, row_begin, row_end, nnz_begin, nnz_end) of every rank."""
        return [(r, *(int(v) for v in self.table[r])) for r in range(self.comm.size())]

    # ---- gemv: local product + gather (gather_gemv_vector) -----------------------
    def gemv(self, root, res, x: torch.Tensor, k: int) -> None:
        """y = A x for k column-major right-hand sides; the result is
        assembled into `res` (m*k, column-major) on `root` only, or on every
        rank when root is None (the reference's no-root gemv).  Every rank's
        block is padded to the largest segment (the reference gathers
        ceil(m/P) rows per rank too).  last_gather_bytes: the bytes this
        rank received in the gather."""
        comm, P = self.comm, self.comm.size()
        rank = comm.rank()
        dev = comm.device()
        rows_max = int((self.table[:, 1] - self.table[:, 0]).max()) if P else 0
        buf = torch.zeros(max(rows_max * k, 1), dtype=self.dtype, device=dev)
        if self.local is not None:
            y = self.local.gemv(x, k)
            buf[: self.rows * k] = y.reshape(-1).to(dtype=self.dtype, device=dev)
        block_bytes = buf.numel() * buf.element_size()
        if root is None:
            parts = [torch.empty_like(buf) for _ in range(P)]
            dist.all_gather(parts, buf, group=comm.group)
            self.last_gather_bytes = (P - 1) * block_bytes
        else:
            root = int(root)
            on_root = rank == root
            parts = [torch.empty_like(buf) for _ in range(P)] if on_root else None
            dist.gather(buf, gather_list=parts, dst=comm.global_rank(root), group=comm.group)
            self.last_gather_bytes = (P - 1) * block_bytes if on_root else 0
            if not on_root:
                return
        _write(res, self._assemble(parts, k))

    def _assemble(self, parts, k: int) -> torch.Tensor:
        """The gathered blocks (rank r: its rows x k, column-major) placed
        into y (m x k, column-major) on their device, in rank order."""
        m = self.m
        out = torch.zeros((k, m), dtype=self.dtype, device=parts[0].device)
        for r in range(len(parts)):
            r0, r1 = int(self.table[r, 0]), int(self.table[r, 1])
            nr = r1 - r0
            if nr <= 0:
                continue
            blk = parts[r][: nr * k].view(k, nr)
            if self.eq:
                # add the first row (a previous rank may hold part of it),
                # copy the rest
                out[:, r0] += blk[:, 0]
                out[:, r0 + 1:r1] = blk[:, 1:]
            else:
                out[:, r0:r1] = blk
        return out.view(-1)

    # ---- entries of every rank (iteration) -----------------------------------------
    def all_entries(self):
        """(rows, cols, values) of the whole matrix in CSR order, gathered
        from the ranks' slices (the reference iterates remote segments)."""
        comm, P = self.comm, self.comm.size()
        dev = comm.device()
        lrp, lci, lv = self.local_csr
        r0 = int(self.table[comm.rank(), 0])
        rows = np.repeat(np.arange(r0, r0 + self.rows), np.diff(lrp.astype(np.int64))) \
            if self.rows > 0 else np.zeros(0, np.int64)
        cnt_max = int((self.table[:, 3] - self.table[:, 2]).max()) if P else 0
        packed = torch.zeros((3, max(cnt_max, 1)), dtype=torch.float64, device=dev)
        c = len(lv)
        packed[0, :c] = torch.from_numpy(rows.astype(np.float64))
        packed[1, :c] = torch.from_numpy(lci.astype(np.float64))
        packed[2, :c] = torch.from_numpy(lv.astype(np.float64))
        parts = [torch.empty_like(packed) for _ in range(P)]
        dist.all_gather(parts, packed, group=comm.group)
        R, Cc, V = [], [], []
        for r in range(P):
            cr = int(self.table[r, 3] - self.table[r, 2])
            p = parts[r].cpu().numpy()
            R.append(p[0, :cr].astype(np.int64))
            Cc.append(p[1, :cr].astype(np.int64))
            V.append(p[2, :cr].astype(self.np_dtype))
        return np.concatenate(R), np.concatenate(Cc), np.concatenate(V)


def _write(res, out: torch.Tensor) -> None:
    """y (a flat tensor) into the caller's result: a numpy array or list on
    the host, or a tensor on any device."""
    if isinstance(res, torch.Tensor):
        res.copy_(out.view(res.shape))
        return
    host = out.cpu().numpy()
    if isinstance(res, np.ndarray):
        res[...] = host.reshape(res.shape)
    else:
        res[:] = host.tolist()


def broadcast_tensor(comm: DistComm, root: int, data, size: int, dtype=None) -> torch.Tensor:
    """The root's `size` elements replicated on every rank (the reference's
    broadcasted_vector::broadcast_data, broadcasted_vector.hpp:17-31), as a
    tensor on comm.device(); the element type is the root's (or `dtype`)."""
    dev = comm.device()
    meta = torch.zeros(1, dtype=torch.int64, device=dev)
    if comm.rank() == root:
        t = torch.as_tensor(np.asarray(data) if not isinstance(data, torch.Tensor) else data)
        if dtype is not None:
            t = t.to(dtype)
        t = t.reshape(-1)[:size].contiguous()
        if t.numel() != size:
            raise ValueError("root_data shorter than data_size")
        meta[0] = {torch.float32: 0, torch.float64: 1}[t.dtype]
    comm.bcast(meta, root)
    tdt = _VDT[int(meta.item())][1]
    if comm.rank() == root:
        buf = t.to(device=dev, dtype=tdt)
    else:
        buf = torch.empty(size, dtype=tdt, device=dev)
    return comm.bcast(buf, root)
