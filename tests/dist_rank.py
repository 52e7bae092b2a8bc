"""One rank of the multi-process gemv tests (test_dist_gloo.py runs
world_size copies of this script; test_gpu_dist.py runs them on the GPU).

Every rank builds the reference tests' matrices through
drb.mp.distributed_sparse_matrix with a torch.distributed communicator and
checks drb.mp.gemv -- root and no-root forms, one vector and a 20-wide
slim matrix, csr_row and csr_eq -- against the oracle's restatement of the
reference's per-rank loops and gather (oracle.gemv_row / gemv_eq with
nseg = world size), and that a gemv with a root moves the partial results
to the root alone (non-root ranks receive no bytes).  With --local oracle
the per-rank product is the oracle's own loop (CPU ranks), so results must
match bit for bit; with
--local device it is this library's GPU kernel, checked within the
reference tests' fp_equal tolerance.  The collectives run over gloo (host
tensors; several ranks may then share one GPU, whose kernels never wait on
one another) or NCCL (one GPU per rank).  Prints "OK" and exits 0, or
prints the failure and exits 1.
"""
import argparse
import os
import sys
from datetime import timedelta

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "distributed-ranges_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

import numpy as np  # noqa: E402
import torch  # noqa: E402
import torch.distributed as dist  # noqa: E402

import oracle  # noqa: E402

GOLD = os.path.join(ROOT, "tests", "golden")
CASES = ["mp_gemv_100x100", "mp_gemv_1000x10", "mp_gemv_10x1000", "band_f64_1000_20_20"]


class OracleBlock:
    """A rank's segment multiplied by the oracle's csr_row loop, in the
    value type (the reference's T accumulation)."""

    def __init__(self, rowptr, colind, values, shape):
        self.rp, self.ci, self.v = rowptr, colind, values
        self.rows, self.n = shape

    def gemv(self, x, k):
        y = oracle.gemv_row(self.rp, self.ci, self.v, x.cpu().numpy(), self.rows, self.n, k,
                            oracle.ACC_T)
        return torch.from_numpy(y)


CHECKS = [0]


def check(cond, what):
    CHECKS[0] += 1
    if not cond:
        raise AssertionError(what)


def run(rank, world, local):
    from drb import mp
    exact = local == "oracle"
    factory = OracleBlock if exact else None
    for name in CASES:
        f = dict(np.load(os.path.join(GOLD, name + ".npz")))
        m, n = int(f["m"]), int(f["n"])
        rp, ci, v = f["rowptr"], f["colind"], f["values"]
        x = f["x"].astype(v.dtype)
        for distr, ref in ((mp.csr_row_distribution, oracle.gemv_row),
                           (mp.csr_eq_distribution, oracle.gemv_eq)):
            tag = f"{name}/{distr.__name__}"
            for root in sorted({0, world - 1}):
                # only the root's view is read
                view = mp.csr_matrix_view(v, rp, ci, (m, n)) if rank == root else None
                a = mp.distributed_sparse_matrix(view, root, distr=distr, local_block=factory)
                check(a.shape() == (m, n) and a.size() == len(v), f"{tag}: shape")
                segs = a.segments()
                check(len(segs) == world and sum(s.size() for s in segs) == len(v),
                      f"{tag}: segments")
                check([s.is_local() for s in segs] == [r == rank for r in range(world)],
                      f"{tag}: is_local")
                b = mp.broadcasted_vector()
                b.broadcast_data(n, root, x if rank == root else None)
                want = ref(rp, ci, v, x, m, n, 1, oracle.ACC_T, world)
                res = np.full(m, 7, v.dtype)
                mp.gemv(root, res, a, b)
                # the gather goes to the root alone (the reference's MPI_Gather)
                got_bytes = a._sharded.last_gather_bytes
                check(got_bytes == 0 if rank != root else got_bytes > 0 or world == 1,
                      f"{tag}: root={root} gather bytes received {got_bytes}")
                if rank == root:
                    if exact:
                        check(np.array_equal(res, want), f"{tag}: root={root} bits")
                    else:
                        check(oracle.fp_equal(want, res), f"{tag}: root={root} fp_equal")
                    if "expected" in f and v.dtype == np.float32:
                        check(oracle.fp_equal(f["expected"], res), f"{tag}: golden")
                else:
                    check((res == 7).all(), f"{tag}: non-root result untouched")
                res2 = np.zeros(m, v.dtype)
                mp.gemv(res2, a, b)  # no root: the result on every rank
                check(a._sharded.last_gather_bytes > 0 or world == 1,
                      f"{tag}: no-root gather reaches every rank")
                check(np.array_equal(res2, want) if exact else oracle.fp_equal(want, res2),
                      f"{tag}: no-root")
                if "x_w20" in f:
                    xs = f["x_w20"].astype(v.dtype)
                    s20 = mp.broadcasted_slim_matrix()
                    s20.broadcast_data(n, 20, root, xs if rank == root else None)
                    w20 = ref(rp, ci, v, xs, m, n, 20, oracle.ACC_T, world)
                    r20 = np.zeros(m * 20, v.dtype)
                    mp.gemv(root, r20, a, s20)
                    if rank == root:
                        check(np.array_equal(r20, w20) if exact else oracle.fp_equal(w20, r20),
                              f"{tag}: width 20")
                if root == 0:
                    got = list(a)
                    src = list(mp.csr_matrix_view(v, rp, ci, (m, n)))
                    check(len(got) == len(src) and all(
                        g[0] == s[0] and v.dtype.type(g[1]) == s[1] for g, s in zip(got, src)),
                        f"{tag}: iteration")
                a.fence()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--rank", type=int, required=True)
    ap.add_argument("--world", type=int, required=True)
    ap.add_argument("--port", type=int, required=True)
    ap.add_argument("--local", choices=["oracle", "device"], default="oracle")
    ap.add_argument("--backend", choices=["gloo", "nccl"], default="gloo")
    a = ap.parse_args()
    backend = a.backend
    if a.local == "device":
        torch.cuda.set_device(a.rank % torch.cuda.device_count())
    dist.init_process_group(backend, init_method=f"tcp://127.0.0.1:{a.port}", rank=a.rank,
                            world_size=a.world, timeout=timedelta(seconds=120))
    rc = 0
    try:
        run(a.rank, a.world, a.local)
        print(f"OK {CHECKS[0]} checks", flush=True)
    except Exception as e:  # report, then leave the group in step with the others
        print(f"FAIL rank {a.rank}: {type(e).__name__}: {e}", flush=True)
        rc = 1
    finally:
        dist.destroy_process_group()
    sys.exit(rc)


if __name__ == "__main__":
    main()
