"""Multi-process gemv (drb.dist) on CPU ranks over gloo: world sizes 2, 3
and 4, csr_row and csr_eq, root and no-root forms, a 20-wide slim matrix,
segments and iteration -- each rank's product is the oracle's loop, so the
assembled results must equal the oracle's restatement of the reference's
per-rank loops and gather bit for bit (see tests/dist_rank.py)."""
import os
import socket
import subprocess
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def run_ranks(world: int, local: str, backend: str, timeout: int = 300):
    port = free_port()
    env = dict(os.environ, CUDA_VISIBLE_DEVICES=os.environ.get("CUDA_VISIBLE_DEVICES", ""))
    if local == "oracle":
        env["CUDA_VISIBLE_DEVICES"] = ""  # CPU ranks
    procs = [subprocess.Popen([sys.executable, os.path.join(HERE, "dist_rank.py"),
                               "--rank", str(r), "--world", str(world), "--port", str(port),
                               "--local", local, "--backend", backend],
                              stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True,
                              env=env) for r in range(world)]
    outs = []
    try:
        for p in procs:
            out, _ = p.communicate(timeout=timeout)
            outs.append((p.returncode, out))
    finally:
        for p in procs:
            if p.poll() is None:
                p.kill()
    return outs


@pytest.mark.parametrize("world", [2, 3, 4])
def test_sharded_gemv_gloo_matches_oracle_bitwise(world):
    outs = run_ranks(world, "oracle", "gloo")
    for rc, out in outs:
        assert rc == 0 and "OK" in out, out[-3000:]
        assert int(out.split("OK")[1].split()[0]) >= 50  # the checks ran
