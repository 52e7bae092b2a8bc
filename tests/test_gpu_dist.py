"""Multi-process gemv with this library's GPU kernels as each rank's local
product: two ranks share the one GPU of a test run and exchange over gloo
(their kernels never wait on one another), running the same cases as
test_dist_gloo.py within the reference tests' fp_equal tolerance."""
import pytest
import torch

from test_dist_gloo import run_ranks

pytestmark = pytest.mark.gpu


def test_sharded_gemv_device_blocks():
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    outs = run_ranks(2, "device", "gloo")
    for rc, out in outs:
        assert rc == 0 and "OK" in out, out[-3000:]
        assert int(out.split("OK")[1].split()[0]) >= 50
