#!/usr/bin/env python
"""Benchmark of the gemv hot path on B200: one JSON line on stdout (rank 0).

Workload (N = 1): plain FP32 CSR SpMV y = A x on the 16,777,216 x 16,777,216
power-law matrix (row lengths ~ Zipf truncated to [1, 16384] with alpha solved
for a mean of 20 nnz/row, uniform distinct sorted columns, values and x
U(-1, 1), int32 indices), seeded synthetic data.  A "step" is one SpMV over
the whole matrix.  The matrix (2.9 GB of algorithmic bytes) is larger than
the 126 MB L2, so no L2 flush is needed between steps.

  value  algorithmic GB/s of the device-resident SpMV
         (bytes = 4*nnz + 4*nnz + 4*(m+1) + 4*n + 4*m, the reference's
         formula from examples/sp/gemv_benchmark.cpp:135-140)
  e2e    the same metric through drb_csr_gemv_host: x copied from pinned host
         memory, SpMV, y copied back, every step
  extra  FP64 SpMV, the adjoint (gemv_backward), the fused residual, dense
         32768^2 gemv, each with its own GB/s; the batched SpMM of 512 CSR
         matrices with 16 right-hand sides (FP32 and BF16, one CUDA-graph
         launch per step)

--impl reference times the reference's CPU algorithm for the same workload
(the csr_row_distribution CPU loop restated in oracle/, one thread per host
core standing in for one MPI rank; the reference itself cannot be built
here: it needs MPI, oneDPL and range-v3).

Multi-GPU: the path does not shard (one handle = one GPU), so --gpus N runs N
independent replicas (weak scaling) and value = total bytes / max time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "distributed-ranges_b200"))
sys.path.insert(0, ROOT)

METRIC = "SpMV GB/s+GFLOP/s (fwd, adjoint) vs HBM peak; BF16/batched vs plain FP32 @err"
M = N_COLS = 16_777_216
ZIPF_HI = 16384
ZIPF_MEAN = 20.0
SEED = 20261205
FALLBACK_HBM = 6650.0


def hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM, "fallback"


def profiled_traffic(name):
    """traffic per launch from the committed ncu summary (a line
    'traffic_bytes_per_launch: N' in profiles/<name>.txt), else None."""
    p = os.path.join(ROOT, "profiles", name + ".txt")
    try:
        for line in open(p):
            if line.startswith("traffic_bytes_per_launch:"):
                return int(float(line.split(":", 1)[1]))
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                                      "--format=csv,noheader,nounits"], capture_output=True,
                                     text=True, timeout=5).stdout.strip()
                if out:
                    self.samples.append([s.strip() for s in out.split(",")])
            except Exception:
                return
            self._stop.wait(0.1)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4)
                          if len(s) > 2 + i and s[2 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.samples)}


def make_workload(nthreads=0):
    import drb
    alpha = drb.gen.zipf_alpha_for_mean(1, ZIPF_HI, ZIPF_MEAN)
    rp, ci, v = drb.gen.powerlaw_csr(M, N_COLS, alpha=alpha, hi=ZIPF_HI, seed=SEED,
                                     nthreads=nthreads)
    x = drb.gen.values(N_COLS, seed=SEED + 1)
    return alpha, rp, ci, v, x


def alg_bytes(m, n, nnz, vb, ib, rb, xb, yb, k=1):
    return vb * nnz + ib * nnz + rb * (m + 1) + xb * n * k + yb * m * k


def cpu_reference(rp, ci, v, x, steps, warmup, budget_s=None):
    """The reference's csr_row CPU loop, one thread per host core."""
    import oracle
    nth = os.cpu_count() or 1
    times = []
    for i in range(warmup + steps):
        _, tl, tg = oracle.gemv_row_threads(rp, ci, v, x, M, N_COLS, 1, nth)
        if i >= warmup:
            times.append(tl + tg)
        if budget_s is not None and i >= warmup and sum(times) > budget_s:
            break
    return nth, times


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    alpha, rp, ci, v, x = make_workload()
    nnz = int(rp[-1])
    bytes_ = alg_bytes(M, N_COLS, nnz, 4, 4, 4, 4, 4)
    nth, times = cpu_reference(rp, ci, v, x, args.steps, args.warmup)
    t = statistics.median(times)
    val = bytes_ / t / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": round(val, 3), "unit": "GB/s",
        "n_gpus": args.gpus, "steps": len(times), "warmup": args.warmup,
        "ms_per_step": round(t * 1e3, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": workload_config(alpha, nnz),
        "gflops": round(2 * nnz / t / 1e9, 3),
        "cpu_baseline": {"value": round(val, 3), "unit": "GB/s", "cores": nth, "kind": "port",
                         "sample": f"{len(times)} full passes over the matrix (csr_row CPU "
                                   f"loop of csr_row_distribution.hpp:116-133, {nth} threads "
                                   f"= {nth} ranks, local phase + gather)"},
        "e2e": {"value": round(val, 3), "unit": "GB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def workload_config(alpha, nnz):
    name = ("csr_powerlaw_16M_fp32" if (M, N_COLS) == (16_777_216, 16_777_216)
            else f"csr_powerlaw_{M}x{N_COLS}_fp32")
    return {"workload": name, "rows": M, "cols": N_COLS, "nnz": nnz,
            "row_len": f"zipf alpha={alpha:.4f} on [1,{ZIPF_HI}] (mean {ZIPF_MEAN})",
            "index": "int32", "values": "U(-1,1) fp32", "x": "U(-1,1) fp32", "k": 1,
            "l2": "inputs (2.9 GB) larger than L2; no flush", "parallelism": "replicas"}


def timed_launches(fn, steps, stream):
    """Per-launch CUDA-event durations (ms) on the launching stream."""
    import torch
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(steps)]
    for i in range(steps):
        ev[i][0].record(stream)
        fn()
        ev[i][1].record(stream)
    stream.synchronize()
    return [a.elapsed_time(b) for a, b in ev]


def run_ours(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    import drb
    from drb import mp
    from drb import _capi as capi

    alpha, rp, ci, v, x = make_workload()
    nnz = int(rp[-1])
    stream = torch.cuda.current_stream()
    A = mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp, ci, (M, N_COLS)), 0,
                                     distr=mp.csr_row_distribution,
                                     adjoint=not args.no_extra, autotune=True)
    vb, cb, rb = A.storage_bytes()
    variant = A.variant()
    bytes_ = alg_bytes(M, N_COLS, nnz, vb, cb, rb, 4, 4)
    xd = torch.from_numpy(x).cuda()
    yd = torch.empty(M, dtype=torch.float32, device="cuda")

    def step():
        A.gemv_device(xd, yd)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    launches0 = capi.launch_count()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        start.record(stream)
        for _ in range(args.steps):
            step()
        end.record(stream)
        torch.cuda.synchronize()
        gpu_launches = capi.launch_count() - launches0  # kernels of the timed region
        per_launch = timed_launches(step, args.steps, stream)
    t_ms = start.elapsed_time(end) / args.steps
    if world > 1:
        tt = torch.tensor([t_ms], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_ms = float(tt.item())
    value = world * bytes_ / (t_ms * 1e-3) / 1e9
    kern_ms = statistics.mean(per_launch)
    peak, peak_kind = hbm_peak()
    achieved = bytes_ / (kern_ms * 1e-3) / 1e9

    # ---- e2e through the host-pointer C ABI (pinned buffers) ----
    xh = torch.from_numpy(x).pin_memory()
    yh = torch.empty(M, dtype=torch.float32).pin_memory()
    for _ in range(max(1, args.warmup)):
        A.gemv_host(xh.numpy(), yh.numpy())
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        A.gemv_host(xh.numpy(), yh.numpy())
    e2e_s = (time.perf_counter() - t0) / args.steps
    if world > 1:
        tt = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_s = float(tt.item())
    e2e_val = world * bytes_ / e2e_s / 1e9
    assert np.array_equal(yh.numpy(), yd.cpu().numpy())

    extra = {}
    if not args.no_extra:
        extra = extras(args, A, rp, ci, v, x, xd, yd, nnz, bytes_, kern_ms, stream)
        if not args.no_batch:
            extra["batched"] = batch_extras(args, stream)

    line = None
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            nth, times = cpu_reference(rp, ci, v, x, steps=30, warmup=1, budget_s=12.0)
            tc = statistics.median(times)
            cpu = {"value": round(bytes_ / tc / 1e9, 3), "unit": "GB/s", "cores": nth,
                   "kind": "port",
                   "sample": f"{len(times)} full passes over the same matrix with the "
                             f"restated csr_row CPU loop, {nth} threads (median)"}
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t_ms, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded, generated on the host)",
            "config": workload_config(alpha, nnz),
            "gflops": round(world * 2 * nnz / (t_ms * 1e-3) / 1e9, 3),
            "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": round(achieved / peak, 4),
                         "traffic": (profiled_traffic("spmv_warp_powerlaw16M_fp32")
                                     if (M, N_COLS) == (16_777_216, 16_777_216) else None),
                         "kernel": "spmv_warp<float,int,int,%d,%d>" % (variant & ~1, variant & 1),
                         "gather_ceiling": {
                             "what": "random x gathers: ~1 L1->crossbar request per SM per "
                                     "clock (288 G/s measured on this B200)",
                             "ceiling_GBps": round(288e9 * bytes_ / nnz / 1e9, 1),
                             "frac": round(achieved / (288e9 * bytes_ / nnz / 1e9), 4)},
                         "alg_bytes_per_launch": bytes_,
                         "kernel_ms": round(kern_ms, 4)},
            "cpu_baseline": cpu,
            "e2e": {"value": round(e2e_val, 3), "unit": "GB/s",
                    "h2d_bytes_per_step": 4 * N_COLS, "d2h_bytes_per_step": 4 * M,
                    "ms_per_step": round(e2e_s * 1e3, 3)},
            "gpu_launches": int(gpu_launches),
            "clocks": clk.summary(),
            "extra": extra,
        }
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    A.destroy()
    if line is not None:
        print(json.dumps(line), flush=True)
    return 0


def extras(args, A, rp, ci, v, x, xd, yd, nnz, bytes32, fwd_ms, stream):
    """Secondary measurements on the same matrix (and a dense gemv)."""
    import torch
    from drb import mp
    out = {}
    peak, _ = hbm_peak()
    steps = max(3, min(args.steps, 10))

    # adjoint: xbar = A^T ybar (CSC plan) and abar = ybar_i x_j
    ybar = yd.clone()
    xbar = torch.empty_like(xd)
    abar = torch.empty(nnz, dtype=torch.float32, device="cuda")
    for _ in range(2):
        mp.gemv_backward(A, ybar, xd, xbar, abar)
    ms = statistics.mean(timed_launches(lambda: mp.gemv_backward(A, ybar, xd, xbar, abar),
                                        steps, stream))
    adj_bytes = bytes32 + (4 * nnz + 4 * nnz + 4 * M + 4 * N_COLS)  # xbar pass + abar pass
    out["adjoint"] = {"ms": round(ms, 4), "ratio_to_fwd": round(ms / fwd_ms, 3),
                      "GBps": round(adj_bytes / (ms * 1e-3) / 1e9, 2),
                      "frac": round(adj_bytes / (ms * 1e-3) / 1e9 / peak, 4)}

    # fused residual ||Ax - b||^2
    b = torch.empty_like(yd).uniform_(-1, 1)
    ms = statistics.mean(timed_launches(lambda: mp.residual_norm2(A, xd, b, yd), steps, stream))
    rb = bytes32 + 4 * M
    out["residual_fused"] = {"ms": round(ms, 4), "GBps": round(rb / (ms * 1e-3) / 1e9, 2)}

    # FP64 SpMV on the same pattern
    A64 = mp.distributed_sparse_matrix(mp.csr_matrix_view(v.astype(np.float64), rp, ci,
                                                          (M, N_COLS)), 0)
    x64 = xd.double()
    y64 = torch.empty(M, dtype=torch.float64, device="cuda")
    A64.gemv_device(x64, y64)
    ms = statistics.mean(timed_launches(lambda: A64.gemv_device(x64, y64), steps, stream))
    b64 = alg_bytes(M, N_COLS, nnz, 8, 4, 4, 8, 8)
    out["spmv_fp64"] = {"ms": round(ms, 4), "GBps": round(b64 / (ms * 1e-3) / 1e9, 2),
                        "frac": round(b64 / (ms * 1e-3) / 1e9 / peak, 4)}
    A64.destroy()
    del x64, y64

    # dense row-major 32768 x 32768 gemv, N(0,1)
    for name, dt, eb in (("dense_fp32", torch.float32, 4), ("dense_fp64", torch.float64, 8)):
        n = 32768
        g = torch.Generator(device="cuda").manual_seed(SEED)
        Ad = torch.randn(n, n, device="cuda", dtype=dt, generator=g)
        xv = torch.randn(n, device="cuda", dtype=dt, generator=g)
        yv = torch.empty(n, device="cuda", dtype=dt)
        mp.dense_gemv(Ad, xv, yv)
        ms = statistics.mean(timed_launches(lambda: mp.dense_gemv(Ad, xv, yv), steps, stream))
        db = eb * n * n + eb * n * 2
        out[name] = {"ms": round(ms, 4), "GBps": round(db / (ms * 1e-3) / 1e9, 2),
                     "frac": round(db / (ms * 1e-3) / 1e9 / peak, 4),
                     "gflops": round(2 * n * n / (ms * 1e-3) / 1e9, 2)}
        del Ad, xv, yv
    torch.cuda.empty_cache()
    return out


BATCH_COUNT = 512
BATCH_K = 16
ROW_GATHER_CEILING = {64: 183e9, 32: 234e9}  # rows/s, register gathers of 64/32-B rows


def batch_extras(args, stream):
    """Batched SpMM: 512 square CSR matrices (rows ~ U[1024, 200000], nnz/row
    ~ U[8, 64], uniform distinct columns, values and X ~ U(-1, 1)), k = 16
    right-hand sides in the reference's column-major layout, one graph launch
    per step; FP32 and BF16 storage (bf16 X, f32 Y)."""
    import torch
    import drb
    from drb import mp
    peak, _ = hbm_peak()
    steps = max(3, min(args.steps, 10))
    k = BATCH_K
    rng = np.random.default_rng(SEED + 5)
    ms_rows = rng.integers(1024, 200001, size=BATCH_COUNT)
    g = torch.Generator(device="cuda").manual_seed(SEED + 6)
    m32, mbf, xs, xbf, ys32, ysbf = [], [], [], [], [], []
    nnz = 0
    t0 = time.time()
    for i, m in enumerate(ms_rows):
        m = int(m)
        rp, ci, v = drb.gen.uniform_rows_csr(m, m, lo=8, hi=64, seed=SEED + 1000 + i)
        nnz += int(rp[-1])
        view = mp.csr_matrix_view(v, rp, ci, (m, m))
        m32.append(mp.distributed_sparse_matrix(view, 0, distr=mp.csr_row_distribution))
        mbf.append(mp.distributed_sparse_matrix(view, 0, distr=mp.csr_row_distribution,
                                                storage=torch.bfloat16))
        x = torch.empty(m * k, device="cuda").uniform_(-1, 1, generator=g)
        xs.append(x)
        xbf.append(x.to(torch.bfloat16))
        ys32.append(torch.empty(m * k, device="cuda"))
        ysbf.append(torch.empty(m * k, device="cuda"))
    gen_s = time.time() - t0
    rows = int(ms_rows.sum())
    out = {"config": {"matrices": BATCH_COUNT, "rows": "U[1024,200000]",
                      "nnz_per_row": "U[8,64]", "k": k, "layout": "column-major X and Y",
                      "total_rows": rows, "total_nnz": nnz,
                      "setup_s": round(gen_s, 1)}}
    res = {}
    for name, mats, xx, yy, vb, xb in (("fp32", m32, xs, ys32, 4, 4),
                                        ("bf16", mbf, xbf, ysbf, 2, 2)):
        b = mp.batch(mats, k, 0)
        b.bind(xx, yy)
        variant = b.autotune()
        for _ in range(2):
            b.gemv()
        ms = statistics.mean(timed_launches(b.gemv, steps, stream))
        byts = nnz * (4 + vb) + (rows + BATCH_COUNT) * 4 + rows * k * (xb + 4)
        gbps = byts / (ms * 1e-3) / 1e9
        rate = nnz / (ms * 1e-3)
        res[name] = ms
        out["batch_" + name] = {
            "ms": round(ms, 3), "GBps": round(gbps, 1), "frac": round(gbps / peak, 4),
            "gflops": round(2 * nnz * k / (ms * 1e-3) / 1e9, 1),
            "gathers_per_s": round(rate / 1e9, 2),
            "gather_ceiling_frac": round(rate / ROW_GATHER_CEILING[k * xb], 4),
            "variant": "cap=%d G=%d" % (128 << (variant >> 4), variant & 15),
            "alg_bytes": byts, "launches_per_step": 2}
        b.destroy()
    torch.cuda.synchronize()
    # bf16 against fp32 on the same inputs: norm-wise relative difference
    num = sum(float(torch.sum((a.double() - c.double()) ** 2)) for a, c in zip(ysbf, ys32))
    den = sum(float(torch.sum(c.double() ** 2)) for c in ys32)
    out["bf16_vs_fp32"] = {"speedup": round(res["fp32"] / res["bf16"], 3),
                           "normwise_rel_diff": float("%.3e" % ((num / den) ** 0.5))}
    for a in m32 + mbf:
        a.destroy()
    del xs, xbf, ys32, ysbf
    torch.cuda.empty_cache()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-extra", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true",
                    help="skip the 512-matrix batched SpMM extra")
    ap.add_argument("--rows", type=int, default=M,
                    help="rows of the power-law matrix (profiling a smaller case)")
    ap.add_argument("--cols", type=int, default=N_COLS,
                    help="columns (keep 16777216 to keep the 64 MB x footprint)")
    args = ap.parse_args()
    globals()["M"] = args.rows
    globals()["N_COLS"] = args.cols
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
