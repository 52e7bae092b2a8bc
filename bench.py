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
         32768^2 gemv, each with its own GB/s; the 131072^2 16-per-row case
         (L2-flushed and warm); L = 0.5||Ax-b||^2 forward and backward on the
         2048^2 Laplacian and a 4M-row power-law matrix with finite-difference
         checks; BF16 / FP32 / compensated FP32 error per row-length bin on the
         8M-row scaled power-law matrix; the batched SpMM of 512 CSR
         matrices with 16 right-hand sides (FP32 and BF16, one CUDA-graph
         launch per step); the tensor-core dense product of 64 BF16 squares
         with 32 right-hand sides

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
    """SM clock and clock-event (throttle) reasons sampled during the timed
    region: through NVML every 2 ms (reads only), else nvidia-smi every 0.1 s.
    The GPU is matched to the CUDA device by UUID."""
    Q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.samples = []  # (sm_mhz, max_mhz, set of active reason names)
        self.source = None
        self._stop = threading.Event()
        self._t = None
        self._nvml = None
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            try:
                uuid = "GPU-" + str(torch.cuda.get_device_properties(gpu_index).uuid)
                h = pynvml.nvmlDeviceGetHandleByUUID(uuid)
            except Exception:
                h = pynvml.nvmlDeviceGetHandleByIndex(gpu_index)
            bits = [pynvml.nvmlClocksEventReasonHwSlowdown,
                    pynvml.nvmlClocksEventReasonHwThermalSlowdown,
                    pynvml.nvmlClocksEventReasonSwThermalSlowdown,
                    pynvml.nvmlClocksEventReasonSwPowerCap]
            self._nvml = (pynvml, h, bits)
            self._nvml_sample()
        except Exception:
            self._nvml = None
            self.samples = []

    def _nvml_sample(self):
        nv, h, bits = self._nvml
        sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
        self.samples.append((float(sm), float(mx),
                             {n for n, b in zip(self.NAMES, bits) if r & b}))

    def _smi_sample(self):
        out = subprocess.run(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                              "--format=csv,noheader,nounits"], capture_output=True,
                             text=True, timeout=5).stdout.strip()
        f = [t.strip() for t in out.split(",")] if out else []
        if len(f) >= 2 and f[0].replace(".", "").isdigit():
            self.samples.append((float(f[0]), float(f[1]) if f[1].replace(".", "").isdigit()
                                 else float("nan"),
                                 {self.NAMES[i] for i in range(4)
                                  if len(f) > 2 + i and f[2 + i].lower().startswith("active")}))

    def _run(self):
        period = 0.002 if self._nvml else 0.1
        while not self._stop.is_set():
            try:
                self._nvml_sample() if self._nvml else self._smi_sample()
            except Exception:
                return
            self._stop.wait(period)

    def __enter__(self):
        self.samples = []
        self.source = "nvml" if self._nvml else "nvidia-smi"
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
        sm = [s[0] for s in self.samples]
        mx = [s[1] for s in self.samples if s[1] == s[1]]
        reasons = sorted(set().union(*[s[2] for s in self.samples]))
        return {"sm_mhz": statistics.median(sm), "sm_min_mhz": min(sm),
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.samples), "source": self.source}


def make_workload(nthreads=0, gen=None):
    """The power-law matrix and x.  gen: the generator module (drb.gen, or
    oracle.gen -- the same source built into the oracle library, which the
    reference arm uses so that it never loads the CUDA library)."""
    if gen is None:
        import drb
        gen = drb.gen
    alpha = gen.zipf_alpha_for_mean(1, ZIPF_HI, ZIPF_MEAN)
    rp, ci, v = gen.powerlaw_csr(M, N_COLS, alpha=alpha, hi=ZIPF_HI, seed=SEED,
                                 nthreads=nthreads)
    x = gen.values(N_COLS, seed=SEED + 1)
    return alpha, rp, ci, v, x


def alg_bytes(m, n, nnz, vb, ib, rb, xb, yb, k=1):
    return vb * nnz + ib * nnz + rb * (m + 1) + xb * n * k + yb * m * k


# Per-row parity of every timed result against the oracle (the csr_row loop
# of csr_row_distribution.hpp:116-133, or a row-dot product for the dense
# cases, accumulated in long double on the host): err = |y - ref| / sum|a x|
# per row and right-hand side, max and mean, with the gate each config is
# held to.  Filled by the legs below; printed as the line's "parity" block.
PARITY = {}
PARITY_RULE = ("per row (and right-hand side): |y - ref| / sum_j |a_ij x_j|, ref = the "
               "oracle's csr_row loop (csr_row_distribution.hpp:116-133) or dense row "
               "product in long double on the same inputs")


def checks_on(args):
    """The per-row oracle checks run on rank 0 only (each uses every host
    thread), and not with --no-parity."""
    return not args.no_parity and int(os.environ.get("RANK", "0")) == 0


def record_parity(name, res, gate=None, **info):
    """res: an oracle.csr_check / dense_check result (or a merge of them)."""
    e = {"max": float("%.3e" % res["max"]), "mean": float("%.3e" % res["mean"]),
         "count": int(res["count"])}
    if gate is not None:
        e["gate"] = gate
        e["pass"] = bool(res["max"] <= gate)
    if res.get("bins"):
        e["per_row_len_bin"] = {k: {"rows": b["rows"], "max": float("%.3e" % b["max"]),
                                    "mean": float("%.3e" % b["mean"])}
                                for k, b in res["bins"].items()}
    e.update(info)
    PARITY[name] = e
    return e


def merge_checks(results):
    """Combine oracle check results of several matrices (a sample)."""
    cnt = sum(r["count"] for r in results)
    return {"max": max(r["max"] for r in results),
            "mean": sum(r["mean"] * r["count"] for r in results) / max(cnt, 1), "count": cnt}


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


def cpu_spread(bytes_, times):
    """GB/s of the slowest, median and fastest pass: the host is shared, so its
    figure moves from run to run."""
    gb = sorted(bytes_ / t / 1e9 for t in times)
    return {"min": round(gb[0], 3), "median": round(statistics.median(gb), 3),
            "max": round(gb[-1], 3), "passes": len(gb)}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import oracle.gen
    alpha, rp, ci, v, x = make_workload(gen=oracle.gen)
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
                                   f"= {nth} ranks, local phase + gather)",
                         "spread": cpu_spread(bytes_, times)},
        "e2e": {"value": round(val, 3), "unit": "GB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def kernel_name(variant):
    """The single-RHS kernel behind a drb_csr_variant code."""
    if variant == 2048:
        return "sell_spmv<float,int>"
    name = "spmv_warp_pipe" if variant & 2 else "spmv_warp"
    return "%s<float,int,int,%d,%d>" % (name, variant & ~3, variant & 1)


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
    if rank == 0 and not args.no_parity:
        import oracle
        t0 = time.time()
        record_parity("spmv_fp32", oracle.csr_check(rp, ci, v, x, M, N_COLS, yh.numpy()),
                      1e-5, matrix=workload_config(alpha, nnz)["workload"],
                      check_s=round(time.time() - t0, 1))

    # the streaming-gather floor on this pattern (column indices and values
    # streamed, x gathered at each, no rows): the roofline of a gather-bound SpMV
    import drb_probe
    drb_probe.gather_probe(A, xd)
    probe_ms = statistics.mean(timed_launches(lambda: drb_probe.gather_probe(A, xd),
                                              args.steps, stream))
    drb_probe.gather_probe(A, xd, False)
    probe_cols_ms = statistics.mean(timed_launches(lambda: drb_probe.gather_probe(A, xd, False),
                                                   args.steps, stream))

    extra = {}
    if not args.no_extra:
        extra = extras(args, A, rp, ci, v, x, xd, yd, nnz, bytes_, kern_ms, stream)
        extra["config1_fixed16"] = config1_extras(args, stream)
        if world == 1:  # 13 GB of host arrays per process
            extra["powerlaw_alpha1_5"] = alpha15_extras(args, stream)
        extra["adjoint_fd"] = adjoint_extras(args, stream)
        extra["precision"] = precision_extras(args, stream)
        extra["cg"] = cg_extras(args, stream)
        if not args.no_batch:
            extra["batched"] = batch_extras(args, stream)
            extra["dense_batch_bf16"] = dense_batch_extras(args, stream)
            b = extra["batched"]
            b["effective_over_plain_fp32_spmv"] = {
                nm: round(b["batch_" + nm]["effective_fp32_spmv_GBps"] / achieved, 2)
                for nm in ("fp32", "bf16")}

    line = None
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            nth, times = cpu_reference(rp, ci, v, x, steps=30, warmup=1, budget_s=12.0)
            tc = statistics.median(times)
            cpu = {"value": round(bytes_ / tc / 1e9, 3), "unit": "GB/s", "cores": nth,
                   "kind": "port",
                   "sample": f"{len(times)} full passes over the same matrix with the "
                             f"restated csr_row CPU loop, {nth} threads (median)",
                   "spread": cpu_spread(bytes_, times)}
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
                         "kernel": kernel_name(variant),
                         "column_blocks": A.column_blocks()[0],
                         "gather_ceiling": {
                             "what": "random x gathers: ~1 L1->crossbar request per SM per "
                                     "clock (288 G/s measured on this B200)",
                             "ceiling_GBps": round(288e9 * bytes_ / nnz / 1e9, 1),
                             "frac": round(achieved / (288e9 * bytes_ / nnz / 1e9), 4)},
                         "stream_gather_floor": {
                             "what": "drb_csr_gather_probe on this matrix: column indices and "
                                     "values streamed with the SpMV's loads, x gathered at "
                                     "each, no rows or y (measured in this run)",
                             "ms": round(probe_ms, 4),
                             "ms_indices_only": round(probe_cols_ms, 4),
                             "frac": round(probe_ms / kern_ms, 4)},
                         "alg_bytes_per_launch": bytes_,
                         "kernel_ms": round(kern_ms, 4)},
            "cpu_baseline": cpu,
            "parity": {"rule": PARITY_RULE,
                       "all_pass": all(e.get("pass", True) for e in PARITY.values()),
                       **PARITY},
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
    mp.residual_norm2(A, xd, b, yd)  # warm-up: the first call allocates the reduction scratch
    ms = statistics.mean(timed_launches(lambda: mp.residual_norm2(A, xd, b, yd), steps, stream))
    rb = bytes32 + 4 * M
    out["residual_fused"] = {"ms": round(ms, 4), "GBps": round(rb / (ms * 1e-3) / 1e9, 2)}

    # k = 16 right-hand sides on the same matrix (column-major X and Y, the
    # broadcasted_slim_matrix layout): the batched kernel on this one handle
    k16 = 16
    X16 = torch.empty(N_COLS * k16, device="cuda").uniform_(-1, 1)
    Y16 = torch.empty(M * k16, device="cuda")
    A.gemv_device(X16, Y16, k16)  # first call: builds the handle's batch
    ms = statistics.mean(timed_launches(lambda: A.gemv_device(X16, Y16, k16), steps, stream))
    b16 = alg_bytes(M, N_COLS, nnz, 4, 4, 4, 4, 4, k16)
    out["spmm_k16"] = {"ms": round(ms, 4), "GBps": round(b16 / (ms * 1e-3) / 1e9, 2),
                       "frac": round(b16 / (ms * 1e-3) / 1e9 / peak, 4),
                       "gflops": round(2 * nnz * k16 / (ms * 1e-3) / 1e9, 2),
                       "vs_16_spmvs": round(16 * fwd_ms / ms, 2)}
    if checks_on(args):
        import oracle
        record_parity("spmm_k16_colmajor", oracle.csr_check(rp, ci, v, X16.cpu().numpy(), M,
                                                            N_COLS, Y16.cpu().numpy(), k=k16),
                      1e-5)
    # Row-major X and Y: no packing pass, the SpMM kernel alone; beside it a
    # plain streaming row gather on the same X (column indices and values
    # streamed in nonzero order, the 64-byte X row gathered at each, no rows
    # or Y): the random 64-byte reads of 1.07 GB of X, not the SM, bound both
    import drb_probe
    from drb import _capi as capi
    X16.copy_(X16.view(k16, N_COLS).t().reshape(-1))
    A.gemv_device(X16, Y16, k16, capi.DRB_ROW_MAJOR)
    rm_ms = statistics.mean(timed_launches(
        lambda: A.gemv_device(X16, Y16, k16, capi.DRB_ROW_MAJOR), steps, stream))
    drb_probe.gather_rows_probe(A, X16, k16)
    probe_ms = statistics.mean(timed_launches(lambda: drb_probe.gather_rows_probe(A, X16, k16),
                                              steps, stream))
    out["spmm_k16"].update({
        "row_major_ms": round(rm_ms, 4),
        "pack_and_y_layout_ms": round(ms - rm_ms, 4),
        "row_gather_probe_ms": round(probe_ms, 4),
        "row_major_vs_probe": round(probe_ms / rm_ms, 4),
        "probe_what": "drb_csr_gather_rows_probe: column indices and values streamed in "
                      "nonzero order, the 64-byte X row gathered at every nonzero (16-byte "
                      "read-only loads, 4 in flight per lane), no rows or Y"})
    if checks_on(args):
        record_parity("spmm_k16_rowmajor", oracle.csr_check(
            rp, ci, v, X16.view(N_COLS, k16).t().contiguous().cpu().numpy().reshape(-1), M,
            N_COLS, Y16.view(M, k16).t().contiguous().cpu().numpy().reshape(-1), k=k16), 1e-5)
    del X16, Y16

    # FP64 SpMV on the same pattern
    A64 = mp.distributed_sparse_matrix(mp.csr_matrix_view(v.astype(np.float64), rp, ci,
                                                          (M, N_COLS)), 0, autotune=True)
    x64 = xd.double()
    y64 = torch.empty(M, dtype=torch.float64, device="cuda")
    A64.gemv_device(x64, y64)
    ms = statistics.mean(timed_launches(lambda: A64.gemv_device(x64, y64), steps, stream))
    b64 = alg_bytes(M, N_COLS, nnz, 8, 4, 4, 8, 8)
    out["spmv_fp64"] = {"ms": round(ms, 4), "GBps": round(b64 / (ms * 1e-3) / 1e9, 2),
                        "frac": round(b64 / (ms * 1e-3) / 1e9 / peak, 4),
                        "column_blocks": A64.column_blocks()[0]}
    if checks_on(args):
        import oracle
        record_parity("spmv_fp64", oracle.csr_check(rp, ci, v.astype(np.float64), x.astype(
            np.float64), M, N_COLS, y64.cpu().numpy()), 1e-12)
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

    # dot / squared norm: 2 x 2 GB streamed, f64 accumulation, fixed order
    for name, dt, eb in (("dot_fp32", torch.float32, 4), ("dot_fp64", torch.float64, 8)):
        n = (1 << 31) // eb
        g = torch.Generator(device="cuda").manual_seed(SEED + 12)
        av = torch.empty(n, device="cuda", dtype=dt).uniform_(-1, 1, generator=g)
        bv = torch.empty(n, device="cuda", dtype=dt).uniform_(-1, 1, generator=g)
        res = torch.empty(1, device="cuda", dtype=torch.float64)
        mp.dot(av, bv, res)
        ms = statistics.mean(timed_launches(lambda: mp.dot(av, bv, res), steps, stream))
        db = 2 * eb * n
        out[name] = {"n": n, "ms": round(ms, 4), "GBps": round(db / (ms * 1e-3) / 1e9, 2),
                     "frac": round(db / (ms * 1e-3) / 1e9 / peak, 4)}
        if name == "dot_fp32":
            # mp::reduce (sum) over a 2 GB distributed_vector's storage
            res32 = torch.empty(1, device="cuda", dtype=torch.float32)
            mp.reduce(av, out=res32)
            ms = statistics.mean(timed_launches(lambda: mp.reduce(av, out=res32), steps,
                                                stream))
            out["reduce_sum_fp32"] = {"n": n, "ms": round(ms, 4),
                                      "GBps": round(4 * n / (ms * 1e-3) / 1e9, 2),
                                      "frac": round(4 * n / (ms * 1e-3) / 1e9 / peak, 4)}
        del av, bv
    torch.cuda.empty_cache()
    return out


BATCH_COUNT = 512
BATCH_K = 16
BATCH_SAMPLE = 16  # matrices of the batch checked against the oracle
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
    # the matrices whose results are checked against the oracle (a seeded sample)
    sample = sorted(int(i) for i in np.random.default_rng(SEED + 9).choice(
        BATCH_COUNT, size=BATCH_SAMPLE, replace=False))
    kept = {}
    for i, m in enumerate(ms_rows):
        m = int(m)
        rp, ci, v = drb.gen.uniform_rows_csr(m, m, lo=8, hi=64, seed=SEED + 1000 + i)
        if i in sample:
            kept[i] = (rp, ci, v)
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
        # the same products as k separate plain FP32 SpMVs per matrix
        eff = k * alg_bytes(rows, rows, nnz, 4, 4, 4, 4, 4) / (ms * 1e-3) / 1e9
        res[name] = ms
        out["batch_" + name] = {
            "ms": round(ms, 3), "GBps": round(gbps, 1), "frac": round(gbps / peak, 4),
            "effective_fp32_spmv_GBps": round(eff, 1),
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
    if checks_on(args):
        import oracle
        chk = {"fp32": [], "bf16": [], "bf16_acc": []}
        for i in sample:
            rp, ci, v = kept[i]
            m = len(rp) - 1
            xh = xs[i].cpu().numpy()
            chk["fp32"].append(oracle.csr_check(rp, ci, v, xh, m, m, ys32[i].cpu().numpy(),
                                                k=k))
            yb = ysbf[i].cpu().numpy()
            chk["bf16"].append(oracle.csr_check(rp, ci, v, xh, m, m, yb, k=k))
            chk["bf16_acc"].append(oracle.csr_check(
                rp, ci, oracle.f32_to_bf16_bits(v),
                xbf[i].view(torch.int16).cpu().numpy().view(np.uint16), m, m, yb, k=k))
        info = {"matrices": sample, "k": k}
        record_parity("batched_fp32_sample", merge_checks(chk["fp32"]), 1e-5, **info)
        u = 2.0 ** -8
        acc = merge_checks(chk["bf16_acc"])
        e2e = merge_checks(chk["bf16"])
        record_parity("batched_bf16_sample", e2e, None,
                      accumulation_only={"max": float("%.3e" % acc["max"]),
                                         "mean": float("%.3e" % acc["mean"])},
                      input_rounding_bound=float("%.3e" % (2 * u + u * u)),
                      within_bound=bool(e2e["max"] <= 2 * u + u * u), **info)
    for a in m32 + mbf:
        a.destroy()
    del xs, xbf, ys32, ysbf
    torch.cuda.empty_cache()
    return out


def l2_flusher():
    """A callable that writes 256 MB (2x the 126 MB L2) on the GPU."""
    import torch
    buf = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    return lambda: buf.fill_(1)


def flushed_launches(fn, steps, stream, flush):
    """Per-launch CUDA-event durations with an L2 flush before each launch
    (the flush itself is outside the events)."""
    import torch
    out = []
    for _ in range(steps):
        flush()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        b.synchronize()
        out.append(a.elapsed_time(b))
    return out


ALPHA_LITERAL = 1.5


def alpha15_extras(args, stream):
    """The power-law matrix with the stated exponent taken literally: 16,777,216
    rows, Zipf alpha = 1.5 on [1, 16384] (mean 98.0 nonzeros per row, about
    1.64e9 nonzeros, 13.2 GB of FP32 CSR), uniform distinct columns, values and
    x U(-1, 1), FP32, int32 indices.  Timed like the headline (inputs far
    larger than L2); y checked per row against the oracle."""
    import torch
    import drb
    from drb import mp
    try:
        import psutil
        avail = psutil.virtual_memory().available
    except Exception:
        avail = None
    if avail is not None and avail < 48e9:
        return {"skipped": f"needs about 48 GB of free host memory ({avail / 1e9:.0f} GB)"}
    m = n = 16_777_216
    peak, _ = hbm_peak()
    steps = max(3, min(args.steps, 10))
    t0 = time.time()
    rp, ci, v = drb.gen.powerlaw_csr(m, n, alpha=ALPHA_LITERAL, hi=ZIPF_HI, seed=SEED + 41)
    x = drb.gen.values(n, seed=SEED + 42)
    gen_s = time.time() - t0
    nnz = int(rp[-1])
    t0 = time.time()
    A = mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp, ci, (m, n)), 0,
                                     distr=mp.csr_row_distribution)
    up_s = time.time() - t0
    vb, cb, rb = A.storage_bytes()
    xd = torch.from_numpy(x).cuda()
    yd = torch.empty(m, device="cuda")
    for _ in range(3):
        A.gemv_device(xd, yd)
    ms = statistics.mean(timed_launches(lambda: A.gemv_device(xd, yd), steps, stream))
    byts = alg_bytes(m, n, nnz, vb, cb, rb, 4, 4)
    out = {"config": {"rows": m, "nnz": nnz,
                      "row_len": f"zipf alpha={ALPHA_LITERAL} on [1,{ZIPF_HI}] "
                                 f"(mean {nnz / m:.1f})",
                      "alg_bytes": byts, "generate_s": round(gen_s, 1),
                      "upload_and_plan_s": round(up_s, 1)},
           "ms": round(ms, 4), "GBps": round(byts / (ms * 1e-3) / 1e9, 1),
           "frac": round(byts / (ms * 1e-3) / 1e9 / peak, 4),
           "gflops": round(2 * nnz / (ms * 1e-3) / 1e9, 1),
           "gathers_per_s_G": round(nnz / (ms * 1e-3) / 1e9, 1)}
    A.destroy()
    if checks_on(args):
        import oracle
        record_parity("powerlaw_alpha1_5_fp32",
                      oracle.csr_check(rp, ci, v, x, m, n, yd.cpu().numpy()), 1e-5)
    del rp, ci, v, x, xd, yd
    torch.cuda.empty_cache()
    return out


def config1_extras(args, stream):
    """131,072^2 CSR with exactly 16 distinct uniform columns per row (the
    reference's own CPU-runnable case): fits in L2, so timed both with an L2
    flush before every launch and L2-warm."""
    import torch
    import drb
    from drb import mp
    n = 131072
    rp, ci, v = drb.gen.fixed_rows_csr(n, n, length=16, seed=SEED + 11)
    A = mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp, ci, (n, n)), 0,
                                     distr=mp.csr_row_distribution, autotune=True)
    x = torch.from_numpy(drb.gen.values(n, seed=SEED + 12)).cuda()
    y = torch.empty(n, device="cuda")
    nnz = int(rp[-1])
    byts = alg_bytes(n, n, nnz, 4, 4, 4, 4, 4)
    for _ in range(3):
        A.gemv_device(x, y)
    steps = max(20, args.steps)
    cold = statistics.median(flushed_launches(lambda: A.gemv_device(x, y), steps, stream,
                                              l2_flusher()))
    warm = statistics.median(timed_launches(lambda: A.gemv_device(x, y), steps, stream))
    if checks_on(args):
        import oracle
        record_parity("config1_fixed16", oracle.csr_check(rp, ci, v, x.cpu().numpy(), n, n,
                                                          y.cpu().numpy()), 1e-5)
    A.destroy()
    return {"config": {"rows": n, "nnz": nnz, "row_len": "exactly 16", "alg_bytes": byts},
            "l2_flushed": {"ms": round(cold, 4), "GBps": round(byts / (cold * 1e-3) / 1e9, 1)},
            "l2_warm": {"ms": round(warm, 4), "GBps": round(byts / (warm * 1e-3) / 1e9, 1)}}


def adjoint_extras(args, stream):
    """L = 0.5 ||A x - b||^2: forward (fused residual) and backward (xbar =
    A^T (A x - b) on the CSC plan, abar = r_i x_j) on the 2048^2 5-point
    Laplacian and on the power-law matrix at 4,194,304 rows, FP64 and FP32;
    FP64 gradients checked by central differences (h = 1e-6) on 1024 seeded
    coordinates of x and 64 of the values."""
    import torch
    import drb
    from drb import mp
    peak, _ = hbm_peak()
    steps = max(3, min(args.steps, 10))
    out = {}
    g = torch.Generator(device="cuda").manual_seed(SEED + 21)
    mats = {"laplacian2048": None, "powerlaw_4M": None}
    rp, ci, v = drb.gen.laplacian2d_csr(2048, value_dtype=np.float64)
    mats["laplacian2048"] = (rp.astype(np.int32), ci, v)
    alpha = drb.gen.zipf_alpha_for_mean(1, ZIPF_HI, ZIPF_MEAN)
    rp, ci, v = drb.gen.powerlaw_csr(4_194_304, 4_194_304, alpha=alpha, hi=ZIPF_HI,
                                     seed=SEED + 22, value_dtype=np.float64)
    mats["powerlaw_4M"] = (rp, ci, v)
    for name, (rp, ci, v) in mats.items():
        m = len(rp) - 1
        nnz = int(rp[-1])
        res = {"rows": m, "nnz": nnz}
        for dt, npdt, eb in (("fp64", np.float64, 8), ("fp32", np.float32, 4)):
            t0 = time.time()
            A = mp.distributed_sparse_matrix(mp.csr_matrix_view(v.astype(npdt), rp, ci, (m, m)),
                                             0, distr=mp.csr_row_distribution, adjoint=True)
            setup = time.time() - t0
            tdt = torch.float64 if dt == "fp64" else torch.float32
            x = torch.randn(m, device="cuda", dtype=torch.float64, generator=g).to(tdt)
            b = torch.randn(m, device="cuda", dtype=torch.float64, generator=g).to(tdt)
            y = torch.empty(m, device="cuda", dtype=tdt)
            xbar = torch.empty_like(x)
            abar = torch.empty(nnz, device="cuda", dtype=tdt)
            fwd = lambda: mp.residual_norm2(A, x, b, y)
            bwd = lambda: mp.gemv_backward(A, r, x, xbar, abar)
            fwd()
            r = y - b
            for _ in range(2):
                bwd()
            f_ms = statistics.mean(timed_launches(fwd, steps, stream))
            b_ms = statistics.mean(timed_launches(bwd, steps, stream))
            fb = alg_bytes(m, m, nnz, eb, 4, 4, eb, eb) + eb * m  # + b for the residual
            bb = (4 * (m + 1) + 8 * nnz + eb * nnz + eb * m + eb * m) \
                + (4 * nnz + eb * m + eb * m + eb * nnz)  # xbar pass + abar pass
            res[dt] = {"fwd_ms": round(f_ms, 4), "bwd_ms": round(b_ms, 4),
                       "bwd_over_fwd": round(b_ms / f_ms, 3),
                       "fwd_GBps": round(fb / (f_ms * 1e-3) / 1e9, 1),
                       "bwd_GBps": round(bb / (b_ms * 1e-3) / 1e9, 1),
                       "bwd_frac": round(bb / (b_ms * 1e-3) / 1e9 / peak, 4),
                       "setup_s_incl_csc_plan": round(setup, 2)}
            if checks_on(args):
                # xbar against the oracle's csr_row loop on the explicitly
                # transposed matrix; abar against r_i x_j elementwise
                import oracle
                cp, ri, vt = oracle.transpose(rp, ci, v.astype(npdt), m, m)
                rh = r.cpu().numpy()
                record_parity(f"adjoint_xbar_{name}_{dt}",
                              oracle.csr_check(cp, ri, vt, rh, m, m, xbar.cpu().numpy()),
                              1e-5 if dt == "fp32" else 1e-12,
                              oracle="csr_row loop on the explicit transpose")
                del cp, ri, vt
                ab_ref = oracle.abar(rp, ci, rh, x.cpu().numpy(), m)
                rel = np.abs(abar.cpu().numpy().astype(np.float64) - ab_ref) / np.maximum(
                    np.abs(ab_ref), 1e-300)
                record_parity(f"adjoint_abar_{name}_{dt}",
                              {"max": float(rel.max()), "mean": float(rel.mean()),
                               "count": len(rel)}, 1e-6 if dt == "fp32" else 1e-15,
                              rule="elementwise |abar_p - r_i x_j| / |r_i x_j|")
                del ab_ref, rel
            if dt == "fp64":
                Aabs = mp.distributed_sparse_matrix(
                    mp.csr_matrix_view(np.abs(v), rp, ci, (m, m)), 0,
                    distr=mp.csr_row_distribution, adjoint=True)
                xscale = torch.empty_like(x)
                mp.gemv_backward(Aabs, r.abs(), None, xscale, None)  # (|A|^T |r|)_i
                Aabs.destroy()
                res[dt]["fd"] = fd_check(A, x, b, r, xbar, abar, xscale, v, rp, m)
                del xscale
            A.destroy()
            del x, b, y, xbar, abar, r
        out[name] = res
    torch.cuda.empty_cache()
    return out


CG_ITERS = 200


def cg_extras(args, stream):
    """Conjugate gradients on the 2048^2 5-point Laplacian (4,194,304 rows,
    SPD), FP64 and FP32: CG_ITERS iterations with rtol = 0 (no early stop)
    through drb_csr_cg, the device-resident loop (SpMV with fused p.Ap,
    x/r update with fused r.r, p update; replayed from a CUDA graph).
    Algorithmic bytes per iteration: the SpMV's (reference formula) + p read
    as the dot weight + 6 vectors (update: read x, p, r, q; write x, r) + 3
    (p update).  Beside it: the same iteration driven from the host as the
    reference's pieces compose (gemv, then each dot returned to the host),
    and the oracle's CPU CG (one thread) on 5 iterations, whose x after 5
    updates is the parity check."""
    import torch
    import drb
    import oracle
    from drb import mp
    peak, _ = hbm_peak()
    rp, ci, v = drb.gen.laplacian2d_csr(2048, value_dtype=np.float64)
    rp = rp.astype(np.int32)
    m = len(rp) - 1
    nnz = int(rp[-1])
    g = torch.Generator(device="cuda").manual_seed(SEED + 31)
    b64 = torch.randn(m, device="cuda", dtype=torch.float64, generator=g)
    out = {"matrix": "laplacian2048", "rows": m, "nnz": nnz, "iterations": CG_ITERS}
    for dt, npdt, eb in (("fp64", np.float64, 8), ("fp32", np.float32, 4)):
        tdt = torch.float64 if dt == "fp64" else torch.float32
        A = mp.distributed_sparse_matrix(mp.csr_matrix_view(v.astype(npdt), rp, ci, (m, m)), 0,
                                         distr=mp.csr_row_distribution)
        b = b64.to(tdt)
        x = torch.zeros(m, device="cuda", dtype=tdt)
        info = mp.conjugate_gradient(A, b, x, max_iters=CG_ITERS, rtol=0.0)  # captures
        times = []
        for _ in range(3):
            x.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            info = mp.conjugate_gradient(A, b, x, max_iters=CG_ITERS, rtol=0.0)
            e1.record(stream)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        it_ms = min(times) / CG_ITERS
        ib = alg_bytes(m, m, nnz, eb, 4, 4, eb, eb) + eb * m + 6 * eb * m + 3 * eb * m
        res = {"ms_per_iter": round(it_ms, 4), "GBps": round(ib / (it_ms * 1e-3) / 1e9, 1),
               "frac_hbm": round(ib / (it_ms * 1e-3) / 1e9 / peak, 4),
               "alg_bytes_per_iter": ib, "iterations_run": info["iterations"],
               "rel_residual": float("%.3e" % (info["residual_norm"] / info["b_norm"]))}
        # host-driven loop: gemv + dot to host per reduction (torch axpys)
        xh = torch.zeros_like(b)
        r = b.clone()
        p = r.clone()
        q = torch.empty_like(b)
        rr = float(mp.dot(r, r).item())
        def host_iter():
            nonlocal rr, p
            A.gemv_device(p, q)
            alpha = rr / float(mp.dot(p, q).item())
            xh.add_(p, alpha=alpha)
            r.sub_(q, alpha=alpha)
            rr1 = float(mp.dot(r, r).item())
            p = r + (rr1 / rr) * p
            rr = rr1
        for _ in range(3):
            host_iter()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(50):
            host_iter()
        torch.cuda.synchronize()
        res["host_loop_ms_per_iter"] = round((time.perf_counter() - t0) / 50 * 1e3, 4)
        res["device_over_host_loop"] = round(res["host_loop_ms_per_iter"] / it_ms, 2)
        if dt == "fp64":
            # parity: x after 5 updates against the oracle's CPU CG
            x.zero_()
            mp.conjugate_gradient(A, b, x, max_iters=5, rtol=0.0)
            bh = b.cpu().numpy()
            t0 = time.perf_counter()
            x_o, it_o, *_ = oracle.cg(rp, ci, v, bh, np.zeros(m), 5, 0.0)
            cpu_s = (time.perf_counter() - t0) / 5
            xd = x.cpu().numpy()
            res["x5_rel_diff_vs_oracle"] = float(
                "%.3e" % (np.linalg.norm(xd - x_o) / np.linalg.norm(x_o)))
            res["cpu_oracle_ms_per_iter_1thread"] = round(cpu_s * 1e3, 2)
        A.destroy()
        del x, xh, r, p, q, b
        out[dt] = res
    torch.cuda.empty_cache()
    return out


def fd_check(A, x, b, r, xbar, abar, xscale, v, rp, m):
    """Central differences of L = 0.5||Ax - b||^2 (h = 1e-6, FP64) against
    xbar on 1024 coordinates and abar on 64 stored entries.  Only the rows
    touched by a perturbation change, so dL is summed row-wise as
    0.5 (y+ - y-)(y+ + y- - 2b), which avoids cancelling two large sums.
    Errors are relative to (|A|^T |r|)_i for xbar (the sum it cancels) and
    to |abar_p| = |r_i x_j| for abar."""
    import torch
    h = 1e-6
    y1 = torch.empty_like(x)
    y2 = torch.empty_like(x)

    def dl(y_p, y_m):
        return float(torch.sum(0.5 * (y_p - y_m) * (y_p + y_m - 2 * b)))
    rng = np.random.default_rng(SEED + 23)
    idx = rng.choice(m, size=1024, replace=False)
    xe = []
    xbh = xbar.cpu().numpy()
    xsh = xscale.cpu().numpy()
    xp = x.clone()
    for i in idx:
        i = int(i)
        xi = float(x[i])
        xp[i] = xi + h
        A.gemv_device(xp, y1)
        xp[i] = xi - h
        A.gemv_device(xp, y2)
        xp[i] = xi
        fd = dl(y1, y2) / (2 * h)
        xe.append(abs(fd - xbh[i]) / max(xsh[i], 1e-300))
    # values: perturb one stored entry at a time through update_values
    nnz = int(rp[-1])
    pidx = rng.choice(nnz, size=64, replace=False)
    ae = []
    abh = abar.cpu().numpy()
    vals = torch.from_numpy(np.ascontiguousarray(v)).cuda()
    for p in pidx:
        p = int(p)
        vp = float(vals[p])
        vals[p] = vp + h
        A.update_values(vals)
        A.gemv_device(x, y1)
        vals[p] = vp - h
        A.update_values(vals)
        A.gemv_device(x, y2)
        vals[p] = vp
        fd = dl(y1, y2) / (2 * h)
        ae.append(abs(fd - abh[p]) / max(abs(abh[p]), 1e-300))
    A.update_values(vals)
    return {"h": h, "x_coords": len(xe), "xbar_max_rel_err": float("%.3e" % max(xe)),
            "value_coords": len(ae), "abar_max_rel_err": float("%.3e" % max(ae))}


PREC_ROWS = 8_388_608
PREC_HI = 65536
PREC_MEAN = 32.0


def precision_extras(args, stream):
    """BF16 storage and FP32 (plain and compensated) on the power-law matrix
    of 8,388,608 rows (Zipf on [1, 65536], mean 32), values N(0,1) * 10^U(-3,3)
    per row, x ~ U(-1,1).  The BF16 mode of this config is bf16 values with
    f32 x (two-sum compensated f32 sums): one bf16 rounding per product, so
    its error against FP64 is bounded by u = 2^-8 = 3.9e-3 relative to
    sum|a x|, inside the 4e-3 gate.  bf16 values and bf16 x round twice
    (bound 2u + u^2 = 7.8e-3) and are reported beside it.  Errors come from the
    oracle (orc_csr_check, long double): end to end against the original FP32
    inputs, and for BF16 also accumulation only, against the bf16-rounded
    inputs the kernel read; max and mean per row-length bin.  Effective
    throughput = FP32-equivalent algorithmic bytes / time."""
    import torch
    import drb
    import oracle
    from drb import mp
    steps = max(3, min(args.steps, 10))
    m = PREC_ROWS
    alpha = drb.gen.zipf_alpha_for_mean(1, PREC_HI, PREC_MEAN)
    rp, ci, v = drb.gen.powerlaw_csr(m, m, alpha=alpha, hi=PREC_HI, seed=SEED + 31,
                                     dist=drb.gen.NORMAL_ROWSCALE)
    nnz = int(rp[-1])
    x = drb.gen.values(m, seed=SEED + 32)
    vbits = oracle.f32_to_bf16_bits(v)
    xbits = oracle.f32_to_bf16_bits(x)
    view = lambda vals: mp.csr_matrix_view(vals, rp, ci, (m, m))
    b32 = alg_bytes(m, m, nnz, 4, 4, 4, 4, 4)
    xd = torch.from_numpy(x).cuda()
    u = 2.0 ** -8
    out = {"config": {"rows": m, "nnz": nnz, "row_len": f"zipf alpha={alpha:.4f} on "
                      f"[1,{PREC_HI}] (mean {PREC_MEAN})", "values": "N(0,1)*10^U(-3,3) per row",
                      "bf16_mode": "bf16_f32x (bf16 values, f32 x, compensated f32 sums)",
                      "reference": "the oracle's csr_row loop in long double (orc_csr_check)"}}
    # name, options, x dtype, value bytes, x bytes, accumulation-only inputs, gate
    variants = [("fp32", dict(), torch.float32, 4, 4, None, None, 1e-5),
                ("fp32_compensated", dict(compensated=True), torch.float32, 4, 4, None, None,
                 1e-5),
                ("bf16_f32x", dict(storage=torch.bfloat16, x_dtype=torch.float32),
                 torch.float32, 2, 4, vbits, x, 4e-3),
                ("bf16", dict(storage=torch.bfloat16), torch.bfloat16, 2, 2, vbits, xbits,
                 None)]
    times = {}
    for name, kw, xdt, vb, xb, vacc, xacc, gate in variants:
        A = mp.distributed_sparse_matrix(view(v), 0, distr=mp.csr_row_distribution,
                                         autotune=True, **kw)
        xin = xd.to(xdt)
        y = torch.empty(m, dtype=torch.float32, device="cuda")
        for _ in range(3):
            A.gemv_device(xin, y)
        ms = statistics.mean(timed_launches(lambda: A.gemv_device(xin, y), steps, stream))
        times[name] = ms
        A.destroy()
        yh = y.cpu().numpy()
        e2e = oracle.csr_check(rp, ci, v, x, m, m, yh)
        nb = alg_bytes(m, m, nnz, vb, 4, 4, xb, 4)
        ent = {"ms": round(ms, 4), "GBps": round(nb / (ms * 1e-3) / 1e9, 1),
               "effective_fp32_GBps": round(b32 / (ms * 1e-3) / 1e9, 1),
               "max_rel_err": float("%.3e" % e2e["max"]),
               "mean_rel_err": float("%.3e" % e2e["mean"])}
        info = {}
        if vacc is not None:
            acc = oracle.csr_check(rp, ci, vacc, xacc, m, m, yh)
            ent["accumulation_only"] = {"max": float("%.3e" % acc["max"]),
                                        "mean": float("%.3e" % acc["mean"])}
            info["accumulation_only"] = ent["accumulation_only"]
        if name == "bf16":
            info["input_rounding_bound"] = float("%.3e" % (2 * u + u * u))
            info["within_bound"] = bool(e2e["max"] <= 2 * u + u * u)
        out[name] = ent
        record_parity("precision_" + name, e2e, gate, **info)
        del yh
    out["speedup_vs_fp32"] = {nm: round(times["fp32"] / times[nm], 3)
                              for nm in ("fp32_compensated", "bf16_f32x", "bf16")}
    out["why_bf16_is_not_faster"] = (
        "x (33.5 MB f32) stays in L2; the product is bound by one random x gather per "
        "nonzero (L1-to-crossbar requests), whatever the width of the values")
    torch.cuda.empty_cache()
    return out


def tensor_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["bf16_tflops"]), "measured"
    except Exception:
        return 1590.0, "fallback"


DENSE_COUNT = 64
DENSE_K = 32
DENSE_SAMPLE = 8  # matrices checked against the oracle


def dense_batch_extras(args, stream):
    """Dense multi-RHS on the tensor cores: 64 square BF16 matrices of side
    ~ U[256, 8192] (rows padded to a multiple of 8 elements), N(0, 1) entries,
    32 right-hand sides column-major, FP32 accumulation and output; one
    launch for all matrices per step (plus the one-launch X layout kernel)."""
    import torch
    from drb import mp
    hbm, _ = hbm_peak()
    tpk, tkind = tensor_peak()
    steps = max(3, min(args.steps, 10))
    k = DENSE_K
    rng = np.random.default_rng(SEED + 7)
    sides = [int(s) for s in rng.integers(256, 8193, size=DENSE_COUNT)]
    g = torch.Generator(device="cuda").manual_seed(SEED + 8)
    As, xs, ys = [], [], []
    for n in sides:
        lda = (n + 7) // 8 * 8
        As.append(torch.empty(n, lda, device="cuda", dtype=torch.bfloat16)
                  .normal_(generator=g))
        xs.append(torch.randn(n * k, device="cuda", generator=g).to(torch.bfloat16))
        ys.append(torch.empty(n * k, device="cuda"))
    P = mp.dense_batch(As, xs, ys, k, 0, ns=sides)
    for _ in range(3):
        P.gemv()
    ms = statistics.mean(timed_launches(P.gemv, steps, stream))
    P.check()
    abytes = sum(2 * n * n for n in sides)
    byts = abytes + sum(2 * n * k + 4 * n * k for n in sides)
    flops = sum(2.0 * n * n * k for n in sides)
    gbps = byts / (ms * 1e-3) / 1e9
    tfl = flops / (ms * 1e-3) / 1e12
    # parity: a seeded sample of the matrices against the oracle's long-double
    # row products of the same bf16 inputs
    sample = sorted(int(i) for i in np.random.default_rng(SEED + 19).choice(
        DENSE_COUNT, size=DENSE_SAMPLE, replace=False))
    if checks_on(args):
        import oracle
        res = []
        for i in sample:
            n = sides[i]
            res.append(oracle.dense_check(
                As[i].view(torch.int16).cpu().numpy().view(np.uint16),
                xs[i].view(torch.int16).cpu().numpy().view(np.uint16),
                ys[i].cpu().numpy(), k=k, n=n))
        record_parity("dense_tc_bf16_sample", merge_checks(res), 1e-5,
                      matrices=sample, sides=[sides[i] for i in sample], k=k)
    out = {"config": {"matrices": DENSE_COUNT, "side": "U[256,8192]", "k": k,
                      "dtype": "bf16 in, fp32 accumulate and out",
                      "A_GB": round(abytes / 1e9, 3)},
           "ms": round(ms, 4), "GBps": round(gbps, 1), "frac_hbm": round(gbps / hbm, 4),
           "tflops": round(tfl, 1), "frac_tensor": round(tfl / tpk, 4),
           "tensor_peak_kind": tkind, "bound": "hbm",
           "launches_per_step": 2, "kernel": "dense_tc (tcgen05.mma M=128 N=32 K=16, TMA ring)"}
    # the same products through torch (cuBLAS), one matmul per matrix, for context
    Xs = [x.view(k, n).t() for x, n in zip(xs, sides)]

    def loop():
        for A, X, n in zip(As, Xs, sides):
            torch.matmul(A[:, :n], X)
    for _ in range(2):
        loop()
    out["torch_matmul_loop_ms"] = round(statistics.mean(timed_launches(loop, 3, stream)), 4)
    P.destroy()
    del As, xs, ys, Xs
    torch.cuda.empty_cache()
    return out


def profile_case(name):
    """A short run of one kernel on a small case of its bench workload, for
    ncu captures (three launches after one warm-up):
      batch16  the batched SpMM on the first 16 matrices of the 512-matrix
               distribution (fp32, k = 16, column-major, default variant);
      dense64  the tensor-core dense batch of the 64 BF16 squares (k = 32);
      dense_f32  the single-matrix dense gemv at 16384 x 16384 FP32 (1 GB,
               above L2), one right-hand side;
      laplacian_f64  the single-RHS SpMV on the 2048^2 5-point Laplacian
               (4,194,304 rows, FP64 values, int32 indices; 335 MB);
      cg_f64   conjugate gradients on that Laplacian, FP64: one warm-up solve
               of 8 iterations, then 24 iterations (rtol 0);
      powerlaw4m  the SpMV kernel variant of DRB_SPMV_VARIANT (default 256,0:
               256-nonzero items, plain product layout) on the first 4,194,304
               rows' worth of the bench distribution (16,777,216 columns, so the
               same 64 MB x, in two column blocks like the bench's handle: one
               spmv_warp launch over the block-major copy, chunk_finish and
               split_combine; DRB_COLSPLIT=0 for the unsplit product);
      residual4m  the fused ||Ax - b||^2 on that matrix (same variant);
      adjoint_lap_f32  gemv_backward (xbar and abar) on the 2048^2 5-point
               Laplacian, FP32, random values;
      dot_f32  the dot kernel on two FP32 vectors of 2^26 elements (2 x 256 MB);
      probe4m  the streaming-gather probe on the powerlaw4m matrix (column
               indices and values streamed, x gathered; the SpMV's floor);
      colsplit_f64_4m  the FP64 SpMV on 4,194,304 rows of the bench
               distribution with 16,777,216 columns (x 128 MB): three column
               blocks in one launch, then split_combine;
      spmm_k16_4m  k = 16 column-major on the powerlaw4m matrix (X 1.07 GB);
      abar4m   the adjoint's abar = ybar_i x_j on the powerlaw4m matrix (FP32,
               the forward product's work items, DRB_SPMV_VARIANT's span);
      batch16_bf16  the batched SpMM of batch16 with BF16 storage and X
               (compensated sums)."""
    import torch
    import drb
    from drb import mp
    if name in ("batch16", "batch16_bf16"):
        k = BATCH_K
        rng = np.random.default_rng(SEED + 5)
        rows = rng.integers(1024, 200001, size=BATCH_COUNT)[:16]
        g = torch.Generator(device="cuda").manual_seed(SEED + 6)
        mats, xs, ys = [], [], []
        for i, m in enumerate(rows):
            m = int(m)
            rp, ci, v = drb.gen.uniform_rows_csr(m, m, lo=8, hi=64, seed=SEED + 1000 + i)
            kw = dict(storage=torch.bfloat16) if name == "batch16_bf16" else {}
            mats.append(mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp, ci, (m, m)), 0,
                                                     distr=mp.csr_row_distribution, **kw))
            xv = torch.empty(m * k, device="cuda").uniform_(-1, 1, generator=g)
            xs.append(xv.to(torch.bfloat16) if kw else xv)
            ys.append(torch.empty(m * k, device="cuda"))
        b = mp.batch(mats, k, 0)
        b.bind(xs, ys)
        for _ in range(4):
            b.gemv()
        torch.cuda.synchronize()
        b.destroy()
    elif name == "dense64":
        k = DENSE_K
        rng = np.random.default_rng(SEED + 7)
        sides = [int(s) for s in rng.integers(256, 8193, size=DENSE_COUNT)]
        g = torch.Generator(device="cuda").manual_seed(SEED + 8)
        As, xs, ys = [], [], []
        for n in sides:
            As.append(torch.empty(n, (n + 7) // 8 * 8, device="cuda", dtype=torch.bfloat16)
                      .normal_(generator=g))
            xs.append(torch.randn(n * k, device="cuda", generator=g).to(torch.bfloat16))
            ys.append(torch.empty(n * k, device="cuda"))
        P = mp.dense_batch(As, xs, ys, k, 0, ns=sides)
        for _ in range(4):
            P.gemv()
        P.check()
        P.destroy()
    elif name == "dense_f32":
        g = torch.Generator(device="cuda").manual_seed(SEED + 9)
        A = torch.randn(16384, 16384, device="cuda", generator=g)
        x = torch.randn(16384, device="cuda", generator=g)
        y = torch.empty(16384, device="cuda")
        for _ in range(4):
            mp.dense_gemv(A, x, y, 1, 0)
        torch.cuda.synchronize()
    elif name == "laplacian_f64":
        rp, ci, v = drb.gen.laplacian2d_csr(2048, value_dtype=np.float64)
        m = len(rp) - 1
        A = mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp.astype(np.int32), ci, (m, m)),
                                         0, distr=mp.csr_row_distribution)
        g = torch.Generator(device="cuda").manual_seed(SEED + 10)
        x = torch.randn(m, device="cuda", dtype=torch.float64, generator=g)
        y = torch.empty(m, device="cuda", dtype=torch.float64)
        for _ in range(4):
            A.gemv_device(x, y)
        A.check()
    elif name == "cg_f64":
        rp, ci, v = drb.gen.laplacian2d_csr(2048, value_dtype=np.float64)
        m = len(rp) - 1
        A = mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp.astype(np.int32), ci, (m, m)),
                                         0, distr=mp.csr_row_distribution)
        g = torch.Generator(device="cuda").manual_seed(SEED + 11)
        b = torch.randn(m, device="cuda", dtype=torch.float64, generator=g)
        x = torch.zeros(m, device="cuda", dtype=torch.float64)
        mp.conjugate_gradient(A, b, x, max_iters=8, rtol=0.0)
        x.zero_()
        mp.conjugate_gradient(A, b, x, max_iters=24, rtol=0.0)
    elif name == "abar4m":
        alpha = drb.gen.zipf_alpha_for_mean(1, ZIPF_HI, ZIPF_MEAN)
        rp, ci, v = drb.gen.powerlaw_csr(4_194_304, N_COLS, alpha=alpha, hi=ZIPF_HI,
                                         seed=SEED)
        A = mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp, ci, (4_194_304, N_COLS)),
                                         0, distr=mp.csr_row_distribution, adjoint=True)
        x = torch.from_numpy(drb.gen.values(N_COLS, seed=SEED + 1)).cuda()
        yb = torch.from_numpy(drb.gen.values(4_194_304, seed=SEED + 2)).cuda()
        abar = torch.empty(len(v), device="cuda")
        for _ in range(4):
            mp.gemv_backward(A, yb, x, None, abar)
        A.check()
    elif name in ("probe4m", "colsplit_f64_4m", "spmm_k16_4m"):
        alpha = drb.gen.zipf_alpha_for_mean(1, ZIPF_HI, ZIPF_MEAN)
        rp, ci, v = drb.gen.powerlaw_csr(4_194_304, N_COLS, alpha=alpha, hi=ZIPF_HI,
                                         seed=SEED)
        dt = np.float64 if name == "colsplit_f64_4m" else np.float32
        if name == "probe4m":
            os.environ["DRB_SPMV_VARIANT"] = "256,1"
        A = mp.distributed_sparse_matrix(mp.csr_matrix_view(v.astype(dt), rp, ci,
                                                            (4_194_304, N_COLS)),
                                         0, distr=mp.csr_row_distribution)
        x = torch.from_numpy(drb.gen.values(N_COLS, seed=SEED + 1).astype(dt)).cuda()
        if name == "probe4m":
            import drb_probe
            for _ in range(4):
                drb_probe.gather_probe(A, x)
        elif name == "colsplit_f64_4m":
            assert A.column_blocks()[0] == 3, A.column_blocks()
            y = torch.empty(4_194_304, device="cuda", dtype=torch.float64)
            for _ in range(4):
                A.gemv_device(x, y)
        else:
            k = 16
            X = torch.empty(N_COLS * k, device="cuda").uniform_(-1, 1)
            Y = torch.empty(4_194_304 * k, device="cuda")
            for _ in range(4):
                A.gemv_device(X, Y, k)
        A.check()
    elif name in ("powerlaw4m", "residual4m"):
        os.environ.setdefault("DRB_SPMV_VARIANT", "256,0")  # or the variant asked for
        alpha = drb.gen.zipf_alpha_for_mean(1, ZIPF_HI, ZIPF_MEAN)
        rp, ci, v = drb.gen.powerlaw_csr(4_194_304, N_COLS, alpha=alpha, hi=ZIPF_HI,
                                         seed=SEED)
        A = mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp, ci, (4_194_304, N_COLS)),
                                         0, distr=mp.csr_row_distribution)
        x = torch.from_numpy(drb.gen.values(N_COLS, seed=SEED + 1)).cuda()
        y = torch.empty(4_194_304, device="cuda")
        b = torch.from_numpy(drb.gen.values(4_194_304, seed=SEED + 2)).cuda()
        for _ in range(4):
            if name == "powerlaw4m":
                A.gemv_device(x, y)
            else:
                mp.residual_norm2(A, x, b, y)
        A.check()
    elif name == "adjoint_lap_f32":
        rp, ci, v = drb.gen.laplacian2d_csr(2048, value_dtype=np.float32)
        m = len(rp) - 1
        v = np.random.default_rng(SEED + 13).uniform(-1, 1, len(v)).astype(np.float32)
        A = mp.distributed_sparse_matrix(mp.csr_matrix_view(v, rp.astype(np.int32), ci, (m, m)),
                                         0, distr=mp.csr_row_distribution, adjoint=True)
        g = torch.Generator(device="cuda").manual_seed(SEED + 14)
        x = torch.randn(m, device="cuda", generator=g)
        yb = torch.randn(m, device="cuda", generator=g)
        xbar = torch.empty(m, device="cuda")
        abar = torch.empty(len(v), device="cuda")
        for _ in range(4):
            mp.gemv_backward(A, yb, x, xbar, abar)
        A.check()
    elif name == "dot_f32":
        g = torch.Generator(device="cuda").manual_seed(SEED + 12)
        a = torch.empty(1 << 26, device="cuda").uniform_(-1, 1, generator=g)
        b = torch.empty(1 << 26, device="cuda").uniform_(-1, 1, generator=g)
        out = torch.empty(1, device="cuda", dtype=torch.float64)
        for _ in range(4):
            mp.dot(a, b, out)
        torch.cuda.synchronize()
    else:
        raise SystemExit(f"unknown profile case {name}")
    print("profile case", name, "done", flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-extra", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the per-row oracle checks of the timed results")
    ap.add_argument("--no-batch", action="store_true",
                    help="skip the batched extras (512 CSR matrices, 64 dense squares)")
    ap.add_argument("--rows", type=int, default=M,
                    help="rows of the power-law matrix (profiling a smaller case)")
    ap.add_argument("--cols", type=int, default=N_COLS,
                    help="columns (keep 16777216 to keep the 64 MB x footprint)")
    ap.add_argument("--profile-case", choices=["batch16", "batch16_bf16", "dense64", "dense_f32",
                                               "laplacian_f64", "cg_f64", "powerlaw4m",
                                               "residual4m", "dot_f32", "adjoint_lap_f32",
                                               "probe4m", "colsplit_f64_4m", "spmm_k16_4m",
                                               "abar4m"],
                    help="run one kernel on a small case (for ncu) and exit")
    args = ap.parse_args()
    if args.profile_case:
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        return profile_case(args.profile_case)
    globals()["M"] = args.rows
    globals()["N_COLS"] = args.cols
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
