"""Benchmark of the clSPARSE hot path on B200: CSR-Adaptive SpMV on the
irregular 2M-row workload (log-normal row lengths mu=2.5 sigma=1.2 plus 50 rows
of 200k nonzeros, columns uniform without replacement, values U[-1,1]; seeded
synthetic input), FP64 (the precision of the reference's published SpM-dV
numbers).

One step = one y = A*x SpMV (alpha=1, beta=0) through clsparseDcsrmv. The
metric is achieved HBM GB/s over the reference's algorithmic byte count
(src/benchmarks/clsparse-bench/functions/clfunc_xSpMdV.hpp:91):
4*(nnz+nrows) + 8*(nnz+ncols+nrows). The matrix (~760 MB) is far larger than
L2 (126 MB), so every step streams it from HBM.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N>1 (torchrun): each rank runs its own replica of the workload on its own GPU
(no data-path collective; weak scaling); the timing is the max over ranks.
--impl reference times the reference algorithm's CPU restatement (the oracle
port; the reference's OpenCL path cannot run on this machine) on all host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "CG time-to-1e-10 rel. residual, learned+mixed vs plain FP64; SpMV HBM GB/s"
WORKLOAD = "irregular SpMV, n=2,000,000, log-normal(2.5,1.2) rows + 50 rows of 200k nnz, FP64 CSR"


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic():
    """dram bytes per launch of the SpMV kernel from the committed ncu summary."""
    p = ROOT / "profiles" / "spmv_irregular_fp64_traffic.json"
    if p.exists():
        return json.loads(p.read_text())
    return None


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.flush()
        self.f.seek(0)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(rp, col, val, seconds=12.0):
    """Oracle port of the reference SpMV on all host cores for ~`seconds`."""
    import oracle
    n = len(rp) - 1
    threads = os.cpu_count() or 1
    x = np.random.default_rng(3).uniform(-1, 1, n)
    y = np.zeros(n)
    nbytes = 4 * (len(col) + n) + 8 * (len(col) + 2 * n)
    oracle.dcsrmv_mt(rp, col, val, 1.0, x, 0.0, y, threads)  # warm
    t0 = time.perf_counter()
    reps = 0
    while True:
        oracle.dcsrmv_mt(rp, col, val, 1.0, x, 0.0, y, threads)
        reps += 1
        el = time.perf_counter() - t0
        if el >= seconds or reps >= 1000:
            break
    gbs = nbytes * reps / el / 1e9
    return {"value": round(gbs, 3), "unit": "GB/s", "cores": threads, "kind": "port",
            "sample": f"{reps} full FP64 SpMVs of the same 2M-row matrix ({el:.1f} s, "
                      f"row ranges balanced by nnz over {threads} threads)"}


def make_matrix():
    from clsparse_b200 import matgen
    return matgen.irregular(2_000_000, mu=2.5, sigma=1.2, n_dense=50, dense_len=200_000, seed=7)


def run_reference(args, rank, world):
    if rank != 0:
        return
    rp, col, val = make_matrix()
    import oracle
    n = len(rp) - 1
    threads = os.cpu_count() or 1
    x = np.random.default_rng(3).uniform(-1, 1, n)
    y = np.zeros(n)
    nbytes = 4 * (len(col) + n) + 8 * (len(col) + 2 * n)
    for _ in range(max(args.warmup, 1)):
        oracle.dcsrmv_mt(rp, col, val, 1.0, x, 0.0, y, threads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        oracle.dcsrmv_mt(rp, col, val, 1.0, x, 0.0, y, threads)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    gbs = nbytes * args.steps / total / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": round(gbs, 3), "unit": "GB/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1e3 * total / args.steps, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": WORKLOAD, "nnz": int(len(col)), "rows": n, "bytes_per_step": nbytes},
        "cpu_baseline": {"value": round(gbs, 3), "unit": "GB/s", "cores": threads, "kind": "port",
                         "sample": f"{args.steps} full FP64 SpMVs (oracle restatement of the reference "
                                   "algorithm; the reference's OpenCL path has no runtime here)"},
        "e2e": {"value": round(gbs, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist

    from clsparse_b200 import api

    torch.cuda.set_device(local_rank)
    rp, col, val = make_matrix()
    n = len(rp) - 1
    nnz = len(col)
    nbytes = 4 * (nnz + n) + 8 * (nnz + n + n)

    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        ctrl = api.Control(stream)
        A = api.CsrMatrix.from_numpy(rp, col, val, dtype=torch.float64)
        A.create_meta(ctrl)
        ctrl.enable_async(True)
        x = torch.tensor(np.random.default_rng(3).uniform(-1, 1, n), device="cuda")
        y = torch.zeros(n, dtype=torch.float64, device="cuda")
        one = torch.ones(1, dtype=torch.float64, device="cuda")
        zero = torch.zeros(1, dtype=torch.float64, device="cuda")

        def step():
            api.csrmv(one, A, x, zero, y, ctrl)

        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        sampler = ClockSampler(local_rank)
        sampler.start()
        time.sleep(0.3)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(args.steps)]
        t_all0 = torch.cuda.Event(enable_timing=True)
        t_all1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        t_all0.record(stream)
        for s, e in ev:
            s.record(stream)
            step()
            e.record(stream)
        t_all1.record(stream)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        per = [s.elapsed_time(e) for s, e in ev]
        total_ms = t_all0.elapsed_time(t_all1)

        # end to end through the C ABI with host buffers: H2D x, SpMV, D2H y
        hx = torch.empty(n, dtype=torch.float64, pin_memory=True)
        hx.copy_(x.cpu())
        hy = torch.empty(n, dtype=torch.float64, pin_memory=True)
        for _ in range(3):
            x.copy_(hx, non_blocking=True)
            step()
            hy.copy_(y, non_blocking=True)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            x.copy_(hx, non_blocking=True)
            step()
            hy.copy_(y, non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_ms = e0.elapsed_time(e1)
        clocks = sampler.stop()

    t = torch.tensor([total_ms, e2e_ms, float(np.mean(per))], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms, e2e_ms, avg_launch_ms = t.tolist()
    if rank != 0:
        ctrl.release()
        return
    value = nbytes * args.steps * world / (total_ms * 1e-3) / 1e9
    e2e_val = nbytes * args.steps * world / (e2e_ms * 1e-3) / 1e9
    achieved = nbytes / (avg_launch_ms * 1e-3) / 1e9
    peak, peak_kind = measured_peak()
    tr = ncu_traffic()
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 5), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": WORKLOAD, "rows": n, "nnz": nnz, "bytes_per_step": nbytes,
                   "l2": "inputs larger than L2 (~760 MB streamed per step)",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                     "traffic": (tr or {}).get("dram_bytes_per_launch"),
                     "algorithmic_bytes_per_launch": nbytes,
                     "kernel": "csr_adaptive_kernel<double,false,0>"},
        "e2e": {"value": round(e2e_val, 2), "unit": "GB/s", "h2d_bytes_per_step": 8 * n,
                "d2h_bytes_per_step": 8 * n},
        "gpu_launches": args.steps,
        "clocks": clocks,
        "gflops": round(2 * nnz * args.steps * world / (total_ms * 1e-3) / 1e9, 2),
    }
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(rp, col, val)
    print(json.dumps(line), flush=True)
    ctrl.release()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    import torch.distributed as dist
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
