"""Benchmark of the multiple-double power-series path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload track|eval|qr]

Prints ONE JSON line (rank 0).  A step is one pass of the hot path over one
batch of seeded synthetic input that is already resident in HBM:
  track -- the batched path tracker on the dense-quadratic n=10 total-degree
           homotopy (1024 paths, degree-8 series + [4/4] Pade predictor,
           3 double-double corrector steps), metric paths/s;
  eval  -- batched eval/diff of 4096 complex double-double systems (n=32,
           32 monomials over <=4 variables, exponents {1,2,3}, degree 31),
           metric systems/s;
  qr    -- 512 quad-double 64x64 block-Toeplitz least-squares solves at
           degree 31, metric instances/s.
Under torchrun each rank runs its own copy of the workload (weak scaling,
no data-path collective: the units are independent); the time is the max
over ranks.  --impl reference times the reference's CPU host code on this
machine's cores (rank 0 only).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default=os.environ.get("PHC_BENCH_WORKLOAD", "track"),
                    choices=["track", "eval", "qr"])
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="budget of the CPU baseline sample")
    ap.add_argument("--no-blocks", action="store_true", help="track: leave out the eval and qr blocks")
    return ap.parse_args()


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["active", "hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names[1:], f[5:9]):
                if v.lower() in ("active", "0x1", "1"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return {}


def fp64_peak_tflops(torch, dev):
    """Dense FP64 throughput measured here: cuBLAS DGEMM 8192^3, best of 5."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    from phcpack_b200 import benchwork

    if args.impl == "reference":
        if rank != 0:
            return 0
        res = benchwork.reference_arm(args)
        print(json.dumps(res), flush=True)
        return 0

    import torch

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    work = benchwork.make(args.workload, dev, rank)
    stream = torch.cuda.Stream(device=dev)
    for _ in range(args.warmup):
        work.step(stream)
    torch.cuda.synchronize()

    clocks = ClockSampler(local)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    launches = 0
    t0.record(stream)
    for k in range(args.steps):
        ev[k][0].record(stream)
        launches += work.step(stream)
        ev[k][1].record(stream)
    t1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    if dist is not None:
        dist.barrier()
    total_s = t0.elapsed_time(t1) / 1e3
    kern_s = [ev[k][0].elapsed_time(ev[k][1]) / 1e3 for k in range(args.steps)]
    from phcpack_b200 import multirank
    total_s = multirank.max_over_ranks(total_s, dist)

    if hasattr(work, "finish"):
        work.finish()
    # end to end through the host entry point (pinned host buffers in, results out)
    e2e = work.e2e(stream, reps=max(3, min(9, args.steps)))
    # whole job: the units of all ranks over the slowest rank's time (every
    # rank takes part in the reduction)
    v = (e2e or {}).get("value") or 0.0
    t_e2e = multirank.max_over_ranks(work.units_per_step / v if v > 0 else float("inf"), dist)
    if e2e and v > 0:
        e2e["value"] = work.units_per_step * world / t_e2e
    check = work.check()

    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0

    units = work.units_per_step * args.steps * world
    value = units / total_s
    peaks = measured_peaks()
    fp64 = fp64_peak_tflops(torch, dev)
    mean_kernel = float(np.mean(kern_s)) / max(1, work.dominant_launches_per_step)
    achieved = work.dominant_flops_per_launch / mean_kernel / 1e12
    traffic = getattr(work, "traffic_bytes_per_launch", None)
    cpu = benchwork.cpu_baseline(args.workload, args.cpu_seconds) if (world == 1 or rank == 0) else None
    out = {
        "metric": work.metric,
        "value": value,
        "unit": work.unit,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": total_s / args.steps * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": work.dtype,
        "data": "synthetic (seeded)",
        "config": dict(work.config, l2="inputs larger than L2" if work.l2_note is None else work.l2_note),
        "roofline": {"bound": "fp64", "achieved": achieved, "peak": fp64, "unit": "TFLOP/s",
                     "frac": achieved / fp64, "traffic": traffic,
                     "peak_source": "measured here: cuBLAS DGEMM 8192^3 (MEASURED_PEAKS.json has no FP64 figure)",
                     "flops_convention": work.flops_note,
                     "hbm_gbs_achieved": work.dominant_bytes_per_launch / mean_kernel / 1e9,
                     "hbm_peak_gbs": peaks.get("hbm_gbs")},
        "e2e": e2e,
        "gpu_launches": launches,
        "cpu_baseline": cpu,
        "clocks": clk,
        "check": check,
    }
    if args.workload == "track" and not args.no_blocks and world == 1:
        out["blocks"] = {name: benchwork.side_block(name, torch, dev, fp64, peaks.get("hbm_gbs"))
                         for name in ("eval", "qr")}
        try:
            out["blocks"]["newton_graph"] = benchwork.newton_graph_block(torch, dev)
        except Exception as e:  # the block is informational; the line stands without it
            out["blocks"]["newton_graph"] = {"error": str(e)[:200]}
    print(json.dumps(out), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
