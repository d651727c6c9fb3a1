"""Workloads of bench.py: seeded synthetic inputs built on the device, one
timed step per batch, the end-to-end host path, and the CPU baseline.

The CPU baseline runs the reference's own host code (oracle/_ref, the
reference sources compiled in place) where that library exists, else the
oracle restatement; both are test infrastructure and are only timed here,
never used by the measured GPU path.
"""
from __future__ import annotations

import os
import platform
import threading
import time

import numpy as np

from . import _lib
from . import workloads as wl

# The reference's cost convention for multiple-double operations
# (Matrices/write_dbl2_qrtimeflops.cpp:51-61, write_dbl4_bstimeflops.cpp:31-61):
# double-double add 20 flops, mul 23; quad-double add 89, mul 336; a complex
# product costs four real ones (Newton/dbl2_systems_kernels.cu:29-37).
MD_ADD = {1: 1, 2: 20, 4: 89}
MD_MUL = {1: 1, 2: 23, 4: 336}


def conv_flops(deg, prec, cplx):
    n1 = deg + 1
    muls = n1 * (n1 + 1) // 2
    adds = deg * n1 // 2
    f = muls * MD_MUL[prec] + adds * MD_ADD[prec]
    return 4 * f if cplx else f


def evaldiff_counts(nvr, exps):
    """(convolutions, series additions) of the common-factor + forward /
    backward / cross evaluation of each monomial."""
    nvr = np.asarray(nvr)
    excess = np.clip(np.asarray(exps) - 1, 0, None).sum(axis=1)
    speel = np.where(nvr == 1, 1, np.where(nvr == 2, 3, 3 * nvr - 3))
    return int((excess + speel).sum()), int((nvr + 1).sum())


def cpu_info():
    model = platform.processor() or ""
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    model = ln.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return model, os.cpu_count() or 1


# --------------------------------------------------------------- eval
def config2_device(torch, dev, nsys=4096, dim=32, deg=31, nmon=32, maxvar=4, expmax=3, seed=2):
    """The 4096-system complex double-double eval/diff workload, generated on
    the device with a seeded torch generator (same distributions as
    workloads.eval_batch)."""
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    n1 = deg + 1
    total = nsys * dim * nmon
    nvr = torch.randint(1, maxvar + 1, (total,), generator=g, device=dev, dtype=torch.int32)
    idx = torch.empty((total, maxvar), dtype=torch.int32, device=dev)
    chunk = 1 << 18
    for c0 in range(0, total, chunk):
        c1 = min(total, c0 + chunk)
        r = torch.rand((c1 - c0, dim), generator=g, device=dev)
        pick = torch.argsort(r, dim=1)[:, :maxvar].to(torch.int32)
        k = nvr[c0:c1].unsqueeze(1)
        col = torch.arange(maxvar, device=dev).unsqueeze(0)
        big = torch.where(col < k, pick, torch.full_like(pick, 1 << 20))
        srt = torch.sort(big, dim=1).values
        idx[c0:c1] = torch.where(col < k, srt, torch.zeros_like(srt))
    exps = torch.randint(1, expmax + 1, (total, maxvar), generator=g, device=dev, dtype=torch.int32)
    col = torch.arange(maxvar, device=dev).unsqueeze(0)
    exps = torch.where(col < nvr.unsqueeze(1), exps, torch.zeros_like(exps))
    mon_off = torch.arange(0, total + 1, nmon, dtype=torch.int32, device=dev)

    def dd_pair(hi):
        lo = hi * (2.0 ** -53) * (torch.rand(hi.shape, generator=g, device=dev, dtype=torch.float64) * 2 - 1)
        s = hi + lo
        e = lo - (s - hi)
        return torch.stack([s, e], dim=-1)

    def unit(shape):
        th = torch.rand(shape, generator=g, device=dev, dtype=torch.float64) * (2 * np.pi)
        return torch.cat([dd_pair(torch.cos(th)), dd_pair(torch.sin(th))], dim=-1).reshape(-1)

    cff = unit((total, n1))
    cst = unit((nsys * dim, n1))
    scale = (2.0 ** -torch.arange(n1, device=dev, dtype=torch.float64))
    re = torch.randn((nsys * dim, n1), generator=g, device=dev, dtype=torch.float64) * scale
    im = torch.randn((nsys * dim, n1), generator=g, device=dev, dtype=torch.float64) * scale
    inp = torch.cat([dd_pair(re), dd_pair(im)], dim=-1).reshape(-1)
    return dict(nsys=nsys, dim=dim, deg=deg, maxvar=maxvar, prec=2, cplx=True, mon_off=mon_off, nvr=nvr, idx=idx,
                exps=exps, cst=cst, cff=cff, input=inp)


EVAL_WORKLOAD = ("eval/diff: 4096 systems, n=32, 32 monomials/polynomial over <=4 variables, exponents {1,2,3}, "
                 "unit-circle coefficients, degree 31, complex dd")


class EvalWork:
    metric = "systems/s, batched eval/diff of polynomial systems at power series (complex double-double)"
    unit = "systems/s"
    dtype = "f64 (complex double-double limbs)"
    kernel_tag = "k_system_evaldiff_config2"
    # DRAM bytes of one launch on the 4096 systems, from the ncu capture of
    # profiles/k_system_evaldiff_config2.md (512 systems, scaled by 8)
    traffic_bytes_per_launch = 1.0808e10
    l2_note = None
    dominant_launches_per_step = 1

    def __init__(self, torch, dev, rank, nsys=4096):
        self.torch = torch
        d = config2_device(torch, dev, nsys=nsys, seed=2 + rank)
        self.d = d
        S = (d["deg"] + 1) * 4
        self.out = torch.empty(d["nsys"] * d["dim"] * (d["dim"] + 1) * S, dtype=torch.float64, device=dev)
        self.units_per_step = d["nsys"]
        nconv, nadd = evaldiff_counts(d["nvr"].cpu().numpy(), d["exps"].cpu().numpy())
        self.dominant_flops_per_launch = float(nconv * conv_flops(d["deg"], 2, True)
                                               + nadd * (d["deg"] + 1) * 2 * MD_ADD[2])
        in_bytes = (d["cff"].numel() + d["cst"].numel() + d["input"].numel()) * 8
        self.dominant_bytes_per_launch = float(in_bytes + self.out.numel() * 8)
        self.flops_note = ("reference op weights: dd add 20, mul 23, complex x4 per convolution; "
                           f"{nconv} convolutions of degree {d['deg']} per step")
        self.config = {"workload": EVAL_WORKLOAD, "systems": d["nsys"], "dim": d["dim"], "degree": d["deg"]}
        self.host = None

    def _args(self, stream_ptr, out_ptr, host=None):
        d = self.d
        src = host if host is not None else d
        return (d["prec"], 1, d["nsys"], d["dim"], d["deg"], d["maxvar"], _lib.ptr(src["mon_off"]),
                _lib.ptr(src["nvr"]), _lib.ptr(src["idx"]), _lib.ptr(src["exps"]), _lib.ptr(src["cst"]),
                _lib.ptr(src["cff"]), _lib.ptr(src["input"]), _lib.ptr(out_ptr), _lib.c_void_p(stream_ptr))

    def step(self, stream):
        _lib.call("phc_system_evaldiff", *self._args(stream.cuda_stream, self.out))
        return 1

    def e2e(self, stream, reps=2):
        torch = self.torch
        if self.host is None:
            self.host = {k: (v.cpu().pin_memory() if hasattr(v, "cpu") else v) for k, v in self.d.items()}
            self.host_out = torch.empty(self.out.numel(), dtype=torch.float64).pin_memory()
        times = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            _lib.call("phc_system_evaldiff_host", *self._args(stream.cuda_stream, self.host_out, self.host))
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1) / 1e3)
        t = float(np.median(times))
        h2d = sum(v.numel() * v.element_size() for v in self.host.values() if hasattr(v, "numel"))
        return {"value": self.units_per_step / t, "unit": self.unit, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(self.host_out.numel() * 8), "path": "phc_system_evaldiff_host"}

    def check(self):
        """Spot check of the timed output against the oracle on 2 systems."""
        try:
            from oracle import pyoracle
            sb = self.sample_batch(2)
            ref = pyoracle.oracle().system_evaldiff(sb)
            S = (sb.deg + 1) * 4
            got = self.out[: 2 * sb.dim * (sb.dim + 1) * S].cpu().numpy()
            err = np.abs(got.reshape(-1, 4)[:, 0] - ref.reshape(-1, 4)[:, 0]).max()
            return {"oracle_systems": 2, "max_abs_hi_diff": float(err)}
        except Exception as e:  # the check never decides the number
            return {"error": str(e)[:200]}

    def sample_batch(self, n):
        d = self.d
        S = (d["deg"] + 1) * 4
        m = n * d["dim"] * 32
        g = lambda t, k: t[:k].cpu().numpy()
        return wl.SystemBatch(n, d["dim"], d["deg"], d["maxvar"], 2, True, g(d["mon_off"], n * d["dim"] + 1),
                              g(d["nvr"], m), g(d["idx"], m), g(d["exps"], m), g(d["cst"], n * d["dim"] * S),
                              g(d["cff"], m * S), g(d["input"], n * d["dim"] * S))


def make(name, dev, rank):
    import torch
    if name == "eval":
        return EvalWork(torch, dev, rank)
    if name == "track":
        from . import trackwork
        return trackwork.TrackWork(torch, dev, rank)
    if name == "qr":
        from . import qrwork
        return qrwork.QRWork(torch, dev, rank)
    raise ValueError(name)


def side_block(name, torch, dev, fp64_tflops, hbm_gbs, steps=3, warm=2):
    """A short timed run of another workload of the path (eval: the
    4096-system eval/diff; qr: the 512-instance quad-double least squares)
    for the track line: CUDA events around each launch, inputs resident,
    inputs larger than L2, and the workload's roofline."""
    from . import autotune
    work = make(name, dev, 0)
    stream = torch.cuda.Stream(device=dev)
    tuned = None
    if name == "eval":
        r = autotune.tune_eval_warps(torch, stream, work._args(stream.cuda_stream, work.out), work.d["dim"],
                                     key="config2")
        tuned = {"eval_warps_per_cta": r["choice"], "seconds": {str(k): round(v, 6) for k, v in r["seconds"].items()}}
    elif name == "qr":
        flag0 = torch.tensor([1, 0, 0, 0, 1], dtype=torch.int32, device=dev).repeat(work.ninst)
        r = autotune.tune_bals_tile(torch, stream, 4, False, work.ninst, 64, 32, work.mat, work.rhs0, work.sol,
                                    work.Q, work.R, work.flags, flag0, work.work, wy=work.wy, reps=1,
                                    cands=tuple(work.tiles))
        work.szt = r["choice"]
        tuned = {"szt": r["choice"], "stage_in_shared_memory": r["stage"] == 2,
                 "seconds": {str(k): round(v, 6) for k, v in r["seconds"].items()}}
    for _ in range(warm):
        work.step(stream)
    torch.cuda.synchronize()
    times = []
    for _ in range(steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        work.step(stream)
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1) / 1e3)
    t = float(np.mean(times))
    achieved = work.dominant_flops_per_launch / t / 1e12
    config = dict(work.config)
    if tuned is not None:
        config["autotuned"] = tuned
    out = {"metric": work.metric, "value": work.units_per_step / t, "unit": work.unit, "steps": steps,
           "ms_per_step": t * 1e3, "config": config,
           "roofline": {"bound": "fp64", "achieved": achieved, "peak": fp64_tflops, "unit": "TFLOP/s",
                        "frac": achieved / fp64_tflops, "flops_convention": work.flops_note,
                        "traffic": getattr(work, "traffic_bytes_per_launch", None),
                        "hbm_gbs_achieved": work.dominant_bytes_per_launch / t / 1e9, "hbm_peak_gbs": hbm_gbs}}
    try:
        out["check"] = work.check()
    except Exception as e:
        out["check"] = {"error": str(e)[:200]}
    del work
    autotune.reset()
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    return out


def newton_graph_block(torch, dev, nsteps=4, reps=20):
    """The power-series Newton method on the shapes of the plain double-double
    workload (one real system, n = 8, 8 monomials per polynomial over <= 3
    variables, exponents {1, 2}, degree 15; 4 steps at fixed working degree
    15, tile 8): a solve launched step by step against the same solve
    captured once in a CUDA graph and replayed (newton.DeviceNewton), CUDA
    events around each solve, median of reps; the replay's series must equal
    the launched solve's bit for bit."""
    from . import newton
    b = wl.eval_batch(11, 1, 8, 15, 8, 3, 2, False, expmax=2)
    dn = newton.DeviceNewton(b, szt=8, device=dev)
    stream = torch.cuda.Stream(device=dev)

    def timed(fn):
        ts = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        return float(np.median(ts))

    t_eager = timed(lambda: dn.solve(nsteps, stream))
    s_eager, _ = dn.result()
    dn.capture(nsteps, stream)
    t_graph = timed(lambda: dn.replay(stream))
    s_graph, _ = dn.result()
    return {"workload": "power-series Newton, one real double-double system n=8 (8 monomials over <=3 variables, "
                        "exponents {1,2}), degree 15, 4 steps at fixed degree 15, tile 8",
            "launched_ms_per_solve": t_eager, "graph_ms_per_solve": t_graph,
            "graph_speedup": t_eager / t_graph, "same_series": bool(np.array_equal(s_eager, s_graph, equal_nan=True))}


# ---------------------------------------------------------- CPU baseline
def _threads_run(fn, nitems, nthreads):
    """Run fn(i) for i < nitems on nthreads Python threads (ctypes calls
    release the GIL, so the C code runs in parallel)."""
    nxt = [0]
    lock = threading.Lock()

    def worker():
        while True:
            with lock:
                i = nxt[0]
                nxt[0] += 1
            if i >= nitems:
                return
            fn(i)

    ts = [threading.Thread(target=worker) for _ in range(nthreads)]
    t0 = time.perf_counter()
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    return time.perf_counter() - t0


def eval_cpu_sample(seconds):
    from oracle import pyoracle
    lib = pyoracle.reference()
    kind = "reference"
    if lib is None:
        lib, kind = pyoracle.oracle(), "port"
    model, cores = cpu_info()
    one = wl.config2(nsys=1, seed=99)
    t = time.perf_counter()
    lib.system_evaldiff(one)
    t1 = time.perf_counter() - t
    n = max(cores, int(seconds / max(t1, 1e-6) * cores * 0.8))
    n = min(n, 64 * cores)
    batches = [wl.config2(nsys=1, seed=1000 + i) for i in range(min(n, 4 * cores))]
    el = _threads_run(lambda i: lib.system_evaldiff(batches[i % len(batches)]), n, cores)
    return {"value": n / el, "unit": "systems/s", "cores": cores, "kind": kind,
            "sample": f"{n} systems of the 4096-system workload (same shapes, seeded), {cores} threads, "
                      f"CPU: {model}"}


def cpu_baseline(workload, seconds, extras=True):
    """extras (track): also the learned-step restatement and the calibration
    against the reference's host code."""
    try:
        if workload == "eval":
            return eval_cpu_sample(seconds)
        if workload == "track":
            from . import trackwork
            return trackwork.cpu_sample(seconds, extras=extras)
        if workload == "qr":
            from . import qrwork
            return qrwork.cpu_sample(seconds)
    except Exception as e:
        return {"value": None, "error": str(e)[:300]}
    return None


def reference_arm(args):
    """bench.py --impl reference: the reference's CPU host implementation of
    the path on this machine's cores, same metric and unit as the GPU arm."""
    vals = []
    res = None
    per = max(2.0, min(20.0, 120.0 / max(1, args.steps + args.warmup)))
    nall = args.warmup + args.steps
    for k in range(nall):
        res = cpu_baseline(args.workload, per, extras=(k == nall - 1))
        if k >= args.warmup and res and res.get("value"):
            vals.append(res["value"])
    v = float(np.median(vals)) if vals else None
    if args.workload == "track":
        from . import trackwork
        metric, unit, config = trackwork.TrackWork.metric, "paths/s", trackwork.static_config()
    elif args.workload == "qr":
        from . import qrwork
        metric, unit, config = qrwork.QRWork.metric, qrwork.QRWork.unit, qrwork.static_config()
    else:
        metric, unit, config = EvalWork.metric, EvalWork.unit, {"workload": EVAL_WORKLOAD}
    return {"impl": "reference", "metric": metric, "value": v, "unit": unit,
            "n_gpus": 0, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "cpu_baseline": dict(res or {}, value=v),
            "e2e": {"value": v, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "config": config}
