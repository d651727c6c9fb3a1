"""bench.py workload 'track': path tracking on the 1024-path dense quadratic
homotopy (n = 10, unit-circle coefficients, total-degree start system,
random complex gamma), degree-8 series, [4/4] Pade, 3 double-double
corrector steps, endpoints refined in double-double.

The measured arm is the batched persistent tracker with the FP64 predictor
and the double-double corrector, using the learned step proposer when a
trained model is available (phcpack_b200/models/step_mlp.npz).  Next to it
the same run is timed as the plain arrangement: all double-double, one path
per launch.
"""
from __future__ import annotations

import os
import time

import numpy as np

from . import _lib
from . import homotopy as hm
from .benchwork import MD_ADD, MD_MUL, _threads_run, cpu_info

MODEL_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "models", "step_mlp.npz")


DEFAULT_K = hm.DEFAULT_IPAR["deg"]


def load_model_bytes():
    if not os.path.exists(MODEL_PATH):
        return None
    with np.load(MODEL_PATH) as z:
        return np.ascontiguousarray(z["model"])


def track_flops(pb: hm.TrackProblem, steps, rejected, pmode=1):
    """Algorithmic work of the tracked paths, a count of complex
    multiply-adds per phase weighted with the reference's convention
    (double-double add 20, mul 23; double 1 and 1; complex product = 4
    multiplications + 2 additions, accumulation 2 additions):
      predictor (Taylor series to degree K, in the predictor's precision):
        the values and Jacobian at the point, the LU of J_0 (n^3/3) and its
        inverse (2 n^3/3); per degree k = 1..K the coefficients k-1 and k of
        every distinct monomial (2k + 1 products for a product of two
        series), the coefficient gathers of the values (2 per term) and the
        product with J_0^{-1} (n^2);
      predictor feedback: one point evaluation of the values;
      corrector: 2 Newton iterations, each a point evaluation of the values
        in double-double and of the Jacobian, its LU (n^3/3) and solve (n^2)
        in the predictor's precision;
      a rejected step costs one feedback and one corrector.
    Returns the total."""
    n = pb.maxdim
    nmono = pb.nmono_max
    nterm = int(np.diff(pb.term_off).mean())
    njg = 2 * nterm  # Jacobian gather entries per equation (quadratic monomials)
    K = DEFAULT_K

    def cma(prec):  # flops of one complex multiply-add in precision prec
        return 4 * MD_MUL[prec] + 4 * MD_ADD[prec]

    v0 = nmono + 2 * n * nterm  # values at a point
    j0 = 2 * n * njg  # Jacobian at a point
    pred = v0 + j0 + n ** 3 + sum(nmono * (2 * k + 1) + 2 * n * nterm + n * n for k in range(1, K + 1))
    pred *= cma(pmode)
    feed = v0 * cma(pmode)
    corr = 2 * (v0 * cma(2) + (j0 + n ** 3 / 3 + n * n) * cma(pmode))
    steps = np.asarray(steps, dtype=np.float64)
    rej = np.asarray(rejected, dtype=np.float64)
    total = float((steps * (pred + feed + corr) + rej * (feed + corr)).sum())
    return total


def static_config(npaths=1024, learned=None, note=None):
    """The benchmark configuration, shared by the GPU and the reference arm."""
    if learned is None:
        learned = os.path.exists(MODEL_PATH)
    if note is None:
        note = hm.config4().note
    return {"workload": "path tracking: dense quadratic n=10, 1024 total-degree paths, degree-8 series, "
                        "[4/4] Pade, 3 dd corrector steps, dd endpoint refinement",
            "paths": npaths, "dim": 10, "predictor": "fp64", "corrector": "double-double",
            "step": "learned (MLP) with plain fallback" if learned else "plain pole step", "system": note}


class TrackWork:
    metric = ("paths/s at endpoint residual <= 1e-24 (double-double), batched + precision-split"
              " + learned-step tracker, 1024-path dense quadratic homotopy")
    unit = "paths/s"
    dtype = "f64 predictor + double-double corrector (complex)"
    kernel_tag = "k_track_config4"
    # DRAM bytes of one launch on the 1024 paths, from the ncu capture of
    # profiles/k_track_config4.md (dram__bytes_read.sum + dram__bytes_write.sum)
    traffic_bytes_per_launch = 5.716e5
    dominant_launches_per_step = 1

    def __init__(self, torch, dev, rank, npaths=1024, tune=True):
        self.torch = torch
        pb = hm.config4(seed=4 + rank)
        if npaths < pb.npaths:
            pb = hm.subset(pb, np.arange(npaths))
        self.pb = pb
        self.dt = hm.DeviceTracker(pb, device=dev)
        self.model = load_model_bytes()
        self.step_mode = 1 if self.model is not None else 0
        if self.model is not None:
            self.dt.set_model(self.model)
        self.units_per_step = pb.npaths
        self.l2_note = "working set (systems, paths, endpoints) < L2; the step is latency bound, not memory bound"
        self.config = static_config(pb.npaths, learned=bool(self.step_mode), note=pb.note)
        self.flops_note = None
        self.dominant_flops_per_launch = 0.0
        self.dominant_bytes_per_launch = float(pb.npaths * pb.maxdim * (16 + 64))
        # the kernel variant of the split tracker, timed on this batch
        if tune:
            from . import autotune
            stream = torch.cuda.Stream(device=dev)
            tv = autotune.tune_track_variant(torch, stream, self.dt, reps=2, pmode=1, rmode=2,
                                             step_mode=self.step_mode)
            self.config["autotuned"] = {"track_variant": tv["choice"], "paths_per_sm": tv["per_sm"],
                                        "seconds": {str(k): round(v, 6) for k, v in tv["seconds"].items()}}

    def step(self, stream):
        self.dt.run(pmode=1, rmode=2, step_mode=self.step_mode, stream=stream)
        return 1

    def finish(self):
        """After the timed steps: per-path counters of the last run give the
        algorithmic flops per launch."""
        r = self.dt.result()
        self.last = r
        self.dominant_flops_per_launch = track_flops(self.pb, r.steps, r.rejected, pmode=1)
        self.flops_note = ("modelled complex multiply-adds per phase (trackwork.track_flops), reference weights "
                           "dd add 20 mul 23, double 1; from the launch's own step and rejection counts")
        return r

    def e2e(self, stream, reps=3):
        torch = self.torch
        times = []
        hm.track_host(self.pb, pmode=1, rmode=2, step_mode=self.step_mode, model=self.model,
                      stream_ptr=stream.cuda_stream)  # warm-up call, untimed
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            r = hm.track_host(self.pb, pmode=1, rmode=2, step_mode=self.step_mode, model=self.model,
                              stream_ptr=stream.cuda_stream)
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1) / 1e3)
        t = float(np.median(times))
        pb = self.pb
        h2d = (pb.dim.nbytes + pb.mono_off.nbytes + pb.mono_nvr.nbytes + pb.mono_idx.nbytes + pb.mono_exp.nbytes
               + pb.eq_off.nbytes + pb.term_off.nbytes + pb.term_mono.nbytes + pb.term_a.nbytes + pb.term_b.nbytes
               + pb.path_sys.nbytes + pb.x0.nbytes)
        d2h = pb.npaths * (pb.maxdim * 64 + 4 * hm.INFO_WORDS + 16)
        return {"value": pb.npaths / t, "unit": self.unit, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "path": "phc_track_host",
                "success": int((r.status == 0).sum())}

    def timed(self, dt, stream, reps=3, **kw):
        """Median CUDA-event seconds of `reps` batched launches of dt.run(**kw)
        after one untimed launch; returns (seconds, result)."""
        torch = self.torch
        dt.run(stream=stream, **kw)
        times = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            dt.run(stream=stream, **kw)
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1) / 1e3)
        return float(np.median(times)), dt.result()

    @staticmethod
    def summary(npaths, t, r):
        ok = r.status == 0
        return {"paths_per_s": npaths / t, "ms": t * 1e3, "success": int(ok.sum()),
                "max_residual_success": float(r.residual[ok].max()) if ok.any() else None,
                "mean_steps": float(r.steps.mean()), "max_steps": int(r.steps.max()),
                "rejected": int(r.rejected.sum()), "steps_pole_curvature_maxsize":
                    [int(r.nbpole.sum()), int(r.nbhess.sum()), int(r.nbmaxm.sum())]}

    def plain(self, stream):
        """The plain arrangement: all double-double, plain step, one path
        per launch."""
        torch = self.torch
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        self.dt.run(pmode=2, rmode=2, step_mode=0, one_per_launch=True, stream=stream)  # warm
        torch.cuda.synchronize()
        e0.record(stream)
        self.dt.run(pmode=2, rmode=2, step_mode=0, one_per_launch=True, stream=stream)
        e1.record(stream)
        e1.synchronize()
        t = e0.elapsed_time(e1) / 1e3
        r = self.dt.result()
        return t, r

    def ablation(self, stream):
        """The three patterns apart on the same 1024 paths, each batched:
        all double-double with the plain step, the precision split with the
        plain step, the precision split with the learned step (the measured
        arm), the measured arm with the predictor's J_0 inverted by
        Householder QR instead of LU, and the plain one-path-per-launch
        all-dd arrangement."""
        n = self.pb.npaths
        out = {}
        t, r = self.timed(self.dt, stream, pmode=2, rmode=2, step_mode=0)
        out["batched_all_dd_plain_step"] = self.summary(n, t, r)
        t, r = self.timed(self.dt, stream, pmode=1, rmode=2, step_mode=0)
        out["batched_split_plain_step"] = self.summary(n, t, r)
        plain_split = r
        if self.step_mode:
            t, r = self.timed(self.dt, stream, pmode=1, rmode=2, step_mode=1)
            out["batched_split_learned_step"] = self.summary(n, t, r)
            out["batched_split_learned_step"]["same_classification_as_plain"] = bool(
                np.array_equal(r.status == 0, plain_split.status == 0))
        # the predictor's J_0 by Householder QR instead of LU (step_mode bit 2)
        t, r = self.timed(self.dt, stream, pmode=1, rmode=2, step_mode=2 | (1 if self.step_mode else 0))
        key = "batched_split_qr_predictor_" + ("learned_step" if self.step_mode else "plain_step")
        out[key] = dict(self.summary(n, t, r), same_classification_as_plain=bool(
            np.array_equal(r.status == 0, plain_split.status == 0)))
        tp, rp = self.plain(stream)
        out["plain_one_path_per_launch"] = dict(self.summary(n, tp, rp), same_classification=bool(
            np.array_equal(rp.status == 0, plain_split.status == 0)))
        return out

    def config5(self, stream):
        """The mixed-size workload: 64 sparse quadratic systems, n in 6..14,
        total-degree paths capped at 256 per system, learned step (when a
        model is present), quad-double endpoint refinement; classification
        against the plain step."""
        pb = hm.config5()
        dt = hm.DeviceTracker(pb, device=self.dt.xend.device)
        out = {"workload": pb.note, "paths": pb.npaths, "dims": [int(pb.dim.min()), int(pb.dim.max())]}
        t0, r0 = self.timed(dt, stream, reps=2, pmode=1, rmode=4, step_mode=0)
        out["plain_step"] = self.summary(pb.npaths, t0, r0)
        if self.step_mode:
            dt.set_model(self.model)
            t1, r1 = self.timed(dt, stream, reps=2, pmode=1, rmode=4, step_mode=1)
            out["learned_step"] = self.summary(pb.npaths, t1, r1)
            out["learned_step"]["same_classification_as_plain"] = bool(np.array_equal(r1.status == 0,
                                                                                      r0.status == 0))
        return out

    def endpoint_errors(self, npaths=16):
        """The error of each result against FP64 and octo-double: end points
        of a sample of paths against an octo-double run of the host oracle
        (same step rule; od refinement), for the GPU's double-double end
        points and for an FP64 run of the same tracker on the host (all
        double, corrector included)."""
        from oracle import pyoracle
        lib = pyoracle.oracle()
        sub = hm.subset(self.pb, np.arange(0, self.pb.npaths, self.pb.npaths // npaths)[:npaths])
        ipar, dpar = hm.params()
        g = hm.track_host(sub, pmode=1, rmode=2)
        x8, i8, _ = pyoracle.track(lib, sub, ipar, dpar, pmode=1, rmode=8, nthreads=npaths)
        _, dp64 = hm.params(restol=1e-12)
        x1, i1, _ = pyoracle.track(lib, sub, ipar, dp64, pmode=1, rmode=1, nthreads=npaths)
        md = sub.maxdim

        def err(xq, limbs_q):
            a = xq.reshape(-1, md, 2, limbs_q)
            b = x8.reshape(-1, md, 2, 8)
            d = np.zeros(a.shape[:3])
            for l in range(limbs_q - 1, -1, -1):
                d = d + (a[..., l] - b[..., l])
            d = d + (-b[..., limbs_q:].sum(axis=-1))
            mag = np.maximum(1.0, np.abs(b[..., 0]).max(axis=(1, 2)))
            return float((np.abs(d).max(axis=(1, 2)) / mag).max())
        ok = (g.status == 0) & (i8.reshape(-1, 6)[:, 0] == 0)
        return {"paths": int(sub.npaths), "all_succeeded": bool(ok.all()),
                "max_rel_error_vs_od_oracle": {"gpu_double_double": err(g.xend, 4),
                                               "host_fp64_run": err(x1, 4)}}

    def check(self):
        torch = self.torch
        out = {}
        r = getattr(self, "last", None) or self.dt.result()
        ok = r.status == 0
        out["success"] = int(ok.sum())
        out["max_residual_success"] = float(r.residual[ok].max()) if ok.any() else None
        out["mean_steps"] = float(r.steps.mean())
        out["rejected"] = int(r.rejected.sum())
        s = torch.cuda.Stream(device=self.dt.xend.device)
        out["ablation"] = self.ablation(s)
        try:
            out["config5"] = self.config5(s)
        except Exception as e:  # a side block never decides the headline
            out["config5"] = {"error": str(e)[:200]}
        try:
            out["endpoint_errors"] = self.endpoint_errors()
        except Exception as e:
            out["endpoint_errors"] = {"error": str(e)[:200]}
        return out


def cpu_sample(seconds, extras=True):
    """The CPU tracker (oracle restatement of the Ada series-Pade tracker) on
    a sample of the 1024 paths, all host cores; with extras also the same
    sample with the learned step and port_calibration()."""
    from oracle import pyoracle
    model, cores = cpu_info()
    pb = hm.config4()
    ipar, dpar = hm.params()
    lib = pyoracle.oracle()
    t = time.perf_counter()
    one = hm.subset(pb, [0])
    pyoracle.track(lib, one, ipar, dpar, pmode=1, rmode=2, nthreads=1)
    t1 = time.perf_counter() - t
    n = int(min(pb.npaths, max(cores, seconds / max(t1, 1e-6) * cores * 0.8)))
    sub = hm.subset(pb, np.arange(n))
    t = time.perf_counter()
    _, info, _ = pyoracle.track(lib, sub, ipar, dpar, pmode=1, rmode=2, nthreads=cores)
    el = time.perf_counter() - t
    ok = int((info.reshape(-1, 6)[:, 0] == 0).sum())
    out = {"value": n / el, "unit": "paths/s", "cores": cores, "kind": "port",
           "sample": f"{n} of the 1024 paths, {ok} successful, {cores} threads (std::thread), CPU: {model}; the "
                     "reference's tracker is Ada (no GNAT here), so this is the C++ restatement"}
    # the same restatement with the learned step (the GPU arm's algorithm):
    # the ratio of the GPU arm to this one is the hardware alone
    if not extras:
        return out
    mdl = load_model_bytes()
    if mdl is not None:
        t = time.perf_counter()
        _, info, _ = pyoracle.track(lib, sub, ipar, dpar, pmode=1, rmode=2, nthreads=cores, step_mode=1, model=mdl)
        el = time.perf_counter() - t
        out["learned_step_paths_per_s"] = n / el
    cal = port_calibration()
    if cal is not None:
        out["calibration"] = cal
    return out


def port_calibration(reps=3):
    """How fast the restatement's host code runs against PHCpack's own host
    code on the same work: one complex double-double system of the eval/diff
    workload (n = 32, degree 31) evaluated and differentiated by the oracle
    (oracle/oracle_core.hpp, the code the CPU tracker is built on) and by the
    reference's CPU_cmplx2_ routines (oracle/_ref), one thread each, best of
    reps.  None where the reference's host code was not built."""
    from oracle import pyoracle
    from . import workloads as wl
    ref = pyoracle.reference()
    if ref is None:
        return None
    port = pyoracle.oracle()
    b = wl.config2(nsys=1, seed=77)

    def best(lib):
        ts = []
        for _ in range(reps):
            t = time.perf_counter()
            lib.system_evaldiff(b)
            ts.append(time.perf_counter() - t)
        return min(ts)

    tp, tr = best(port), best(ref)
    return {"work": "eval/diff of one complex double-double system (n=32, 32 monomials per polynomial, degree 31), "
                    "one thread", "port_s": tp, "reference_s": tr, "port_time_over_reference_time": tp / tr}
