"""bench.py workload 'qr': 512 block lower-triangular Toeplitz least-squares
problems in quad-double, 64 x 64 Jacobian blocks, degree 31 (32 blocks),
tile 32: the blocked Householder QR of A_0 (WY trailing products on the FP64
tensor cores by Ozaki splitting) and the tail of 31 stages.  Entries of
A_k: leading limb N(0,1), lower limbs random at 2^-53 relative scale.
Metric instances/s; the CUDA-core WY variant is timed beside it.
"""
from __future__ import annotations

import time

import numpy as np

from . import _lib
from . import dense
from .benchwork import MD_ADD, MD_MUL, _threads_run, cpu_info

NINST, DIM, DEGP1, SZT, PREC = 512, 64, 32, 32, 4


def static_config():
    return {"workload": "block-Toeplitz least squares: 512 instances, 64x64 quad-double blocks, degree 31, "
                        "tile 32, WY products as Ozaki-split FP64 tensor-core products",
            "instances": NINST, "dim": DIM, "degree": DEGP1 - 1, "tile": SZT}


def bals_flops(n=DIM, degp1=DEGP1, prec=PREC):
    """Algorithmic work per instance with the reference's weights (qd mul 336,
    add 89): QR with explicit Q, 8/3 n^3 multiply-adds; the tail
    sum_s (d+1-s) n^2; Q^T b and back substitution d (n^2 + n^2/2)."""
    d = degp1 - 1
    ma = (8.0 / 3.0) * n ** 3 + (d * (d + 1) / 2) * n * n + d * 1.5 * n * n
    return ma * (MD_MUL[prec] + MD_ADD[prec])


def make_inputs(torch, dev, seed, ninst=NINST):
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    f64 = dict(dtype=torch.float64, device=dev)

    def qd(shape):
        hi = torch.randn(shape, generator=g, **f64)
        limbs = [hi]
        for _ in range(3):
            limbs.append(limbs[-1] * (2.0 ** -53) * (torch.rand(shape, generator=g, **f64) * 2 - 1))
        # renormalise each (hi, lo) pair from the bottom
        for i in range(3, 0, -1):
            s = limbs[i - 1] + limbs[i]
            e = limbs[i] - (s - limbs[i - 1])
            limbs[i - 1], limbs[i] = s, e
        return torch.stack(limbs, dim=-1).reshape(-1)

    mat = qd((ninst, DEGP1, DIM, DIM))
    rhs = qd((ninst, DEGP1, DIM))
    return mat, rhs


class QRWork:
    metric = "instances/s, quad-double block-Toeplitz least squares (64x64 blocks, degree 31)"
    unit = "instances/s"
    dtype = "f64 (quad-double limbs, real)"
    kernel_tag = "k_bals_solve_qd64"
    # DRAM bytes of one launch on the 512 instances, from the ncu capture of
    # profiles/k_bals_solve_qd64.md (scaled to 512 instances)
    traffic_bytes_per_launch = 2.5731e9
    dominant_launches_per_step = 1
    l2_note = "inputs (2.1 GB of A_k) larger than L2"

    def __init__(self, torch, dev, rank, ninst=NINST, wy=1):
        self.torch = torch
        self.ninst, self.wy = ninst, wy
        self.mat, self.rhs0 = make_inputs(torch, dev, 3 + rank, ninst)
        f64 = dict(dtype=torch.float64, device=dev)
        self.rhs = torch.empty_like(self.rhs0)
        self.sol = torch.zeros(ninst * DEGP1 * DIM * PREC, **f64)
        self.Q = torch.zeros(ninst * DIM * DIM * PREC, **f64)
        self.R = torch.zeros(ninst * DIM * DIM * PREC, **f64)
        self.flags = torch.zeros(ninst * 5, dtype=torch.int32, device=dev)
        self.flag0 = torch.tensor([1, 0, 0, 0, 1], dtype=torch.int32, device=dev).repeat(ninst)
        # workspace for every tile size the autotuner may pick
        self.tiles = [t for t in (8, 16, 32, 64) if DIM % t == 0]
        nb = max(dense.workspace_bytes_wy(PREC, False, DIM, t, w) for t in self.tiles for w in (0, 1))
        self.work = torch.zeros(ninst * nb // 8, **f64)
        self.szt = SZT
        self.units_per_step = ninst
        self.dominant_flops_per_launch = bals_flops() * ninst
        self.dominant_bytes_per_launch = float(self.mat.numel() * 8)
        self.flops_note = "reference weights qd mul 336 add 89; QR 8/3 n^3, tail d(d+1)/2 n^2, solves 1.5 d n^2"
        self.config = static_config()

    def step(self, stream, wy=None):
        wy = self.wy if wy is None else wy
        with self.torch.cuda.stream(stream):
            self.rhs.copy_(self.rhs0)
            self.flags.copy_(self.flag0)
        _lib.call("phc_bals_solve_wy", PREC, 0, self.ninst, DIM, DEGP1, self.szt, 1, _lib.ptr(self.mat),
                  _lib.ptr(self.rhs), _lib.ptr(self.sol), _lib.ptr(self.Q), _lib.ptr(self.R), _lib.ptr(self.flags),
                  _lib.ptr(self.work), int(wy), _lib.c_void_p(stream.cuda_stream))
        return 1

    def e2e(self, stream, reps=2):
        torch = self.torch
        mat_h = self.mat.cpu().numpy()
        rhs_h = self.rhs0.cpu().numpy()
        times = []
        for _ in range(reps):
            t0 = time.perf_counter()
            sol, _, _, _, fl = dense.bals_solve_host(PREC, False, mat_h, rhs_h, self.ninst, DIM, DEGP1, SZT)
            times.append(time.perf_counter() - t0)
        t = float(np.median(times))
        return {"value": self.ninst / t, "unit": self.unit, "h2d_bytes_per_step": int(mat_h.nbytes + rhs_h.nbytes),
                "d2h_bytes_per_step": int(sol.nbytes), "path": "phc_bals_solve_host (CUDA-core WY products), "
                "wall clock"}

    def check(self):
        torch = self.torch
        s = torch.cuda.Stream(device=self.mat.device)
        x1 = self.sol.clone()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        self.step(s, wy=0)
        e1.record(s)
        e1.synchronize()
        t0 = e0.elapsed_time(e1) / 1e3
        x0 = self.sol.clone()
        # leading limbs, per (instance, degree) block relative to max(1, |x|):
        # the solutions of these random systems grow by orders of magnitude
        # with the degree
        a = x1.view(self.ninst * DEGP1, DIM, PREC)[..., 0]
        b = x0.view(self.ninst * DEGP1, DIM, PREC)[..., 0]
        rel = ((a - b).abs().amax(dim=1) / b.abs().amax(dim=1).clamp(min=1.0)).max().item()
        return {"cuda_core_wy_instances_per_s": self.ninst / t0,
                "max_rel_diff_vs_cuda_core_per_block_lead_limb": float(rel)}


def cpu_sample(seconds):
    """The reference's own CPU_dbl4_qrbs_solve (oracle/_ref) on a sample of
    instances, all host cores."""
    from oracle import pyoracle
    lib = pyoracle.reference()
    kind = "reference"
    if lib is None:
        lib, kind = pyoracle.oracle(), "port"
    model, cores = cpu_info()
    rng = np.random.default_rng(7)
    from . import workloads as wl
    mat = wl.random_numbers(rng, (DEGP1, DIM, DIM), PREC, False, "normal")
    rhs = wl.random_numbers(rng, (DEGP1, DIM), PREC, False, "normal")
    t = time.perf_counter()
    lib.bals_solve(PREC, False, DIM, DEGP1, 1, mat, rhs)
    t1 = time.perf_counter() - t
    n = int(max(cores, min(4 * cores * 8, seconds / max(t1, 1e-6) * cores * 0.8)))
    el = _threads_run(lambda i: lib.bals_solve(PREC, False, DIM, DEGP1, 1, mat, rhs), n, cores)
    return {"value": n / el, "unit": "instances/s", "cores": cores, "kind": kind,
            "sample": f"{n} instances (64x64 qd, degree 31), {cores} threads, CPU_dbl4_qrbs_solve, CPU: {model}"}
