"""Host mirror of the Newton layer: Newton's method on power series.

Mirrors PHCpack's ``dbl2_row_newton_qrstep`` (src/GPU/Newton/
dbl2_newton_method.cpp:429) and the step loop of ``test_dbl2_row_newton``
(:1455-1492), batched over systems.  A system is given as a
``workloads.SystemBatch``; its ``input`` holds the start series.
"""
from __future__ import annotations

import numpy as np

from . import _lib
from .workloads import SystemBatch


def newton_host(b: SystemBatch, nsteps: int, szt: int | None = None, schedule: int = 0):
    """Run Newton on every system of b; returns (series, flags) with flags
    (zeroQ, noqr, upidx, bsidx, tailidx) per system."""
    b.validate()
    szt = b.dim if szt is None else szt
    ser = np.array(b.input, dtype=np.float64, copy=True)
    flags = np.zeros(5 * b.nsys, np.int32)
    _lib.call("phc_newton_host", b.prec, int(b.cplx), b.nsys, b.dim, b.deg, szt, b.maxvar, _lib.ptr(b.mon_off),
              _lib.ptr(b.nvr), _lib.ptr(b.idx), _lib.ptr(b.exps), _lib.ptr(b.cst), _lib.ptr(b.cff), _lib.ptr(ser),
              nsteps, schedule, _lib.ptr(flags), _lib.c_void_p(0))
    return ser, flags


class DeviceNewton:
    """A batch of systems resident on the device for repeated Newton solves at
    a fixed working degree: each step is phc_newton_step (evaluate and
    differentiate, linearise, block-Toeplitz least squares, update; four
    launches and a memset, all on one stream, no host synchronisation), and
    the steps of one solve, from the start series on, can be captured once in
    a CUDA graph and replayed: one graph launch per solve instead of five
    launches per step.  The start series and the skip-rule flags (zeroQ = 1,
    noqr = 0, tail index 1, as phc_newton_host starts them) are restored on
    the device at the start of every solve."""

    def __init__(self, b: SystemBatch, szt: int | None = None, device="cuda"):
        import torch
        b.validate()
        self.torch = torch
        self.b = b
        self.szt = b.dim if szt is None else szt
        dev = torch.device(device)

        def t(a):
            return torch.from_numpy(np.ascontiguousarray(a)).to(dev)

        self.mon_off, self.nvr, self.idx, self.exps = t(b.mon_off), t(b.nvr), t(b.idx), t(b.exps)
        self.cst, self.cff = t(b.cst), t(b.cff)
        self.start = t(b.input)
        self.series = self.start.clone()
        nm = b.nsys * b.dim * b.dim * b.width
        self.Q = torch.zeros(nm, dtype=torch.float64, device=dev)
        self.R = torch.zeros(nm, dtype=torch.float64, device=dev)
        self.flags0 = torch.tensor([1, 0, 0, 0, 1] * b.nsys, dtype=torch.int32, device=dev)
        self.flags = self.flags0.clone()
        f = _lib.lib().phc_newton_workspace_bytes
        f.restype = _lib.ctypes.c_longlong
        nbytes = int(f(b.prec, int(b.cplx), b.nsys, b.dim, b.deg, self.szt, _lib.ctypes.c_longlong(b.nmon)))
        if nbytes < 0:
            raise _lib.PhcError("phc_newton_workspace_bytes", nbytes, "bad sizes")
        self.work = torch.empty(max(1, nbytes // 8), dtype=torch.float64, device=dev)
        self.graph = None
        self.graph_steps = 0

    def reset(self, stream):
        with self.torch.cuda.stream(stream):
            self.series.copy_(self.start)
            self.flags.copy_(self.flags0)

    def step(self, stream):
        b = self.b
        _lib.call("phc_newton_step", b.prec, int(b.cplx), b.nsys, b.dim, b.deg, b.deg, self.szt, b.maxvar,
                  _lib.ptr(self.mon_off), _lib.ctypes.c_longlong(b.nmon), _lib.ptr(self.nvr), _lib.ptr(self.idx),
                  _lib.ptr(self.exps), _lib.ptr(self.cst), _lib.ptr(self.cff), _lib.ptr(self.series),
                  _lib.ptr(self.Q), _lib.ptr(self.R), _lib.ptr(self.flags), _lib.ptr(self.work),
                  _lib.c_void_p(stream.cuda_stream))

    def solve(self, nsteps: int, stream):
        """nsteps Newton steps from the start series, launch by launch."""
        self.reset(stream)
        for _ in range(nsteps):
            self.step(stream)

    def capture(self, nsteps: int, stream):
        """Capture a solve of nsteps steps (restoring the start series first)
        in a CUDA graph on stream; one eager solve runs first, so that the
        library's one-time set-up (function attributes) happens outside the
        capture."""
        torch = self.torch
        self.solve(nsteps, stream)
        stream.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=stream, capture_error_mode="thread_local"):
            self.solve(nsteps, stream)
        self.graph = g
        self.graph_steps = nsteps
        return g

    def replay(self, stream):
        """One captured solve, launched on stream (ordered after the work
        already queued there)."""
        if self.graph is None:
            raise RuntimeError("DeviceNewton.replay: capture() first")
        with self.torch.cuda.stream(stream):
            self.graph.replay()

    def result(self):
        """(series, flags) as numpy arrays, the layout of newton_host."""
        self.torch.cuda.synchronize()
        return self.series.cpu().numpy().copy(), self.flags.cpu().numpy().copy()
