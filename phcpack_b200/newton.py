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
