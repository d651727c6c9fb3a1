"""Error measures for limb-interleaved multiple-double arrays (tests only)."""
from __future__ import annotations

import numpy as np

from phcpack_b200.workloads import SystemBatch


def parts(flat, prec, cplx):
    W = prec * (2 if cplx else 1)
    return np.asarray(flat, dtype=np.float64).reshape(-1, W)


def absdiff(a, b, prec, cplx):
    """|a - b| per number, summing the limb differences in double (the limbs
    are non-overlapping, so this is accurate to a few ulps of the error)."""
    A, B = parts(a, prec, cplx), parts(b, prec, cplx)
    ngroups = 2 if cplx else 1
    out = np.zeros(A.shape[0])
    for q in range(ngroups):
        d = np.zeros(A.shape[0])
        for l in range(prec - 1, -1, -1):
            d = d + (A[:, q * prec + l] - B[:, q * prec + l])
        out = np.maximum(out, np.abs(d))
    return out


def lead(b, prec, cplx):
    B = parts(b, prec, cplx)
    if cplx:
        return np.hypot(B[:, 0], B[:, prec])
    return np.abs(B[:, 0])


def abs_batch(b: SystemBatch) -> SystemBatch:
    """The same supports with every coefficient and input replaced by the
    modulus of its leading limb, in plain double: evaluating it gives, per
    output coefficient, the sum of the absolute values of the terms, the
    natural scale of the rounding error."""
    f = lambda a: lead(a, b.prec, b.cplx)
    return SystemBatch(b.nsys, b.dim, b.deg, b.maxvar, 1, False, b.mon_off, b.nvr, b.idx, b.exps,
                       f(b.cst), f(b.cff), f(b.input))


def check_scaled(a, b, scale, prec, cplx, rtol):
    """max |a-b| / scale over all numbers; returns the worst ratio / rtol."""
    d = absdiff(a, b, prec, cplx)
    s = np.maximum(np.asarray(scale, dtype=np.float64).reshape(-1), 1e-300)
    return float((d / s).max()) / rtol


def rel_series(a, b, prec, cplx, n1):
    """normwise relative error per series of n1 numbers (max over series)"""
    d = absdiff(a, b, prec, cplx).reshape(-1, n1)
    m = lead(b, prec, cplx).reshape(-1, n1).max(axis=1)
    m = np.where(m > 0, m, 1.0)
    return float((d.max(axis=1) / m).max())
