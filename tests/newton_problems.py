"""Known-answer problems of the Newton layer (test infrastructure: the
constant terms come from the oracle's evaluation of the exact solution)."""
from __future__ import annotations

import numpy as np

from oracle import pyoracle
from phcpack_b200 import workloads as wl
from phcpack_b200.workloads import SystemBatch


def exponential_test_system(seed, nsys, dim, deg, nmon, maxvar, prec, cplx, expmax=2, oracle_lib=None):
    """Known-answer problem of Newton/dbl2_monomial_systems.cpp:16-39 and
    dbl2_newton_method.cpp:868-873: the solution is x_i(t) = exp(c_i t) with
    random |c_i| in [63/64, 1]; constant coefficients uniform in [-1, 1]
    (unit circle when complex) and constant terms chosen so that the series
    solves the system.  Returns (batch with the start series in input,
    the exact solution series).  The start series is the solution's leading
    coefficient plus 1e-16, higher coefficients zero
    (Newton/dbl2_newton_testers.cpp:25-41)."""
    rng = np.random.default_rng(seed)
    mon_off, nvr, idx, exps = wl.random_supports(rng, nsys, dim, nmon, maxvar, 1, expmax)
    n1 = deg + 1
    W = prec * (2 if cplx else 1)
    nm = len(nvr)
    # constant coefficient series
    c0 = wl.random_numbers(rng, (nm,), prec, cplx, "unit" if cplx else "uniform", tail=False).reshape(nm, W)
    cff = np.zeros((nm, n1, W))
    cff[:, 0, :] = c0
    # solution series: exp(c t) = sum c^k/k! t^k, coefficients in double then
    # widened with zero lower limbs (exact as given)
    mag = rng.uniform(63 / 64, 1.0, size=(nsys * dim,))
    sol = np.zeros((nsys * dim, n1, W))
    if cplx:
        ang = rng.uniform(0, 2 * np.pi, size=(nsys * dim,))
        c = mag * np.exp(1j * ang)
    else:
        c = mag * rng.choice([-1.0, 1.0], size=(nsys * dim,))
    fact = 1.0
    for k in range(n1):
        if k > 0:
            fact *= k
        v = c ** k / fact
        sol[:, k, 0] = np.real(v)
        if cplx:
            sol[:, k, prec] = np.imag(v)
    zero_cst = np.zeros(nsys * dim * n1 * W)
    tmp = SystemBatch(nsys, dim, deg, maxvar, prec, cplx, mon_off, nvr, idx, exps, zero_cst, cff.reshape(-1),
                      sol.reshape(-1))
    if oracle_lib is None:
        oracle_lib = pyoracle.oracle()
    val = oracle_lib.system_evaldiff(tmp).reshape(nsys * dim, dim + 1, n1, W)[:, dim]
    cst = -val  # negating every limb negates the number exactly
    start = np.zeros((nsys * dim, n1, W))
    start[:, 0, :] = sol[:, 0, :]
    if prec > 1:
        hi, lo = start[:, 0, 0], start[:, 0, 1] + 1e-16
        s_ = hi + lo
        start[:, 0, 1] = lo - (s_ - hi)
        start[:, 0, 0] = s_
    else:
        start[:, 0, 0] += 1e-16
    b = SystemBatch(nsys, dim, deg, maxvar, prec, cplx, mon_off, nvr, idx, exps, cst.reshape(-1), cff.reshape(-1),
                    start.reshape(-1))
    return b, sol.reshape(-1)


def config1(seed=1, nsys=1):
    """n=8 real double-double systems, 8 monomials per polynomial over <= 3
    distinct variables, exponents in {1, 2}, coefficients uniform in [-1, 1],
    degree 15, with a known exponential-series solution."""
    return exponential_test_system(seed, nsys, 8, 15, 8, 3, 2, False, expmax=2)
