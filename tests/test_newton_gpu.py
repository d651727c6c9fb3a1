"""GPU parity of the batched power-series Newton method against the oracle
on the reference's known-answer problem (exponential-series solutions,
Newton/dbl2_monomial_systems.cpp:16-39, start = leading coefficients +
1e-16 as in dbl2_newton_testers.cpp:25-41).

Each coefficient x_k is solved from the lower ones, so rounding errors are
amplified order by order by the system's ||J_0^-1|| ||J_j||; the accuracy
attainable at coefficient k is a property of the problem.  The criterion is
therefore relative to the oracle's own error: per coefficient,
|gpu - exact| <= 10 |oracle - exact| + 1e3 eps_md, eps_md = 1e-32 (dd),
1e-64 (qd), and the tail indices (skip-rule outcome) must agree."""
import numpy as np
import pytest

from mdcheck import absdiff
from oracle import pyoracle
from phcpack_b200 import newton
from newton_problems import exponential_test_system

pytestmark = pytest.mark.gpu
ORC = pyoracle.oracle()
EPS = {2: 1e-32, 4: 1e-64}


def check(gpu, orc, exact, prec, cplx, nsys, dim, n1):
    # errors per (system, degree), maximised over the variables
    eg = absdiff(gpu, exact, prec, cplx).reshape(nsys, dim, n1).max(axis=1)
    eo = absdiff(orc, exact, prec, cplx).reshape(nsys, dim, n1).max(axis=1)
    return bool((eg <= 10 * eo + 1e3 * EPS[prec]).all())


@pytest.mark.parametrize("prec,cplx", [(2, False), (2, True), (4, False), (4, True)])
def test_newton_schedule_vs_oracle_known_answer(prec, cplx):
    # the n=8, degree-15 workload: <= 3 variables per monomial, exponents {1,2}
    b, sol = exponential_test_system(7, 4, 8, 15, 8, 3, prec, cplx)
    ser, fl = newton.newton_host(b, 14, szt=4, schedule=1)
    so, flo = pyoracle.newton_steps(ORC, b, b.deg, 14, schedule=1)
    assert np.array_equal(fl.reshape(-1, 5)[:, 4], flo.reshape(-1, 5)[:, 4])
    assert (fl.reshape(-1, 5)[:, 4] >= b.deg).all()
    assert check(ser, so, sol, prec, cplx, b.nsys, b.dim, b.deg + 1)


@pytest.mark.parametrize("prec,cplx", [(2, False), (4, True)])
def test_newton_fixed_degree_four_steps_vs_oracle(prec, cplx):
    # 4 steps at fixed working degree 15 (tile 8), started from the series
    # after 6 steps of the reference schedule
    b, sol = exponential_test_system(5, 3, 8, 15, 8, 3, prec, cplx)
    so6, _ = pyoracle.newton_steps(ORC, b, b.deg, 6, schedule=1)
    b.input = so6
    ser, fl = newton.newton_host(b, 4, szt=8, schedule=0)
    so, flo = pyoracle.newton_steps(ORC, b, b.deg, 4, schedule=0)
    assert np.array_equal(fl.reshape(-1, 5)[:, [0, 1, 4]], flo.reshape(-1, 5)[:, [0, 1, 4]])
    assert check(ser, so, sol, prec, cplx, b.nsys, b.dim, b.deg + 1)


def test_newton_known_answer_accuracy_double_double():
    # a system whose error amplification is mild: the exponential series is
    # recovered to double-double accuracy through degree 15
    b, sol = exponential_test_system(7, 4, 8, 15, 8, 3, 2, False)
    ser, _ = newton.newton_host(b, 14, szt=8, schedule=1)
    err = absdiff(ser, sol, 2, False).reshape(4, -1).max(axis=1)
    assert err[1] < 1e-22


@pytest.mark.parametrize("prec,cplx,tol", [(2, False, 1e-28), (2, True, 1e-28), (4, False, 1e-60), (4, True, 1e-60)])
def test_newton_coefficients_equal_oracle_directly(prec, cplx, tol):
    """The GPU's series against the oracle's, coefficient by coefficient (not
    through the exact solution): |gpu - oracle| <= 1e-28 (dd) / 1e-60 (qd)
    times max(1, |x|) at every coefficient that the problem determines to
    that accuracy (the oracle's own error against the exact series is below
    a tenth of the tolerance), after 1, 3 and 6 steps of the reference's
    schedule.  Each order amplifies the rounding of the lower ones by
    ||J_0^-1|| ||J_j|| in any implementation (on seed 11 from 1e-35 at order
    0 to 1e-21 at order 12), so the high orders of these random systems are
    determined less accurately than 1e-28; there the criterion relative to
    the oracle's own error above applies.  After 6 steps the first two
    coefficients of every series (dd; the constant terms in qd) must be
    among the coefficients compared."""
    b, sol = exponential_test_system(11, 3, 8, 15, 8, 3, prec, cplx)
    W = prec * (2 if cplx else 1)
    n1 = b.deg + 1
    for nsteps in (1, 3, 6):
        ser, _ = newton.newton_host(b, nsteps, szt=4, schedule=1)
        so, _ = pyoracle.newton_steps(ORC, b, b.deg, nsteps, schedule=1)
        d = absdiff(ser, so, prec, cplx).reshape(-1, n1)
        eo = absdiff(so, sol, prec, cplx).reshape(-1, n1)
        mag = np.maximum(np.abs(so.reshape(-1, n1, W)[:, :, 0]), 1.0)
        if cplx:
            mag = np.maximum(mag, np.abs(so.reshape(-1, n1, W)[:, :, prec]))
        determined = eo <= 0.1 * tol * mag
        if nsteps == 6:
            first = 2 if prec == 2 else 1
            assert determined[:, :first].all(), eo[:, :first].max()
        assert (d[determined] <= tol * mag[determined]).all(), (nsteps, float((d / mag)[determined].max()))


def test_newton_long_series_vs_oracle_known_answer():
    # degree 63 (series longer than a warp in the evaluation): the
    # reference's schedule reaches degree 63 in 11 steps; same skip-rule
    # outcome as the oracle, errors within the criterion above
    b, sol = exponential_test_system(9, 2, 8, 63, 8, 3, 2, False)
    ser, fl = newton.newton_host(b, 12, szt=8, schedule=1)
    so, flo = pyoracle.newton_steps(ORC, b, b.deg, 12, schedule=1)
    assert np.array_equal(fl.reshape(-1, 5)[:, 4], flo.reshape(-1, 5)[:, 4])
    assert check(ser, so, sol, 2, False, b.nsys, b.dim, b.deg + 1)
