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
    b, sol = newton.exponential_test_system(7, 4, 8, 15, 8, 3, prec, cplx)
    ser, fl = newton.newton_host(b, 14, szt=4, schedule=1)
    so, flo = pyoracle.newton_steps(ORC, b, b.deg, 14, schedule=1)
    assert np.array_equal(fl.reshape(-1, 5)[:, 4], flo.reshape(-1, 5)[:, 4])
    assert (fl.reshape(-1, 5)[:, 4] >= b.deg).all()
    assert check(ser, so, sol, prec, cplx, b.nsys, b.dim, b.deg + 1)


@pytest.mark.parametrize("prec,cplx", [(2, False), (4, True)])
def test_newton_fixed_degree_four_steps_vs_oracle(prec, cplx):
    # 4 steps at fixed working degree 15 (tile 8), started from the series
    # after 6 steps of the reference schedule
    b, sol = newton.exponential_test_system(5, 3, 8, 15, 8, 3, prec, cplx)
    so6, _ = pyoracle.newton_steps(ORC, b, b.deg, 6, schedule=1)
    b.input = so6
    ser, fl = newton.newton_host(b, 4, szt=8, schedule=0)
    so, flo = pyoracle.newton_steps(ORC, b, b.deg, 4, schedule=0)
    assert np.array_equal(fl.reshape(-1, 5)[:, [0, 1, 4]], flo.reshape(-1, 5)[:, [0, 1, 4]])
    assert check(ser, so, sol, prec, cplx, b.nsys, b.dim, b.deg + 1)


def test_newton_known_answer_accuracy_double_double():
    # a system whose error amplification is mild: the exponential series is
    # recovered to double-double accuracy through degree 15
    b, sol = newton.exponential_test_system(7, 4, 8, 15, 8, 3, 2, False)
    ser, _ = newton.newton_host(b, 14, szt=8, schedule=1)
    err = absdiff(ser, sol, 2, False).reshape(4, -1).max(axis=1)
    assert err[1] < 1e-22
