"""The WY trailing products as Ozaki-split products on the FP64 tensor
cores (wy=1) against the oracle and against the CUDA-core products (wy=0),
with the tolerances of the other dense tests: QR factors within
1e3 * eps_md (* max|R| for R), least-squares blocks within
1e4 * eps_md * max(1, |x|), eps_md = 1e-28 (dd), 1e-60 (qd)."""
import numpy as np
import pytest

import golden_io
from mdcheck import absdiff, lead
from oracle import pyoracle
from phcpack_b200 import dense
from phcpack_b200 import workloads as wl

pytestmark = pytest.mark.gpu
ORC = pyoracle.oracle()
EPS = {1: 1e-14, 2: 1e-28, 4: 1e-60}


@pytest.mark.parametrize("prec,n,szt", [(4, 64, 32), (2, 64, 32), (4, 32, 8), (2, 24, 8), (4, 16, 16), (1, 64, 16)])
def test_qr_tensor_core_products_vs_oracle(prec, n, szt):
    rng = np.random.default_rng(100 + n + szt + prec)
    ninst = 2
    As = [wl.random_numbers(rng, (n, n), prec, False, "normal") for _ in range(ninst)]
    Q, R = dense.blocked_houseqr_wy(prec, False, np.concatenate(As), ninst, n, n, szt, wy=1)
    W = prec
    for k in range(ninst):
        Qo, Ro = ORC.blocked_houseqr(prec, False, n, n, szt, n // szt, As[k])
        q = Q[k * n * n * W:(k + 1) * n * n * W]
        r = R[k * n * n * W:(k + 1) * n * n * W]
        assert absdiff(q, Qo, prec, False).max() <= 1e3 * EPS[prec]
        assert absdiff(r, Ro, prec, False).max() <= 1e3 * EPS[prec] * lead(Ro, prec, False).max()


@pytest.mark.parametrize("name", [n for n in golden_io.names("baqr_") if "_r" in n])
def test_qr_tensor_core_products_vs_golden(name):
    d = golden_io.load(name)
    prec, n, szt = int(d["prec"]), int(d["n"]), int(d["szt"])
    Q, R = dense.blocked_houseqr_wy(prec, False, d["A"], 1, n, n, szt, wy=1)
    assert absdiff(Q, d["Q"], prec, False).max() <= 1e3 * EPS[prec]
    assert absdiff(R, d["R"], prec, False).max() <= 1e3 * EPS[prec] * lead(d["R"], prec, False).max()


def test_least_squares_tensor_core_vs_cuda_core_quad_double():
    # the 64 x 64 quad-double degree-31 least-squares workload, 2 instances
    prec, n, degp1, szt, ninst = 4, 64, 32, 32, 2
    rng = np.random.default_rng(31)
    mat = wl.random_numbers(rng, (ninst, degp1, n, n), prec, False, "normal")
    rhs = wl.random_numbers(rng, (ninst, degp1, n), prec, False, "normal")
    x1, f1 = dense.bals_solve_wy(prec, False, mat, rhs, ninst, n, degp1, szt, wy=1)
    x0, f0 = dense.bals_solve_wy(prec, False, mat, rhs, ninst, n, degp1, szt, wy=0)
    assert np.array_equal(f1, f0)
    s = lead(x0, prec, False).reshape(ninst * degp1, n).max(axis=1)
    e = absdiff(x1, x0, prec, False).reshape(ninst * degp1, n).max(axis=1)
    assert (e <= 1e4 * EPS[prec] * np.maximum(s, 1.0)).all()
    so, _, _, _, _ = ORC.bals_solve(prec, False, n, degp1, 1, mat[:degp1 * n * n * prec], rhs[:degp1 * n * prec])
    e = absdiff(x1[:degp1 * n * prec], so, prec, False).reshape(degp1, n).max(axis=1)
    assert (e <= 1e4 * EPS[prec] * np.maximum(s[:degp1], 1.0)).all()
