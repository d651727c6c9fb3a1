"""The oracle restatement pinned against PHCpack's own host code: the golden
fixtures (outputs of the reference's CPU_* routines) and, where the
reference tree is present, the compiled reference itself on fresh inputs."""
import numpy as np
import pytest

import golden_io
from mdcheck import absdiff, abs_batch, check_scaled, lead
from oracle import pyoracle
from phcpack_b200 import workloads as wl

ORC = pyoracle.oracle()


def tol(prec):
    return {1: 1e-14, 2: 1e-28, 4: 1e-60}[prec]


@pytest.mark.parametrize("name", golden_io.names("eval_"))
def test_eval_oracle_vs_golden(name):
    d = golden_io.load(name)
    b = golden_io.batch(d)
    out = ORC.system_evaldiff(b)
    if not b.cplx:
        # real arithmetic follows the reference operation by operation
        assert np.array_equal(out, d["output"])
    scale = ORC.system_evaldiff(abs_batch(b))
    assert check_scaled(out, d["output"], scale, b.prec, b.cplx, tol(b.prec)) <= 1.0


@pytest.mark.parametrize("name", golden_io.names("baqr_"))
def test_baqr_oracle_vs_golden(name):
    d = golden_io.load(name)
    prec, cplx, n, szt = int(d["prec"]), bool(d["cplx"]), int(d["n"]), int(d["szt"])
    Q, R = ORC.blocked_houseqr(prec, cplx, n, n, szt, n // szt, d["A"])
    if not cplx:
        assert np.array_equal(Q, d["Q"]) and np.array_equal(R, d["R"])
    assert absdiff(Q, d["Q"], prec, cplx).max() <= 50 * tol(prec)
    assert absdiff(R, d["R"], prec, cplx).max() <= 50 * tol(prec) * lead(d["R"], prec, cplx).max()


@pytest.mark.parametrize("name", golden_io.names("tabs_"))
def test_tabs_oracle_vs_golden(name):
    d = golden_io.load(name)
    prec, cplx, n, szt = int(d["prec"]), bool(d["cplx"]), int(d["n"]), int(d["szt"])
    x, U2, b2 = ORC.upper_tiled_solver(prec, cplx, n, szt, n // szt, d["U"], d["b"])
    scale = lead(d["x"], prec, cplx).max()
    assert absdiff(x, d["x"], prec, cplx).max() <= 100 * tol(prec) * scale
    # like the reference, the diagonal tiles of U are overwritten by their inverses
    assert absdiff(U2, d["U_after"], prec, cplx).max() <= 100 * tol(prec) * lead(d["U_after"], prec, cplx).max()


@pytest.mark.parametrize("name", golden_io.names("bals_"))
def test_bals_oracle_vs_golden(name):
    d = golden_io.load(name)
    prec, cplx, n, degp1 = int(d["prec"]), bool(d["cplx"]), int(d["n"]), int(d["degp1"])
    sol, _, _, _, fl = ORC.bals_solve(prec, cplx, n, degp1, 1, d["mat"], d["rhs"])
    assert np.array_equal(fl, d["flags"])
    if not cplx:
        assert np.array_equal(sol, d["sol"])
    s = lead(d["sol"], prec, cplx).reshape(degp1, n).max(axis=1)
    err = absdiff(sol, d["sol"], prec, cplx).reshape(degp1, n).max(axis=1)
    assert (err <= 1e4 * tol(prec) * np.maximum(s, 1.0)).all()


@pytest.mark.skipif(pyoracle.reference() is None, reason="reference tree not present")
@pytest.mark.parametrize("prec,cplx", [(2, False), (2, True), (4, False), (4, True)])
def test_eval_oracle_vs_reference_fresh(prec, cplx):
    b = wl.eval_batch(101 + prec + int(cplx), 2, 7, 12, 7, 5, prec, cplx, expmax=3)
    ref = pyoracle.reference().system_evaldiff(b)
    out = ORC.system_evaldiff(b)
    scale = ORC.system_evaldiff(abs_batch(b))
    assert check_scaled(out, ref, scale, prec, cplx, tol(prec)) <= 1.0


def test_od_oracle_vs_golden():
    """Octo-double add, mul, div and multiply-by-double of the oracle equal the
    reference's (Norms/octo_double_functions.cpp) bit for bit."""
    import os
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "od_ops.npz"))
    a, b = d["a"], d["b"]
    for op, key in enumerate(("add", "mul", "div", "mul_d")):
        assert np.array_equal(ORC.od_binop(op, a, b), d[key]), key


def test_od_oracle_vs_reference_fresh():
    ref = pyoracle.reference()
    if ref is None:
        pytest.skip("the reference tree is not available here")
    rng = np.random.default_rng(77)
    raw = np.zeros((500, 8))
    for k in range(500):
        limbs = [rng.standard_normal() * 10.0 ** rng.integers(-20, 20)]
        for _ in range(7):
            limbs.append(limbs[-1] * 2.0 ** -53 * rng.uniform(-1, 1))
        raw[k] = limbs
    a = ref.od_binop(0, raw, np.zeros_like(raw))
    b = ref.od_binop(0, raw[::-1].copy(), np.zeros_like(raw))
    for op in range(4):
        assert np.array_equal(ORC.od_binop(op, a, b), ref.od_binop(op, a, b)), op
