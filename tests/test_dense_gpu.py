"""GPU parity of the batched blocked Householder QR, tiled back substitution
and block-Toeplitz least squares against the golden fixtures from PHCpack's
host code and against the oracle.

Tolerances: QR factors within 1e3 * eps_md * max|R| (the GPU accumulates the
WY products in a different association than the host); solutions within
1e4 * eps_md relative to max(1, |x|) per block, eps_md = 1e-28 (dd),
1e-60 (qd), 1e-14 (double)."""
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


def batch_of(arrs):
    return np.concatenate([np.asarray(a).reshape(-1) for a in arrs])


@pytest.mark.parametrize("name", golden_io.names("baqr_"))
def test_baqr_gpu_vs_golden(name):
    d = golden_io.load(name)
    prec, cplx, n, szt = int(d["prec"]), bool(d["cplx"]), int(d["n"]), int(d["szt"])
    Q, R = dense.blocked_houseqr_host(prec, cplx, d["A"], 1, n, n, szt)
    sR = lead(d["R"], prec, cplx).max()
    assert absdiff(Q, d["Q"], prec, cplx).max() <= 1e3 * EPS[prec]
    assert absdiff(R, d["R"], prec, cplx).max() <= 1e3 * EPS[prec] * sR


@pytest.mark.parametrize("prec,cplx,n,szt", [(2, False, 64, 32), (2, True, 32, 8), (4, False, 64, 32),
                                             (4, True, 32, 16), (1, True, 10, 5), (2, False, 24, 8)])
def test_baqr_gpu_batch_vs_oracle(prec, cplx, n, szt):
    rng = np.random.default_rng(n + szt + prec)
    ninst = 3
    As = [wl.random_numbers(rng, (n, n), prec, cplx, "normal") for _ in range(ninst)]
    Q, R = dense.blocked_houseqr_host(prec, cplx, batch_of(As), ninst, n, n, szt)
    W = dense.width(prec, cplx)
    for k in range(ninst):
        Qo, Ro = ORC.blocked_houseqr(prec, cplx, n, n, szt, n // szt, As[k])
        q = Q[k * n * n * W:(k + 1) * n * n * W]
        r = R[k * n * n * W:(k + 1) * n * n * W]
        assert absdiff(q, Qo, prec, cplx).max() <= 1e3 * EPS[prec]
        assert absdiff(r, Ro, prec, cplx).max() <= 1e3 * EPS[prec] * lead(Ro, prec, cplx).max()


@pytest.mark.parametrize("name", golden_io.names("tabs_"))
def test_tabs_gpu_vs_golden(name):
    d = golden_io.load(name)
    prec, cplx, n, szt = int(d["prec"]), bool(d["cplx"]), int(d["n"]), int(d["szt"])
    x, U2, b2 = dense.upper_tiled_solver_host(prec, cplx, d["U"], d["b"], 1, n, szt)
    assert absdiff(x, d["x"], prec, cplx).max() <= 1e3 * EPS[prec] * max(1.0, lead(d["x"], prec, cplx).max())
    assert absdiff(U2, d["U_after"], prec, cplx).max() <= 1e3 * EPS[prec] * lead(d["U_after"], prec, cplx).max()
    assert absdiff(b2, d["b_after"], prec, cplx).max() <= 1e3 * EPS[prec] * max(1.0, lead(d["b_after"], prec, cplx).max())


def check_bals(sol, ref, prec, cplx, degp1, n):
    s = lead(ref, prec, cplx).reshape(degp1, n).max(axis=1)
    err = absdiff(sol, ref, prec, cplx).reshape(degp1, n).max(axis=1)
    return (err <= 1e4 * EPS[prec] * np.maximum(s, 1.0)).all()


@pytest.mark.parametrize("name", golden_io.names("bals_"))
def test_bals_gpu_vs_golden(name):
    d = golden_io.load(name)
    prec, cplx, n, degp1 = int(d["prec"]), bool(d["cplx"]), int(d["n"]), int(d["degp1"])
    szt = n // 2
    sol, _, _, _, fl = dense.bals_solve_host(prec, cplx, d["mat"], d["rhs"], 1, n, degp1, szt)
    assert np.array_equal(fl, d["flags"])
    assert check_bals(sol, d["sol"], prec, cplx, degp1, n)


@pytest.mark.parametrize("prec,cplx,n,szt,degp1", [(4, False, 64, 32, 32), (2, True, 16, 8, 9), (1, True, 10, 10, 9),
                                                   (4, True, 8, 4, 5)])
def test_bals_gpu_batch_vs_oracle(prec, cplx, n, szt, degp1):
    # the quad-double 64x64, degree-31 least-squares workload at a small batch
    rng = np.random.default_rng(degp1 + n)
    ninst = 2
    mats = [wl.random_numbers(rng, (degp1, n, n), prec, cplx, "normal") for _ in range(ninst)]
    rhss = [wl.random_numbers(rng, (degp1, n), prec, cplx, "normal") for _ in range(ninst)]
    sol, _, _, _, fl = dense.bals_solve_host(prec, cplx, batch_of(mats), batch_of(rhss), ninst, n, degp1, szt)
    W = dense.width(prec, cplx)
    blk = degp1 * n * W
    for k in range(ninst):
        so, _, _, _, flo = ORC.bals_solve(prec, cplx, n, degp1, 1, mats[k], rhss[k])
        assert np.array_equal(fl[5 * k:5 * k + 5], flo)
        assert check_bals(sol[k * blk:(k + 1) * blk], so, prec, cplx, degp1, n)


def test_bals_skip_rules():
    # right hand sides that vanish past degree 2 exercise the skip-update and
    # skip-back-substitution rules; a zero b_0 with zeroQ=0 skips the QR
    prec, cplx, n, degp1 = 2, False, 8, 6
    rng = np.random.default_rng(9)
    mat = wl.random_numbers(rng, (degp1, n, n), prec, cplx, "normal")
    A1 = mat.reshape(degp1, n, n, 2)
    A1[1:] = 0.0
    rhs = wl.random_numbers(rng, (degp1, n), prec, cplx, "normal").reshape(degp1, n, 2)
    rhs[2:] = 0.0
    sol, _, Q, R, fl = dense.bals_solve_host(prec, cplx, A1.reshape(-1), rhs.reshape(-1), 1, n, degp1, 4)
    so, _, Qo, Ro, flo = ORC.bals_solve(prec, cplx, n, degp1, 1, A1.reshape(-1), rhs.reshape(-1))
    assert np.array_equal(fl, flo) and fl[3] == degp1 - 2 and fl[4] == 1
    assert check_bals(sol, so, prec, cplx, degp1, n)
    # second call: b_0 = 0 and zeroQ = 0 -> the QR of the previous call is reused
    rhs2 = rhs.copy()
    rhs2[0] = 0.0
    sol2, _, _, _, fl2 = dense.bals_solve_host(prec, cplx, A1.reshape(-1), rhs2.reshape(-1), 1, n, degp1, 4,
                                               flags=np.array([0, 0, 0, 0, 1], np.int32), Q=Q, R=R)
    so2, _, _, _, flo2 = ORC.bals_solve(prec, cplx, n, degp1, 1, A1.reshape(-1), rhs2.reshape(-1),
                                        flags=(0, 0, 0, 0, 1), Q=Qo, R=Ro)
    assert fl2[1] == 1 and np.array_equal(fl2, flo2)
    assert check_bals(sol2, so2, prec, cplx, degp1, n)


def test_bals_host_entry_matches_device_entry():
    # 70 instances through the host entry and through the device entry:
    # solutions and flags equal bit for bit
    prec, cplx, n, szt, degp1, ninst = 2, True, 8, 4, 4, 70
    rng = np.random.default_rng(70)
    mat = batch_of([wl.random_numbers(rng, (degp1, n, n), prec, cplx, "normal") for _ in range(ninst)])
    rhs = batch_of([wl.random_numbers(rng, (degp1, n), prec, cplx, "normal") for _ in range(ninst)])
    sol, _, _, _, fl = dense.bals_solve_host(prec, cplx, mat.copy(), rhs.copy(), ninst, n, degp1, szt)
    sol2, fl2 = dense.bals_solve_wy(prec, cplx, mat, rhs, ninst, n, degp1, szt, wy=0)
    assert np.array_equal(fl, fl2)
    assert np.array_equal(sol, sol2)


@pytest.mark.parametrize("prec,cplx", [(2, False), (2, True), (4, False), (4, True)])
@pytest.mark.parametrize("tailidx", [0, 1, 3])
def test_linear_residue_vs_reference(prec, cplx, tailidx):
    """phc_linear_residue_host against the reference's own host code
    (CPU_dbl2_linear_residue and twins, Newton/dbl2_bals_host.cpp:548,
    through oracle/_ref): the residual entries agree within 1e2 * eps_md
    of the largest product magnitude and the per-limb maximum is that of the
    same entry (rows below tailidx stay as they were given)."""
    ref = pyoracle.reference()
    if ref is None:
        pytest.skip("the reference's host code was not built here")
    n, degp1, ninst = 8, 5, 3
    W = prec * (2 if cplx else 1)
    rng = np.random.default_rng(100 + 10 * prec + tailidx + (5 if cplx else 0))
    mats = [wl.random_numbers(rng, (degp1, n, n), prec, cplx, "normal") for _ in range(ninst)]
    rhss = [wl.random_numbers(rng, (degp1, n), prec, cplx, "normal") for _ in range(ninst)]
    sols = [wl.random_numbers(rng, (degp1, n), prec, cplx, "normal") for _ in range(ninst)]
    prev = [wl.random_numbers(rng, (degp1, n), prec, cplx, "normal") for _ in range(ninst)]
    res, mx = dense.linear_residue_host(prec, cplx, batch_of(mats), batch_of(rhss), batch_of(sols), ninst, n, degp1,
                                        tailidx, res=batch_of(prev))
    res = res.reshape(ninst, -1)
    mx = mx.reshape(ninst, prec)
    for q in range(ninst):
        r_ref, mx_ref = ref.linear_residue(prec, cplx, n, degp1, tailidx, mats[q], rhss[q], sols[q], res=prev[q])
        scale = 2.0 * n * degp1  # |A|, |x| ~ 1: sums of n * degp1 products
        assert absdiff(res[q], r_ref, prec, cplx).max() <= 1e2 * EPS[prec] * scale
        rows = res[q].reshape(degp1, n * W)
        assert np.array_equal(rows[:tailidx], np.asarray(prev[q]).reshape(degp1, n * W)[:tailidx])
        assert abs(mx[q, 0] - mx_ref[0]) <= 1e-12 * mx_ref[0]
