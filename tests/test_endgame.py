"""End-game diagnostics on the CPU: the oracle's restatement of Newton-Fabry
and of the Hessian distance against closed forms, the classification of
the Fabry estimate, and the argument checks of the C ABI (no device work).

Closed form: h(x, t) = x^2 - 1 + w t has the path x(t) = sqrt(1 - w t),
whose series at t0 has the coefficients c_k = sqrt(A) binom(1/2, k)
(-w/A)^k, A = 1 - w t0.  Fabry's ratio with offset 1 at degree K is then
c_{K-2}/c_{K-1} = (K-1)/(K-5/2) A/w, the next ratio K/(K-3/2) A/w, and
J = 2x, H = 2, so eta = 2 sigma_min(J) / sigma_max(H) = 2 |x|."""
import ctypes

import numpy as np
import pytest

from oracle import pyoracle
from phcpack_b200 import _lib
from phcpack_b200 import endgame as eg
from phcpack_b200 import homotopy as hm

ORC = pyoracle.oracle()


def sqrt_problem(w, t0):
    p = [[(((0, 2),), 1.0 + 0j), ((), complex(-1.0 + w))]]
    q = [[(((0, 2),), 1.0 + 0j), ((), -1.0 + 0j)]]
    x0 = np.sqrt(complex(1.0 - w * t0))
    return hm.homotopy_problem([(p, q)], 1.0, [(0, [x0])]), x0


def closed_form(w, t0, K):
    A = 1.0 - w * t0
    z = (K - 1) / (K - 2.5) * A / w
    e = abs(z - K / (K - 1.5) * A / w) * (K - 1)
    return z, e


@pytest.mark.parametrize("pmode", [1, 2, 4])
@pytest.mark.parametrize("w,t0", [(1.0, 0.5), (0.6 + 0.8j, 0.25), (2.0, 0.0)])
def test_oracle_fabry_closed_form(pmode, w, t0):
    pb, x0 = sqrt_problem(w, t0)
    K = 8
    ipar, dpar = eg.params(pmode, deg=K)
    r = pyoracle.series_diagnostics(ORC, pb, np.array([x0.real, x0.imag]), 1, np.array([t0]), ipar, dpar, pmode)
    z, e = closed_form(w, t0, K)
    assert r["status"][0] == 0 and r["fail"][0] == 0
    assert abs(r["z"][0] - z) <= 1e-13 * abs(z)
    assert abs(r["err"][0] - e) <= 1e-12 * abs(z) * K
    assert abs(r["radius"][0] - abs(z)) <= 1e-14 * abs(z)
    # the series coefficients against the binomial series
    A = 1.0 - w * t0
    b, c = 1.0, []
    for k in range(K + 1):
        c.append(np.sqrt(complex(A)) * b * (-w / A) ** k)
        b *= (0.5 - k) / (k + 1)
    L = pmode
    got = r["series"][0, 0, :, 0] + 1j * r["series"][0, 0, :, L]
    assert np.abs(got - np.array(c)).max() <= 1e-13
    sj = np.linalg.svd(r["J"][0], compute_uv=False)
    sh = np.linalg.svd(r["H"][0, 0], compute_uv=False)
    assert abs(2 * sj.min() / sh.max() - 2 * abs(x0)) <= 1e-14


@pytest.mark.parametrize("offset", [0, 1, 2])
def test_oracle_fabry_offsets(offset):
    # offset 0: c_{K-1}/c_K; offset j > 0: c_{K-1-j}/c_{K-j}
    pb, x0 = sqrt_problem(1.0, 0.5)
    K = 9
    ipar, dpar = eg.params(2, deg=K, offset=offset)
    r = pyoracle.series_diagnostics(ORC, pb, np.array([x0.real, x0.imag]), 1, np.array([0.5]), ipar, dpar, 2)
    A = 0.5
    j = K - 1 - offset  # z = c_j / c_{j+1} = (j+1)/(j-1/2) A
    assert abs(r["z"][0] - (j + 1) / (j - 0.5) * A) <= 1e-13


def test_oracle_singular_point():
    # h = x^2 at t = 1 (start x^2 - 1): the Jacobian 2x vanishes at x = 0
    p = [[(((0, 2),), 1.0 + 0j)]]
    q = [[(((0, 2),), 1.0 + 0j), ((), -1.0 + 0j)]]
    pb = hm.homotopy_problem([(p, q)], 1.0, [(0, [0j])])
    ipar, dpar = eg.params(2)
    r = pyoracle.series_diagnostics(ORC, pb, np.zeros(2), 1, np.array([1.0]), ipar, dpar, 2)
    assert r["status"][0] == 1 and r["fail"][0] == 1 and np.isinf(r["radius"][0])
    assert np.abs(r["J"][0]).max() == 0.0


def test_classify_approach_to_singular_endpoint():
    """x(t) = sqrt(1 - t): at t = 1 - d the singular point estimate is
    t + (K-1)/(K-5/2) d, which closes in on t = 1."""
    K = 8
    ts, zs = [], []
    for d in (1e-1, 1e-2, 1e-3):
        z, _ = closed_form(1.0, 1.0 - d, K)
        ts.append(1.0 - d)
        zs.append(z)
    n = len(ts)
    diag = eg.Diagnostics(np.array(zs, complex), np.abs(zs), np.zeros(n), np.ones(n), np.ones(n), np.ones(n),
                          np.ones(n), np.ones(n), np.zeros(n), np.zeros(n, np.int32), np.zeros(n, np.int32))
    assert eg.classify(ts, diag) == ["singular at t = 1"] * n
    # a pole far off the interval, and one inside it away from 1
    diag.z[:] = [3.0 + 0j, 0.01j, 1.5 + 1.0j]
    diag.radius[:] = np.abs(diag.z)
    assert eg.classify([0.5, 0.2, 0.0], diag) == ["regular", "interior singularity", "regular"]
    diag.status[0] = 1
    assert eg.classify([0.5, 0.2, 0.0], diag)[0] == "no series"


def _host_args(pb, ipar, dpar, pmode, xlimbs=1):
    xpt = np.zeros(pb.npaths * pb.maxdim * 2 * xlimbs)
    tpt = np.zeros(pb.npaths)
    dout = np.zeros(pb.npaths * 10)
    iout = np.zeros(pb.npaths * 2, np.int32)
    p = _lib.ptr
    return (pb.nsys, p(pb.dim), pb.maxvar, p(pb.mono_off), p(pb.mono_nvr), p(pb.mono_idx), p(pb.mono_exp),
            p(pb.eq_off), p(pb.term_off), p(pb.term_mono), p(pb.term_a), p(pb.term_b), pb.npaths, p(pb.path_sys),
            p(xpt), xlimbs, p(tpt), p(np.asarray(ipar, np.int32)), p(np.asarray(dpar, np.float64)), pmode,
            ctypes.c_void_p(0), p(dout), p(iout))


@pytest.mark.parametrize("change,match", [
    (dict(pmode=3), "precision"),
    (dict(xlimbs=3), "xlimbs"),
    (dict(ipar=[2, 1, 1, 0, 4]), "deg"),
    (dict(ipar=[8, 6, 3, 1, 4]), "numdeg + dendeg"),
    (dict(ipar=[8, 5, 1, 7, 4]), "offset"),
    (dict(ipar=[8, 5, 1, 1, 65]), "newton_steps"),
])
def test_diagnostics_host_rejects_bad_arguments(change, match):
    pb, _ = sqrt_problem(1.0, 0.5)
    ipar, dpar = eg.params(2)
    ipar = change.get("ipar", ipar)
    f = _lib.lib().phc_series_diagnostics_host
    f.restype = ctypes.c_int
    rc = f(*_host_args(pb, ipar, dpar, change.get("pmode", 2), change.get("xlimbs", 1)))
    msg = _lib.lib().phc_last_error().decode()
    assert rc < 0 and match in msg, msg


def test_diagnostics_refuses_shared_memory_beyond_the_limit():
    """n = 32 in quad-double needs more than 227 KB of shared memory per
    point: refused before any device work (null device pointers suffice)."""
    f = _lib.lib().phc_series_diagnostics
    f.restype = ctypes.c_int
    dim = np.array([32], np.int32)
    ipar = np.array([8, 5, 1, 1, 4], np.int32)
    dpar = np.array([1e-48, 0.005])
    N = ctypes.c_void_p(0)
    rc = f(1, _lib.ptr(dim), 2, 32, 600, N, N, N, N, N, N, N, N, N, N, N, N, 0, 1, N, N, 1, N, _lib.ptr(ipar),
           _lib.ptr(dpar), 4, N, N, N, N)
    msg = _lib.lib().phc_last_error().decode()
    assert rc < 0 and "shared memory" in msg, msg
