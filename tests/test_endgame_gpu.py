"""GPU parity of the end-game diagnostics (phc_series_diagnostics) with the
oracle's restatement, and with closed forms.

Tolerances: the series coefficient k of a component against the oracle's
within rtol * (max_j |c_j| of that component), rtol 1e-10 in double, 1e-24
in double-double, 1e-48 in quad-double (times 100); Fabry's z and radius
within 1e-6 relative in double, 1e-14 otherwise (a ratio of the smallest
coefficients); the singular values (one-sided Jacobi on the GPU) against numpy's
SVD of the oracle's Jacobian and Hessians within 1e-11 of the largest
singular value; eta and the curvature step within 1e-9 relative."""
import numpy as np
import pytest

from oracle import pyoracle
from phcpack_b200 import endgame as eg
from phcpack_b200 import homotopy as hm

pytestmark = pytest.mark.gpu
ORC = pyoracle.oracle()
RTOL = {1: 1e-10, 2: 1e-24, 4: 1e-48}
ZTOL = {1: 1e-6, 2: 1e-14, 4: 1e-14}


def sqrt_problem(w, t0):
    p = [[(((0, 2),), 1.0 + 0j), ((), complex(-1.0 + w))]]
    q = [[(((0, 2),), 1.0 + 0j), ((), -1.0 + 0j)]]
    x0 = np.sqrt(complex(1.0 - w * t0))
    return hm.homotopy_problem([(p, q)], 1.0, [(0, [x0])]), x0


def check_against_oracle(pb, xpt, xlimbs, tpt, pmode, **kw):
    d = eg.series_diagnostics(pb, xpt, tpt, xlimbs=xlimbs, pmode=pmode, want_series=True, **kw)
    ipar, dpar = eg.params(pmode, **kw)
    r = pyoracle.series_diagnostics(ORC, pb, xpt, xlimbs, tpt, ipar, dpar, pmode)
    assert np.array_equal(d.status, r["status"]) and np.array_equal(d.fail, r["fail"])
    rt = RTOL[pmode]
    K = int(ipar[0])
    L = pmode
    ok = d.status != 1
    for p in range(pb.npaths):
        n = int(pb.dim[pb.path_sys[p]])
        for i in range(n):
            g = d.series[p, i]
            o = r["series"][p, i]
            scale = np.abs(o[:, 0] + 1j * o[:, L]).max()
            # the differences of the limbs, summed (exact for the leading
            # limbs of two close numbers)
            dl = g - o
            diff = np.abs(dl[:, :L].sum(1) + 1j * dl[:, L:].sum(1))
            assert diff.max() <= max(rt, 1e-30) * max(scale, 1.0) * 1e2, (p, i, diff.max(), scale)
    f = ok & (d.fail == 0)
    zt = ZTOL[pmode]
    assert np.all(np.abs(d.z[f] - r["z"][f]) <= zt * np.abs(r["z"][f]))
    assert np.allclose(d.radius[f], r["radius"][f], rtol=zt)
    assert np.allclose(d.pade_norm, r["padenorm"], rtol=1e-9)
    for p in range(pb.npaths):
        n = int(pb.dim[pb.path_sys[p]])
        sj = np.linalg.svd(r["J"][p, :n, :n], compute_uv=False)
        sh = np.array([np.linalg.svd(r["H"][p, i, :n, :n], compute_uv=False).max() for i in range(n)])
        assert abs(d.sigma_min[p] - sj.min()) <= 1e-11 * sj.max(), (p, d.sigma_min[p], sj.min())
        hn = np.sqrt((sh ** 2).sum())
        assert abs(d.hessian_norm[p] - hn) <= 1e-11 * max(hn, 1e-300)
        if hn > 0 and sj.min() > 1e-6 * sj.max():
            eta = 2 * sj.min() / hn
            assert abs(d.eta[p] - eta) <= 1e-9 * eta
            step = (dpar[1] * eta / r["padenorm"][p]) ** (1.0 / K)
            assert abs(d.curv_step[p] - step) <= 1e-9 * step
    return d, r


@pytest.mark.parametrize("pmode", [1, 2, 4])
def test_closed_form(pmode):
    K = 8
    for w, t0 in [(1.0, 0.5), (0.6 + 0.8j, 0.25)]:
        pb, x0 = sqrt_problem(w, t0)
        d = eg.series_diagnostics(pb, np.array([x0.real, x0.imag]), [t0], pmode=pmode, deg=K)
        A = 1.0 - w * t0
        z = (K - 1) / (K - 2.5) * A / w
        e = abs(z - K / (K - 1.5) * A / w) * (K - 1)
        assert d.status[0] == 0 and d.fail[0] == 0
        assert abs(d.z[0] - z) <= 1e-13 * abs(z) and abs(d.err[0] - e) <= 1e-11
        assert abs(d.sigma_min[0] - 2 * abs(x0)) <= 1e-14 and abs(d.hessian_norm[0] - 2.0) <= 1e-14
        assert abs(d.eta[0] - 2 * abs(x0)) <= 1e-14


@pytest.mark.parametrize("pmode", [1, 2, 4])
def test_start_points_dense_quadratic(pmode):
    rng = np.random.default_rng(11)
    n = 6
    pb = hm.total_degree_problem([hm.dense_quadratic(rng, n)], complex(hm.unit(rng)))
    pb = hm.subset(pb, np.arange(24))
    check_against_oracle(pb, pb.x0, 1, np.zeros(pb.npaths), pmode)


@pytest.mark.parametrize("pmode", [2, 4])
def test_tracked_end_points(pmode):
    rng = np.random.default_rng(12)
    n = 5
    pb = hm.total_degree_problem([hm.dense_quadratic(rng, n)], complex(hm.unit(rng)))
    res = hm.track_host(pb, pmode=1, rmode=4)
    assert (res.status == 0).all()
    d, _ = check_against_oracle(pb, res.xend, res.limbs, res.t, pmode)
    assert (d.status == 0).all() and (d.lastdx <= 1e-20).all()


def test_staged_partials_and_several_systems():
    # cubic monomials stage their partials; two systems of different sizes
    rng = np.random.default_rng(13)
    polys3 = [[(((0, 3),), 1.0 + 0j), (((1, 1), (2, 2)), 0.5 - 0.2j), ((), -1.0 + 0j)],
              [(((1, 3),), 1.0 + 0j), (((0, 2), (2, 1)), -0.3 + 0.4j), ((), -2.0 + 0j)],
              [(((2, 3),), 1.0 + 0j), (((0, 1), (1, 1), (2, 1)), 0.7j), ((), -0.5 + 0j)]]
    polys2 = [hm.dense_quadratic(rng, 2)[0], hm.dense_quadratic(rng, 2)[1]]
    pb = hm.total_degree_problem([polys3, polys2], complex(hm.unit(rng)), maxvar=3)
    check_against_oracle(pb, pb.x0, 1, np.zeros(pb.npaths), 2)


def test_singular_jacobian():
    p = [[(((0, 2),), 1.0 + 0j)]]
    q = [[(((0, 2),), 1.0 + 0j), ((), -1.0 + 0j)]]
    pb = hm.homotopy_problem([(p, q)], 1.0, [(0, [0j])])
    d = eg.series_diagnostics(pb, np.zeros(2), [1.0], pmode=2)
    assert d.status[0] == 1 and d.fail[0] == 1 and np.isinf(d.radius[0])
    assert d.sigma_min[0] == 0.0 and d.eta[0] == 0.0
    assert eg.classify([1.0], d) == ["no series"]


def test_approach_to_singular_end_point():
    """h = x^2 - (1 - t): the path sqrt(1 - t) ends at a double root; at
    t = 1 - d the singular point estimate t + z closes in on 1 and eta =
    2 sqrt(d) goes to zero."""
    p = [[(((0, 2),), 1.0 + 0j)]]
    q = [[(((0, 2),), 1.0 + 0j), ((), -1.0 + 0j)]]
    ds = np.array([1e-1, 1e-2, 1e-3, 1e-4])
    pb = hm.homotopy_problem([(p, q)] * 1, 1.0, [(0, [np.sqrt(d)]) for d in ds])
    xpt = np.stack([np.sqrt(ds), np.zeros_like(ds)], axis=1).reshape(-1)
    d = eg.series_diagnostics(pb, xpt, 1.0 - ds, pmode=2)
    ts = 1.0 - ds + d.z
    assert np.all(np.abs(ts - 1.0) <= 0.3 * ds)
    assert np.allclose(d.eta, 2 * np.sqrt(ds), rtol=1e-12)
    assert eg.classify(1.0 - ds, d) == ["singular at t = 1"] * len(ds)


@pytest.mark.parametrize("n", [1, 32])
def test_dimension_extremes(n):
    rng = np.random.default_rng(14 + n)
    # x_i^2 - c_i with a linear coupling: diagonal dominant, regular
    polys = []
    for i in range(n):
        poly = [(((i, 2),), 1.0 + 0j), ((), complex(-1.0 - 0.5 * rng.random()))]
        if n > 1:
            poly.append(((((i + 1) % n, 1),), complex(0.1 * rng.standard_normal())))
        polys.append(poly)
    pb = hm.total_degree_problem([polys], complex(hm.unit(rng)), max_paths_per_system=4, rng=rng)
    check_against_oracle(pb, pb.x0, 1, np.zeros(pb.npaths), 2)


def test_device_entry_point_matches_host_entry_point():
    import torch
    rng = np.random.default_rng(15)
    pb = hm.total_degree_problem([hm.dense_quadratic(rng, 5)], complex(hm.unit(rng)))
    pb = hm.subset(pb, np.arange(16))
    dt = hm.DeviceTracker(pb)
    tpt = torch.zeros(pb.npaths, dtype=torch.float64, device="cuda")
    dout, iout = eg.series_diagnostics_device(dt, dt.arr["x0"], tpt, 1, 2)
    torch.cuda.synchronize()
    dev = eg.Diagnostics.from_arrays(dout.cpu().numpy(), iout.cpu().numpy())
    host = eg.series_diagnostics(pb, pb.x0, np.zeros(pb.npaths), pmode=2)
    assert np.array_equal(dev.status, host.status) and np.array_equal(dev.fail, host.fail)
    for f in ("z", "radius", "err", "sigma_min", "hessian_norm", "eta", "pade_norm", "curv_step"):
        assert np.array_equal(getattr(dev, f), getattr(host, f)), f
