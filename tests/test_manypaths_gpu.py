"""The tracker's drop-in entry points through the C ABI: the systems and the
start solutions go into the containers, gpumanypaths_dd / _qd track with the
reference's arguments (mode, verbose, regamma, imgamma), and the end points
read back from the solution container are those of phc_track_host on the
same homotopy: same status per path, same end points (the same kernel on
the same arrays), on cyclic 5-roots (120 total-degree paths) and on the
1024-path dense quadratic n = 10 workload."""
import numpy as np
import pytest

from phcpack_b200 import homotopy as hm
from phcpack_b200 import manypaths, phcio

pytestmark = pytest.mark.gpu


def cyclic_text(n):
    x = [f"x{i + 1}" for i in range(n)]
    rows = [" + ".join("*".join(x[(i + j) % n] for j in range(k)) for i in range(n)) + ";" for k in range(1, n)]
    return f"{n}\n" + "\n".join(rows) + "\n" + "*".join(x) + " - 1;\n"


def start_solutions(degs):
    pts = hm.total_degree_solutions(degs)
    x = np.zeros((len(pts), len(degs), 2, 1))
    for s, p in enumerate(pts):
        x[s, :, 0, 0] = p.real
        x[s, :, 1, 0] = p.imag
    return pts, x


def drop_in_vs_host(target, gamma, prec, capfd=None):
    n = len(target)
    q, degs = hm.total_degree_start(target)
    pts, x = start_solutions(degs)
    manypaths.clear()
    manypaths.set_system("target", target, n)
    manypaths.set_system("start", q, n)
    manypaths.set_solutions(x)
    assert manypaths.track(2, 1 if capfd else 0, gamma.real, gamma.imag, prec=prec) == 0
    if capfd:
        out = capfd.readouterr().out
        assert f"number of solutions : {len(pts)}" in out and "Mode of execution : 2" in out
    got = manypaths.get_solutions(limbs=4)
    pb = hm.homotopy_problem([(target, q)], gamma, [(0, p) for p in pts])
    rmode = 4 if prec == 4 else 2
    h = hm.track_host(pb, pmode=1, rmode=rmode)
    assert np.array_equal(got["status"], h.status)
    assert np.array_equal(got["x"].reshape(-1), h.xend)
    assert np.array_equal(got["res"], h.residual) and np.array_equal(got["t"], h.t)
    manypaths.clear()
    return h


def test_drop_in_cyclic5(capfd):
    polys, sym = phcio.parse_system(cyclic_text(5))
    gamma = complex(np.exp(0.7j))
    h = drop_in_vs_host(polys, gamma, 2, capfd)
    assert (h.status == 0).sum() >= 60


def test_drop_in_dense_quadratic_1024_paths():
    rng = np.random.default_rng(4)
    target = hm.dense_quadratic(rng, 10)
    gamma = complex(hm.unit(rng))
    h = drop_in_vs_host(target, gamma, 2)
    assert (h.status == 0).all()


def test_drop_in_quad_double():
    rng = np.random.default_rng(9)
    target = hm.dense_quadratic(rng, 4)
    gamma = complex(hm.unit(rng))
    h = drop_in_vs_host(target, gamma, 4)
    assert (h.status == 0).all()
