"""Text-in/text-out tracking (phcpack_b200.phcio.manypaths, the counterpart of
gpumanypaths_dd / _qd) on the GPU."""
from decimal import Decimal, getcontext
from fractions import Fraction

import numpy as np
import pytest

from phcpack_b200 import homotopy as hm
from phcpack_b200 import phcio

pytestmark = pytest.mark.gpu


def _inv_sqrt2(digits=160):
    getcontext().prec = digits
    return Fraction(Decimal(1) / Decimal(2).sqrt())


RESTOL = {2: 1e-24, 4: 1e-48, 8: 1e-100}


@pytest.mark.parametrize("rmode,tol", [(2, 1e-30), (4, 1e-60), (8, 1e-120)])
def test_circle_and_line_dd_qd_od(rmode, tol):
    text, r = phcio.manypaths("2\n x^2 + y^2 - 1;\n x - y;\n", rmode=rmode, restol=RESTOL[rmode])
    assert (r.status == 0).all()
    sols = phcio.parse_solutions(text, symbols=["x", "y"], nlimbs=rmode)
    assert len(sols) == 2
    c = _inv_sqrt2()
    signs = sorted(np.sign(s["x"][0, 0, 0]) for s in sols)
    assert signs == [-1.0, 1.0]
    for s in sols:
        sg = 1 if s["x"][0, 0, 0] > 0 else -1
        for j in range(2):
            re_ = phcio.limbs_to_fraction(s["x"][j, 0])
            im_ = phcio.limbs_to_fraction(s["x"][j, 1])
            assert abs(re_ - sg * c) <= tol and abs(im_) <= tol
        assert s["t"] == 1.0 and s["res"] <= RESTOL[rmode]


def cyclic_text(n):
    x = [f"x{i + 1}" for i in range(n)]
    rows = [" + ".join("*".join(x[(i + j) % n] for j in range(k)) for i in range(n)) + ";" for k in range(1, n)]
    return f"{n}\n" + "\n".join(rows) + "\n" + "*".join(x) + " - 1;\n"


def test_cyclic5_endpoints():
    """cyclic 5-roots: 120 total-degree paths, 70 isolated regular roots;
    the other paths diverge.  Every path classified as success ends at a
    root (residual <= 1e-24 in double-double) and the roots found are
    distinct solutions of the system."""
    text, r = phcio.manypaths(cyclic_text(5), seed=2, maxsteps=2000)
    polys, sym = phcio.parse_system(cyclic_text(5))
    sols = phcio.parse_solutions(text, symbols=sym)
    assert len(sols) == 120
    ok = np.flatnonzero(r.status == 0)
    assert len(ok) >= 60
    pts = np.array([sols[p]["x"] for p in ok])
    for p in ok:
        assert sols[p]["res"] <= 1e-24
    # distinct roots among the successes
    d = np.abs(pts[:, None, :] - pts[None, :, :]).max(axis=2) + np.eye(len(ok))
    assert (d > 1e-6).all()
    # root accounting: the successes are regular roots, the rest diverged
    a = r.accounting
    assert a["regular"] == len(ok) and a["singular"] == 0 and a["clustered"] == 0
    assert a["regular"] + a["infinity"] + a["failures"] == 120
    assert all(sols[p]["m"] == 1 for p in ok)
    # the end game places the singular point of the failed paths at t = 1
    assert len(r.endgame) == 120 - len(ok)
    assert list(r.endgame.values()).count("singular at t = 1") >= 0.8 * len(r.endgame)


def test_given_start_system_and_solutions_match_total_degree():
    target = "3\n x^2 + y*z - 1;\n y^2 + x - 2*i;\n z^2 + x*y - 3;\n"
    polys, sym = phcio.parse_system(target)
    q, degs = hm.total_degree_start(polys)
    start = phcio.write_system(q, sym)
    sols = [dict(t=0.0, m=1, x=x, err=0.0, rco=1.0, res=0.0) for x in hm.total_degree_solutions(degs)]
    start_sols = phcio.write_solutions(sols, sym, digits=17)
    g = complex(hm.unit(np.random.default_rng(0)))
    t1, r1 = phcio.manypaths(target, gamma=g)
    t2, r2 = phcio.manypaths(target, start, start_sols, gamma=g)
    assert np.array_equal(r1.status, r2.status)
    assert np.abs(r1.endpoints(3) - r2.endpoints(3)).max() <= 1e-28


def test_linear_product_start_eigenproblem():
    """(A - lam I) v = 0, c . v = 1 has total degree 2^n but n solutions, the
    2-homogeneous Bezout number for the partition {lam}{v}: tracked from a
    linear-product start system, every path converges and the lam
    coordinates are the eigenvalues of A."""
    rng = np.random.default_rng(6)
    n = 6
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    c = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    rows = []
    for i in range(n):
        terms = [f"({float(A[i, j].real)!r} + {float(A[i, j].imag)!r}*i)*v{j + 1}" for j in range(n)]
        rows.append(" + ".join(terms) + f" - lam*v{i + 1};")
    rows.append(" + ".join(f"({float(c[j].real)!r} + {float(c[j].imag)!r}*i)*v{j + 1}" for j in range(n)) + " - 1;")
    target = f"{n + 1}\n" + "\n".join(rows) + "\n"
    text, r = phcio.manypaths(target, start="linear-product")
    assert r.status.shape == (n,) and (r.status == 0).all()
    polys, sym = phcio.parse_system(target)
    sols = phcio.parse_solutions(text, symbols=sym)
    lam = sym.index("lam")
    got = np.sort_complex(np.array([s["x"][lam] for s in sols]))
    want = np.sort_complex(np.linalg.eigvals(A))
    assert np.abs(got - want).max() <= 1e-10
    assert all(s["res"] <= 1e-24 for s in sols)


def test_mixed_volume_start_cyclic5():
    """cyclic 5-roots from a start system with its supports: the mixed
    volume, 70, is the number of paths (against 120 total-degree paths),
    and every path ends at a distinct root."""
    from phcpack_b200 import rootcounts
    polys, sym = phcio.parse_system(cyclic_text(5))
    assert rootcounts.mixed_volume(polys, len(sym)) == 70
    text, r = phcio.manypaths(cyclic_text(5), start="mixed-volume", seed=3, maxsteps=2000)
    assert r.status.shape == (70,) and (r.status == 0).all()
    sols = phcio.parse_solutions(text, symbols=sym)
    pts = np.array([s["x"] for s in sols])
    d = np.abs(pts[:, None, :] - pts[None, :, :]).max(axis=2) + np.eye(len(pts))
    assert (d > 1e-6).all()
    assert all(s["res"] <= 1e-24 for s in sols)
