"""PHCpack text formats (phcpack_b200.phcio): the readers pinned against the
reference's example systems and their solution lists (tests/golden/
phcio_demo.json, made by tests/golden/make_phcio_golden.py), the grammar,
exact number output and round trips.  CPU only."""
import json
import os
from decimal import Decimal, getcontext
from fractions import Fraction

import numpy as np
import pytest

from phcpack_b200 import homotopy as hm
from phcpack_b200 import phcio

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "phcio_demo.json")


def test_reference_demo_systems_and_solutions():
    d = json.load(open(GOLDEN))
    assert len(d) >= 120
    unparsed = sorted(k for k, v in d.items() if not v["parsed"])
    assert unparsed == ["READ_ME"]  # the directory's description, not a system
    mismatch = {k: (v["total_degree"], v["stated_total_degree"]) for k, v in d.items()
                if v["parsed"] and v["stated_total_degree"] is not None
                and v["stated_total_degree"] != v["total_degree"]}
    # d1 states 4068; its degrees 2,2,2,2,2,2,1,2,2,2,3,3 multiply to 4608
    assert mismatch == {"d1": (4608, 4068)}
    assert d["d1"]["degrees"] == [2, 2, 2, 2, 2, 2, 1, 2, 2, 2, 3, 3]
    checked = sum(1 for v in d.values() if v["parsed"] and v["stated_total_degree"] is not None)
    assert checked >= 100
    with_sols = [v for v in d.values() if "solutions" in v]
    assert len(with_sols) >= 100 and not any("solutions_error" in v for v in d.values())
    assert sum(v["solutions_at_t1"] for v in with_sols) > 14000
    for v in with_sols:
        assert v["at_t1_residuals_below_1e-8"] == v["solutions_at_t1"]
    c5 = d["cyclic5"]
    assert (c5["neq"], c5["nvar"], c5["terms"], c5["degrees"]) == (5, 5, [5, 5, 5, 5, 2], [1, 2, 3, 4, 5])


def cyclic_text(n):
    x = [f"x{i + 1}" for i in range(n)]
    rows = []
    for k in range(1, n):
        rows.append(" + ".join("*".join(x[(i + j) % n] for j in range(k)) for i in range(n)) + ";")
    rows.append("*".join(x) + " - 1;")
    return f"{n}\n" + "\n".join(rows) + "\n"


def test_cyclic5_matches_the_demo_summary():
    polys, sym = phcio.parse_system(cyclic_text(5))
    c5 = json.load(open(GOLDEN))["cyclic5"]
    assert [len(p) for p in polys] == c5["terms"]
    assert [hm.degree(p) for p in polys] == c5["degrees"]
    assert sym == ["x1", "x2", "x3", "x4", "x5"]


def as_dict(polys):
    return [dict(p) for p in polys]


def test_grammar():
    txt = """2 2
    -x^2 + 3*y**2 - 1/2*x*y + 1.5E-01;
    (x - y)*(x + 2*y) - (1 + 2*i)*x^(2)*y + 4*i - (x+y)^2 + x*-2;
    TITLE : not part of the system
    """
    polys, sym = phcio.parse_system(txt)
    assert sym == ["x", "y"]
    X, Y = (0, 1), (1, 1)
    p0, p1 = as_dict(polys)
    assert p0 == {((0, 2),): -1, ((1, 2),): 3, (X, Y): -0.5, (): 0.15}
    # (x - y)(x + 2y) = x^2 + xy - 2y^2; -(x + y)^2 = -x^2 - 2xy - y^2; -2x
    assert p1 == {(X, Y): -1, ((1, 2),): -3, ((0, 2), Y): -(1 + 2j), (): 4j, (X,): -2}


def test_grammar_errors():
    with pytest.raises(phcio.ParseError):
        phcio.parse_system("2\n x + y;\n")  # one polynomial short
    with pytest.raises(phcio.ParseError):
        phcio.parse_system("1\n x + y;\n")  # two variables, the line says one
    with pytest.raises(phcio.ParseError):
        phcio.parse_system("1\n x^y;\n")  # exponent not an integer
    with pytest.raises(phcio.ParseError):
        phcio.parse_system("1\n x $ 1;\n")
    with pytest.raises(phcio.ParseError):
        phcio.parse_system("1\n (x + 1;\n")
    with pytest.raises(phcio.ParseError):
        phcio.parse_system("x + 1;\n")  # no dimension line


def test_system_round_trip():
    rng = np.random.default_rng(3)
    for n in (1, 3, 6):
        polys = hm.dense_quadratic(rng, n)
        polys = [[(m, c * (10.0 ** rng.integers(-20, 20))) for m, c in p] for p in polys]
        sym = [f"z{i}" for i in range(n)]
        text = phcio.write_system(polys, sym)
        back, sym2 = phcio.parse_system(text)
        assert sym2 == sym
        assert as_dict(back) == [dict((tuple(sorted(m)), c) for m, c in p) for p in polys]


def exact_decimal(limbs, digits):
    getcontext().prec = 400
    v = sum((Decimal(float(x)) for x in limbs), Decimal(0))
    return f"{v:.{digits - 1}E}"


def test_format_number_is_exact_and_rounds_half_even():
    rng = np.random.default_rng(5)
    for _ in range(200):
        hi = float(rng.standard_normal() * 10.0 ** rng.integers(-30, 30))
        lo = hi * 2.0 ** -53 * float(rng.uniform(-1, 1))
        for digits in (17, 32, 40):
            s = phcio.format_number([hi, lo], digits)
            ref = exact_decimal([hi, lo], digits)
            assert Decimal(s.strip()) == Decimal(ref), (s, ref)
    assert phcio.format_number([0.125], 2) == " 1.2E-01"  # half to even
    assert phcio.format_number([0.375], 2) == " 3.8E-01"
    assert phcio.format_number([-2.5], 1) == "-2.E+00"
    assert phcio.format_number([0.0], 4) == " 0.000E+00"


def test_parse_number_limbs():
    third = Fraction(1, 3)
    s = "3.333333333333333333333333333333333333333333333333333333333333333E-01"
    for nl in (1, 2, 4):
        limbs = phcio.parse_number(s, nl)
        err = abs(phcio.limbs_to_fraction(limbs) - third)
        assert err <= Fraction(1, 3) * Fraction(2) ** (-52 * nl) + Fraction(10) ** -64


def test_solutions_round_trip_dd_and_names():
    rng = np.random.default_rng(9)
    sym = ["x", "y", "z"]
    sols = []
    for _ in range(5):
        hi = rng.standard_normal((3, 2))
        lo = hi * 2.0 ** -53 * rng.uniform(-1, 1, (3, 2))
        x = np.stack([hi + lo, (hi - (hi + lo)) + lo], axis=-1)  # normalised (hi, lo)
        sols.append(dict(t=1.0, m=1, x=x, err=1e-30, rco=0.25, res=3e-31))
    text = phcio.write_solutions(sols, sym, digits=32)
    back = phcio.parse_solutions(text, symbols=sym, nlimbs=2)
    assert len(back) == 5
    for s, b in zip(sols, back):
        for j in range(3):
            for part in range(2):
                a = phcio.limbs_to_fraction(s["x"][j, part])
                c = phcio.limbs_to_fraction(b["x"][j, part])
                assert abs(a - c) <= abs(a) * Fraction(10) ** -31
        assert b["res"] == pytest.approx(3e-31) and b["rco"] == pytest.approx(0.25)
    # coordinates listed in another order are placed by name
    lines = text.splitlines()
    k = lines.index("the solution for t :")
    lines[k + 1], lines[k + 3] = lines[k + 3], lines[k + 1]
    back2 = phcio.parse_solutions("\n".join(lines), symbols=sym, nlimbs=2)
    assert np.array_equal(back2[0]["x"], back[0]["x"])


def test_explicit_total_degree_start_matches_builder():
    rng = np.random.default_rng(11)
    polys = hm.sparse_quadratic(rng, 4)
    gamma = complex(hm.unit(rng))
    a = hm.total_degree_problem([polys], gamma, maxvar=2)
    q, degs = hm.total_degree_start(polys)
    b = hm.homotopy_problem([(polys, q)], gamma, [(0, x) for x in hm.total_degree_solutions(degs)], maxvar=2)
    for k in ("dim", "mono_off", "mono_nvr", "mono_idx", "mono_exp", "eq_off", "term_off", "term_mono", "term_a",
              "term_b", "path_sys", "x0"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k


def test_mhom_bezout_numbers_match_the_reference_demo_statements():
    d = json.load(open(GOLDEN))
    stated = [x for v in d.values() for x in v.get("mhom_bezout", [])]
    assert len(stated) >= 60
    assert all(x["computed"] == x["stated"] for x in stated)


def eigen_text(A, c):
    """(A - lam I) v = 0, c . v = 1: n + 1 equations in v1..vn, lam."""
    n = A.shape[0]
    rows = []
    for i in range(n):
        terms = [f"({float(A[i, j].real)!r} + {float(A[i, j].imag)!r}*i)*v{j + 1}" for j in range(n)]
        rows.append(" + ".join(terms) + f" - lam*v{i + 1};")
    rows.append(" + ".join(f"({float(c[j].real)!r} + {float(c[j].imag)!r}*i)*v{j + 1}" for j in range(n)) + " - 1;")
    return f"{n + 1}\n" + "\n".join(rows) + "\n"


def test_linear_product_start_system():
    from phcpack_b200 import rootcounts
    rng = np.random.default_rng(4)
    n = 4
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    c = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    polys, sym = phcio.parse_system(eigen_text(A, c))
    lam = sym.index("lam")
    vs = [k for k in range(len(sym)) if k != lam]
    assert rootcounts.bezout_number(polys, [list(range(len(sym)))]) == 2 ** n
    assert rootcounts.bezout_number(polys, [[lam], vs]) == n
    part, b = rootcounts.best_partition(polys, len(sym))
    assert b == n and sorted(map(sorted, part)) == sorted([[lam], sorted(vs)])
    q, roots, _ = rootcounts.linear_product_start(polys, part, np.random.default_rng(0))
    assert len(roots) == n
    for x in roots:
        for poly in q:
            v = sum(cf * np.prod([x[j] ** e for j, e in m]) for m, cf in poly)
            assert abs(v) <= 1e-10
    assert np.min(np.abs(np.subtract.outer(np.array(roots)[:, 0], np.array(roots)[:, 0])) + np.eye(n)) > 1e-8


def test_root_accounting():
    sols = [
        dict(x=np.array([1.0 + 0j, -2.0 + 1e-15j]), rco=0.3, res=1e-30),          # real regular
        dict(x=np.array([1.0 + 1j, 2.0 + 0j]), rco=1e-12, res=1e-30),            # complex singular, with #3
        dict(x=np.array([1.0 + 1j, 2.0 + 1e-14j]), rco=1e-11, res=1e-30),        # complex singular, with #2
        dict(x=np.array([3.0 + 1j, 4.0 + 0j]), rco=0.2, res=1e-30),              # complex regular, clustered
        dict(x=np.array([3.0 + 1j, 4.0 + 0j]), rco=0.2, res=1e-30),              # complex regular, clustered
        dict(x=np.array([1e9 + 0j, 1.0 + 0j]), rco=0.1, res=1.0),                # at infinity
        dict(x=np.array([0.5 + 0.5j, 0.1 + 0j]), rco=0.1, res=1e-3),             # failed path
        dict(x=np.array([7.0 + 0j, 5.0 - 3j]), rco=1e-9, res=1e-30),             # complex singular, alone
    ]
    fail = np.array([0, 0, 0, 0, 0, 1, 1, 0], bool)
    cnt = phcio.root_accounting(sols, fail)
    kinds = [s["kind"] for s in sols]
    assert kinds == ["real regular", "complex singular", "complex singular", "complex regular", "complex regular",
                     "at infinity", "no solution", "complex singular"]
    assert [s.get("m") for s in sols] == [None, 2, 2, -5, -4, None, 0, 0]
    assert cnt == dict(total=8, regular=3, singular=3, real=1, complex=5, clustered=2, infinity=1, failures=1)
    text = phcio.write_solutions([dict(s, t=1.0) for s in sols], ["x", "y"], digits=20)
    assert "= res :  1.000E-30 = real regular ==" in text and "= at infinity ==" in text
    back = phcio.parse_solutions(text, symbols=["x", "y"])
    assert [b["m"] for b in back][:3] == [1, 2, 2]
    assert "Number of solutions at infinity : 1." in phcio.accounting_text(cnt)
