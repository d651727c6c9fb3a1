"""PHCpack's text formats for polynomial systems and solution lists, and a
text-in/text-out driver of the batched tracker.

The tracker entry ``gpumanypaths_dd(mode, verbose, regamma, imgamma)``
(Ada/PHCtoC/gpumanypaths_dd.h:27) reads the target system, the start system
and the start solutions from PHCpack's containers and writes the end points
back (gpumanypaths_dd.cpp:25-61, through lib2path_read_*_sys/_sols and
lib2path_write_*_sols, GPU/Path/Host/lib2path.h:37-69).  ``manypaths`` does
the same with the containers' text forms, so that a caller without the Ada
runtime can hand over what ``phc`` reads and writes:

* systems: a first line with the number of polynomials (optionally followed
  by the number of variables), then each polynomial terminated by ';' --
  sums of terms with '+', '-', '*', '^' or '**' integer powers, parentheses,
  floating-point numbers and quotients of numbers (1/2), 'i' or 'I' for the
  imaginary unit (standard_parse_numbers.adb:388-400), and variables
  named by symbols, numbered in order of first appearance (the grammar of
  Parse_Polynomial, Math_Lib/Polynomials/standard_complex_poly_strings.adb
  :312-414);
* solution lists: "len dim", a bar of '=', then per solution "solution k :",
  "t : re im", "m : mult", "the solution for t :", one line "name : re im"
  per variable and the diagnostics "== err : e = rco : r = res : s ==",
  followed by "=" (Deformations/Solutions/dobldobl_complex_solutions_io.adb
  :215-230, :331-356 and put_bar of standard_complex_solutions_io.adb:553).

Numbers are written with 32 (double-double) or 64 (quad-double) significant
digits from the exact sum of their limbs; numbers are read exactly and
rounded to the nearest multiple-double.  The tracker's coefficients and
start points are doubles (include/phc_b200.h, phc_track), so coefficients
and start solutions are rounded to double on the way in.
"""
from __future__ import annotations

import re
from fractions import Fraction

import numpy as np

from . import homotopy as hm

_TOKEN = re.compile(r"""\s*(?:
    (?P<num>(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?) |
    (?P<sym>[A-Za-z_][A-Za-z0-9_\[\]]*) |
    (?P<op>\*\*|[-+*/^();])
)""", re.VERBOSE)


class ParseError(ValueError):
    pass


def _tokens(text):
    out, pos = [], 0
    text = text.rstrip()
    while pos < len(text):
        m = _TOKEN.match(text, pos)
        if m is None or m.end() == pos:
            raise ParseError(f"unexpected character {text[pos]!r} at offset {pos}")
        kind = m.lastgroup
        out.append((kind, m.group(kind), m.start(kind)))
        pos = m.end()
    return out


# polynomials during parsing: dict {monomial: complex}, a monomial a sorted
# tuple of (variable, exponent) with exponent >= 1

def _padd(p, q, sign=1):
    r = dict(p)
    for m, c in q.items():
        r[m] = r.get(m, 0) + sign * c
    return r


def _pmul(p, q):
    r = {}
    for m1, c1 in p.items():
        for m2, c2 in q.items():
            e = dict(m1)
            for v, k in m2:
                e[v] = e.get(v, 0) + k
            m = tuple(sorted(e.items()))
            r[m] = r.get(m, 0) + c1 * c2
    return r


def _ppow(p, d):
    r = {(): 1.0 + 0j}
    for _ in range(d):
        r = _pmul(r, p)
    return r


class _Parser:
    def __init__(self, toks, symbols):
        self.t, self.k, self.sym = toks, 0, symbols

    def peek(self):
        return self.t[self.k] if self.k < len(self.t) else (None, None, -1)

    def take(self, val=None):
        tok = self.peek()
        if tok[0] is None or (val is not None and tok[1] != val):
            raise ParseError(f"expected {val!r} at token {self.k}, found {tok[1]!r}")
        self.k += 1
        return tok

    def poly(self):
        sign = 1
        if self.peek()[1] in ("+", "-"):
            sign = -1 if self.take()[1] == "-" else 1
        acc = _padd({}, self.term(), sign)
        while self.peek()[1] in ("+", "-"):
            sign = -1 if self.take()[1] == "-" else 1
            acc = _padd(acc, self.term(), sign)
        return acc

    def term(self):
        acc = self.factor()
        while self.peek()[1] == "*":
            self.take()
            acc = _pmul(acc, self.factor())
        return acc

    def factor(self):
        base = self.atom()
        if self.peek()[1] in ("^", "**"):
            self.take()
            if self.peek()[1] == "(":
                self.take()
                d = self.integer()
                self.take(")")
            else:
                d = self.integer()
            base = _ppow(base, d)
        return base

    def integer(self):
        kind, val, _ = self.take()
        if kind != "num" or not val.isdigit():
            raise ParseError(f"expected a nonnegative integer exponent, found {val!r}")
        return int(val)

    def atom(self):
        kind, val, _ = self.take()
        if kind == "num":
            v = float(val)
            if self.peek()[1] == "/":  # a quotient of numbers, as in 1/2*x
                self.take()
                kind2, val2, _ = self.take()
                if kind2 != "num":
                    raise ParseError(f"expected a number after '/', found {val2!r}")
                v = v / float(val2)
            return {(): complex(v)}
        if kind == "sym":
            if val in ("i", "I"):
                return {(): 1j}
            if val not in self.sym:
                self.sym.append(val)
            return {((self.sym.index(val), 1),): 1.0 + 0j}
        if val == "(":
            p = self.poly()
            self.take(")")
            return p
        if val == "-":  # a signed factor, as in x*-2
            return _padd({}, self.factor(), -1)
        raise ParseError(f"unexpected {val!r}")


def parse_polynomial(text, symbols):
    """One polynomial (no ';') over the symbol list, which grows with new
    names; returns a list of (monomial, coefficient), zero terms dropped."""
    ps = _Parser(_tokens(text), symbols)
    p = ps.poly()
    if ps.k != len(ps.t):
        raise ParseError(f"trailing input at token {ps.k}: {ps.t[ps.k][1]!r}")
    return [(m, complex(c)) for m, c in sorted(p.items()) if c != 0]


def parse_system(text, symbols=None):
    """A polynomial system in PHCpack's format (text after the last
    polynomial is ignored).  Returns (polynomials, symbols): polynomials as
    lists of (monomial, coefficient), monomials as tuples of (variable
    index, exponent), variables numbered by first appearance (after any
    names given in symbols)."""
    symbols = list(symbols or [])
    head, _, rest = text.strip().partition("\n")
    nums = head.split()
    try:
        neq = int(nums[0])
        nvar = int(nums[1]) if len(nums) > 1 else neq
    except (ValueError, IndexError):
        raise ParseError("the first line must hold the number of polynomials") from None
    if len(nums) > 2:
        raise ParseError("the first line holds at most two numbers")
    parts = rest.split(";")
    if len(parts) < neq + 1:
        raise ParseError(f"expected {neq} polynomials terminated by ';'")
    # what follows the last polynomial (titles, root counts, solutions) is
    # not part of the system
    polys = [parse_polynomial(parts[i], symbols) for i in range(neq)]
    if len(symbols) != nvar:
        raise ParseError(f"{len(symbols)} variables occur, the first line says {nvar}")
    return polys, symbols


def _num_str(x, digits=15):
    return f"{x:+.{digits - 1}E}"


def write_polynomial(poly, symbols):
    out = []
    for m, c in poly:
        coef = f"({_num_str(c.real, 17)} {_num_str(c.imag, 17)}*i)"
        mon = "".join(f"*{symbols[v]}" + (f"^{e}" if e > 1 else "") for v, e in m)
        out.append(f" + {coef}{mon}")
    return "".join(out) if out else " 0"


def write_system(polys, symbols):
    """PHCpack's format: the dimension line, then one polynomial per line."""
    lines = [f"{len(polys)}" + ("" if len(symbols) == len(polys) else f" {len(symbols)}")]
    lines += [write_polynomial(p, symbols) + ";" for p in polys]
    return "\n".join(lines) + "\n"


# ----------------------------------------------------------- numbers

def limbs_to_fraction(limbs):
    return sum((Fraction(float(v)) for v in limbs), Fraction(0))


def fraction_to_limbs(q, nlimbs):
    """The nearest multiple-double: greedy, each limb the double nearest to
    what is left."""
    out = []
    for _ in range(nlimbs):
        v = float(q)
        out.append(v)
        q -= Fraction(v)
    return out


def format_number(limbs, digits):
    """The exact value of a sum of doubles in scientific notation with
    digits significant digits, rounded half to even, PHCpack's style (a
    blank for the sign of positive numbers, E and a signed two-digit
    exponent)."""
    q = limbs_to_fraction(limbs)
    if q == 0:
        return " 0." + "0" * (digits - 1) + "E+00"
    sign = "-" if q < 0 else " "
    q = abs(q)
    e = len(str(q.numerator)) - len(str(q.denominator))
    while q >= Fraction(10) ** (e + 1):
        e += 1
    while q < Fraction(10) ** e:
        e -= 1
    scaled = q * Fraction(10) ** (digits - 1 - e)
    n = scaled.numerator // scaled.denominator
    rem = scaled - n
    if rem > Fraction(1, 2) or (rem == Fraction(1, 2) and n % 2 == 1):
        n += 1
    if n >= 10 ** digits:
        n //= 10
        e += 1
    s = str(n)
    return f"{sign}{s[0]}.{s[1:]}E{'+' if e >= 0 else '-'}{abs(e):02d}"


def parse_number(text, nlimbs=1):
    return fraction_to_limbs(Fraction(text.strip()), nlimbs)


# ----------------------------------------------------------- solutions

_SOL_LINE = re.compile(r"^\s*(\S+)\s*:\s*(\S+)\s+(\S+)\s*$")


def parse_solutions(text, symbols=None, nlimbs=1):
    """A solution list in PHCpack's format.  Returns a list of dicts with t
    (complex), m (int), x (nlimbs == 1: complex vector; else an array of
    shape (dim, 2, nlimbs) of limbs), names, err, rco, res.  Each solution
    is anchored on its "the solution for t :" line; its t and m lines are
    the last ones before it (t = 0 and m = 1 when absent).  With symbols,
    the coordinates are placed by name (as Symbol_Table lookups do in
    get_vector); otherwise in the order written."""
    lines = text.splitlines()
    k = 0
    while k < len(lines) and not lines[k].strip():
        k += 1
    head = lines[k].split()
    length, dim = int(head[0]), int(head[1])
    k += 1
    sols = []
    t, mult = 0j, 1
    while len(sols) < length:
        while k < len(lines) and "the solution for t" not in lines[k]:
            ln = lines[k].strip()
            if ln.startswith("t :"):
                m = _SOL_LINE.match(lines[k])
                t = complex(float(Fraction(m.group(2))), float(Fraction(m.group(3))))
            elif ln.startswith("m :"):
                mult = int(ln.split(":")[1].split()[0])
            k += 1
        if k >= len(lines):
            raise ParseError(f"found {len(sols)} of {length} solutions")
        k += 1
        names, vals = [], []
        for _ in range(dim):
            m = _SOL_LINE.match(lines[k]) if k < len(lines) else None
            if m is None:
                raise ParseError(f"line {k + 1}: expected 'name : re im'")
            names.append(m.group(1))
            vals.append((parse_number(m.group(2), nlimbs), parse_number(m.group(3), nlimbs)))
            k += 1
        diag = {}
        for key in ("err", "rco", "res"):
            g = re.search(key + r"\s*:\s*(\S+)", lines[k]) if k < len(lines) else None
            diag[key] = float(g.group(1)) if g else 0.0
        k += 1
        order = list(range(dim))
        if symbols is not None and sorted(names) == sorted(symbols[:dim]):
            order = [names.index(sname) for sname in symbols[:dim]]
            names = list(symbols[:dim])
        vals = [vals[i] for i in order]
        if nlimbs == 1:
            x = np.array([complex(re_[0], im_[0]) for re_, im_ in vals])
        else:
            x = np.array([[re_, im_] for re_, im_ in vals], dtype=np.float64)
        sols.append(dict(t=t, m=mult, x=x, names=names, **diag))
        t, mult = 0j, 1
    return sols


def write_solutions(sols, symbols, digits=32):
    """PHCpack's solution list format.  Each solution: t (complex), m, x
    (complex vector, or limbs of shape (dim, 2, nlimbs)), err, rco, res."""
    dim = len(symbols)
    out = [f"{len(sols)} {dim}", "=" * 75]
    for k, s in enumerate(sols, 1):
        x = np.asarray(s["x"])
        out.append(f"solution {k} :")
        t = complex(s.get("t", 1.0))
        out.append(f"t : {format_number([t.real], digits)}  {format_number([t.imag], digits)}")
        out.append(f"m : {int(s.get('m', 1))}")
        out.append("the solution for t :")
        for j in range(dim):
            if x.ndim == 1:
                re_, im_ = [x[j].real], [x[j].imag]
            else:
                re_, im_ = x[j, 0], x[j, 1]
            out.append(f" {symbols[j]} : {format_number(re_, digits)}  {format_number(im_, digits)}")
        kind = f" {s['kind']} ==" if "kind" in s else "="
        out.append("== err : " + f"{s.get('err', 0.0): .3E}" + " = rco : " + f"{s.get('rco', 1.0): .3E}" +
                   " = res : " + f"{s.get('res', 0.0): .3E}" + " =" + kind)
    return "\n".join(out) + "\n"


# ----------------------------------------------------------- root accounting

def root_accounting(sols, fail, tolsing=1e-8, tolclus=1e-12, tolreal=1e-13, infinity=1e8):
    """Classify end points as PHCpack's root refiners do (Write_Type and
    Multiplicity of Deformations/Newton/dobldobl_root_refiners.adb:53-111,
    At_Infinity and Is_Real of Solutions/dobldobl_solution_diagnostics.adb):
    a coordinate above `infinity` in modulus puts the point at infinity; a
    failed path is "no solution" (m = 0); otherwise the point is real when
    every imaginary part is at most tolreal, singular when rco < tolsing.  A
    singular point's multiplicity is the number of points equal to it within
    tolclus per coordinate (0 when it stands alone); regular points that
    coincide are marked clustered with m = -(index of the other, 1-based).
    Sets s["kind"] and s["m"] in place; returns the counts of
    Write_Global_Info."""
    pts = [np.asarray(s["x"]) for s in sols]
    pts = [p if p.ndim == 1 else p[:, 0, 0] + 1j * p[:, 1, 0] for p in pts]
    cnt = dict(total=len(sols), regular=0, singular=0, real=0, complex=0, clustered=0, infinity=0, failures=0)

    def equal(a, b):
        return bool(np.all(np.abs(a - b) <= tolclus))

    for k, s in enumerate(sols):
        x = pts[k]
        if np.any(~np.isfinite(x)) or np.any(np.abs(x) > infinity):
            s["kind"] = "at infinity"
            cnt["infinity"] += 1
            continue
        if fail[k]:
            s["kind"] = "no solution"
            s["m"] = 0
            cnt["failures"] += 1
            continue
        real = bool(np.all(np.abs(x.imag) <= tolreal))
        singular = s.get("rco", 1.0) < tolsing
        cnt["real" if real else "complex"] += 1
        cnt["singular" if singular else "regular"] += 1
        s["kind"] = ("real " if real else "complex ") + ("singular" if singular else "regular")
        others = [j for j in range(len(sols)) if j != k and not fail[j] and equal(x, pts[j])]
        if singular:
            s["m"] = len(others) + 1 if others else 0
        elif others:
            s["m"] = -(others[0] + 1)
            cnt["clustered"] += 1
    return cnt


def accounting_text(cnt):
    """The summary PHCpack writes after refining (Write_Global_Info)."""
    bar = "=" * 75
    rows = [("regular solutions", "regular"), ("singular solutions", "singular"), ("real solutions", "real"),
            ("complex solutions", "complex"), ("clustered solutions", "clustered"),
            ("solutions at infinity", "infinity"), ("failures", "failures")]
    out = [bar, f"A list of {cnt['total']} solutions has been refined :"]
    out += [f"Number of {name:<22}: {cnt[key]}." for name, key in rows]
    return "\n".join(out + [bar]) + "\n"


# ----------------------------------------------------------- the driver

def _eval_jac(polys, x):
    n = len(polys)
    J = np.zeros((n, len(x)), complex)
    for i, p in enumerate(polys):
        for m, c in p:
            for a, (v, e) in enumerate(m):
                d = c * e * x[v] ** (e - 1)
                for b, (u, f) in enumerate(m):
                    if b != a:
                        d = d * x[u] ** f
                J[i, v] += d
    return J


def manypaths(target, start=None, start_solutions=None, gamma=None, rmode=2, pmode=1, step_mode=0, model=None,
              seed=0, partition=None, endgame=True, **kw):
    """Track all paths of (1 - t) gamma q + t p from the start solutions of
    q to p on the GPU, in PHCpack's text formats: the counterpart of
    gpumanypaths_dd (rmode 2) and gpumanypaths_qd (rmode 4), and an
    octo-double refinement (rmode 8), with the containers replaced by text.
    target, start: systems (text).  Without a start system the total-degree
    start system x_i^{d_i} - 1 and all its roots-of-unity solutions are
    used; start="linear-product" builds a random linear-product start system
    and all its roots for a partition of the variables (partition: lists of
    variable names; default the partition with the smallest m-homogeneous
    Bezout number, phcpack_b200.rootcounts); start="mixed-volume" a system
    with the target's supports and random coefficients whose roots with
    nonzero coordinates, as many as the mixed volume, are found first on the
    GPU (rootcounts.mixed_volume_start).  gamma: complex (default:
    random on the unit circle from seed).  Returns (solution list text of
    the end points at t = 1, the TrackResult with the counts of
    root_accounting in its `accounting` attribute).  err is the forward
    error estimate |J^{-1}|_inf * res and rco the reciprocal 1-norm
    condition number of the Jacobian at the end point (both in double); the
    diagnostics line of each solution carries its kind ("complex regular",
    "at infinity", ...).  endgame: the paths that failed get the end-game
    diagnostics at their last point (phcpack_b200.endgame): the result's
    `endgame` maps each to "singular at t = 1" (diverging, or ending at a
    singular solution), "interior singularity", "regular" or "no series",
    and the accounting counts them under "endgame"."""
    polys, symbols = parse_system(target)
    if len(polys) != len(symbols):
        raise ParseError("the tracker needs as many polynomials as variables")
    if gamma is None:
        gamma = complex(hm.unit(np.random.default_rng(seed)))
    if start is None:
        q, degs = hm.total_degree_start(polys)
        xs = hm.total_degree_solutions(degs)
    elif start == "linear-product":
        from . import rootcounts
        if partition is None:
            part, _ = rootcounts.best_partition(polys, len(symbols))
        else:
            part = [[symbols.index(v) for v in st] for st in partition]
        q, xs, _ = rootcounts.linear_product_start(polys, part, np.random.default_rng(seed + 1))
    elif start == "mixed-volume":
        from . import rootcounts
        q, xs, _ = rootcounts.mixed_volume_start(polys, len(symbols), np.random.default_rng(seed + 1))
    else:
        q, _ = parse_system(start, symbols=list(symbols))
        if start_solutions is None:
            raise ValueError("a start system needs its start solutions")
        xs = [s["x"] for s in parse_solutions(start_solutions, symbols=symbols)]
    pb = hm.homotopy_problem([(polys, q)], gamma, [(0, x) for x in xs])
    r = hm.track_host(pb, pmode=pmode, rmode=rmode, step_mode=step_mode, model=model, **kw)
    n = len(symbols)
    nl = rmode
    xe = r.xend.reshape(pb.npaths, pb.maxdim, 2, r.limbs)[:, :n, :, :nl]
    sols = []
    for p in range(pb.npaths):
        x = r.endpoints(pb.maxdim)[p, :n]
        J = _eval_jac(polys, x)
        try:
            Ji = np.linalg.inv(J)
            rco = 1.0 / (np.abs(J).sum(axis=0).max() * np.abs(Ji).sum(axis=0).max())
            err = float(np.abs(Ji).sum(axis=1).max() * r.residual[p])
        except np.linalg.LinAlgError:
            rco, err = 0.0, float("inf")
        # a successful path's end point is refined at t = 1 exactly
        t_end = 1.0 if r.status[p] == 0 else float(r.t[p])
        sols.append(dict(t=complex(t_end), m=1, x=xe[p], err=err, rco=rco, res=float(r.residual[p])))
    r.accounting = root_accounting(sols, r.status != 0)
    # the end game of the failed paths: where is the nearest singular point?
    r.endgame = {}
    bad = np.flatnonzero(r.status != 0)
    if endgame and len(bad):
        from . import endgame as eg
        xe = r.xend.reshape(pb.npaths, -1)[bad]
        d = eg.series_diagnostics(hm.subset(pb, bad), xe, r.t[bad], xlimbs=r.limbs, pmode=2)
        r.endgame = {int(p): c for p, c in zip(bad, eg.classify(r.t[bad], d))}
        counts = {}
        for c in r.endgame.values():
            counts[c] = counts.get(c, 0) + 1
        r.accounting["endgame"] = counts
    return write_solutions(sols, symbols, digits={2: 32, 4: 64, 8: 128}[rmode]), r
