"""Multi-homogeneous root counts and linear-product start systems, the
feeders of paths into the batched tracker besides the total-degree start.

For a partition of the variables into m sets (set j with k_j variables) and
the degree d_ij of polynomial i in the variables of set j, the
m-homogeneous Bezout number is the sum over all assignments of polynomials
to sets with set j chosen exactly k_j times of the products of the d_ij
(Root_Counts/Product/m_homogeneous_bezout_numbers.adb).  A linear-product
start system with that many regular roots replaces polynomial i by a
product of d_ij random linear forms in the variables of set j, over all j
(Root_Counts/Product/m_homogeneous_start_systems.adb): its roots are found by
choosing one linear factor per polynomial consistently with the
assignment and solving the linear systems, one block of k_j equations in
the k_j variables of each set.
"""
from __future__ import annotations

import itertools
from functools import lru_cache

import numpy as np

from . import homotopy as hm


def degree_table(polys, partition):
    """d[i][j] = the degree of polynomial i in the variables of set j."""
    where = {}
    for j, part in enumerate(partition):
        for v in part:
            where[v] = j
    d = np.zeros((len(polys), len(partition)), dtype=np.int64)
    for i, p in enumerate(polys):
        for m, _ in p:
            deg = np.zeros(len(partition), dtype=np.int64)
            for v, e in m:
                deg[where[v]] += e
            d[i] = np.maximum(d[i], deg)
    return d


def bezout_number(polys, partition):
    """The m-homogeneous Bezout number of the system for the partition (a
    list of lists of variable indices)."""
    d = degree_table(polys, partition)
    sizes = tuple(len(p) for p in partition)
    n = len(polys)
    if sum(sizes) != n:
        raise ValueError("the partition must cover as many variables as there are polynomials")

    @lru_cache(maxsize=None)
    def count(i, left):
        if i == n:
            return 1
        total = 0
        for j, k in enumerate(left):
            if k > 0 and d[i, j] > 0:
                rest = left[:j] + (k - 1,) + left[j + 1:]
                total += int(d[i, j]) * count(i + 1, rest)
        return total

    return count(0, sizes)


def _set_partitions(items):
    if not items:
        yield []
        return
    first, rest = items[0], items[1:]
    for part in _set_partitions(rest):
        for i in range(len(part)):
            yield part[:i] + [[first] + part[i]] + part[i + 1:]
        yield [[first]] + part


def best_partition(polys, nvar, max_vars=9):
    """The partition of the variables with the smallest m-homogeneous Bezout
    number, by enumeration of all set partitions (nvar <= max_vars);
    larger systems get the 1-homogeneous (total degree) partition."""
    if nvar > max_vars:
        part = [list(range(nvar))]
        return part, bezout_number(polys, part)
    best, best_b = None, None
    for part in _set_partitions(list(range(nvar))):
        part = [sorted(p) for p in part]
        b = bezout_number(polys, part)
        if best_b is None or b < best_b or (b == best_b and len(part) < len(best)):
            best, best_b = part, b
    return sorted(best, key=lambda p: p[0]), best_b


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


def linear_product_start(polys, partition, rng):
    """A random linear-product start system for the partition and all its
    roots.  Returns (start polynomials as lists of (monomial, coefficient),
    list of start points, the linear forms)."""
    n = len(polys)
    d = degree_table(polys, partition)
    forms = []  # forms[i][j][r] = (constant, {variable: coefficient})
    q = []
    for i in range(n):
        fi = []
        prod = {(): 1.0 + 0j}
        for j, part in enumerate(partition):
            fij = []
            for _ in range(int(d[i, j])):
                c = hm.unit(rng, len(part) + 1)
                lin = {(): complex(c[0])}
                for v, cv in zip(part, c[1:]):
                    lin[((v, 1),)] = complex(cv)
                fij.append((complex(c[0]), dict(zip(part, (complex(x) for x in c[1:])))))
                prod = _pmul(prod, lin)
            fi.append(fij)
        forms.append(fi)
        q.append([(m, complex(c)) for m, c in sorted(prod.items()) if c != 0])
    sizes = [len(p) for p in partition]
    roots = []
    # assignments of polynomials to sets with set j used sizes[j] times
    for assign in itertools.product(range(len(partition)), repeat=n):
        if any(assign.count(j) != sizes[j] for j in range(len(partition))):
            continue
        if any(d[i, assign[i]] == 0 for i in range(n)):
            continue
        for choice in itertools.product(*[range(int(d[i, assign[i]])) for i in range(n)]):
            x = np.zeros(n, complex)
            for j, part in enumerate(partition):
                rows = [i for i in range(n) if assign[i] == j]
                A = np.zeros((len(rows), len(part)), complex)
                b = np.zeros(len(rows), complex)
                for a, i in enumerate(rows):
                    c0, cv = forms[i][j][choice[i]]
                    b[a] = -c0
                    for col, v in enumerate(part):
                        A[a, col] = cv[v]
                xs = np.linalg.solve(A, b)
                for col, v in enumerate(part):
                    x[v] = xs[col]
            roots.append(x)
    return q, roots, forms


def linear_product_problem(polys, partition, gamma, rng) -> hm.TrackProblem:
    """The homotopy (1 - t) gamma q + t p from a linear-product start system
    q for the partition, with all of q's roots as start points."""
    q, roots, _ = linear_product_start(polys, partition, rng)
    return hm.homotopy_problem([(polys, q)], gamma, [(0, x) for x in roots])


# ------------------------------------------------------------ mixed volume
# The BKK bound: the number of isolated roots with nonzero coordinates of a
# system with generic coefficients is the mixed volume of its Newton
# polytopes, computed natively by phc_mixed_volume (include/phc_b200.h; the
# method of MixedVol, Root_Counts/MixedVol/mixedvol_algorithm.adb: random
# lifting, lower edges, relation table, depth-first search of the mixed
# cells with LP feasibility tests).

def _supports(polys, nvar):
    out = []
    for p in polys:
        pts = set()
        for m, c in p:
            if c == 0:
                continue
            e = [0] * nvar
            for v, k in m:
                e[v] += k
            pts.add(tuple(e))
        out.append(np.array(sorted(pts), dtype=np.int64).reshape(-1, nvar))
    return out


def mixed_cells(supports, seed=0, max_cells=1 << 16):
    """Mixed volume and mixed cells of a random lifting of n supports (arrays
    of exponent vectors in n variables).  Returns (mixed volume, cells): a
    cell is an n x 2 array of point indices, one edge per support."""
    from . import _lib
    n = len(supports)
    if any(np.asarray(a).reshape(-1, n).shape[1] != n for a in supports):
        raise ValueError("mixed_cells: need n supports in n variables")
    counts = np.array([len(a) for a in supports], np.int32)
    pts = np.ascontiguousarray(np.concatenate([np.asarray(a, np.int64).reshape(-1, n) for a in supports])
                               .astype(np.int32).reshape(-1))
    cells = np.zeros(max(1, max_cells) * 2 * n, np.int32)
    nc = np.zeros(1, np.int64)
    lib = _lib.lib()
    f = lib.phc_mixed_volume
    f.restype = _lib.ctypes.c_longlong
    mv = int(f(n, _lib.ptr(counts), _lib.ptr(pts), _lib.ctypes.c_ulonglong(seed), int(max_cells), _lib.ptr(cells),
               _lib.ptr(nc)))
    if mv < 0:
        raise _lib.PhcError("phc_mixed_volume", mv, lib.phc_last_error().decode(errors="replace"))
    k = int(min(nc[0], max_cells))
    return mv, cells[:k * 2 * n].reshape(k, n, 2)


def mixed_volume(polys, nvar=None, seed=0):
    """The mixed volume of the Newton polytopes of a square system (a list
    of polynomials as lists of (monomial, coefficient))."""
    nvar = len(polys) if nvar is None else nvar
    mv, _ = mixed_cells(_supports(polys, nvar), seed, max_cells=0)
    return mv


def _monomial(e):
    return tuple((v, int(k)) for v, k in enumerate(e) if k > 0)


def mixed_volume_start(polys, nvar, rng, pmode=1, rmode=2, **kw):
    """A start system with as many paths as the mixed volume: q has the
    supports of polys and random coefficients on the unit circle, and its
    roots with nonzero coordinates (as many as the mixed volume, for generic
    coefficients) are found once by the total-degree homotopy on the GPU.
    q then starts the linear homotopy (1 - t) gamma q + t p to polys, or to
    any system with the same supports (a cheater's homotopy), with one path
    per root instead of one per total-degree start point.  Returns (q, the
    distinct roots of q with nonzero coordinates, the mixed volume)."""
    S = _supports(polys, nvar)
    mv = mixed_volume(polys, nvar)
    q = [[(_monomial(e), complex(hm.unit(rng))) for e in S[i]] for i in range(len(polys))]
    qq, degs = hm.total_degree_start(q)
    pb = hm.homotopy_problem([(q, qq)], complex(hm.unit(rng)), [(0, x) for x in hm.total_degree_solutions(degs)])
    r = hm.track_host(pb, pmode=pmode, rmode=rmode, **kw)
    x = r.endpoints(pb.maxdim)[r.status == 0, :nvar]
    x = x[np.abs(x).min(axis=1) > 1e-8] if len(x) else x
    roots = []
    for v in x:
        if all(np.abs(v - w).max() > 1e-8 * max(1.0, np.abs(v).max()) for w in roots):
            roots.append(v)
    return q, roots, mv
