"""The mixed volume (phc_mixed_volume, rootcounts.mixed_volume) against the
mixed volumes that the reference's example systems state
(tests/golden/mixed_volume_demo.json, made by make_mixed_volume_golden.py
from src/Demo), recomputed here from the stored supports, and against
closed forms."""
import ctypes
import json
import os

import numpy as np
import pytest

from phcpack_b200 import _lib
from phcpack_b200 import homotopy as hm
from phcpack_b200 import rootcounts as rc

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "mixed_volume_demo.json")))


def test_fixture_agrees_with_the_stated_mixed_volumes():
    done = {k: v for k, v in GOLD.items() if "computed" in v}
    assert len(done) >= 100
    bad = {k: (v["stated"], v["computed"]) for k, v in done.items() if v["stated"] != v["computed"]}
    assert not bad, bad


FAST = sorted(k for k, v in GOLD.items() if "computed" in v and v["seconds"] <= 0.05)


@pytest.mark.parametrize("name", FAST)
def test_recompute_from_supports(name):
    g = GOLD[name]
    S = [np.array(s, dtype=np.int64).reshape(-1, g["nvar"]) for s in g["supports"]]
    mv, cells = rc.mixed_cells(S, seed=3)
    assert mv == g["stated"]
    # the cells' volumes add up to the mixed volume
    vol = sum(abs(round(np.linalg.det(np.array([S[i][q] - S[i][p] for i, (p, q) in enumerate(c)], float))))
              for c in cells)
    assert vol == mv


def test_closed_forms():
    rng = np.random.default_rng(0)
    # dense quadratics: the mixed volume is the Bezout number 2^n
    assert rc.mixed_volume(hm.dense_quadratic(rng, 4)) == 16
    # (A - lam I) v = 0, c . v = 1: n eigenpairs
    n = 5
    polys = []
    for i in range(n):
        p = [(((j, 1),), 1.0 + 0j) for j in range(n)]
        p.append((((i, 1), (n, 1)), -1.0 + 0j))
        polys.append(p)
    polys.append([(((j, 1),), 1.0 + 0j) for j in range(n)] + [((), -1.0 + 0j)])
    assert rc.mixed_volume(polys, n + 1) == n
    # a support of one point: no roots with nonzero coordinates
    assert rc.mixed_volume([[(((0, 1),), 1.0 + 0j)], [(((1, 1),), 1.0 + 0j), ((), 1.0 + 0j)]]) == 0


def test_rejects_bad_sizes():
    f = _lib.lib().phc_mixed_volume
    f.restype = ctypes.c_longlong
    counts = np.array([2], np.int32)
    pts = np.zeros(2, np.int32)
    assert f(0, _lib.ptr(counts), _lib.ptr(pts), ctypes.c_ulonglong(0), 0, ctypes.c_void_p(0),
             ctypes.c_void_p(0)) < 0
    assert "bad sizes" in _lib.lib().phc_last_error().decode()


def test_error_is_raised_as_phc_error():
    with pytest.raises(_lib.PhcError, match="phc_mixed_volume"):
        rc.mixed_cells([np.zeros((2, 65), np.int64)] * 65)
