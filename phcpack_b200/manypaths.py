"""Host side of the tracker's drop-in entry points gpumanypaths_d / _dd / _qd
(Ada/PHCtoC/gpumanypaths_dd.h:27): the containers they read and write, and
the call with the reference's arguments.  phcpy's py2c_gpu_manypaths_dd
(Mod/phcpy2cpath_dd.cpp:4593) maps onto ``track(mode, verbose, regamma,
imgamma, prec=2)`` after the systems and the start solutions are stored."""
from __future__ import annotations

import numpy as np

from . import _lib

ENTRY = {1: "gpumanypaths_d", 2: "gpumanypaths_dd", 4: "gpumanypaths_qd"}


def _flat_system(polys, nvar):
    """Polynomials as lists of (monomial, coefficient), a monomial a tuple of
    (variable, exponent) pairs: the container arrays (terms per polynomial,
    exponent vectors, complex coefficients)."""
    nterms, exps, cff = [], [], []
    for poly in polys:
        nterms.append(len(poly))
        for mono, c in poly:
            e = [0] * nvar
            for v, k in mono:
                e[v] += k
            exps.extend(e)
            cff.extend([complex(c).real, complex(c).imag])
    return (np.asarray(nterms, np.int32), np.asarray(exps if exps else [0], np.int32),
            np.asarray(cff if cff else [0.0], np.float64))


def set_system(which, polys, nvar):
    """which: 'target' or 'start'."""
    nt, ex, cf = _flat_system(polys, nvar)
    _lib.call(f"phc_container_set_{which}", len(polys), nvar, _lib.ptr(nt), _lib.ptr(ex), _lib.ptr(cf))


def set_solutions(x):
    """x: array (nsols, nvar, 2, limbs) of limbs (real part, imaginary part)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    nsols, nvar, _, limbs = x.shape
    _lib.call("phc_container_set_solutions", nsols, nvar, limbs, _lib.ptr(x.reshape(-1)))


def number_of_solutions():
    n = np.zeros(1, np.int32)
    _lib.call("phc_container_number_of_solutions", _lib.ptr(n))
    return int(n[0])


def dimension():
    n = np.zeros(1, np.int32)
    _lib.call("phc_container_dimension", _lib.ptr(n))
    return int(n[0])


def get_solutions(limbs=2):
    """The solutions in the container: dict with x (nsols, nvar, 2, limbs),
    t, status and res per solution."""
    ns = number_of_solutions()
    nvar = dimension()
    x = np.zeros(ns * nvar * 2 * limbs)
    t = np.zeros(max(ns, 1))
    st = np.zeros(max(ns, 1), np.int32)
    res = np.zeros(max(ns, 1))
    _lib.call("phc_container_get_solutions", limbs, _lib.ptr(x), _lib.ptr(t), _lib.ptr(st), _lib.ptr(res))
    return {"x": x.reshape(ns, nvar, 2, limbs), "t": t[:ns], "status": st[:ns], "res": res[:ns]}


def set_parameters(ipar, dpar):
    ipar = np.ascontiguousarray(ipar, dtype=np.int32)
    dpar = np.ascontiguousarray(dpar, dtype=np.float64)
    _lib.call("phc_container_set_parameters", _lib.ptr(ipar), _lib.ptr(dpar))


def clear():
    _lib.lib().phc_container_clear()


def track(mode, verbose, regamma, imgamma, prec=2):
    """Call gpumanypaths_d (prec 1), _dd (2) or _qd (4) with the reference's
    arguments; returns its status (0: tracked)."""
    return _lib.call(ENTRY[prec], int(mode), int(verbose), _lib.c_double(regamma), _lib.c_double(imgamma))
