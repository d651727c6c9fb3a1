"""Argument checks of the C ABI, on the CPU: every entry point rejects bad
sizes, precisions and system descriptions with a negative status and a
message from phc_last_error() before it touches the device, and
phc_track_prepare (host only) builds the Jacobian gather lists with the slot
codes documented in include/phc_b200.h."""
import ctypes

import numpy as np
import pytest

from phcpack_b200 import _lib
from phcpack_b200 import homotopy as hm

NULL = ctypes.c_void_p(0)


def rejected(name, *args, match=None):
    f = getattr(_lib.lib(), name)
    f.restype = ctypes.c_int
    rc = f(*args)
    msg = _lib.lib().phc_last_error().decode()
    assert rc < 0, f"{name} accepted bad arguments"
    if match is not None:
        assert match in msg, msg
    return rc


def test_dense_entry_points_reject_bad_sizes():
    assert rejected("phc_blocked_houseqr", 3, 0, 1, 8, 8, 4, NULL, NULL, NULL, NULL, NULL,
                    match="precision") == -1
    rejected("phc_blocked_houseqr", 2, 0, 1, 8, 6, 4, NULL, NULL, NULL, NULL, NULL, match="ncols")
    rejected("phc_upper_tiled_solver", 2, 0, 1, 10, 4, NULL, NULL, NULL, NULL, NULL, match="szt")
    rejected("phc_bals_solve", 2, 0, 1, 8, 4, 4, 0, NULL, NULL, NULL, NULL, NULL, NULL, NULL, NULL,
             match="tailidx")
    rejected("phc_bals_solve", 2, 0, 1, 8, 4, 4, 9, NULL, NULL, NULL, NULL, NULL, NULL, NULL, NULL,
             match="tailidx")


def test_eval_rejects_bad_precision_and_sizes():
    rejected("phc_system_evaldiff", 3, 1, 1, 4, 3, 2, NULL, NULL, NULL, NULL, NULL, NULL, NULL, NULL, NULL,
             match="precision")
    rejected("phc_system_evaldiff", 2, 1, 1, 0, 3, 2, NULL, NULL, NULL, NULL, NULL, NULL, NULL, NULL, NULL,
             match="sizes")


def small_problem(n=3, npaths=4):
    rng = np.random.default_rng(1)
    pb = hm.total_degree_problem([hm.dense_quadratic(rng, n)], complex(hm.unit(rng)))
    return hm.subset(pb, np.arange(npaths))


def track_args(pb, pmode=1, rmode=2, ipar=None):
    ip, dp = hm.params()
    if ipar is not None:
        ip = np.array(ipar, dtype=np.int32)
    xend = np.zeros(pb.npaths * pb.maxdim * 16)
    info = np.zeros(pb.npaths * 6, np.int32)
    dinfo = np.zeros(pb.npaths * 2)
    p = _lib.ptr
    return (pb.nsys, p(pb.dim), pb.maxvar, p(pb.mono_off), p(pb.mono_nvr), p(pb.mono_idx), p(pb.mono_exp),
            p(pb.eq_off), p(pb.term_off), p(pb.term_mono), p(pb.term_a), p(pb.term_b), pb.npaths, p(pb.path_sys),
            p(pb.x0), p(ip), p(dp), pmode, rmode, 0, NULL, p(xend), p(info), p(dinfo), NULL)


def test_track_host_rejects_bad_modes_and_parameters():
    pb = small_problem()
    rejected("phc_track_host", *track_args(pb, pmode=3), match="predictor precision")
    rejected("phc_track_host", *track_args(pb, rmode=3), match="refinement precision")
    # numdeg + dendeg must equal deg
    rejected("phc_track_host", *track_args(pb, ipar=[8, 3, 4, 4, 3, 100, 4]), match="numdeg")


def test_track_prepare_rejects_malformed_systems():
    pb = small_problem()
    bad = pb.mono_idx.copy()
    bad[bad.argmax()] = pb.maxdim + 5  # a variable index out of range
    p = _lib.ptr
    neq = int(pb.eq_off[-1])
    jg_off = np.zeros(neq * pb.maxdim + 1, np.int32)
    jg = np.zeros(4096, np.int32)
    rejected("phc_track_prepare", pb.nsys, p(pb.dim), pb.maxvar, p(pb.mono_off), p(pb.mono_nvr), p(bad),
             p(pb.mono_exp), p(pb.eq_off), p(pb.term_off), p(pb.term_mono), pb.maxdim, p(jg_off), p(jg), p(jg),
             match="out of range")
    dim = pb.dim.copy()
    dim[0] = pb.maxdim + 1  # more variables than equations listed
    rejected("phc_track_prepare", pb.nsys, p(dim), pb.maxvar, p(pb.mono_off), p(pb.mono_nvr), p(pb.mono_idx),
             p(pb.mono_exp), p(pb.eq_off), p(pb.term_off), p(pb.term_mono), pb.maxdim + 1, p(jg_off), p(jg),
             p(jg), match="equations")


def test_gather_slot_codes():
    """Dense quadratic systems: every partial is read in place (no staging):
    codes -1 (the constant 1 of a linear monomial), -2 (2 x_j of x_j^2) and
    -3-l (x_l of x_j x_l); each (equation, variable) list holds the linear
    term, the square and the n-1 mixed products."""
    n = 4
    pb = small_problem(n=n)
    jg_off, jg_term, jg_slot, staged = hm.gather_lists(pb)
    assert staged == 0
    counts = np.diff(jg_off).reshape(n, pb.maxdim)
    assert (counts == n + 1).all()
    for e in range(n):
        for j in range(n):
            codes = jg_slot[jg_off[e * pb.maxdim + j]:jg_off[e * pb.maxdim + j + 1]]
            assert sorted(codes[codes >= -2].tolist()) == [-2, -1]
            assert sorted((-codes[codes <= -3] - 3).tolist()) == sorted(set(range(n)) - {j})


def test_gather_slot_codes_stage_higher_degrees():
    # x0^2 x1 - 1 and x1^3 - x0: partials of degree-3 monomials are staged
    polys = [[(((0, 2), (1, 1)), 1.0 + 0j), ((), -1.0 + 0j)], [(((1, 3),), 1.0 + 0j), (((0, 1),), -1.0 + 0j)]]
    pb = hm.total_degree_problem([polys], complex(0.6, 0.8), maxvar=2)
    jg_off, jg_term, jg_slot, staged = hm.gather_lists(pb)
    assert staged >= 2 and (jg_slot >= 0).sum() == staged
