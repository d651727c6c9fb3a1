"""GPU parity of the batched series eval/diff (phc_system_evaldiff) against
the golden fixtures from PHCpack's host code and against the oracle.

Tolerance: per output coefficient |gpu - ref| <= rtol * A, where A is the same
coefficient of the evaluation with every input replaced by its absolute value
(the sum of the absolute values of the terms, the scale of rounding error);
rtol = 1e-28 for double-double, 1e-60 for quad-double, 1e-14 for double."""
import numpy as np
import pytest

import golden_io
from mdcheck import abs_batch, check_scaled
from oracle import pyoracle
from phcpack_b200 import series
from phcpack_b200 import workloads as wl

pytestmark = pytest.mark.gpu
ORC = pyoracle.oracle()
RTOL = {1: 1e-14, 2: 1e-28, 4: 1e-60}


def run_device(b):
    import torch
    db = series.DeviceBatch(b)
    out = db.evaldiff()
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("name", golden_io.names("eval_"))
def test_eval_gpu_vs_golden(name):
    d = golden_io.load(name)
    b = golden_io.batch(d)
    out = run_device(b)
    scale = ORC.system_evaldiff(abs_batch(b))
    assert check_scaled(out, d["output"], scale, b.prec, b.cplx, RTOL[b.prec]) <= 1.0


@pytest.mark.parametrize("prec,cplx", [(1, False), (1, True), (2, False), (2, True), (4, False), (4, True)])
def test_eval_gpu_vs_oracle_config2_shape(prec, cplx):
    # the eval/diff workload's shapes (n=32, 32 monomials over <= 4 variables,
    # exponents {1,2,3}, degree 31) at a batch the oracle finishes quickly
    b = wl.eval_batch(7 + prec, 3 if prec < 4 else 1, 32, 31, 32, 4, prec, cplx, expmax=3)
    out = run_device(b)
    ref = ORC.system_evaldiff(b)
    scale = ORC.system_evaldiff(abs_batch(b))
    assert check_scaled(out, ref, scale, prec, cplx, RTOL[prec]) <= 1.0


@pytest.mark.parametrize("prec,cplx", [(2, False), (2, True), (4, True)])
def test_eval_gpu_long_monomials(prec, cplx):
    # monomials of 20..32 distinct variables at degree 31: the scratch of a
    # warp (2*32-1 series) no longer fits 8 warps per CTA, so fewer
    # polynomials share a CTA
    b = wl.eval_batch(40 + prec, 1, 32, 31, 6, 32, prec, cplx, expmax=1, minvar=20)
    out = run_device(b)
    ref = ORC.system_evaldiff(b)
    scale = ORC.system_evaldiff(abs_batch(b))
    assert check_scaled(out, ref, scale, prec, cplx, RTOL[prec]) <= 1.0


@pytest.mark.parametrize("deg", [0, 1, 2, 7, 8, 15, 30])
def test_eval_gpu_degrees(deg):
    b = wl.eval_batch(100 + deg, 5, 6, deg, 5, 4, 2, True, expmax=3)
    out = run_device(b)
    ref = ORC.system_evaldiff(b)
    scale = ORC.system_evaldiff(abs_batch(b))
    assert check_scaled(out, ref, scale, 2, True, RTOL[2]) <= 1.0


def test_eval_gpu_ragged_supports():
    # uneven monomial counts, empty polynomials, one-variable monomials,
    # up to 8 variables per monomial, dim not a multiple of the warp group
    rng = np.random.default_rng(3)
    nsys, dim, deg, maxvar = 3, 11, 9, 8
    counts = rng.integers(0, 9, size=nsys * dim)
    counts[0] = 0
    mon_off = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
    nm = int(mon_off[-1])
    nvr = rng.integers(1, maxvar + 1, size=nm).astype(np.int32)
    idx = np.zeros((nm, maxvar), np.int32)
    exps = np.zeros((nm, maxvar), np.int32)
    for m in range(nm):
        idx[m, :nvr[m]] = rng.choice(dim, nvr[m], replace=False)
        exps[m, :nvr[m]] = rng.integers(1, 3, nvr[m])
    cff = wl.random_numbers(rng, (nm, deg + 1), 2, True, "unit")
    cst = wl.random_numbers(rng, (nsys * dim, deg + 1), 2, True, "unit")
    inp = wl.random_numbers(rng, (nsys * dim, deg + 1), 2, True, "normal")
    b = wl.SystemBatch(nsys, dim, deg, maxvar, 2, True, mon_off, nvr, idx, exps, cst, cff, inp)
    out = run_device(b)
    ref = ORC.system_evaldiff(b)
    scale = ORC.system_evaldiff(abs_batch(b))
    assert check_scaled(out, ref, scale, 2, True, RTOL[2]) <= 1.0


def test_eval_host_entry_point_matches_device():
    b = wl.eval_batch(5, 4, 12, 15, 10, 4, 2, True, expmax=3)
    a = series.system_evaldiff_host(b)
    c = run_device(b)
    assert np.array_equal(a, c)


def test_eval_host_entry_point_pipelined_chunks():
    # 70 systems: the host entry copies and evaluates them in 8 uneven
    # chunks on two streams; the result equals one device launch bit for bit
    b = wl.eval_batch(6, 70, 6, 7, 5, 3, 2, True, expmax=2)
    a = series.system_evaldiff_host(b)
    c = run_device(b)
    assert np.array_equal(a, c)


def test_eval_reference_shaped_single_polynomial():
    d = golden_io.load("eval_dd_real")
    b = golden_io.batch(d)
    S = (b.deg + 1) * b.width
    m0, m1 = int(b.mon_off[0]), int(b.mon_off[1])
    out = series.gpu_poly_evaldiff(2, False, b.dim, m1 - m0, b.deg, b.nvr[m0:m1], b.idx[m0:m1],
                                   b.cst[:S], b.cff[m0 * S:m1 * S], b.input[:b.dim * S], exps=b.exps[m0:m1])
    scale = ORC.system_evaldiff(abs_batch(b))[:(b.dim + 1) * (b.deg + 1)]
    assert check_scaled(out, d["output"][:(b.dim + 1) * S], scale, 2, False, RTOL[2]) <= 1.0


@pytest.mark.parametrize("deg,prec,cplx", [(32, 2, True), (47, 2, False), (63, 2, True), (100, 4, False),
                                           (100, 1, True), (191, 2, True), (191, 4, True)])
def test_eval_gpu_long_series_vs_oracle(deg, prec, cplx):
    # series longer than a warp (the large-degree kernel), up to the
    # reference's largest degree 191; exponents {1,2,3}, up to 4 variables
    b = wl.eval_batch(200 + deg, 2, 6, deg, 5, 4, prec, cplx, expmax=3)
    out = run_device(b)
    ref = ORC.system_evaldiff(b)
    scale = ORC.system_evaldiff(abs_batch(b))
    assert check_scaled(out, ref, scale, prec, cplx, RTOL[prec]) <= 1.0


def test_eval_rejects_degree_beyond_limit():
    from phcpack_b200._lib import PhcError
    b = wl.eval_batch(1, 1, 3, 192, 2, 2, 2, False)
    with pytest.raises(PhcError):
        run_device(b)
