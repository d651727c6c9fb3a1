"""The autotuner (phcpack_b200/autotune.py) on the device: every launch shape
it may pick gives the result of the built-in rule, and the choice it makes is
one of the candidates.  Eval/diff and the tracker must agree bit for bit
across shapes (the arithmetic of each polynomial and each path is the same;
only the grouping into CTAs changes); the least squares with another tile
size rounds differently, so it is compared with the oracle at the tolerance
of tests/test_dense_gpu.py."""
import numpy as np
import pytest

from mdcheck import absdiff, lead
from oracle import pyoracle
from phcpack_b200 import _lib, autotune, dense, homotopy as hm, series
from phcpack_b200 import workloads as wl

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _restore_rules():
    yield
    autotune.reset()


def test_eval_warps_choice_does_not_change_results():
    import torch
    b = wl.eval_batch(31, 6, 16, 15, 12, 4, 2, True, expmax=3)
    db = series.DeviceBatch(b)
    autotune.reset()
    ref = db.evaldiff().cpu().numpy()
    for w in (1, 2, 4, 8):
        autotune.set_knob(autotune.KNOB_EVAL_WARPS, w)
        assert autotune.get_knob(autotune.KNOB_EVAL_WARPS) == w
        out = db.evaldiff().cpu().numpy()
        assert np.array_equal(out, ref), w
    stream = torch.cuda.Stream()
    args = (b.prec, int(b.cplx), b.nsys, b.dim, b.deg, b.maxvar, _lib.ptr(db.mon_off), _lib.ptr(db.nvr),
            _lib.ptr(db.idx), _lib.ptr(db.exps), _lib.ptr(db.cst), _lib.ptr(db.cff), _lib.ptr(db.input),
            _lib.ptr(db.output), _lib.c_void_p(stream.cuda_stream))
    res = autotune.tune_eval_warps(torch, stream, args, b.dim, key="test")
    assert res["choice"] in (1, 2, 4, 8) and autotune.get_knob(autotune.KNOB_EVAL_WARPS) == res["choice"]
    torch.cuda.synchronize()
    assert np.array_equal(db.output.cpu().numpy(), ref)


def test_track_variant_choice_does_not_change_results():
    import torch
    pb = hm.subset(hm.config4(), np.arange(192))
    dt = hm.DeviceTracker(pb)
    results = {}
    for v, k in ((1, 0), (2, 0), (2, 3), (1, 5)):
        autotune.set_knob(autotune.KNOB_TRACK_VARIANT, v)
        autotune.set_knob(autotune.KNOB_TRACK_PER_SM, k)
        dt.run(pmode=1, rmode=2)
        results[(v, k)] = dt.result()
    a = results[(1, 0)]
    for b in results.values():
        assert np.array_equal(a.status, b.status) and np.array_equal(a.steps, b.steps)
        assert np.array_equal(a.xend, b.xend)
    stream = torch.cuda.Stream()
    res = autotune.tune_track_variant(torch, stream, dt, reps=1, per_sm=(4, 8), pmode=1, rmode=2)
    assert res["choice"] in (1, 2) and autotune.get_knob(autotune.KNOB_TRACK_VARIANT) == res["choice"]
    assert res["per_sm"] in (4, 8) and autotune.get_knob(autotune.KNOB_TRACK_PER_SM) == res["per_sm"]


def test_bals_tile_choice_is_valid_and_accurate():
    import torch
    prec, cplx, n, degp1, ninst = 2, False, 32, 4, 16
    rng = np.random.default_rng(33)
    mats = [wl.random_numbers(rng, (degp1, n, n), prec, cplx, "normal") for _ in range(ninst)]
    rhss = [wl.random_numbers(rng, (degp1, n), prec, cplx, "normal") for _ in range(ninst)]
    f64 = dict(dtype=torch.float64, device="cuda")
    W = prec
    mat = torch.from_numpy(np.concatenate([m.reshape(-1) for m in mats])).cuda()
    rhs0 = torch.from_numpy(np.concatenate([r.reshape(-1) for r in rhss])).cuda()
    sol = torch.zeros(ninst * degp1 * n * W, **f64)
    Q = torch.zeros(ninst * n * n * W, **f64)
    R = torch.zeros(ninst * n * n * W, **f64)
    flags = torch.zeros(ninst * 5, dtype=torch.int32, device="cuda")
    flag0 = torch.tensor([1, 0, 0, 0, 1], dtype=torch.int32, device="cuda").repeat(ninst)
    work = torch.zeros(ninst * dense.workspace_bytes_wy(prec, cplx, n, 8, 0) // 8, **f64)
    stream = torch.cuda.Stream()
    res = autotune.tune_bals_tile(torch, stream, prec, cplx, ninst, n, degp1, mat, rhs0, sol, Q, R, flags, flag0,
                                  work, wy=0, reps=1)
    assert res["choice"] in (8, 16, 32) and res["stage"] in (1, 2)
    assert set(res["seconds"]) == {f"{t}/{g}" for t in (8, 16, 32) for g in (1, 2)}
    assert autotune.get_knob(autotune.KNOB_DENSE_STAGE) == res["stage"]
    # the solution with the chosen tile against the oracle
    sol_t, _ = dense.bals_solve_wy(prec, cplx, mat.cpu().numpy(), rhs0.cpu().numpy(), ninst, n, degp1,
                                   res["choice"], wy=0)
    orc = pyoracle.oracle()
    for q in range(ninst):
        so = orc.bals_solve(prec, cplx, n, degp1, 1, mats[q].reshape(-1), rhss[q].reshape(-1))[0]
        got = sol_t.reshape(ninst, -1)[q]
        s = lead(so, prec, cplx).reshape(degp1, n).max(axis=1)
        err = absdiff(got, so, prec, cplx).reshape(degp1, n).max(axis=1)
        assert np.all(err <= 1e4 * 1e-28 * np.maximum(1.0, s)), (q, err, s)


@pytest.mark.parametrize("prec,cplx,n,szt", [(4, False, 64, 16), (2, True, 32, 8), (2, False, 64, 32)])
def test_staged_panels_give_the_same_solution(prec, cplx, n, szt):
    """The least squares with the WY panels and the column panel of R in
    shared memory (knob 3 = 2) equals the one with them in global memory
    (knob 3 = 1) bit for bit: the same operations in the same order."""
    degp1, ninst = 3, 6
    rng = np.random.default_rng(n + szt)
    mat = np.concatenate([wl.random_numbers(rng, (degp1, n, n), prec, cplx, "normal").reshape(-1)
                          for _ in range(ninst)])
    rhs = np.concatenate([wl.random_numbers(rng, (degp1, n), prec, cplx, "normal").reshape(-1) for _ in range(ninst)])
    out = {}
    for g in (1, 2):
        autotune.set_knob(autotune.KNOB_DENSE_STAGE, g)
        out[g] = dense.bals_solve_host(prec, cplx, mat, rhs, ninst, n, degp1, szt)
    for a, b in zip(out[1], out[2]):
        assert np.array_equal(a, b)
