"""GPU path tracker against the CPU tracker restatement (oracle).

Criteria: identical success/failure classification per path; endpoints of
successful paths agree to 1e-26 absolute per component (both are refined in
double-double at t = 1; quad-double refinement: 1e-50); endpoint residuals
<= 1e-24; the one-path-per-launch arrangement gives bitwise the same
results as the batched persistent kernel (same code per path)."""
import numpy as np
import pytest

from oracle import pyoracle
from phcpack_b200 import homotopy as hm

pytestmark = pytest.mark.gpu
ORC = pyoracle.oracle()


def endpoint_diff(pb, xa, xb, limbs, width=4):
    a = xa.reshape(-1, pb.maxdim, 2 * width)
    b = xb.reshape(-1, pb.maxdim, 2 * width)
    d = np.zeros(a.shape[:2])
    for part in (0, width):
        acc = np.zeros(a.shape[:2])
        for l in range(limbs - 1, -1, -1):
            acc = acc + (a[..., part + l] - b[..., part + l])
        d = np.maximum(d, np.abs(acc))
    return d.max(axis=1)


def compare_with_oracle(pb, g, xo, io, max_step_diff):
    """Identical classification, end points within 1e-26, residuals <= 1e-24,
    and per-path step counts and step-rule counts close to the oracle's."""
    io = io.reshape(-1, 6)
    assert np.array_equal(g.status, io[:, 0])
    ok = g.status == 0
    assert (g.residual[ok] <= 1e-24).all()
    assert (endpoint_diff(pb, g.xend, xo, 2)[ok] <= 1e-26).all()
    # the same step rules; rounding may move a few decisions of a path
    assert np.abs(g.steps - io[:, 1]).max() <= max_step_diff
    assert abs(g.steps.mean() - io[:, 1].mean()) <= 0.05 * io[:, 1].mean()
    # one step-size decision (pole, curvature or maxsize) per predictor step
    assert np.array_equal((g.nbpole + g.nbhess + g.nbmaxm)[ok], g.steps[ok])
    assert abs(g.nbhess.sum() - io[:, 4].sum()) <= 0.05 * max(1, io[:, 4].sum())
    return ok


@pytest.mark.parametrize("step_mode", [0, 1])
def test_track_config4_all_paths_vs_oracle(step_mode):
    """All 1024 paths of the dense quadratic n = 10 workload with the FP64
    predictor and the double-double corrector, with the plain step and with
    the learned step (the committed model) against the oracle's run with the
    same step rule and the same network."""
    from phcpack_b200 import trackwork
    pb = hm.config4()
    ipar, dpar = hm.params()
    model = trackwork.load_model_bytes() if step_mode else None
    if step_mode:
        assert model is not None
    g = hm.track_host(pb, pmode=1, rmode=2, step_mode=step_mode, model=model)
    xo, io, _ = pyoracle.track(ORC, pb, ipar, dpar, pmode=1, rmode=2, nthreads=16, step_mode=step_mode,
                               model=model)
    ok = compare_with_oracle(pb, g, xo, io, max_step_diff=4)
    assert ok.all()


@pytest.mark.parametrize("step_mode", [2, 3])
def test_track_qr_predictor_vs_oracle(step_mode):
    """The predictor's J_0 inverted by Householder QR in double (step_mode
    bit 2; with bit 1 the learned step as well) on 256 paths of the dense
    quadratic n = 10 workload against the oracle's run with the same QR:
    same classification, end points and step counts as for the LU predictor,
    and the QR predictor's series agree with the LU predictor's (the step
    counts of the two modes are close)."""
    from phcpack_b200 import trackwork
    pb = hm.subset(hm.config4(), np.arange(0, 1024, 4))
    ipar, dpar = hm.params()
    model = trackwork.load_model_bytes() if step_mode & 1 else None
    g = hm.track_host(pb, pmode=1, rmode=2, step_mode=step_mode, model=model)
    xo, io, _ = pyoracle.track(ORC, pb, ipar, dpar, pmode=1, rmode=2, nthreads=16, step_mode=step_mode,
                               model=model)
    ok = compare_with_oracle(pb, g, xo, io, max_step_diff=4)
    assert ok.all()
    lu = hm.track_host(pb, pmode=1, rmode=2, step_mode=step_mode & 1, model=model)
    assert np.array_equal(lu.status, g.status)
    assert abs(lu.steps.mean() - g.steps.mean()) <= 0.05 * lu.steps.mean()
    assert (endpoint_diff(pb, g.xend, lu.xend, 2)[ok] <= 1e-26).all()


def test_track_qr_predictor_needs_the_double_predictor():
    from phcpack_b200 import _lib
    pb = hm.subset(hm.config4(), np.arange(4))
    with pytest.raises(_lib.PhcError):
        hm.track_host(pb, pmode=2, rmode=2, step_mode=2)


@pytest.mark.parametrize("pmode", [1, 2])
def test_track_config4_sample_vs_oracle(pmode):
    pb = hm.subset(hm.config4(), np.arange(0, 1024, 16))
    ipar, dpar = hm.params()
    g = hm.track_host(pb, pmode=pmode, rmode=2)
    xo, io, do = pyoracle.track(ORC, pb, ipar, dpar, pmode=pmode, rmode=2, nthreads=8)
    io = io.reshape(-1, 6)
    assert np.array_equal(g.status, io[:, 0])
    ok = g.status == 0
    assert ok.mean() > 0.9
    assert (g.residual[ok] <= 1e-24).all()
    assert (endpoint_diff(pb, g.xend, xo, 2)[ok] <= 1e-26).all()
    # step counts follow the same rules; rounding may move a few decisions
    assert np.abs(g.steps - io[:, 1]).max() <= 3


def test_track_quad_double_refinement():
    pb = hm.subset(hm.config4(), [1, 77, 300, 901])
    ipar, dpar = hm.params(restol=1e-50)
    g = hm.track_host(pb, pmode=1, rmode=4, restol=1e-50)
    xo, io, _ = pyoracle.track(ORC, pb, ipar, dpar, pmode=1, rmode=4)
    assert np.array_equal(g.status, io.reshape(-1, 6)[:, 0])
    ok = g.status == 0
    assert ok.all()
    assert (endpoint_diff(pb, g.xend, xo, 4)[ok] <= 1e-50).all()


def test_track_octo_double_refinement():
    """Octo-double refinement at t = 1 (rmode 8): the same classification as
    the oracle, end points within 1e-110 of the oracle's, residuals
    <= 1e-100."""
    pb = hm.subset(hm.config4(), [3, 150, 600, 1000])
    ipar, dpar = hm.params(restol=1e-100, refine_steps=6)
    g = hm.track_host(pb, pmode=1, rmode=8, restol=1e-100, refine_steps=6)
    xo, io, _ = pyoracle.track(ORC, pb, ipar, dpar, pmode=1, rmode=8)
    assert np.array_equal(g.status, io.reshape(-1, 6)[:, 0])
    ok = g.status == 0
    assert ok.all()
    assert (g.residual <= 1e-100).all()
    assert (endpoint_diff(pb, g.xend, xo, 8, width=8)[ok] <= 1e-110).all()


def test_one_path_per_launch_matches_batched():
    import torch
    pb = hm.subset(hm.config4(), np.arange(0, 1024, 64))
    dt = hm.DeviceTracker(pb)
    dt.run(pmode=2, rmode=2)
    torch.cuda.synchronize()
    a = dt.result()
    dt.run(pmode=2, rmode=2, one_per_launch=True)
    torch.cuda.synchronize()
    b = dt.result()
    assert np.array_equal(a.xend, b.xend) and np.array_equal(a.status, b.status)
    assert np.array_equal(a.steps, b.steps)


def test_track_mixed_sizes_vs_oracle():
    # the 64-system mixed-size workload, a few paths of several systems
    pb5 = hm.config5()
    pick = np.concatenate([np.nonzero(pb5.path_sys == s)[0][:3] for s in range(0, 64, 8)])
    pb = hm.subset(pb5, pick)
    ipar, dpar = hm.params()
    g = hm.track_host(pb, pmode=1, rmode=2)
    xo, io, do = pyoracle.track(ORC, pb, ipar, dpar, pmode=1, rmode=2, nthreads=8)
    # success / failure classification; on diverging paths (solutions at
    # infinity of these sparse systems) the failure mode itself (step below
    # minsize or a large residual at t = 1) depends on rounding
    assert np.array_equal(g.status == 0, io.reshape(-1, 6)[:, 0] == 0)
    ok = g.status == 0
    assert (endpoint_diff(pb, g.xend, xo, 2)[ok] <= 1e-26 * np.maximum(1, np.abs(g.endpoints(pb.maxdim)).max(axis=1)[ok])).all()


def test_track_device_entry_matches_host_entry():
    import torch
    pb = hm.subset(hm.config4(), [5, 6, 7, 8])
    h = hm.track_host(pb, pmode=1, rmode=2)
    dt = hm.DeviceTracker(pb)
    dt.run(pmode=1, rmode=2)
    torch.cuda.synchronize()
    d = dt.result()
    assert np.array_equal(h.xend, d.xend) and np.array_equal(h.status, d.status)


@pytest.mark.parametrize("n", [1, 2, 24, 32])
def test_track_dimension_extremes_vs_oracle(n):
    """The smallest and largest dimensions the kernel takes (n = 1 and the
    32 of one warp per LU): a seeded weakly coupled quadratic system, a
    sample of its total-degree paths, same classification as the oracle and
    end points within 1e-26 (relative to their size)."""
    rng = np.random.default_rng(100 + n)
    # x_i^2 - a_i plus a weak coupling to three other variables: 2^n regular
    # roots near the (+-) square roots of a_i, all reached from x_i^2 - 1
    target = []
    for i in range(n):
        poly = [(((i, 2),), 1.0 + 0j), ((), complex(-rng.uniform(1.0, 3.0)))]
        if n > 1:
            for j in rng.choice([k for k in range(n) if k != i], size=min(3, n - 1), replace=False):
                poly.append((((int(j), 1),), complex(0.1 * hm.unit(rng))))
        target.append(poly)
    gamma = complex(hm.unit(rng))
    cap = min(8, 2 ** n)
    pb = hm.total_degree_problem([target], gamma, max_paths_per_system=cap, rng=rng)
    ipar, dpar = hm.params()
    g = hm.track_host(pb, pmode=1, rmode=2)
    xo, io, _ = pyoracle.track(ORC, pb, ipar, dpar, pmode=1, rmode=2)
    io = io.reshape(-1, 6)
    assert np.array_equal(g.status == 0, io[:, 0] == 0)
    ok = (g.status == 0) & (io[:, 0] == 0)
    assert ok.any()
    assert (g.residual[ok] <= 1e-24).all()
    scale = np.maximum(1.0, np.abs(g.endpoints(pb.maxdim)).max(axis=1))
    assert (endpoint_diff(pb, g.xend, xo, 2)[ok] <= 1e-26 * scale[ok]).all()
    if n == 1:
        a = -target[0][1][1].real
        x = g.endpoints(pb.maxdim)[:, 0]
        assert np.allclose(np.sort(x.real), [-np.sqrt(a), np.sqrt(a)], atol=1e-14)


def test_track_batch_beyond_one_wave_matches_smaller_batches():
    """1,200 paths are more than the GPU holds at 7 paths per SM, so they run
    in the 8-paths-per-SM (64-register) variant; two batches of 600 fit and run
    in the 72-register variant.  Both give the same classification and end
    points."""
    pb5 = hm.config5()
    pb = hm.subset(pb5, np.arange(1200))
    whole = hm.track_host(pb, pmode=1, rmode=2)
    a = hm.track_host(hm.subset(pb5, np.arange(600)), pmode=1, rmode=2)
    b = hm.track_host(hm.subset(pb5, np.arange(600, 1200)), pmode=1, rmode=2)
    status = np.concatenate([a.status, b.status])
    assert np.array_equal(whole.status, status)
    ok = whole.status == 0
    assert ok.sum() >= 200  # most paths of these sparse systems diverge
    d = endpoint_diff(pb, whole.xend, np.concatenate([a.xend, b.xend]), 2)
    scale = np.maximum(1.0, np.abs(whole.endpoints(pb.maxdim)).max(axis=1))
    assert (d[ok] <= 1e-26 * scale[ok]).all()


def test_track_curvature_step_binding_vs_oracle():
    """With a tiny cbeta the curvature step is the smallest step nearly
    everywhere, so the tracker computes the singular values of the Jacobian
    and of the Hessians at every step (its bound never settles the minimum):
    same classification as the oracle, end points within 1e-26, and about
    as many curvature-step decisions."""
    pb = hm.subset(hm.config4(), np.arange(0, 1024, 128))
    ipar, dpar = hm.params(cbeta=1e-16)
    g = hm.track_host(pb, pmode=1, rmode=2, cbeta=1e-16)
    xo, io, _ = pyoracle.track(ORC, pb, ipar, dpar, pmode=1, rmode=2, nthreads=8)
    io = io.reshape(-1, 6)
    assert np.array_equal(g.status, io[:, 0]) and (g.status == 0).all()
    assert (endpoint_diff(pb, g.xend, xo, 2) <= 1e-26).all()
    assert g.nbhess.sum() >= 0.6 * g.steps.sum()
    assert abs(g.nbhess.sum() - io[:, 4].sum()) <= 0.02 * io[:, 4].sum()
    assert np.abs(g.steps - io[:, 1]).max() <= 4
