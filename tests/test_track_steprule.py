"""The tracker oracle's step rule (CPU): the curvature step of Hesse_Pade
next to the pole step, counted the way the reference's Minimum counts, and
the learned step mode restated from the device's network."""
import numpy as np

from oracle import mlp_oracle, pyoracle
from phcpack_b200 import homotopy as hm
from phcpack_b200 import trackwork

ORC = pyoracle.oracle()


def test_one_step_rule_decision_per_step():
    pb = hm.subset(hm.config4(), np.arange(0, 1024, 64))
    ipar, dpar = hm.params()
    _, info, dinfo = pyoracle.track(ORC, pb, ipar, dpar, pmode=1, rmode=2, nthreads=4)
    io = info.reshape(-1, 6)
    assert (io[:, 0] == 0).all()
    # every predictor step takes the pole step, the curvature step or maxsize
    assert np.array_equal(io[:, 3] + io[:, 4] + io[:, 5], io[:, 1])
    # on this workload the pole step decides most steps, and maxsize bounds
    # the early ones
    assert io[:, 3].sum() > 0 and io[:, 5].sum() > 0


def test_curvature_step_binds_with_small_cbeta_and_not_with_large():
    """cbeta scales the curvature step (cbeta eta / |err|)^(1/K): a tiny cbeta
    makes it the smallest step on most steps, a huge one never."""
    pb = hm.subset(hm.config4(), [0, 100, 200])
    ipar, dpar_small = hm.params(cbeta=1e-16)
    _, i_small, _ = pyoracle.track(ORC, pb, ipar, dpar_small, pmode=1, rmode=2)
    ipar, dpar_big = hm.params(cbeta=1e12)
    _, i_big, _ = pyoracle.track(ORC, pb, ipar, dpar_big, pmode=1, rmode=2)
    s, b = i_small.reshape(-1, 6), i_big.reshape(-1, 6)
    assert (s[:, 0] == 0).all() and (b[:, 0] == 0).all()
    assert (s[:, 4] >= 0.6 * s[:, 1]).all()  # most steps the curvature step
    assert (b[:, 4] == 0).all()
    assert (s[:, 1] > b[:, 1]).all()  # smaller steps, more of them


def test_oracle_rejects_nonpositive_cbeta():
    pb = hm.subset(hm.config4(), [0])
    ipar, dpar = hm.params(cbeta=0.0)
    try:
        pyoracle.track(ORC, pb, ipar, dpar, pmode=1, rmode=2)
    except AssertionError:
        return
    raise AssertionError("cbeta = 0 accepted")


def test_learned_mode_uses_the_network():
    """step_mode 1 with the committed model: same end points as the plain
    step (both refined at t = 1), fewer steps."""
    model = trackwork.load_model_bytes()
    assert model is not None
    pb = hm.subset(hm.config4(), np.arange(0, 1024, 128))
    ipar, dpar = hm.params()
    xp, ip, _ = pyoracle.track(ORC, pb, ipar, dpar, pmode=1, rmode=2, nthreads=4)
    xl, il, _ = pyoracle.track(ORC, pb, ipar, dpar, pmode=1, rmode=2, nthreads=4, step_mode=1, model=model)
    ip, il = ip.reshape(-1, 6), il.reshape(-1, 6)
    assert (ip[:, 0] == 0).all() and (il[:, 0] == 0).all()
    a, b = xp.reshape(-1, 8), xl.reshape(-1, 8)
    assert np.abs((a[:, 0] - b[:, 0]) + (a[:, 1] - b[:, 1])).max() < 1e-26
    assert il[:, 1].mean() < ip[:, 1].mean()
