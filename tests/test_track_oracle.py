"""The CPU tracker restatement on the 1024-path dense quadratic workload:
sampled paths end at solutions of the target system (checked independently
in numpy), and the endpoint classification is self-consistent."""
import numpy as np

from oracle import pyoracle
from phcpack_b200 import homotopy as hm

ORC = pyoracle.oracle()


def target_residual(pb, xend, p):
    """max |p_i(x)| of the target (t = 1) in complex128, from the flat arrays"""
    md = pb.maxdim
    x = (xend.reshape(-1, md, 8)[p, :, 0] + 1j * xend.reshape(-1, md, 8)[p, :, 4])
    s = pb.path_sys[p]
    r = 0.0
    for e in range(pb.eq_off[s], pb.eq_off[s + 1]):
        v = 0j
        for tr in range(pb.term_off[e], pb.term_off[e + 1]):
            m = pb.term_mono[tr]
            c = complex(*pb.term_b[2 * tr:2 * tr + 2])  # the coefficient at t = 1
            for u in range(pb.mono_nvr[m]):
                c *= x[pb.mono_idx[m * pb.maxvar + u]] ** pb.mono_exp[m * pb.maxvar + u]
            v += c
        r = max(r, abs(v))
    return r, np.abs(x[:pb.dim[s]]).max()


def test_oracle_tracker_config4_sample():
    pb = hm.subset(hm.config4(), np.arange(0, 1024, 128))
    ipar, dpar = hm.params()
    xe, info, di = pyoracle.track(ORC, pb, ipar, dpar, pmode=1, rmode=2, nthreads=4)
    info = info.reshape(-1, 6)
    di = di.reshape(-1, 2)
    assert (info[:, 0] == 0).all()
    assert (di[:, 1] <= 1e-24).all()
    assert (np.abs(di[:, 0] - 1.0) < 1e-12).all()
    for p in range(pb.npaths):
        r, mx = target_residual(pb, xe, p)
        assert r <= 1e-12 * max(1.0, mx) ** 2


def test_oracle_tracker_all_dd_predictor_same_endpoints():
    pb = hm.subset(hm.config4(), [3, 500, 1000])
    ipar, dpar = hm.params()
    x1, i1, _ = pyoracle.track(ORC, pb, ipar, dpar, pmode=1, rmode=2)
    x2, i2, _ = pyoracle.track(ORC, pb, ipar, dpar, pmode=2, rmode=2)
    assert np.array_equal(i1.reshape(-1, 6)[:, 0], i2.reshape(-1, 6)[:, 0])
    e1 = x1.reshape(-1, 8)
    e2 = x2.reshape(-1, 8)
    assert np.abs((e1[:, 0] - e2[:, 0]) + (e1[:, 1] - e2[:, 1])).max() < 1e-26


def test_oracle_qr_predictor_matches_lu_predictor():
    """The oracle's predictor with J_0 inverted by Householder QR (step_mode
    bit 2) reaches the same end points as with LU, in about as many steps:
    both give J_0^{-1} to double accuracy, only their rounding differs."""
    pb = hm.subset(hm.config4(), np.arange(0, 1024, 128))
    ipar, dpar = hm.params()
    xl, il, dl = pyoracle.track(ORC, pb, ipar, dpar, pmode=1, rmode=2, nthreads=4, step_mode=0)
    xq, iq, dq = pyoracle.track(ORC, pb, ipar, dpar, pmode=1, rmode=2, nthreads=4, step_mode=2)
    il, iq = il.reshape(-1, 6), iq.reshape(-1, 6)
    assert (iq[:, 0] == 0).all() and (il[:, 0] == 0).all()
    assert np.abs(iq[:, 1] - il[:, 1]).max() <= 3
    a = xl.reshape(-1, pb.maxdim, 8)
    b = xq.reshape(-1, pb.maxdim, 8)
    for part in (0, 4):
        d = (a[..., part] - b[..., part]) + (a[..., part + 1] - b[..., part + 1])
        assert np.abs(d).max() <= 1e-26
    # the QR mode is refused with the double-double predictor
    import pytest
    with pytest.raises(AssertionError):
        pyoracle.track(ORC, pb, ipar, dpar, pmode=2, rmode=2, nthreads=1, step_mode=2)
