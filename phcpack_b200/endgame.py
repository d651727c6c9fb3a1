"""End-game diagnostics of paths: the series of a path at a point (x, t) of
the homotopy, the nearest singular point in t by Fabry's ratio theorem, and
the Hessian distance to the nearest singular solution, batched on the GPU
(include/phc_b200.h, phc_series_diagnostics).

The reference computes these one solution at a time on the host:
Newton_Fabry (Ada Deformations/Curves/dobldobl_fabry_on_homotopy.adb:30-83,
Fabry in Math_Lib/Circuits/convergence_radius_estimates.adb:392-425) and
the step bounds of its series trackers (Hesse_Pade and Distance,
Deformations/Curves/dobldobl_predictor_convolutions.adb:368-406,
singular_values_of_hessians.adb:190-211).  ``classify`` reads the Fabry
estimate at the last point of a path: a singular point that closes in on
t = 1 as t approaches 1 marks a path that ends at a singular solution or
diverges; one at a distance from t = 1 marks a path that passed near a
singularity inside the interval.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _lib

DEFAULT_IPAR = dict(deg=8, numdeg=5, dendeg=1, offset=1, newton_steps=4)
DEFAULT_TOLRES = {1: 1e-12, 2: 1e-24, 4: 1e-48}
DEFAULT_BETA2 = 0.005
FIELDS = ("zre", "zim", "radius", "err", "sigma_min", "hessian_norm", "eta", "pade_norm", "curv_step", "lastdx")
STATUS = {0: "ok", 1: "singular Jacobian", 2: "Newton above tolres"}


def params(pmode=2, **kw):
    ip = dict(DEFAULT_IPAR)
    dp = dict(tolres=DEFAULT_TOLRES[pmode], beta2=DEFAULT_BETA2)
    for k, v in kw.items():
        if k in ip:
            ip[k] = v
        elif k in dp:
            dp[k] = v
        else:
            raise KeyError(k)
    ipar = np.array([ip[k] for k in ("deg", "numdeg", "dendeg", "offset", "newton_steps")], np.int32)
    dpar = np.array([dp["tolres"], dp["beta2"]], np.float64)
    return ipar, dpar


@dataclass
class Diagnostics:
    z: np.ndarray            # the singular point is at t + z (complex)
    radius: np.ndarray       # |z|
    err: np.ndarray          # Fabry's error estimate
    sigma_min: np.ndarray    # smallest singular value of the Jacobian
    hessian_norm: np.ndarray # 2-norm of the largest singular values of the Hessians
    eta: np.ndarray          # 2 sigma_min / hessian_norm
    pade_norm: np.ndarray    # 2-norm of the Pade error estimates
    curv_step: np.ndarray    # (beta2 eta / pade_norm)^(1/deg)
    lastdx: np.ndarray       # Newton's last max |dx|
    fail: np.ndarray         # 1: no Fabry estimate
    status: np.ndarray       # 0 ok, 1 singular Jacobian, 2 Newton above tolres
    series: np.ndarray | None = None  # points x maxdim x (deg+1) x 2*pmode limbs

    @staticmethod
    def from_arrays(dout, iout, series=None):
        d = dout.reshape(-1, len(FIELDS))
        return Diagnostics(d[:, 0] + 1j * d[:, 1], d[:, 2].copy(), d[:, 3].copy(), d[:, 4].copy(), d[:, 5].copy(),
                           d[:, 6].copy(), d[:, 7].copy(), d[:, 8].copy(), d[:, 9].copy(), iout[0::2].copy(),
                           iout[1::2].copy(), series)


def series_diagnostics(pb, xpt, tpt, xlimbs=1, pmode=2, want_series=False, **kw) -> Diagnostics:
    """Diagnostics at one point per path of the TrackProblem pb: xpt holds
    maxdim complex numbers per path with xlimbs limbs per part (real limbs,
    then imaginary limbs: 1 for complex doubles, 4 or 8 for the end points of
    the tracker), tpt the values of t.  Host arrays in and out."""
    ipar, dpar = params(pmode, **kw)
    K = int(ipar[0])
    xpt = np.ascontiguousarray(xpt, dtype=np.float64).reshape(-1)
    tpt = np.ascontiguousarray(tpt, dtype=np.float64).reshape(-1)
    if xpt.size != pb.npaths * pb.maxdim * 2 * xlimbs or tpt.size != pb.npaths:
        raise ValueError("series_diagnostics: xpt or tpt does not match the paths")
    dout = np.zeros(pb.npaths * len(FIELDS))
    iout = np.zeros(pb.npaths * 2, np.int32)
    series = np.zeros(pb.npaths * pb.maxdim * (K + 1) * 2 * pmode) if want_series else None
    _lib.call("phc_series_diagnostics_host", pb.nsys, _lib.ptr(pb.dim), pb.maxvar, _lib.ptr(pb.mono_off),
              _lib.ptr(pb.mono_nvr), _lib.ptr(pb.mono_idx), _lib.ptr(pb.mono_exp), _lib.ptr(pb.eq_off),
              _lib.ptr(pb.term_off), _lib.ptr(pb.term_mono), _lib.ptr(pb.term_a), _lib.ptr(pb.term_b), pb.npaths,
              _lib.ptr(pb.path_sys), _lib.ptr(xpt), int(xlimbs), _lib.ptr(tpt), _lib.ptr(ipar), _lib.ptr(dpar),
              pmode, _lib.ptr(series), _lib.ptr(dout), _lib.ptr(iout))
    if series is not None:
        series = series.reshape(pb.npaths, pb.maxdim, K + 1, 2 * pmode)
    return Diagnostics.from_arrays(dout, iout, series)


def at_endpoints(pb, result, pmode=2, **kw) -> Diagnostics:
    """Diagnostics at the last points of the paths a tracker run reached
    (homotopy.TrackResult: end points at t = result.t)."""
    return series_diagnostics(pb, result.xend, result.t, xlimbs=result.limbs, pmode=pmode, **kw)


def classify(t, diag: Diagnostics, near=0.5):
    """Read the Fabry estimate at points t of the paths: "no series" when
    the Jacobian is singular at the point; "singular at t = 1" when the
    nearest singular point t + z lies within 2 |1 - t| of the point and
    within near * |z| of t = 1 (it closes in on 1 as the point does: the
    path ends at a singular solution or diverges); "interior singularity"
    when the nearest singular point is closer than t = 1 but away from it;
    "regular" otherwise."""
    t = np.asarray(t, dtype=np.float64)
    out = []
    for p in range(t.size):
        if diag.status[p] == 1:
            out.append("no series")
            continue
        if diag.fail[p]:
            out.append("regular")
            continue
        ts = t[p] + diag.z[p]
        gap = abs(1.0 - t[p])
        r = diag.radius[p]
        if r <= 2.0 * gap and abs(ts - 1.0) <= near * r:
            out.append("singular at t = 1")
        elif r < gap:
            out.append("interior singularity")
        else:
            out.append("regular")
    return out


def series_diagnostics_device(dt, xpt, tpt, xlimbs=1, pmode=2, dout=None, iout=None, stream=None, **kw):
    """phc_series_diagnostics on a problem resident on the device
    (homotopy.DeviceTracker dt) with device tensors xpt and tpt; dout
    (points x 10 doubles) and iout (points x 2 ints) are device tensors,
    allocated when not given.  Returns (dout, iout); does not synchronise."""
    import torch
    pb = dt.pb
    ipar, dpar = params(pmode, **kw)
    a = dt.arr
    dev = a["x0"].device
    if dout is None:
        dout = torch.zeros(pb.npaths * len(FIELDS), dtype=torch.float64, device=dev)
    if iout is None:
        iout = torch.zeros(pb.npaths * 2, dtype=torch.int32, device=dev)
    s = 0 if stream is None else stream.cuda_stream
    _lib.call("phc_series_diagnostics", pb.nsys, _lib.ptr(a["dim"]), pb.maxvar, pb.maxdim, pb.nmono_max,
              _lib.ptr(a["mono_off"]), _lib.ptr(a["mono_nvr"]), _lib.ptr(a["mono_idx"]), _lib.ptr(a["mono_exp"]),
              _lib.ptr(a["eq_off"]), _lib.ptr(a["term_off"]), _lib.ptr(a["term_mono"]), _lib.ptr(a["term_a"]),
              _lib.ptr(a["term_b"]), _lib.ptr(a["jg_off"]), _lib.ptr(a["jg_term"]), _lib.ptr(a["jg_slot"]),
              dt.gstaged, pb.npaths, _lib.ptr(a["path_sys"]), _lib.ptr(xpt), int(xlimbs), _lib.ptr(tpt),
              _lib.ptr(ipar), _lib.ptr(dpar), pmode, _lib.c_void_p(0), _lib.ptr(dout), _lib.ptr(iout),
              _lib.c_void_p(s))
    return dout, iout
