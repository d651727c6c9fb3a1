"""ctypes bindings of the CPU oracle (test infrastructure only).

Two libraries with the same flat-array conventions:
  * ``liboracle.so``      -- this project's restatement (oracle_capi.cpp);
  * ``_ref/libphcref.so`` -- PHCpack's own host code behind ref_harness.cpp,
    present only where it was built from the reference tree.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libphcref.so")
# the reference's src/GPU tree, where the reference is present (unset: the
# reference-backed library is not built)
REF_TREE = os.environ.get("PHC_REFERENCE_GPU", "")

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


SHIM_BIN = os.path.join(HERE, "_ref", "test_dbl2_polynomials")
# the reference's matrix, Newton and quad double polynomial test programs
# linked with ref_shim_matrices.cu, ref_shim_newton.cu and ref_shim_polynomials.cu
SHIM_MATRIX_BINS = {name: os.path.join(HERE, "_ref", name) for name in ("test_dbl2_baqr", "test_dbl4_baqr",
                                                                        "test_dbl2_tabs", "test_dbl2_newton",
                                                                        "test_dbl4_newton", "test_dbl4_polynomials")}


def build(ref: bool = True) -> None:
    """Compile liboracle.so and, where the reference tree exists,
    _ref/libphcref.so and the reference's test programs for polynomials,
    blocked QR, tiled back substitution and Newton linked with this library
    through the ref_shim_*.cu files (needs phcpack_b200/libphcb200.so built
    first)."""
    targets = ["liboracle.so"]
    if ref and REF_TREE and os.path.isdir(REF_TREE):
        targets.append("_ref/libphcref.so")
        if os.path.exists(os.path.join(HERE, "..", "phcpack_b200", "libphcb200.so")):
            targets += ["shim"]
    subprocess.run(["make", "-s", "-C", HERE, f"REF={REF_TREE}"] + targets, check=True)


def _dp(a):
    return a.ctypes.data_as(_D)


def _ip(a):
    return a.ctypes.data_as(_I)


class Lib:
    def __init__(self, path: str, prefix: str):
        self.lib = ctypes.CDLL(path)
        self.prefix = prefix

    def _fn(self, name):
        f = getattr(self.lib, f"{self.prefix}_{name}")
        f.restype = ctypes.c_int
        return f

    def system_evaldiff(self, b) -> np.ndarray:
        out = np.zeros(b.output_size())
        rc = self._fn("system_evaldiff")(
            b.prec, int(b.cplx), b.nsys, b.dim, b.deg, b.maxvar, _ip(b.mon_off), _ip(b.nvr), _ip(b.idx),
            _ip(b.exps), _dp(b.cst), _dp(b.cff), _dp(b.input), _dp(out))
        assert rc == 0
        return out

    def blocked_houseqr(self, prec, cplx, nrows, ncols, szt, nbt, A):
        W = prec * (2 if cplx else 1)
        A = np.ascontiguousarray(A, dtype=np.float64)
        Q = np.zeros(nrows * nrows * W)
        R = np.zeros(nrows * ncols * W)
        rc = self._fn("blocked_houseqr")(prec, int(cplx), nrows, ncols, szt, nbt, _dp(A), _dp(Q), _dp(R))
        assert rc == 0
        return Q, R

    def upper_tiled_solver(self, prec, cplx, dim, szt, nbt, U, b):
        W = prec * (2 if cplx else 1)
        U = np.array(U, dtype=np.float64, copy=True)
        b = np.array(b, dtype=np.float64, copy=True)
        x = np.zeros(dim * W)
        rc = self._fn("upper_tiled_solver")(prec, int(cplx), dim, szt, nbt, _dp(U), _dp(b), _dp(x))
        assert rc == 0
        return x, U, b

    def bals_solve(self, prec, cplx, dim, degp1, tailidx, mat, rhs, flags=(1, 0, 0, 0, 1), Q=None, R=None):
        W = prec * (2 if cplx else 1)
        mat = np.ascontiguousarray(mat, dtype=np.float64)
        rhs = np.array(rhs, dtype=np.float64, copy=True)
        sol = np.zeros(degp1 * dim * W)
        Q = np.zeros(dim * dim * W) if Q is None else np.array(Q, dtype=np.float64, copy=True)
        R = np.zeros(dim * dim * W) if R is None else np.array(R, dtype=np.float64, copy=True)
        fl = np.array(flags, dtype=np.int32)
        rc = self._fn("bals_solve")(prec, int(cplx), dim, degp1, tailidx, _dp(mat), _dp(rhs), _dp(sol), _dp(Q),
                                    _dp(R), _ip(fl))
        assert rc == 0
        return sol, rhs, Q, R, fl


    def linear_residue(self, prec, cplx, dim, degp1, tailidx, mat, rhs, sol, res=None):
        """Reference library only: CPU_dbl2_linear_residue and its twins."""
        W = prec * (2 if cplx else 1)
        mat = np.ascontiguousarray(mat, dtype=np.float64)
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        sol = np.ascontiguousarray(sol, dtype=np.float64)
        res = np.zeros(degp1 * dim * W) if res is None else np.array(res, dtype=np.float64, copy=True)
        mx = np.zeros(prec)
        rc = self._fn("linear_residue")(prec, int(cplx), dim, degp1, tailidx, _dp(mat), _dp(rhs), _dp(sol), _dp(res),
                                        _dp(mx))
        assert rc == 0
        return res, mx

    def od_binop(self, op, a, b):
        """Octo-double add (0), mul (1), div (2) or multiply by a double (3,
        b[k, 0]) of rows of eight limbs."""
        a = np.ascontiguousarray(a, dtype=np.float64).reshape(-1, 8)
        b = np.ascontiguousarray(b, dtype=np.float64).reshape(-1, 8)
        out = np.zeros_like(a)
        rc = self._fn("od_binop")(op, a.shape[0], _dp(a), _dp(b), _dp(out))
        assert rc == 0
        return out


_oracle = None
_ref = None


def oracle() -> Lib:
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO):
            build(ref=False)
        _oracle = Lib(ORACLE_SO, "orc")
    return _oracle


def reference() -> Lib | None:
    """PHCpack's own host code, or None where it was never built."""
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO) and REF_TREE and os.path.isdir(REF_TREE):
            build(ref=True)
        if not os.path.exists(REF_SO):
            return None
        _ref = Lib(REF_SO, "ref")
    return _ref


def newton_steps(lib: Lib, b, deg, nsteps, schedule=0):
    """Newton on power series for every system of batch b (series of degree
    deg in b.input, updated copy returned) with the oracle's single-system
    step (oracle_capi.cpp newton_t); flags per system as in the C ABI."""
    W = b.width
    n1 = deg + 1
    out = np.array(b.input, dtype=np.float64, copy=True)
    flags_all = []
    f = lib._fn("newton_step")
    for s in range(b.nsys):
        m0, m1 = int(b.mon_off[s * b.dim]), int(b.mon_off[(s + 1) * b.dim])
        off = (b.mon_off[s * b.dim:(s + 1) * b.dim + 1] - m0).astype(np.int32)
        ser = np.ascontiguousarray(out[s * b.dim * n1 * W:(s + 1) * b.dim * n1 * W])
        cst = np.ascontiguousarray(b.cst[s * b.dim * n1 * W:(s + 1) * b.dim * n1 * W])
        cff = np.ascontiguousarray(b.cff[m0 * n1 * W:m1 * n1 * W])
        nvr = np.ascontiguousarray(b.nvr[m0:m1])
        idx = np.ascontiguousarray(b.idx.reshape(-1, b.maxvar)[m0:m1])
        exps = np.ascontiguousarray(b.exps.reshape(-1, b.maxvar)[m0:m1])
        Q = np.zeros(b.dim * b.dim * W)
        R = np.zeros(b.dim * b.dim * W)
        fl = np.array([1, 0, 0, 0, 1], np.int32)
        wrk = 0 if schedule else deg
        for _ in range(nsteps):
            rc = f(b.prec, int(b.cplx), b.dim, wrk, deg, b.maxvar, _ip(off), _ip(nvr), _ip(idx), _ip(exps), _dp(cst),
                   _dp(cff), _dp(ser), _dp(Q), _dp(R), _ip(fl))
            assert rc == 0
            if schedule:
                if fl[4] >= deg:
                    break
                wrk = min(deg, wrk + 1 + wrk // 2)
        out[s * b.dim * n1 * W:(s + 1) * b.dim * n1 * W] = ser
        flags_all.append(fl.copy())
    return out, np.concatenate(flags_all)


def track(lib: Lib, pb, ipar, dpar, pmode=1, rmode=2, nthreads=1, step_mode=0, model=None):
    """Track the paths of a homotopy TrackProblem on the CPU (the tracker
    restatement of tracker_oracle.cpp); step_mode 1 with a model buffer
    (uint8 array, the device layout) uses the learned step.  Returns (xend,
    info, dinfo) with the layout of the C ABI (16 doubles per complex end
    point coordinate for rmode 8, 8 otherwise; 6 ints of info per path)."""
    xend = np.zeros(pb.npaths * pb.maxdim * (16 if rmode == 8 else 8))
    info = np.zeros(pb.npaths * 6, np.int32)
    m = None if model is None else np.ascontiguousarray(model)
    dinfo = np.zeros(pb.npaths * 2)
    f = lib._fn("track")
    rc = f(pb.nsys, _ip(pb.dim), pb.maxvar, _ip(pb.mono_off), _ip(pb.mono_nvr), _ip(pb.mono_idx), _ip(pb.mono_exp),
           _ip(pb.eq_off), _ip(pb.term_off), _ip(pb.term_mono), _dp(pb.term_a), _dp(pb.term_b), pb.npaths,
           _ip(pb.path_sys), pb.maxdim, _dp(pb.x0), _ip(ipar), _dp(dpar), pmode, rmode, int(step_mode),
           None if m is None else m.ctypes.data_as(ctypes.c_void_p), nthreads,
           _dp(xend), _ip(info), _dp(dinfo))
    assert rc == 0
    return xend, info, dinfo


def series_diagnostics(lib: Lib, pb, xpt, xlimbs, tpt, ipar, dpar, pmode=2):
    """End-game diagnostics of tracker_oracle.cpp at the points (xpt, tpt)
    of a TrackProblem's homotopies: the series, Fabry's ratio, the Pade error
    norm, and the Jacobian and Hessians in complex double (their singular
    values are left to the caller).  Returns a dict of arrays."""
    K = int(ipar[0])
    W = 2 * pmode
    n = pb.maxdim
    series = np.zeros(pb.npaths * n * (K + 1) * W)
    dout = np.zeros(pb.npaths * 6)
    iout = np.zeros(pb.npaths * 2, np.int32)
    J = np.zeros(pb.npaths * n * n * 2)
    H = np.zeros(pb.npaths * n * n * n * 2)
    xpt = np.ascontiguousarray(xpt, dtype=np.float64)
    tpt = np.ascontiguousarray(tpt, dtype=np.float64)
    ipar = np.ascontiguousarray(ipar, dtype=np.int32)
    dpar = np.ascontiguousarray(dpar, dtype=np.float64)
    f = lib._fn("series_diagnostics")
    rc = f(pb.nsys, _ip(pb.dim), pb.maxvar, _ip(pb.mono_off), _ip(pb.mono_nvr), _ip(pb.mono_idx), _ip(pb.mono_exp),
           _ip(pb.eq_off), _ip(pb.term_off), _ip(pb.term_mono), _dp(pb.term_a), _dp(pb.term_b), pb.npaths,
           _ip(pb.path_sys), n, _dp(xpt), int(xlimbs), _dp(tpt), _ip(ipar), _dp(dpar), pmode, _dp(series),
           _dp(dout), _ip(iout), _dp(J), _dp(H))
    assert rc == 0
    d = dout.reshape(-1, 6)
    Jc = J.reshape(pb.npaths, n, n, 2)
    Hc = H.reshape(pb.npaths, n, n, n, 2)
    return dict(series=series.reshape(pb.npaths, n, K + 1, W), z=d[:, 0] + 1j * d[:, 1], radius=d[:, 2],
                err=d[:, 3], padenorm=d[:, 4], lastdx=d[:, 5], fail=iout[0::2].copy(), status=iout[1::2].copy(),
                J=Jc[..., 0] + 1j * Jc[..., 1], H=Hc[..., 0] + 1j * Hc[..., 1])
