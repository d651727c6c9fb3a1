"""Host mirror of the Matrices and Newton least-squares layers.

Mirrors PHCpack's ``GPU_dbl2_blocked_houseqr`` (src/GPU/Matrices/
dbl2_baqr_kernels.cu:3520), ``GPU_dbl2_upper_tiled_solver``
(dbl2_tabs_kernels.cu:952) and ``GPU_dbl2_bals_solve``
(Newton/dbl2_bals_kernels.cu:554), batched over instances.  Arrays are flat,
row-major and limb-interleaved (see include/phc_b200.h).
"""
from __future__ import annotations

import numpy as np

from . import _lib


def width(prec, cplx):
    return prec * (2 if cplx else 1)


def workspace_bytes(prec, cplx, n, szt):
    f = _lib.lib().phc_dense_workspace_bytes
    f.restype = _lib.ctypes.c_longlong
    return int(f(prec, int(cplx), n, szt))


def blocked_houseqr_host(prec, cplx, A, ninst, nrows, ncols, szt):
    W = width(prec, cplx)
    A = np.ascontiguousarray(A, dtype=np.float64)
    Q = np.empty(ninst * nrows * nrows * W)
    R = np.empty(ninst * nrows * ncols * W)
    _lib.call("phc_blocked_houseqr_host", prec, int(cplx), ninst, nrows, ncols, szt, _lib.ptr(A), _lib.ptr(Q),
              _lib.ptr(R), _lib.c_void_p(0))
    return Q, R


def upper_tiled_solver_host(prec, cplx, U, b, ninst, dim, szt):
    """Returns x, and U, b as the reference leaves them (diagonal tiles of U
    inverted, b updated)."""
    W = width(prec, cplx)
    U = np.array(U, dtype=np.float64, copy=True)
    b = np.array(b, dtype=np.float64, copy=True)
    x = np.empty(ninst * dim * W)
    _lib.call("phc_upper_tiled_solver_host", prec, int(cplx), ninst, dim, szt, _lib.ptr(U), _lib.ptr(b),
              _lib.ptr(x), _lib.c_void_p(0))
    return x, U, b


def bals_solve_host(prec, cplx, mat, rhs, ninst, dim, degp1, szt, tailidx=1, flags=None, sol=None, Q=None, R=None):
    """Block-Toeplitz least squares; flags per instance (zeroQ, noqr, upidx,
    bsidx, newtail), default zeroQ=1, noqr=0 as the reference's Newton
    drivers start.  Returns sol, rhs (overwritten), Q, R, flags."""
    W = width(prec, cplx)
    mat = np.ascontiguousarray(mat, dtype=np.float64)
    rhs = np.array(rhs, dtype=np.float64, copy=True)
    sol = np.zeros(ninst * degp1 * dim * W) if sol is None else np.array(sol, dtype=np.float64, copy=True)
    Q = np.zeros(ninst * dim * dim * W) if Q is None else np.array(Q, dtype=np.float64, copy=True)
    R = np.zeros(ninst * dim * dim * W) if R is None else np.array(R, dtype=np.float64, copy=True)
    if flags is None:
        flags = np.tile(np.array([1, 0, 0, 0, tailidx], np.int32), ninst)
    flags = np.array(flags, dtype=np.int32, copy=True)
    _lib.call("phc_bals_solve_host", prec, int(cplx), ninst, dim, degp1, szt, tailidx, _lib.ptr(mat), _lib.ptr(rhs),
              _lib.ptr(sol), _lib.ptr(Q), _lib.ptr(R), _lib.ptr(flags), _lib.c_void_p(0))
    return sol, rhs, Q, R, flags


def linear_residue_host(prec, cplx, mat, rhs, sol, ninst, dim, degp1, tailidx, res=None):
    """Residual rhs_i - sum_j A_j sol_{i-j} of the linearised system for
    tailidx <= i < degp1 (phc_linear_residue_host); returns res (rows below
    tailidx as given) and resmax (prec doubles per instance)."""
    W = width(prec, cplx)
    mat = np.ascontiguousarray(mat, dtype=np.float64)
    rhs = np.ascontiguousarray(rhs, dtype=np.float64)
    sol = np.ascontiguousarray(sol, dtype=np.float64)
    res = np.zeros(ninst * degp1 * dim * W) if res is None else np.array(res, dtype=np.float64, copy=True)
    resmax = np.zeros(ninst * prec)
    _lib.call("phc_linear_residue_host", prec, int(cplx), ninst, dim, degp1, tailidx, _lib.ptr(mat), _lib.ptr(rhs),
              _lib.ptr(sol), _lib.ptr(res), _lib.ptr(resmax), _lib.c_void_p(0))
    return res, resmax


class DeviceBals:
    """Resident buffers for repeated batched solves (torch CUDA tensors as
    device memory)."""

    def __init__(self, prec, cplx, ninst, dim, degp1, szt, device="cuda"):
        import torch
        self.prec, self.cplx, self.ninst, self.dim, self.degp1, self.szt = prec, cplx, ninst, dim, degp1, szt
        W = width(prec, cplx)
        f64 = dict(dtype=torch.float64, device=device)
        self.mat = torch.zeros(ninst * degp1 * dim * dim * W, **f64)
        self.rhs = torch.zeros(ninst * degp1 * dim * W, **f64)
        self.sol = torch.zeros(ninst * degp1 * dim * W, **f64)
        self.Q = torch.zeros(ninst * dim * dim * W, **f64)
        self.R = torch.zeros(ninst * dim * dim * W, **f64)
        self.flags = torch.zeros(ninst * 5, dtype=torch.int32, device=device)
        nb = workspace_bytes(prec, cplx, dim, szt)
        self.work = torch.zeros(ninst * nb // 8, **f64)

    def reset_flags(self, tailidx=1):
        import torch
        f = torch.tensor([1, 0, 0, 0, tailidx], dtype=torch.int32)
        self.flags.copy_(f.repeat(self.ninst))

    def solve(self, tailidx=1, stream=None):
        s = 0 if stream is None else stream.cuda_stream
        _lib.call("phc_bals_solve", self.prec, int(self.cplx), self.ninst, self.dim, self.degp1, self.szt, tailidx,
                  _lib.ptr(self.mat), _lib.ptr(self.rhs), _lib.ptr(self.sol), _lib.ptr(self.Q), _lib.ptr(self.R),
                  _lib.ptr(self.flags), _lib.ptr(self.work), _lib.c_void_p(s))


def workspace_bytes_wy(prec, cplx, n, szt, wy):
    f = _lib.lib().phc_dense_workspace_bytes_wy
    f.restype = _lib.ctypes.c_longlong
    return int(f(prec, int(cplx), n, szt, int(wy)))


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda")


def blocked_houseqr_wy(prec, cplx, A, ninst, nrows, ncols, szt, wy=1):
    """Blocked QR with the WY trailing products on the FP64 tensor cores
    (wy=1, Ozaki splitting) or on the CUDA cores (wy=0); device buffers
    through torch, host arrays in and out."""
    import torch
    W = width(prec, cplx)
    dA = _dev(np.asarray(A, np.float64))
    dQ = torch.zeros(ninst * nrows * nrows * W, dtype=torch.float64, device="cuda")
    dR = torch.zeros(ninst * nrows * ncols * W, dtype=torch.float64, device="cuda")
    work = torch.zeros(ninst * workspace_bytes_wy(prec, cplx, nrows, szt, wy) // 8, dtype=torch.float64,
                       device="cuda")
    _lib.call("phc_blocked_houseqr_wy", prec, int(cplx), ninst, nrows, ncols, szt, _lib.ptr(dA), _lib.ptr(dQ),
              _lib.ptr(dR), _lib.ptr(work), int(wy), _lib.c_void_p(0))
    torch.cuda.synchronize()
    return dQ.cpu().numpy(), dR.cpu().numpy()


def bals_solve_wy(prec, cplx, mat, rhs, ninst, dim, degp1, szt, wy=1, tailidx=1):
    import torch
    W = width(prec, cplx)
    dm, db = _dev(np.asarray(mat, np.float64)), _dev(np.asarray(rhs, np.float64))
    f64 = dict(dtype=torch.float64, device="cuda")
    dx = torch.zeros(ninst * degp1 * dim * W, **f64)
    dQ = torch.zeros(ninst * dim * dim * W, **f64)
    dR = torch.zeros(ninst * dim * dim * W, **f64)
    fl = _dev(np.tile(np.array([1, 0, 0, 0, tailidx], np.int32), ninst))
    work = torch.zeros(ninst * workspace_bytes_wy(prec, cplx, dim, szt, wy) // 8, **f64)
    _lib.call("phc_bals_solve_wy", prec, int(cplx), ninst, dim, degp1, szt, tailidx, _lib.ptr(dm), _lib.ptr(db),
              _lib.ptr(dx), _lib.ptr(dQ), _lib.ptr(dR), _lib.ptr(fl), _lib.ptr(work), int(wy), _lib.c_void_p(0))
    torch.cuda.synchronize()
    return dx.cpu().numpy(), fl.cpu().numpy()
