"""Host mirror of the Polynomials layer: evaluation and differentiation of
polynomial systems at truncated power series on the GPU.

Mirrors PHCpack's ``GPU_dbl2_poly_evaldiff`` family
(src/GPU/Polynomials/dbl2_polynomials_kernels.cu:1577) and the host-mode
``CPU_dbl2_poly_evaldiff`` (dbl2_polynomials_host.cpp:259) argument meaning:
``nvr``/``idx`` supports, ``cst`` constant series, ``cff`` coefficient
series, ``input`` the series of the variables, ``output`` dim+1 series per
polynomial with the value in row ``dim``.  Batched over systems.
"""
from __future__ import annotations

import numpy as np

from . import _lib
from .workloads import SystemBatch


class DeviceBatch:
    """A SystemBatch resident in device memory (torch CUDA tensors used as
    plain device buffers)."""

    def __init__(self, b: SystemBatch, device="cuda"):
        import torch

        self.b = b.validate()
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)
        self.mon_off, self.nvr = t(b.mon_off), t(b.nvr)
        self.idx, self.exps = t(b.idx), t(b.exps)
        self.cst, self.cff, self.input = t(b.cst), t(b.cff), t(b.input)
        self.output = torch.empty(b.output_size(), dtype=torch.float64, device=device)

    def evaldiff(self, stream=None):
        """Enqueue the batched eval/diff on ``stream`` (a torch stream or None)."""
        b = self.b
        s = 0 if stream is None else stream.cuda_stream
        _lib.call("phc_system_evaldiff", b.prec, int(b.cplx), b.nsys, b.dim, b.deg, b.maxvar,
                  _lib.ptr(self.mon_off), _lib.ptr(self.nvr), _lib.ptr(self.idx), _lib.ptr(self.exps),
                  _lib.ptr(self.cst), _lib.ptr(self.cff), _lib.ptr(self.input), _lib.ptr(self.output),
                  _lib.c_void_p(s))
        return self.output


def system_evaldiff_host(b: SystemBatch, out: np.ndarray | None = None) -> np.ndarray:
    """Host arrays in, host arrays out (the reference's GPU_* driver shape)."""
    b.validate()
    if out is None:
        out = np.empty(b.output_size())
    _lib.call("phc_system_evaldiff_host", b.prec, int(b.cplx), b.nsys, b.dim, b.deg, b.maxvar,
              _lib.ptr(b.mon_off), _lib.ptr(b.nvr), _lib.ptr(b.idx), _lib.ptr(b.exps), _lib.ptr(b.cst),
              _lib.ptr(b.cff), _lib.ptr(b.input), _lib.ptr(out), _lib.c_void_p(0))
    return out


def split_limbs(flat: np.ndarray, prec: int, cplx: bool, shape) -> list[np.ndarray]:
    """Flat limb-interleaved array -> list of separate limb arrays in the
    reference's order (hi, lo / hihi, lohi, hilo, lolo; real then imaginary)."""
    W = prec * (2 if cplx else 1)
    a = np.asarray(flat).reshape(tuple(shape) + (W,))
    return [np.ascontiguousarray(a[..., c]) for c in range(W)]


def join_limbs(parts, prec: int, cplx: bool) -> np.ndarray:
    """Inverse of split_limbs."""
    return np.ascontiguousarray(np.stack(parts, axis=-1)).reshape(-1)


def gpu_poly_evaldiff(prec: int, cplx: bool, dim: int, nbr: int, deg: int, nvr, idx, cst, cff, inp, exps=None):
    """One polynomial, reference argument order: ``nbr`` monomials with
    ``nvr[m]`` variables ``idx[m]``, constant series ``cst`` (deg+1 numbers),
    coefficient series ``cff`` (nbr x (deg+1)), input series (dim x (deg+1)),
    all limb-interleaved.  Returns output (dim+1 series, value in row dim).
    The reference's polynomial kernels take exponent 1 only; ``exps``
    extends that with the common-factor method."""
    nvr = np.asarray(nvr, dtype=np.int32)
    maxvar = max(1, int(nvr.max()) if nbr else 1)
    idx2 = np.zeros((nbr, maxvar), dtype=np.int32)
    exp2 = np.ones((nbr, maxvar), dtype=np.int32)
    for m in range(nbr):
        idx2[m, :nvr[m]] = idx[m][:nvr[m]]
        if exps is not None:
            exp2[m, :nvr[m]] = exps[m][:nvr[m]]
    b = SystemBatch(1, dim, deg, maxvar, prec, cplx, np.array([0] * 0 + [0, nbr] + [nbr] * (dim - 1), np.int32),
                    nvr, idx2, exp2,
                    np.concatenate([np.asarray(cst, np.float64).reshape(-1),
                                    np.zeros((dim - 1) * (deg + 1) * prec * (2 if cplx else 1))]),
                    np.asarray(cff, np.float64).reshape(-1), np.asarray(inp, np.float64).reshape(-1))
    out = system_evaldiff_host(b)
    S = (deg + 1) * prec * (2 if cplx else 1)
    return out[: (dim + 1) * S]
