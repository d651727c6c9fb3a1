"""Seeded synthetic inputs for the multiple-double power-series path.

Every array is float64, flat and limb-interleaved: a number in precision
``prec`` (1 double, 2 double-double, 4 quad-double) occupies ``prec``
consecutive doubles, a complex number ``2*prec`` (real limbs, then imaginary
limbs).  A series of degree ``deg`` is ``deg+1`` consecutive numbers.

The generators stand in for the inputs PHCpack's test drivers draw from
libc ``rand()`` (src/GPU/Norms/random_numbers.cpp:10-17); the shapes and
value distributions are the ones named for each workload (systems of
polynomials with supports over a few distinct variables, unit-circle or
uniform coefficients, series decaying as 2^-k).
"""
from __future__ import annotations

import numpy as np

TWO_M53 = 2.0 ** -53


def _quick_renorm(limbs: np.ndarray) -> np.ndarray:
    """Renormalise a stack of limbs (last axis) so that each limb is at most
    half an ulp of the one before (a non-overlapping expansion)."""
    out = limbs.copy()
    L = out.shape[-1]
    for _ in range(2):
        for i in range(L - 1, 0, -1):
            a = out[..., i - 1]
            b = out[..., i]
            s = a + b
            e = b - (s - a)
            out[..., i - 1] = s
            out[..., i] = e
    return out


def md_from_double(x: np.ndarray, prec: int, rng: np.random.Generator | None = None,
                   tail: bool = True) -> np.ndarray:
    """Turn doubles into ``prec``-limb numbers.  With ``tail`` the lower limbs
    are random at 2^-53 scale relative to the limb above."""
    x = np.asarray(x, dtype=np.float64)
    out = np.zeros(x.shape + (prec,))
    out[..., 0] = x
    if prec > 1 and tail:
        assert rng is not None
        for i in range(1, prec):
            out[..., i] = out[..., i - 1] * TWO_M53 * rng.uniform(-1.0, 1.0, size=x.shape)
        out = _quick_renorm(out)
    return out


def pack(re: np.ndarray, im: np.ndarray | None) -> np.ndarray:
    """Interleave real and imaginary limb stacks (shape (..., prec))."""
    if im is None:
        return np.ascontiguousarray(re).reshape(-1)
    return np.ascontiguousarray(np.concatenate([re, im], axis=-1)).reshape(-1)


def random_numbers(rng, shape, prec, cplx, kind="unit", scale=None, tail=True):
    """``kind``: 'unit' (unit circle / +-1 uniform), 'uniform' (U[-1,1]),
    'normal' (N(0,1)).  ``scale`` multiplies the leading limb."""
    shape = tuple(shape)
    if cplx:
        if kind == "unit":
            th = rng.uniform(0.0, 2.0 * np.pi, size=shape)
            re, im = np.cos(th), np.sin(th)
        elif kind == "normal":
            re, im = rng.standard_normal(shape), rng.standard_normal(shape)
        else:
            re, im = rng.uniform(-1, 1, shape), rng.uniform(-1, 1, shape)
        if scale is not None:
            re, im = re * scale, im * scale
        return pack(md_from_double(re, prec, rng, tail), md_from_double(im, prec, rng, tail))
    if kind == "normal":
        re = rng.standard_normal(shape)
    else:
        re = rng.uniform(-1, 1, shape)
    if scale is not None:
        re = re * scale
    return pack(md_from_double(re, prec, rng, tail), None)


class SystemBatch:
    """A batch of ``nsys`` polynomial systems of dimension ``dim``.

    Polynomial (s, p) owns monomials ``mon_off[s*dim+p] .. mon_off[s*dim+p+1]-1``;
    monomial m has ``nvr[m]`` distinct variables ``idx[m, :nvr[m]]`` with
    exponents ``exps[m, :nvr[m]]`` and a coefficient series ``cff[m]``.
    ``cst`` holds one constant series per polynomial; ``input`` one series per
    variable per system.
    """

    def __init__(self, nsys, dim, deg, maxvar, prec, cplx, mon_off, nvr, idx, exps, cst, cff, inp):
        self.nsys, self.dim, self.deg, self.maxvar = nsys, dim, deg, maxvar
        self.prec, self.cplx = prec, cplx
        self.mon_off = np.ascontiguousarray(mon_off, dtype=np.int32)
        self.nvr = np.ascontiguousarray(nvr, dtype=np.int32)
        self.idx = np.ascontiguousarray(idx, dtype=np.int32)
        self.exps = np.ascontiguousarray(exps, dtype=np.int32)
        self.cst = np.ascontiguousarray(cst, dtype=np.float64)
        self.cff = np.ascontiguousarray(cff, dtype=np.float64)
        self.input = np.ascontiguousarray(inp, dtype=np.float64)

    @property
    def width(self):
        return self.prec * (2 if self.cplx else 1)

    @property
    def nmon(self):
        return int(self.mon_off[-1])

    def validate(self):
        """Raise ValueError on supports a kernel could not evaluate."""
        npoly = self.nsys * self.dim
        if self.mon_off.shape != (npoly + 1,) or self.mon_off[0] != 0 or (np.diff(self.mon_off) < 0).any():
            raise ValueError("mon_off must be nondecreasing with nsys*dim+1 entries starting at 0")
        nm = self.nmon
        if self.nvr.shape[0] < nm or self.idx.reshape(-1).shape[0] < nm * self.maxvar:
            raise ValueError("supports shorter than mon_off[-1] monomials")
        k = self.nvr[:nm]
        if (k < 1).any() or (k > self.maxvar).any():
            raise ValueError("nvr out of [1, maxvar]")
        idx = self.idx.reshape(-1, self.maxvar)[:nm]
        ex = self.exps.reshape(-1, self.maxvar)[:nm]
        used = np.arange(self.maxvar)[None, :] < k[:, None]
        if ((idx < 0) | (idx >= self.dim))[used].any() or (ex < 1)[used].any():
            raise ValueError("variable index or exponent out of range")
        for m in np.nonzero(k > 1)[0][:100000]:
            if len(set(idx[m, :k[m]].tolist())) != k[m]:
                raise ValueError(f"monomial {m} repeats a variable (use exponents)")
        return self

    def output_size(self):
        return self.nsys * self.dim * (self.dim + 1) * (self.deg + 1) * self.width


def random_supports(rng, nsys, dim, nmon, maxvar, minvar=1, expmax=1, expmin=1):
    """Per polynomial ``nmon`` monomials, each over a uniform number of
    distinct variables in [minvar, maxvar] chosen without replacement,
    exponents uniform in [expmin, expmax]."""
    total = nsys * dim * nmon
    mon_off = np.arange(0, total + 1, nmon, dtype=np.int32)
    nvr = rng.integers(minvar, maxvar + 1, size=total).astype(np.int32)
    idx = np.zeros((total, maxvar), dtype=np.int32)
    exps = np.zeros((total, maxvar), dtype=np.int32)
    for m in range(total):
        k = nvr[m]
        idx[m, :k] = np.sort(rng.choice(dim, size=k, replace=False))
        exps[m, :k] = rng.integers(expmin, expmax + 1, size=k)
    return mon_off, nvr, idx, exps


def eval_batch(seed, nsys, dim, deg, nmon, maxvar, prec, cplx, expmax=1, minvar=1,
               cff_kind="unit", decay=True) -> SystemBatch:
    """Batched eval/diff workload: series inputs x_{i,k} ~ N(0,1)*2^-k with
    lower limbs at 2^-53 relative scale, coefficient and constant series
    with every coefficient on the unit circle (complex) or U[-1,1] (real)."""
    rng = np.random.default_rng(seed)
    mon_off, nvr, idx, exps = random_supports(rng, nsys, dim, nmon, maxvar, minvar, expmax)
    n1 = deg + 1
    kind = cff_kind if cplx else "uniform"
    cff = random_numbers(rng, (len(nvr), n1), prec, cplx, kind)
    cst = random_numbers(rng, (nsys * dim, n1), prec, cplx, kind)
    scale = (2.0 ** -np.arange(n1)) if decay else None
    inp = random_numbers(rng, (nsys * dim, n1), prec, cplx, "normal",
                         scale=np.broadcast_to(scale, (nsys * dim, n1)) if decay else None)
    return SystemBatch(nsys, dim, deg, maxvar, prec, cplx, mon_off, nvr, idx, exps, cst, cff, inp)


def config2(nsys=4096, seed=2, dim=32, deg=31, nmon=32, maxvar=4):
    """4096 systems n=32, 32 monomials per polynomial over <= 4 variables with
    exponents in {1,2,3}, unit-circle coefficients, degree 31, complex dd."""
    return eval_batch(seed, nsys, dim, deg, nmon, maxvar, prec=2, cplx=True, expmax=3)
