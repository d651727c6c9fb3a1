"""Generate the golden fixtures of tests/golden from PHCpack's own host code.

Run where the reference tree is present:
    python tests/golden/make_golden.py
It builds oracle/_ref/libphcref.so (the reference's host sources compiled in
place, see oracle/Makefile) and stores, for seeded inputs, the outputs of the
reference's CPU_dbl{2,4}_* and CPU_cmplx{2,4}_* routines.  The fixtures are
small .npz files; the GPU box has no reference tree and reads only these.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import pyoracle  # noqa: E402
from phcpack_b200 import workloads as wl  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def save(name, **arrays):
    np.savez_compressed(os.path.join(OUT, name + ".npz"), **arrays)
    size = os.path.getsize(os.path.join(OUT, name + ".npz"))
    print(f"{name}.npz  {size} bytes")


def batch_arrays(b):
    return dict(nsys=b.nsys, dim=b.dim, deg=b.deg, maxvar=b.maxvar, prec=b.prec, cplx=int(b.cplx),
                mon_off=b.mon_off, nvr=b.nvr, idx=b.idx, exps=b.exps, cst=b.cst, cff=b.cff, input=b.input)


def main():
    ref = pyoracle.reference()
    if ref is None:
        raise SystemExit("the reference tree is not available here")
    # eval/diff: real dd (the n=8, <=3 variables, exponents {1,2} workload at
    # degree 15), complex dd (n=32-like supports at degree 31, exponents
    # {1,2,3}), complex qd
    cases = [
        ("eval_dd_real", wl.eval_batch(11, 2, 8, 15, 8, 3, 2, False, expmax=2)),
        ("eval_dd_cplx", wl.eval_batch(12, 2, 8, 31, 8, 4, 2, True, expmax=3)),
        ("eval_qd_real", wl.eval_batch(13, 1, 6, 15, 6, 4, 4, False, expmax=2)),
        ("eval_qd_cplx", wl.eval_batch(14, 1, 6, 15, 6, 4, 4, True, expmax=3)),
        ("eval_dd_cplx_k8", wl.eval_batch(15, 1, 10, 8, 12, 6, 2, True, expmax=2, minvar=4)),
    ]
    for name, b in cases:
        out = ref.system_evaldiff(b)
        save(name, output=out, **batch_arrays(b))
    # blocked Householder QR (Matrices/dbl{2,4}_baqr_host.cpp)
    rng = np.random.default_rng(21)
    for prec, cplx, n, szt in [(2, False, 16, 8), (2, True, 16, 8), (4, False, 32, 16), (4, True, 16, 8)]:
        A = wl.random_numbers(rng, (n, n), prec, cplx, "normal")
        Q, R = ref.blocked_houseqr(prec, cplx, n, n, szt, n // szt, A)
        save(f"baqr_p{prec}_{'c' if cplx else 'r'}{n}", A=A, Q=Q, R=R, prec=prec, cplx=int(cplx), n=n, szt=szt)
    # tiled back substitution (Matrices/dbl{2,4}_tabs_host.cpp)
    for prec, cplx, n, szt in [(2, False, 16, 4), (4, True, 16, 8)]:
        A = wl.random_numbers(rng, (n, n), prec, cplx, "normal")
        _, R = ref.blocked_houseqr(prec, cplx, n, n, szt, n // szt, A)
        b = wl.random_numbers(rng, (n,), prec, cplx, "normal")
        x, U2, b2 = ref.upper_tiled_solver(prec, cplx, n, szt, n // szt, R, b)
        save(f"tabs_p{prec}_{'c' if cplx else 'r'}{n}", U=R, b=b, x=x, U_after=U2, b_after=b2, prec=prec,
             cplx=int(cplx), n=n, szt=szt)
    # block Toeplitz least squares (Newton/dbl{2,4}_bals_host.cpp)
    for prec, cplx, n, degp1 in [(2, False, 8, 8), (2, True, 8, 9), (4, True, 8, 8)]:
        M = wl.random_numbers(rng, (degp1, n, n), prec, cplx, "normal")
        rhs = wl.random_numbers(rng, (degp1, n), prec, cplx, "normal")
        sol, rhs2, Q, R, fl = ref.bals_solve(prec, cplx, n, degp1, 1, M, rhs)
        save(f"bals_p{prec}_{'c' if cplx else 'r'}{n}", mat=M, rhs=rhs, sol=sol, flags=fl, prec=prec,
             cplx=int(cplx), n=n, degp1=degp1)


def make_od():
    """Octo-double add, mul, div and multiply-by-double of the reference
    (Norms/octo_double_functions.cpp) on seeded random normalised inputs."""
    ref = pyoracle.reference()
    if ref is None:
        raise SystemExit("the reference tree is not available here")
    rng = np.random.default_rng(31)
    n = 256

    def rand_od():
        out = np.zeros((n, 8))
        for k in range(n):
            limbs = [rng.standard_normal() * 10.0 ** rng.integers(-8, 8)]
            for _ in range(7):
                limbs.append(limbs[-1] * 2.0 ** -53 * rng.uniform(-1, 1))
            out[k] = limbs
        return ref.od_binop(0, out, np.zeros((n, 8)))  # renormalised by the reference's odf_add

    a, b = rand_od(), rand_od()
    save("od_ops", a=a, b=b, add=ref.od_binop(0, a, b), mul=ref.od_binop(1, a, b), div=ref.od_binop(2, a, b),
         mul_d=ref.od_binop(3, a, b))


if __name__ == "__main__":
    import sys
    if sys.argv[1:] == ["od"]:
        make_od()
    else:
        main()
        make_od()
