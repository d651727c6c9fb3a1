"""PHCpack's own polynomial test program (Polynomials/test_dbl2_polynomials.cpp
and its tester, unchanged) linked with oracle/ref_shim_polynomials.cu in place
of the reference's GPU code: GPU_dbl2_poly_evaldiff, GPU_cmplx2_poly_evaldiff
and GPU_cmplx2vectorized_poly_evaldiff with the reference's signatures, on
this library.  In its mode 2 the reference's tester evaluates random
polynomials on its CPU code and through the GPU entry points and sums all
differences; it passes when both sums (real and complex double-double data)
stay below 1e-24.  The program is built from the reference tree
(oracle/Makefile, target shim); without it the test is skipped."""
import os
import subprocess

import pytest

from oracle import pyoracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dim,nterms,deg,seed", [(8, 16, 15, 7), (16, 32, 31, 11), (32, 64, 31, 3), (8, 16, 63, 5),
                                                   (8, 16, 191, 9)])
def test_reference_tester_through_the_shim(dim, nterms, deg, seed):
    if not os.path.exists(pyoracle.SHIM_BIN):
        pytest.skip("the reference's test program was not built here")
    # seed, dimension, random polynomial (0), number of terms, degree,
    # verbose level 1, mode 2 (GPU and CPU)
    stdin = f"{seed}\n{dim}\n0\n{nterms}\n{deg}\n1\n2\n"
    run = subprocess.run([pyoracle.SHIM_BIN], input=stdin, capture_output=True, text=True, timeout=300)
    out = run.stdout
    assert run.returncode == 0, run.stderr[-2000:]
    assert "on real data" in out and "on complex data" in out, out[-2000:]
    assert "All tests passed." in out, out[-3000:]


def run_program(name, stdin):
    path = pyoracle.SHIM_MATRIX_BINS[name]
    if not os.path.exists(path):
        pytest.skip(f"the reference's {name} was not built here")
    run = subprocess.run([path], input=stdin, capture_output=True, text=True, timeout=600)
    assert run.returncode == 0, run.stderr[-2000:]
    assert "failed" not in run.stderr, run.stderr[-2000:]
    return run.stdout


@pytest.mark.parametrize("name,szt,nbt,nrows", [("test_dbl2_baqr", 8, 2, 16), ("test_dbl2_baqr", 8, 4, 40),
                                                ("test_dbl4_baqr", 32, 2, 64), ("test_dbl4_baqr", 8, 3, 30)])
def test_reference_blocked_qr_tester_through_the_shim(name, szt, nbt, nrows):
    """PHCpack's test_dbl2_baqr / test_dbl4_baqr (Matrices/, unchanged) with
    GPU_dbl{2,4}_blocked_houseqr and GPU_cmplx{2,4}_blocked_houseqr of
    oracle/ref_shim_matrices.cu: in mode 2 the tester factors a random real
    and a random complex matrix on its CPU code and through the GPU entry
    points and probes Q^T A = R and the orthogonality of Q at its own
    tolerance (1e-20 dd, 1e-40 qd) for each: four passes."""
    one = f"7\n{szt}\n{nbt}\n{nrows}\n0\n2\n"
    out = run_program(name, one + one)
    assert out.count("The test succeeded.") == 4, out[-3000:]
    assert "The test failed" not in out


def sums(out, label):
    import re
    return [float(v) for v in re.findall(re.escape(label) + r"\s*:\s*([0-9.eE+-]+)", out)]


@pytest.mark.parametrize("dim,szt,nbt", [(8, 8, 4), (16, 16, 2), (12, 4, 6)])
def test_reference_tiled_solver_tester_through_the_shim(dim, szt, nbt):
    """PHCpack's test_dbl2_tabs (Matrices/, unchanged) with
    GPU_dbl2_upper_inverse, GPU_cmplx2_upper_inverse,
    GPU_dbl2_upper_tiled_solver and GPU_cmplx2_upper_tiled_solver of the
    shim: random upper triangular matrices (real and complex), the GPU
    inverse of one tile and the tiled solve.  The tester prints the sums of
    the differences between its CPU results and the GPU's (inverse, the
    inverted diagonal tiles) and the errors of both solutions against the
    exact one; the GPU's are at double-double rounding level."""
    stdin = f"{dim}\n0\n{dim}\n0\n{szt}\n{nbt}\n0\n1\n{szt}\n{nbt}\n0\n1\n"
    out = run_program("test_dbl2_tabs", stdin)
    inv = sums(out, "Sum of errors on inverse")
    diag = sums(out, "Sum of errors on diagonal tiles")
    cpu = sums(out, "Sum of CPU errors on solution")
    gpu = sums(out, "Sum of GPU errors on solution")
    assert len(inv) == 2 and len(diag) == 2 and len(cpu) == 2 and len(gpu) == 2, out[-3000:]
    assert max(inv) <= 1e-20 and max(diag) <= 1e-20, (inv, diag)
    for c, g in zip(cpu, gpu):
        assert g <= max(100 * c, 1e-26), (cpu, gpu)


def newton_steps(out):
    import re
    return re.findall(r"up_h : (\d+)\s+bs_h : (\d+)\s+tail_h : (\d+)\s+up_d : (\d+)\s+bs_d : (\d+)\s+tail_d : (\d+)", out)


def newton_tester(name, tol, drift, cdata, dim, deg, problem, extra, szt, nbt, nbsteps=8):
    """Runs one of the reference's Newton test programs in mode 2 and checks
    its host-versus-device sums: at the first Newton step (same input on
    both sides) every sum is at most tol, the reference's own tolerance; the
    host and the device then iterate independently, so later sums are the
    first step's rounding differences as the iteration carries them, bounded
    by drift; the skipped updates, skipped back substitutions and tail
    indices agree at every step."""
    if problem == -3:  # the number of columns comes after the Newton steps
        stdin = f"7\n{cdata}\n{dim}\n{deg}\n1\n{problem}\n{nbsteps}\n4\n2\n{nbt}\n{szt}\n"
    else:
        stdin = f"7\n{cdata}\n{dim}\n{deg}\n1\n{problem}\n{extra}{nbsteps}\n2\n{nbt}\n{szt}\n"
    out = run_program(name, stdin)
    steps = newton_steps(out)
    blocks = out.split("up_h :")
    assert len(steps) >= 3 and len(blocks) == len(steps) + 1, out[-3000:]
    first = sums(blocks[0], "sum of errors")
    errs = sums(out, "sum of errors")
    assert len(first) >= 3 and len(errs) >= 3 * len(steps), out[-3000:]
    assert max(first) <= tol, first
    assert max(errs) <= drift, [e for e in errs if e > drift][:10]
    for s in steps:
        assert s[0:3] == s[3:6], steps
    assert int(steps[-1][5]) >= deg, steps[-1]


# seed 7, complex data, dimension, degree, verbose level 1, test problem
# (3: unimodular monomial system, -1: lower triangular ones, -2: decoupled
# monomials, -3: the columns of cyclic n-roots, -4: a 2-column system, -5:
# the polynomials of cyclic n-roots in row form), [size of the numbers |
# number of columns], 8 Newton steps, mode 2 (host and device), tiles, tile size
@pytest.mark.parametrize("cdata,dim,deg,problem,extra,szt,nbt", [
    (0, 8, 8, 3, "2\n", 4, 2), (1, 8, 8, 3, "2\n", 4, 2), (0, 8, 8, -1, "", 8, 1), (0, 8, 8, -2, "", 4, 2),
    (0, 8, 8, -3, None, 4, 2), (1, 8, 8, -3, None, 4, 2), (1, 8, 8, -4, "", 4, 2), (0, 8, 8, -5, "", 4, 2),
    (1, 8, 8, -5, "", 2, 4), (0, 16, 15, 3, "2\n", 8, 2)])
def test_reference_newton_tester_through_the_shim(cdata, dim, deg, problem, extra, szt, nbt):
    """PHCpack's test_dbl2_newton (Newton/, unchanged) with every device
    entry point it calls taken from the shims: GPU_{dbl2,cmplx2}_bals_solve,
    GPU_{dbl2,cmplx2}_linear_residue, GPU_dbl2_evaluate_monomials,
    GPU_cmplx2vectorized_evaluate_monomials, GPU_{dbl2,cmplx2}_evaluate_columns
    (oracle/ref_shim_newton.cu) and the polynomial evaluation of
    oracle/ref_shim_polynomials.cu.  In mode 2 the tester runs each Newton
    step on its CPU code and on the device path and prints the sum of the
    differences of the evaluated system, Jacobian, right hand sides, Q, R,
    updated right hand sides, solution update and series; all stay below
    the reference's own tolerance 1e-20 (for the columns of cyclic n-roots
    at the first step, the later steps drifting apart as the iteration
    amplifies the first step's rounding differences, to about 1e-18 after
    eight steps), and the skipped updates, skipped back substitutions and
    tail indices of the host and device agree at every step."""
    newton_tester("test_dbl2_newton", 1e-20, 1e-20 if problem != -3 else 1e-15, cdata, dim, deg, problem, extra,
                  szt, nbt, nbsteps=12)


@pytest.mark.parametrize("cdata,dim,deg,problem,extra,szt,nbt", [
    (0, 8, 8, 3, "2\n", 4, 2), (1, 8, 8, 3, "2\n", 4, 2), (0, 8, 8, -3, None, 4, 2), (1, 8, 8, -4, "", 8, 1),
    (0, 8, 8, -5, "", 4, 2), (1, 8, 8, -5, "", 4, 2)])
def test_reference_quad_double_newton_tester_through_the_shim(cdata, dim, deg, problem, extra, szt, nbt):
    """PHCpack's test_dbl4_newton (Newton/, unchanged) with the quad double
    twins of the Newton-layer entry points (ref_shim_newton.cu and
    ref_shim_polynomials.cu compiled with -DSHIM_NEWTON4 / -DSHIM_POLY4):
    at the first step every host-versus-device sum stays below the
    tester's own tolerance 1e-50, and the skip counts and tail indices agree
    at every step.  The tester sums differences limb by limb, so two
    quad-doubles equal to 1e-63 but normalised differently (a leading limb
    one ulp apart, the next limb compensating) count as about one ulp of the
    leading limb; later steps are held to 1e-30 for that reason (seen once:
    9.6e-35 from a Jacobian entry of -3.88e-19 whose two values differ by
    9e-64)."""
    newton_tester("test_dbl4_newton", 1e-50, 1e-30, cdata, dim, deg, problem, extra, szt, nbt, nbsteps=12)


@pytest.mark.parametrize("dim,nterms,deg,seed", [(8, 16, 15, 7), (16, 32, 31, 11), (8, 16, 100, 13)])
def test_reference_quad_double_polynomial_tester_through_the_shim(dim, nterms, deg, seed):
    """PHCpack's test_dbl4_polynomials (Polynomials/, unchanged) with
    GPU_dbl4_poly_evaldiff, GPU_cmplx4_poly_evaldiff and
    GPU_cmplx4vectorized_poly_evaldiff of the shim; the tester's own
    tolerance is 1e-56 on the sums of the differences."""
    stdin = f"{seed}\n{dim}\n0\n{nterms}\n{deg}\n1\n2\n"
    out = run_program("test_dbl4_polynomials", stdin)
    assert "on real data" in out and "on complex data" in out, out[-2000:]
    assert "All tests passed." in out, out[-3000:]
