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


@pytest.mark.parametrize("dim,nterms,deg,seed", [(8, 16, 15, 7), (16, 32, 31, 11), (32, 64, 31, 3)])
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
