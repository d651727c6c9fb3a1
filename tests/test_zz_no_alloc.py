"""The allocation-free block-Toeplitz solve (phc_bals_solve_static).

Callers that cannot afford cudaFree's device-wide synchronisation, hand all
device memory to their own allocator, or must not allocate once set up
cannot let the library allocate; this entry point takes its
workspace from a static device array instead.  Checked through the C ABI
against phc_bals_solve with a caller-provided workspace, on two calls in a
row of the same shape, and on two calls in a row of different shapes and
precisions (the shared array keeps the previous call's contents), within
the tolerance of the other least-squares tests: per degree block,
1e4 * eps_md * max(1, |x|)."""
import numpy as np
import pytest

from mdcheck import absdiff, lead
from phcpack_b200 import _lib, dense
from phcpack_b200 import workloads as wl

pytestmark = pytest.mark.gpu
EPS = {1: 1e-14, 2: 1e-28, 4: 1e-60}


def run(static, prec, cplx, ninst, n, degp1, szt, mat, rhs):
    import torch
    dev = "cuda"
    W = dense.width(prec, cplx)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    d_mat, d_rhs = t(mat), t(rhs)
    d_sol = torch.zeros(ninst * degp1 * n * W, dtype=torch.float64, device=dev)
    d_Q = torch.zeros(ninst * n * n * W, dtype=torch.float64, device=dev)
    d_R = torch.zeros(ninst * n * n * W, dtype=torch.float64, device=dev)
    d_fl = t(np.tile(np.array([1, 0, 0, 0, 1], np.int32), ninst))
    if static:
        _lib.call("phc_bals_solve_static", prec, int(cplx), ninst, n, degp1, szt, 1, _lib.ptr(d_mat),
                  _lib.ptr(d_rhs), _lib.ptr(d_sol), _lib.ptr(d_Q), _lib.ptr(d_R), _lib.ptr(d_fl), _lib.c_void_p(0))
    else:
        work = torch.zeros(ninst * dense.workspace_bytes(prec, cplx, n, szt) // 8, dtype=torch.float64, device=dev)
        _lib.call("phc_bals_solve", prec, int(cplx), ninst, n, degp1, szt, 1, _lib.ptr(d_mat), _lib.ptr(d_rhs),
                  _lib.ptr(d_sol), _lib.ptr(d_Q), _lib.ptr(d_R), _lib.ptr(d_fl), _lib.ptr(work), _lib.c_void_p(0))
    torch.cuda.synchronize()
    return d_sol.cpu().numpy(), d_fl.cpu().numpy()


def agree(a, b, prec, cplx, ninst, degp1, n):
    s = lead(b, prec, cplx).reshape(ninst * degp1, n).max(axis=1)
    e = absdiff(a, b, prec, cplx).reshape(ninst * degp1, n).max(axis=1)
    return bool((e <= 1e4 * EPS[prec] * np.maximum(s, 1.0)).all())


@pytest.mark.parametrize("shape", [(4, False, 3, 64, 8, 32), (2, True, 5, 16, 9, 8)])
def test_static_workspace_matches_allocating_entry_point_twice(shape):
    prec, cplx, ninst, n, degp1, szt = shape
    rng = np.random.default_rng(n * degp1)
    for call in range(2):  # two calls in a row share the static array
        mat = wl.random_numbers(rng, (ninst, degp1, n, n), prec, cplx, "normal")
        rhs = wl.random_numbers(rng, (ninst, degp1, n), prec, cplx, "normal")
        xs, fs = run(True, prec, cplx, ninst, n, degp1, szt, mat, rhs)
        xr, fr = run(False, prec, cplx, ninst, n, degp1, szt, mat, rhs)
        assert np.array_equal(fs, fr)
        assert agree(xs, xr, prec, cplx, ninst, degp1, n)


def test_static_workspace_two_shapes_back_to_back():
    """A quad-double real call, then a double-double complex call of another
    shape right after it, each against the allocating entry point."""
    rng = np.random.default_rng(77)
    for prec, cplx, ninst, n, degp1, szt in [(4, False, 3, 64, 8, 32), (2, True, 5, 16, 9, 8)]:
        mat = wl.random_numbers(rng, (ninst, degp1, n, n), prec, cplx, "normal")
        rhs = wl.random_numbers(rng, (ninst, degp1, n), prec, cplx, "normal")
        xs, fs = run(True, prec, cplx, ninst, n, degp1, szt, mat, rhs)
        xr, fr = run(False, prec, cplx, ninst, n, degp1, szt, mat, rhs)
        assert np.array_equal(fs, fr)
        assert agree(xs, xr, prec, cplx, ninst, degp1, n)


def test_static_workspace_rejects_requests_beyond_its_capacity():
    f = _lib.lib().phc_bals_solve_static_capacity_bytes
    f.restype = _lib.ctypes.c_longlong
    cap = int(f())
    per = dense.workspace_bytes(4, True, 64, 32)
    too_many = cap // per + 1
    with pytest.raises(_lib.PhcError) as e:
        _lib.call("phc_bals_solve_static", 4, 1, too_many, 64, 8, 32, 1, _lib.c_void_p(0), _lib.c_void_p(0),
                  _lib.c_void_p(0), _lib.c_void_p(0), _lib.c_void_p(0), _lib.c_void_p(0), _lib.c_void_p(0))
    assert e.value.rc == -3
