"""Failures injected on the host (no GPU fault): inputs that make numerical
work fail come back as per-path or per-instance status codes, the other
items of the batch are unaffected, and nothing faults or hangs.

  * a homotopy with a NaN / an infinite coefficient: those paths fail;
  * a start point where the Jacobian is singular (a zero pivot of LU);
  * a least-squares instance whose A_0 has a zero column (beta = 0 for that
    Householder reflector) and one that is entirely zero;
  * the learned step with proposals scaled by 1e6: every proposal fails
    the feedback or the corrector and is redone with the plain step, so the
    classification is that of the plain step."""
import numpy as np
import pytest

from phcpack_b200 import dense
from phcpack_b200 import homotopy as hm
from phcpack_b200 import trackwork
from phcpack_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def small(n=3, npaths=8, seed=1):
    rng = np.random.default_rng(seed)
    pb = hm.total_degree_problem([hm.dense_quadratic(rng, n)], complex(hm.unit(rng)))
    return hm.subset(pb, np.arange(npaths))


def two_systems_one_poisoned(value):
    """Two copies of a small homotopy, the second with one coefficient set
    to value; returns (problem, paths of system 1)."""
    rng = np.random.default_rng(2)
    target = hm.dense_quadratic(rng, 3)
    gamma = complex(hm.unit(rng))
    pb = hm.total_degree_problem([target, target], gamma)
    e = int(pb.eq_off[1])  # first equation of the second system
    tr = int(pb.term_off[e]) + 1
    pb.term_b[2 * tr] = value
    return pb, np.flatnonzero(pb.path_sys == 1)


@pytest.mark.parametrize("value", [np.nan, np.inf])
def test_nonfinite_coefficient_fails_its_paths_only(value):
    pb, bad = two_systems_one_poisoned(value)
    r = hm.track_host(pb, pmode=1, rmode=2)
    good = np.setdiff1d(np.arange(pb.npaths), bad)
    assert (r.status[bad] != 0).all()
    assert (r.status[good] == 0).all() and (r.residual[good] <= 1e-24).all()
    # the same good paths tracked alone give the same end points
    alone = hm.track_host(hm.subset(pb, good), pmode=1, rmode=2)
    assert np.array_equal(alone.xend, r.xend.reshape(pb.npaths, -1)[good].reshape(-1))


def test_singular_start_jacobian_fails_that_path():
    """x = 0 for the start system x_i^2 - 1: J = diag(2 x_i) is singular
    (a zero pivot in the first column) and h(0, 0) != 0."""
    pb = small()
    x0 = pb.x0.reshape(pb.npaths, -1).copy()
    x0[3] = 0.0
    pb.x0 = np.ascontiguousarray(x0.reshape(-1))
    r = hm.track_host(pb, pmode=1, rmode=2)
    assert r.status[3] != 0
    others = np.delete(np.arange(pb.npaths), 3)
    assert (r.status[others] == 0).all()


def test_least_squares_zero_column_and_zero_block():
    """Instance 1 has a zero column in A_0 (its reflector has beta = 0),
    instance 2 an A_0 that is zero; instances 0 and 3 are regular and solved
    bit for bit as if alone."""
    prec, cplx, ninst, n, degp1, szt = 2, False, 4, 8, 4, 4
    rng = np.random.default_rng(5)
    W = dense.width(prec, cplx)
    mat = wl.random_numbers(rng, (ninst, degp1, n, n), prec, cplx, "normal").reshape(ninst, degp1, n, n, W)
    mat[1, 0, :, 2, :] = 0.0
    mat[2, 0] = 0.0
    mat = mat.reshape(-1)
    rhs = wl.random_numbers(rng, (ninst, degp1, n), prec, cplx, "normal")
    sol, _, _, _, flags = dense.bals_solve_host(prec, cplx, mat, rhs, ninst, n, degp1, szt)
    assert np.isfinite(sol.reshape(ninst, -1)[[0, 3]]).all()
    for k in (0, 3):
        m1 = mat.reshape(ninst, -1)[k]
        r1 = rhs.reshape(ninst, -1)[k]
        s1, _, _, _, f1 = dense.bals_solve_host(prec, cplx, m1, r1, 1, n, degp1, szt)
        assert np.array_equal(s1, sol.reshape(ninst, -1)[k]) and np.array_equal(f1, flags.reshape(ninst, 5)[k])
    # a zero column of A_0 leaves a zero on the diagonal of R (beta = 0 for
    # that reflector, as in the reference), and the inverted diagonal tile
    # of the back substitution is not finite: the solutions of instances 1
    # and 2 report it by their non-finite entries, as the reference's do
    for k in (1, 2):
        assert not np.isfinite(sol.reshape(ninst, -1)[k]).all()


def test_learned_proposals_all_rejected_fall_back_to_plain():
    model = trackwork.load_model_bytes()
    assert model is not None
    pb = hm.subset(hm.config4(), np.arange(0, 1024, 32))
    plain = hm.track_host(pb, pmode=1, rmode=2, step_mode=0)
    wild = hm.track_host(pb, pmode=1, rmode=2, step_mode=1, model=model, learn_scale=1e6)
    assert np.array_equal(plain.status, wild.status)
    assert (wild.status == 0).all() and (wild.residual <= 1e-24).all()
    # every proposal (at least maxsize > plain step) is rejected at least once
    assert (wild.rejected > 0).all()
