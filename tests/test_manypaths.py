"""The containers of the tracker's drop-in entry points (gpumanypaths_*):
what is stored is what is read back, and the argument checks come before
any device work (CPU only)."""
import numpy as np
import pytest

from phcpack_b200 import _lib, manypaths


def test_solutions_round_trip_in_all_limb_counts():
    rng = np.random.default_rng(3)
    for limbs in (1, 2, 4):
        x = rng.standard_normal((5, 3, 2, limbs))
        manypaths.set_solutions(x)
        assert manypaths.number_of_solutions() == 5
        got = manypaths.get_solutions(limbs)
        assert np.array_equal(got["x"], x)
        assert (got["status"] == 0).all() and (got["t"] == 0).all()
    manypaths.clear()
    assert manypaths.number_of_solutions() == 0


def test_system_checks():
    with pytest.raises(_lib.PhcError, match="neq"):
        _lib.call("phc_container_set_target", 0, 2, _lib.c_void_p(0), _lib.c_void_p(0), _lib.c_void_p(0))
    nt = np.array([1], np.int32)
    ex = np.array([-1, 0], np.int32)
    cf = np.array([1.0, 0.0])
    with pytest.raises(_lib.PhcError, match="negative exponent"):
        _lib.call("phc_container_set_target", 1, 2, _lib.ptr(nt), _lib.ptr(ex), _lib.ptr(cf))


def test_drop_in_refuses_cpu_mode_and_empty_containers():
    manypaths.clear()
    with pytest.raises(_lib.PhcError, match="containers"):
        manypaths.track(2, 0, 1.0, 0.0)
    with pytest.raises(_lib.PhcError, match="CPU only"):
        manypaths.track(1, 0, 1.0, 0.0)
    with pytest.raises(_lib.PhcError, match="mode 7"):
        manypaths.track(7, 0, 1.0, 0.0, prec=4)


def test_square_dimension_check():
    p = [[(((0, 2),), 1.0 + 0j), ((), -1.0 + 0j)], [(((1, 2),), 1.0 + 0j), ((), -2.0 + 0j)]]
    manypaths.set_system("target", p, 2)
    manypaths.set_system("start", p[:1], 2)
    manypaths.set_solutions(np.zeros((1, 2, 2, 1)))
    with pytest.raises(_lib.PhcError, match="square"):
        manypaths.track(2, 0, 1.0, 0.0)
    manypaths.clear()
