"""CUDA-graph-captured Newton solves (newton.DeviceNewton): the steps of a
solve at fixed working degree, captured once and replayed, give bit for bit
the series and skip-rule flags of the same steps run through
phc_newton_host (schedule 0), on the known-answer problem in real
double-double (n = 8, degree 15, tile 8, the plain workload's shapes) and in
complex quad-double; a second replay repeats the first."""
import numpy as np
import pytest

from newton_problems import exponential_test_system
from phcpack_b200 import newton

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec,cplx,szt", [(2, False, 8), (4, True, 4)])
def test_graph_replay_equals_host_loop(prec, cplx, szt):
    import torch
    b, _ = exponential_test_system(5, 3, 8, 15, 8, 3, prec, cplx)
    ser_h, fl_h = newton.newton_host(b, 4, szt=szt, schedule=0)
    dn = newton.DeviceNewton(b, szt=szt)
    s = torch.cuda.Stream()
    dn.capture(4, s)
    for _ in range(2):
        dn.replay(s)
        ser_g, fl_g = dn.result()
        assert np.array_equal(ser_g, ser_h.reshape(ser_g.shape))
        assert np.array_equal(fl_g, fl_h.reshape(fl_g.shape))


def test_launched_solve_equals_host_loop():
    import torch
    b, _ = exponential_test_system(6, 2, 8, 15, 8, 3, 2, False)
    ser_h, fl_h = newton.newton_host(b, 3, szt=8, schedule=0)
    dn = newton.DeviceNewton(b, szt=8)
    s = torch.cuda.Stream()
    dn.solve(3, s)
    ser_d, fl_d = dn.result()
    assert np.array_equal(ser_d, ser_h.reshape(ser_d.shape))
    assert np.array_equal(fl_d, fl_h.reshape(fl_d.shape))
