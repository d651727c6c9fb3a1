"""The FP64 network oracle's gradient formulas against central finite
differences (without the BF16 rounding, which has no derivative)."""
import numpy as np

from oracle import mlp_oracle
from phcpack_b200 import learn


def test_oracle_gradient_finite_differences():
    rng = np.random.default_rng(0)
    X = rng.standard_normal((20, 24))
    y = rng.standard_normal(20)
    P = learn.init_params(1).astype(np.float64)
    P[-1] = 0.2
    mean, inv_std = np.zeros(24), np.ones(24)
    G, _ = mlp_oracle.grad(P, mean, inv_std, X, y, rounding=False)
    h = 1e-6
    for i in rng.choice(P.size, 40, replace=False).tolist() + [P.size - 1]:
        Pp, Pm = P.copy(), P.copy()
        Pp[i] += h
        Pm[i] -= h
        lp = np.mean((mlp_oracle.forward(Pp.astype(np.float64), mean, inv_std, X, False)[0] - y) ** 2)
        lm = np.mean((mlp_oracle.forward(Pm.astype(np.float64), mean, inv_std, X, False)[0] - y) ** 2)
        assert abs((lp - lm) / (2 * h) - G[i]) <= 1e-6 + 1e-4 * abs(G[i])


def test_bf16_rounding_is_nearest_even():
    # bfloat16 keeps 7 fraction bits: the spacing next to 1 is 2^-7
    a = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -7 + 2 ** -10], np.float32)
    r = mlp_oracle.bf16(a)
    assert r[0] == 1.0
    assert r[1] == 1.0                 # tie: to the even neighbour below
    assert r[2] == 1.0 + 2 ** -6       # tie: to the even neighbour above
    assert r[3] == 1.0 + 2 ** -7       # below the tie: down
