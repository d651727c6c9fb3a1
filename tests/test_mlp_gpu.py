"""The learned step proposer: BF16 inference and training kernels against
an FP64 oracle of the same network (weights rounded to BF16 as on the
device), and what the trained network gains in the tracker.

Tolerances: forward outputs and gradients within 1e-3 relative to the
largest magnitude (FP32 accumulation over at most 128 terms against FP64)."""
import numpy as np
import pytest

from oracle import mlp_oracle
from phcpack_b200 import _lib, learn
from phcpack_b200 import homotopy as hm

pytestmark = pytest.mark.gpu


def setup(seed=3, nb=300):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((nb, 24)).astype(np.float32) * 2 + 1
    y = np.tanh(X[:, 0] * 0.3 - X[:, 5] * 0.2).astype(np.float32)
    tr = learn.Trainer(X, y, seed=seed)
    P = learn.init_params(seed)
    P[128 * 24:128 * 24 + 128] = rng.standard_normal(128) * 0.1  # nonzero biases
    P[-1] = 0.3
    tr.P.copy_(__import__("torch").from_numpy(P).to(tr.dev))
    return tr, X, y, P


def test_forward_matches_fp64_oracle():
    tr, X, y, P = setup()
    tr.pack()
    out = tr.predict(X)
    ref, _ = mlp_oracle.forward(P, tr.mean.cpu().numpy(), tr.inv_std.cpu().numpy(), X)
    assert np.abs(out - ref).max() <= 1e-3 * max(1.0, np.abs(ref).max())


def test_gradient_matches_fp64_oracle():
    import torch
    tr, X, y, P = setup(nb=257)
    tr.pack()
    Xd, yd = tr.X.contiguous(), tr.y.contiguous()
    _lib.call("phc_mlp_grad", _lib.ptr(tr.model), X.shape[0], _lib.ptr(Xd), _lib.ptr(yd), _lib.ptr(tr.G),
              _lib.ptr(tr.loss), _lib.c_void_p(0))
    torch.cuda.synchronize()
    G = tr.G.cpu().numpy().astype(np.float64)
    Gr, loss = mlp_oracle.grad(P, tr.mean.cpu().numpy(), tr.inv_std.cpu().numpy(), X, y)
    assert np.abs(G - Gr).max() <= 1e-3 * np.abs(Gr).max()
    assert abs(float(tr.loss.item()) - loss) <= 1e-3 * loss


def test_training_reduces_loss():
    rng = np.random.default_rng(5)
    X = rng.standard_normal((4096, 24)).astype(np.float32)
    y = (0.5 * X[:, 1] - 0.25 * X[:, 7] + 0.1 * X[:, 2] * X[:, 3]).astype(np.float32)
    tr = learn.Trainer(X, y, seed=5)
    hist = tr.fit(epochs=15, batch=256, lr=2e-3)
    assert hist[-1] < 0.2 * hist[0]


def test_learned_step_gains_over_plain_with_same_classification():
    # train on tracker logs of other systems, track 128 paths of the
    # benchmark homotopy with and without the proposer
    X, yv, R = learn.collect([hm.config4(seed=100), hm.config4(seed=101)])
    assert X.shape[0] > 1000 and (yv > 0).mean() > 0.5  # larger steps pass the feedback
    tr = learn.Trainer(X, yv, seed=0)
    tr.fit(epochs=20)
    model = tr.model_array()
    pb = hm.subset(hm.config4(), np.arange(0, 1024, 8))
    plain = hm.track_host(pb, pmode=1, rmode=2, step_mode=0)
    lrn = hm.track_host(pb, pmode=1, rmode=2, step_mode=1, model=model)
    assert np.array_equal(plain.status == 0, lrn.status == 0)
    ok = lrn.status == 0
    assert (lrn.residual[ok] <= 1e-24).all()
    assert lrn.steps.mean() < 0.8 * plain.steps.mean()
