"""The learned step proposer: data from the plain tracker, training on the
GPU with the library's own BF16 kernels, and the model file.

Data: the tracker in logging mode records per accepted step the 24
features of the predictor's series, the accepted step, the plain pole step
and the largest probed multiple of the pole step (1.5, 2, 3, 4, 6 times, at
most maxsize) whose Pade prediction still passes the predictor feedback.
The target is log(largest passing step / pole step): the network learns how
much further than the conservative pole step the predictor can be trusted.
At run time the corrector judges every proposal; a rejected one is redone
with the plain step, so the learned step never changes which paths succeed.

    python -m phcpack_b200.learn --out step_mlp.npz
"""
from __future__ import annotations

import argparse
import os

import numpy as np

from . import _lib
from . import homotopy as hm

NPARAM = 128 * 24 + 128 + 128 * 128 + 128 + 128 + 1


def model_bytes():
    f = _lib.lib().phc_mlp_model_bytes
    f.restype = _lib.ctypes.c_longlong
    return int(f())


def collect(problems, device="cuda", cap_per_problem=200000):
    """Run the plain batched tracker with logging on each problem; returns
    (X [N,24] float32, y [N] float32, raw records [N,32])."""
    import torch
    recs = []
    for pb in problems:
        dt = hm.DeviceTracker(pb, device=device, log_cap=cap_per_problem)
        dt.run(pmode=1, rmode=2, step_mode=0)
        torch.cuda.synchronize()
        cnt = min(int(dt.log_count.item()), cap_per_problem)
        recs.append(dt.log[:cnt * 32].reshape(cnt, 32).cpu().numpy())
    R = np.concatenate(recs, axis=0)
    X = R[:, :24].astype(np.float32)
    y = np.log(np.maximum(R[:, 28], 1e-30) / np.maximum(R[:, 25], 1e-30)).astype(np.float32)
    y = np.clip(y, -3.0, 3.0)
    return X, y, R


def init_params(seed=0):
    """He-uniform initial weights, zero biases (FP32 master layout)."""
    rng = np.random.default_rng(seed)
    P = np.zeros(NPARAM, np.float32)
    o = 0
    W1 =rng.uniform(-1, 1, (128, 24)) * np.sqrt(6.0 / 24)
    W2 = rng.uniform(-1, 1, (128, 128)) * np.sqrt(6.0 / 128)
    W3 = rng.uniform(-1, 1, (128,)) * np.sqrt(6.0 / 128) * 0.1
    P[o:o + W1.size] = W1.reshape(-1)
    o += W1.size + 128
    P[o:o + W2.size] = W2.reshape(-1)
    o += W2.size + 128
    P[o:o + 128] = W3
    return P


class Trainer:
    """FP32 master parameters and Adam state on the device; every step packs
    the BF16 model the tracker uses and differentiates through it."""

    def __init__(self, X, y, seed=0, device="cuda"):
        import torch
        self.torch = torch
        self.dev = device
        mean = X.mean(axis=0).astype(np.float32)
        std = np.maximum(X.std(axis=0), 1e-3).astype(np.float32)
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)
        self.mean, self.inv_std = t(mean), t((1.0 / std).astype(np.float32))
        self.X, self.y = t(X.astype(np.float32)), t(y.astype(np.float32))
        self.P = t(init_params(seed))
        self.G = torch.zeros(NPARAM, dtype=torch.float32, device=device)
        self.m = torch.zeros_like(self.G)
        self.v = torch.zeros_like(self.G)
        self.loss = torch.zeros(1, dtype=torch.float32, device=device)
        self.model = torch.zeros(model_bytes(), dtype=torch.uint8, device=device)
        self.step_count = 0
        self.rng = np.random.default_rng(seed + 1)

    def pack(self):
        _lib.call("phc_mlp_pack", _lib.ptr(self.P), _lib.ptr(self.mean), _lib.ptr(self.inv_std),
                  _lib.ptr(self.model), _lib.c_void_p(0))

    def step(self, idx, lr=1e-3):
        torch = self.torch
        self.pack()
        Xb = self.X[idx].contiguous()
        yb = self.y[idx].contiguous()
        _lib.call("phc_mlp_grad", _lib.ptr(self.model), int(idx.numel()), _lib.ptr(Xb), _lib.ptr(yb),
                  _lib.ptr(self.G), _lib.ptr(self.loss), _lib.c_void_p(0))
        self.step_count += 1
        _lib.call("phc_mlp_adam", _lib.ptr(self.P), _lib.ptr(self.G), _lib.ptr(self.m), _lib.ptr(self.v),
                  _lib.ctypes.c_float(lr), _lib.ctypes.c_float(0.9), _lib.ctypes.c_float(0.999),
                  _lib.ctypes.c_float(1e-8), self.step_count, _lib.c_void_p(0))

    def fit(self, epochs=20, batch=1024, lr=1e-3):
        torch = self.torch
        n = self.X.shape[0]
        hist = []
        for ep in range(epochs):
            perm = torch.from_numpy(self.rng.permutation(n)).to(self.dev)
            self.loss.zero_()
            nb = 0
            for b0 in range(0, n, batch):
                self.step(perm[b0:b0 + batch], lr=lr)
                nb += 1
            hist.append(float(self.loss.item()) / max(1, nb))
        self.pack()
        return hist

    def predict(self, X):
        torch = self.torch
        Xd = torch.from_numpy(np.ascontiguousarray(X, dtype=np.float32)).to(self.dev)
        out = torch.zeros(X.shape[0], dtype=torch.float32, device=self.dev)
        _lib.call("phc_mlp_forward", _lib.ptr(self.model), int(X.shape[0]), _lib.ptr(Xd), _lib.ptr(out),
                  _lib.c_void_p(0))
        return out.cpu().numpy()

    def model_array(self):
        self.pack()
        self.torch.cuda.synchronize()
        return self.model.cpu().numpy()


def training_problems():
    """Tracker runs the data comes from: the dense quadratic n = 10 system
    with other seeds than the benchmark's (seeds 100..103) and a sample of
    the sparse mixed-size systems."""
    probs = [hm.config4(seed=100 + k) for k in range(4)]
    pb5 = hm.config5(seed=105)
    probs.append(hm.subset(pb5, np.arange(0, pb5.npaths, 4)))
    return probs


def train_default(seed=0, epochs=30, device="cuda"):
    X, y, R = collect(training_problems(), device=device)
    tr = Trainer(X, y, seed=seed, device=device)
    hist = tr.fit(epochs=epochs)
    return tr, X, y, hist


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default="step_mlp.npz")
    ap.add_argument("--epochs", type=int, default=30)
    a = ap.parse_args()
    tr, X, y, hist = train_default(epochs=a.epochs)
    os.makedirs(os.path.dirname(a.out) or ".", exist_ok=True)
    np.savez(a.out, model=tr.model_array(), loss=np.array(hist, np.float32), nsamples=X.shape[0],
             target_mean=float(y.mean()))
    print(f"samples {X.shape[0]}, target mean {y.mean():.3f}, loss first {hist[0]:.4f} last {hist[-1]:.4f}")


if __name__ == "__main__":
    main()
