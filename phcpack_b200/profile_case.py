"""Run one hot-path launch at a chosen size, for ncu captures.

    python -m phcpack_b200.profile_case eval --nsys 512
    python -m phcpack_b200.profile_case bals --ninst 64
    python -m phcpack_b200.profile_case track --paths 256 [--variant 2]
    python -m phcpack_b200.profile_case diag --paths 1024

Builds the seeded workload on the device, runs the kernel ``--warm`` times
untimed and then ``--reps`` more times, and exits (``diag``: the end-game
diagnostics in double-double at the start points of the dense quadratic
n=10 homotopy, with the time of the timed launches printed).  The sizes keep a
capture to a few GB on the device while the inputs still exceed the L2.
"""
from __future__ import annotations

import argparse
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["eval", "bals", "track", "diag"])
    ap.add_argument("--nsys", type=int, default=512)
    ap.add_argument("--ninst", type=int, default=64)
    ap.add_argument("--paths", type=int, default=256)
    ap.add_argument("--warm", type=int, default=1)
    ap.add_argument("--reps", type=int, default=1)
    ap.add_argument("--variant", type=int, default=2,
                    help="track: kernel variant of the split tracker (1 narrow, 2 wide, 0 the built-in rule)")
    a = ap.parse_args()
    import torch

    from phcpack_b200 import benchwork

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    if a.case == "eval":
        w = benchwork.EvalWork(torch, dev, 0, nsys=a.nsys)
    elif a.case == "bals":
        from phcpack_b200 import qrwork
        w = qrwork.QRWork(torch, dev, 0, ninst=a.ninst)
    elif a.case == "diag":
        return diag(torch, dev, a)
    else:
        from phcpack_b200 import autotune, trackwork
        autotune.set_knob(autotune.KNOB_TRACK_VARIANT, a.variant)
        w = trackwork.TrackWork(torch, dev, 0, npaths=a.paths, tune=False)
    s = torch.cuda.Stream(device=dev)
    for _ in range(a.warm + a.reps):
        w.step(s)
    torch.cuda.synchronize()
    print(f"{a.case}: ok")


def diag(torch, dev, a):
    import numpy as np

    from phcpack_b200 import endgame
    from phcpack_b200 import homotopy as hm
    pb = hm.config4()
    pb = hm.subset(pb, np.arange(min(a.paths, pb.npaths)))
    dt = hm.DeviceTracker(pb, device=dev)
    tpt = torch.zeros(pb.npaths, dtype=torch.float64, device=dev)
    s = torch.cuda.Stream(device=dev)
    out = None
    for _ in range(a.warm):
        out = endgame.series_diagnostics_device(dt, dt.arr["x0"], tpt, 1, 2, stream=s)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(a.reps):
        out = endgame.series_diagnostics_device(dt, dt.arr["x0"], tpt, 1, 2, stream=s)
    e1.record(s)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / max(1, a.reps)
    st = out[1].cpu().numpy()[1::2]
    print(f"diag: ok, {pb.npaths} points, {ms:.3f} ms per launch, {pb.npaths / ms * 1e3:.0f} points/s, "
          f"status counts {np.bincount(st, minlength=3).tolist()}")


if __name__ == "__main__":
    main()
