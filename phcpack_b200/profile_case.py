"""Run one hot-path launch at a chosen size, for ncu captures.

    python -m phcpack_b200.profile_case eval --nsys 512
    python -m phcpack_b200.profile_case bals --ninst 64
    python -m phcpack_b200.profile_case track --paths 256

Builds the seeded workload on the device, runs the kernel ``--warm`` times
untimed and then ``--reps`` more times, and exits.  The sizes keep a
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
    ap.add_argument("case", choices=["eval", "bals", "track"])
    ap.add_argument("--nsys", type=int, default=512)
    ap.add_argument("--ninst", type=int, default=64)
    ap.add_argument("--paths", type=int, default=256)
    ap.add_argument("--warm", type=int, default=1)
    ap.add_argument("--reps", type=int, default=1)
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
    else:
        from phcpack_b200 import trackwork
        w = trackwork.TrackWork(torch, dev, 0, npaths=a.paths)
    s = torch.cuda.Stream(device=dev)
    for _ in range(a.warm + a.reps):
        w.step(s)
    torch.cuda.synchronize()
    print(f"{a.case}: ok")


if __name__ == "__main__":
    main()
