"""Loading of the golden fixtures (tests only)."""
from __future__ import annotations

import glob
import os

import numpy as np

from phcpack_b200.workloads import SystemBatch

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def names(prefix):
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, prefix + "*.npz")))


def batch(d) -> SystemBatch:
    return SystemBatch(int(d["nsys"]), int(d["dim"]), int(d["deg"]), int(d["maxvar"]), int(d["prec"]),
                       bool(d["cplx"]), d["mon_off"], d["nvr"], d["idx"], d["exps"], d["cst"], d["cff"], d["input"])
