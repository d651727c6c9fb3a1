"""Autotuner of the library's launch shapes, run on the device.

Three choices are swept once per shape and cached for the process:

* the warps (polynomials) per CTA of ``phc_system_evaldiff`` (knob 0 of
  ``phc_tune_set``), over 1, 2, 4 and 8;
* the tile size ``szt`` of the blocked QR / least squares
  (``phc_bals_solve``), over the divisors of the dimension among
  8, 16, 32 and 64 (a call argument, returned to the caller), with the
  WY panels and the column panel of R in global or in shared memory
  (knob 3);
* the variant of the split tracker's kernel (knob 1), 1 the 64-register
  kernel at 8 paths per SM, 2 the 72-register kernel at 7 paths per SM,
  together with the paths tracked at once per SM (knob 2), 4 to 8.

Every candidate is timed with CUDA events on the caller's stream after one
untimed run; the fastest is kept (ties to the built-in rule's choice).  The
knobs change launch shapes only: results are the same for every choice
(the tests check this).
"""
from __future__ import annotations

import numpy as np

from . import _lib

KNOB_EVAL_WARPS = 0
KNOB_TRACK_VARIANT = 1
KNOB_TRACK_PER_SM = 2
KNOB_DENSE_STAGE = 3

_cache: dict = {}


def set_knob(knob: int, value: int) -> None:
    _lib.call("phc_tune_set", int(knob), int(value))


def get_knob(knob: int) -> int:
    return _lib.call("phc_tune_get", int(knob))


def _time(torch, stream, fn, reps: int = 3) -> float:
    """Median CUDA-event seconds of fn() on stream, after one untimed run."""
    fn()
    times = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1) / 1e3)
    return float(np.median(times))


def tune_eval_warps(torch, stream, args, dim: int, key=None, reps: int = 3) -> dict:
    """Sweep the warps per CTA of phc_system_evaldiff; args: the argument
    tuple of the call (device pointers, the stream last).  Sets knob 0 to the
    fastest and returns {"choice", "seconds": {warps: s}}."""
    key = ("eval", key if key is not None else dim)
    if key in _cache:
        set_knob(KNOB_EVAL_WARPS, _cache[key]["choice"])
        return _cache[key]
    cands = [w for w in (1, 2, 4, 8) if w <= max(1, dim)]
    secs = {}
    for w in cands:
        set_knob(KNOB_EVAL_WARPS, w)
        secs[w] = _time(torch, stream, lambda: _lib.call("phc_system_evaldiff", *args), reps)
    best = min(cands, key=lambda w: (secs[w], -w))
    set_knob(KNOB_EVAL_WARPS, best)
    _cache[key] = {"choice": best, "seconds": secs}
    return _cache[key]


def tune_bals_tile(torch, stream, prec, cplx, ninst, dim, degp1, mat, rhs0, sol, Q, R, flags, flag0, work,
                   wy: int = 0, reps: int = 3, cands=(8, 16, 32, 64), stages=(1, 2)) -> dict:
    """Sweep the tile size of phc_bals_solve_wy and the staging of its panels
    (knob 3: 1 global memory, 2 shared memory where they fit) on resident
    device buffers (rhs and flags are restored from rhs0 and flag0 before
    every run; work must hold the workspace of every tile).  Sets knob 3 and
    returns {"choice": tile, "stage", "seconds"}; the caller passes the tile
    as szt."""
    key = ("bals", prec, cplx, ninst, dim, degp1, wy, tuple(cands), tuple(stages))
    if key in _cache:
        set_knob(KNOB_DENSE_STAGE, _cache[key]["stage"])
        return _cache[key]
    tiles = [t for t in cands if dim % t == 0 and t <= dim]
    if not tiles:
        tiles = [dim]
    rhs = torch.empty_like(rhs0)

    def run(szt):
        with torch.cuda.stream(stream):
            rhs.copy_(rhs0)
            flags.copy_(flag0)
        _lib.call("phc_bals_solve_wy", prec, int(cplx), ninst, dim, degp1, szt, 1, _lib.ptr(mat), _lib.ptr(rhs),
                  _lib.ptr(sol), _lib.ptr(Q), _lib.ptr(R), _lib.ptr(flags), _lib.ptr(work), int(wy),
                  _lib.c_void_p(stream.cuda_stream))

    secs = {}
    for g in stages:
        set_knob(KNOB_DENSE_STAGE, g)
        for t in tiles:
            secs[(t, g)] = _time(torch, stream, lambda t=t: run(t), reps)
    best = min(secs, key=lambda tg: (secs[tg], tg[0], tg[1]))
    set_knob(KNOB_DENSE_STAGE, best[1])
    _cache[key] = {"choice": best[0], "stage": best[1], "seconds": {f"{t}/{g}": v for (t, g), v in secs.items()}}
    return _cache[key]


def tune_track_variant(torch, stream, tracker, reps: int = 2, per_sm=(4, 5, 6, 7, 8), **run_kw) -> dict:
    """Time the kernel variants of the split tracker and the paths per SM on
    a DeviceTracker's own batch (tracker.run(**run_kw)); set knobs 1 and 2
    to the fastest pair.  choice: the variant; per_sm: the paths per SM."""
    key = ("track", tracker.pb.npaths, tracker.pb.maxdim, tuple(per_sm), tuple(sorted(run_kw.items())))
    if key in _cache:
        set_knob(KNOB_TRACK_VARIANT, _cache[key]["choice"])
        set_knob(KNOB_TRACK_PER_SM, _cache[key]["per_sm"])
        return _cache[key]
    secs = {}
    for v in (1, 2):
        set_knob(KNOB_TRACK_VARIANT, v)
        for k in per_sm:
            set_knob(KNOB_TRACK_PER_SM, k)
            secs[(v, k)] = _time(torch, stream, lambda: tracker.run(stream=stream, **run_kw), reps)
    best = min(secs, key=lambda vk: (secs[vk], -vk[1]))
    set_knob(KNOB_TRACK_VARIANT, best[0])
    set_knob(KNOB_TRACK_PER_SM, best[1])
    _cache[key] = {"choice": best[0], "per_sm": best[1], "seconds": {f"{v}/{k}": t for (v, k), t in secs.items()}}
    return _cache[key]


def reset() -> None:
    """Back to the built-in rules; the cache is kept."""
    set_knob(KNOB_EVAL_WARPS, 0)
    set_knob(KNOB_TRACK_VARIANT, 0)
    set_knob(KNOB_TRACK_PER_SM, 0)
    set_knob(KNOB_DENSE_STAGE, 0)
