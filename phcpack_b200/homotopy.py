"""Homotopies and path tracking: host mirror of the tracker interface.

Builds total-degree homotopies h(x, t) = (1 - t) gamma q(x) + t p(x) with
the start system q_i = x_i^{d_i} - 1 and its roots-of-unity start solutions
(Ada Root_Counts/Product/total_degree_start_systems.adb:108-160; the
homotopy as in Path/Path_GPU/eval_coef.cu:27-28), flattens them into the
arrays of include/phc_b200.h phc_track, and runs the GPU tracker.  The
tracker's entry points mirror ``gpumanypaths_dd(mode, verbose, regamma,
imgamma)`` (Ada/PHCtoC/gpumanypaths_dd.h:27): systems and start solutions in,
end points and per-path success flags out.
"""
from __future__ import annotations

import itertools
from dataclasses import dataclass, field

import numpy as np

from . import _lib

# Defaults of the Ada series-Pade tracker (Curves/homotopy_continuation_
# parameters.adb:6-24), with the series degree and Pade degrees of the
# 1024-path benchmark workload: degree-8 series, [4/4] Pade, 3 corrector steps.
DEFAULT_IPAR = dict(deg=8, numdeg=4, dendeg=4, nit=4, corsteps=3, maxsteps=1000, refine_steps=4)
DEFAULT_DPAR = dict(pbeta=0.5, alpha=1e-3, maxsize=0.1, minsize=1e-6, tolres=1e-8, epsilon=1e-12,
                    restol=1e-24, learn_scale=1.0, cbeta=0.005)
# ints per path in the tracker's info output: status, steps, rejected steps,
# and the times the step was the pole step, the curvature step and maxsize
INFO_WORDS = 6
STATUS = {0: "success", 1: "step below minsize", 2: "maxsteps reached", 3: "residual above restol"}


def params(**kw):
    ip = dict(DEFAULT_IPAR)
    dp = dict(DEFAULT_DPAR)
    for k, v in kw.items():
        if k in ip:
            ip[k] = v
        elif k in dp:
            dp[k] = v
        else:
            raise KeyError(k)
    ipar = np.array([ip[k] for k in ("deg", "numdeg", "dendeg", "nit", "corsteps", "maxsteps", "refine_steps")],
                    np.int32)
    dpar = np.array([dp[k] for k in ("pbeta", "alpha", "maxsize", "minsize", "tolres", "epsilon", "restol",
                                     "learn_scale", "cbeta")], np.float64)
    return ipar, dpar


# A polynomial: list of (monomial, coefficient); a monomial is a tuple of
# (variable, exponent) pairs with distinct variables in increasing order.
def unit(rng, size=None):
    return np.exp(1j * rng.uniform(0.0, 2.0 * np.pi, size=size))


def dense_quadratic(rng, n):
    """All monomials of degree <= 2 in n variables, unit-circle coefficients."""
    mons = [()] + [((j, 1),) for j in range(n)]
    for j in range(n):
        for k in range(j, n):
            mons.append(((j, 2),) if j == k else ((j, 1), (k, 1)))
    return [[(m, complex(c)) for m, c in zip(mons, unit(rng, len(mons)))] for _ in range(n)]


def sparse_quadratic(rng, n, mmin=3, mmax=6):
    """Each polynomial: a uniform number in [mmin, mmax] of distinct random
    monomials of degree 1 or 2 (at least one of degree 2), unit-circle
    coefficients, plus a constant term."""
    polys = []
    for _ in range(n):
        m = int(rng.integers(mmin, mmax + 1))
        mons = set()
        while len(mons) < m:
            if rng.random() < 0.5 or len(mons) == m - 1 and not any(sum(e for _, e in x) == 2 for x in mons):
                j, k = sorted(rng.choice(n, 2, replace=True).tolist())
                mons.add(((j, 2),) if j == k else ((j, 1), (k, 1)))
            else:
                mons.add(((int(rng.integers(n)), 1),))
        mons = sorted(mons)
        coef = unit(rng, len(mons) + 1)
        polys.append([((), complex(coef[0]))] + [(mm, complex(c)) for mm, c in zip(mons, coef[1:])])
    return polys


def degree(poly):
    return max(sum(e for _, e in m) for m, _ in poly)


@dataclass
class TrackProblem:
    """Flat homotopies and start points, the arrays of phc_track."""
    nsys: int
    maxvar: int
    dim: np.ndarray
    mono_off: np.ndarray
    mono_nvr: np.ndarray
    mono_idx: np.ndarray
    mono_exp: np.ndarray
    eq_off: np.ndarray
    term_off: np.ndarray
    term_mono: np.ndarray
    term_a: np.ndarray
    term_b: np.ndarray
    path_sys: np.ndarray
    x0: np.ndarray
    note: str = ""
    extra: dict = field(default_factory=dict)

    @property
    def maxdim(self):
        return int(self.dim.max())

    @property
    def npaths(self):
        return int(self.path_sys.shape[0])

    @property
    def nmono_max(self):
        return int(np.diff(self.mono_off).max())


def homotopy_problem(pairs, gamma, starts, maxvar=None) -> TrackProblem:
    """Flatten homotopies h = (1 - t) gamma q + t p for a list of (p, q)
    pairs (target and start systems, polynomials as lists of (monomial,
    coefficient), a monomial a tuple of (variable, exponent)) with start
    points starts = [(system index, complex vector), ...].  maxvar: the most
    distinct variables in a monomial (None: from the systems)."""
    if maxvar is None:
        maxvar = max(1, max(len(m) for p, q in pairs for poly in list(p) + list(q) for m, _ in poly))
    dim, mono_off, nvr, idx, exps = [], [0], [], [], []
    eq_off, term_off, term_mono, ta, tb = [0], [0], [], [], []
    maxdim = max(len(p) for p, _ in pairs)
    for s, (polys, qpolys) in enumerate(pairs):
        n = len(polys)
        if len(qpolys) != n:
            raise ValueError(f"system {s}: {n} target and {len(qpolys)} start polynomials")
        # distinct monomials of the system: the constant, then target and
        # start monomials in order of appearance
        table = {}

        def mono_id(m):
            if m not in table:
                table[m] = len(table)
            return table[m]

        mono_id(())
        for p in list(polys) + list(qpolys):
            for m, _ in p:
                mono_id(m)
        base = mono_off[-1]
        for m, k in sorted(table.items(), key=lambda kv: kv[1]):
            if len(m) > maxvar:
                raise ValueError("monomial with more than maxvar variables")
            nvr.append(len(m))
            idx.append([v for v, _ in m] + [0] * (maxvar - len(m)))
            exps.append([e for _, e in m] + [0] * (maxvar - len(m)))
        mono_off.append(base + len(table))
        for i in range(n):
            cp, cq = {}, {}
            for m, c in polys[i]:
                cp[m] = cp.get(m, 0) + c
            for m, c in qpolys[i]:
                cq[m] = cq.get(m, 0) + c
            for m in sorted(set(cp) | set(cq), key=lambda mm: table[mm]):
                a = gamma * cq.get(m, 0.0)
                b = complex(cp.get(m, 0.0))
                term_mono.append(base + table[m])
                ta.append([a.real, a.imag])
                tb.append([b.real, b.imag])
            term_off.append(len(term_mono))
        eq_off.append(eq_off[-1] + n)
        dim.append(n)
    path_sys, x0 = [], []
    for s, pt in starts:
        v = np.zeros(maxdim, complex)
        v[:len(pt)] = pt
        path_sys.append(s)
        x0.append(np.stack([v.real, v.imag], axis=-1).reshape(-1))
    i32 = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.int32))
    f64 = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1))
    return TrackProblem(len(pairs), maxvar, i32(dim), i32(mono_off), i32(nvr), i32(idx).reshape(-1),
                        i32(exps).reshape(-1), i32(eq_off), i32(term_off), i32(term_mono), f64(ta), f64(tb),
                        i32(path_sys), f64(x0))


def total_degree_start(polys):
    """The total-degree start system q_i = x_i^{d_i} - 1 of a target system
    (Root_Counts/Product/total_degree_start_systems.adb:108-160) and its
    degrees."""
    degs = [degree(p) for p in polys]
    return [[(((i, d),), 1.0), ((), -1.0)] for i, d in enumerate(degs)], degs


def total_degree_solutions(degs, pick=None):
    """All products of roots of unity (the start solutions of
    x_i^{d_i} - 1), or those with the flat indices in pick (the index runs
    fastest over the first variable)."""
    roots = [np.exp(2j * np.pi * np.arange(d) / d) for d in degs]
    total = int(np.prod(degs))
    out = []
    for flat in (range(total) if pick is None else pick):
        rem = int(flat)
        pt = np.zeros(len(degs), complex)
        for i, d in enumerate(degs):
            pt[i] = roots[i][rem % d]
            rem //= d
        out.append(pt)
    return out


def total_degree_problem(targets, gamma, max_paths_per_system=None, rng=None, maxvar=2) -> TrackProblem:
    """Total-degree homotopies for a list of target systems.  Start
    solutions are all products of roots of unity; when a system has more
    than max_paths_per_system of them, a seeded uniform sample (without
    replacement, rng) of that many is kept."""
    pairs, starts = [], []
    for s, polys in enumerate(targets):
        q, degs = total_degree_start(polys)
        pairs.append((polys, q))
        total = int(np.prod(degs))
        pick = None
        if max_paths_per_system is not None and total > max_paths_per_system:
            pick = np.sort(rng.choice(total, size=max_paths_per_system, replace=False))
        starts.extend((s, pt) for pt in total_degree_solutions(degs, pick))
    return homotopy_problem(pairs, gamma, starts, maxvar=maxvar)


def config4(seed=4):
    """The 1024-path workload: one seeded dense quadratic system, n = 10,
    unit-circle coefficients, total-degree homotopy with random complex
    gamma."""
    rng = np.random.default_rng(seed)
    target = dense_quadratic(rng, 10)
    gamma = complex(unit(rng))
    pb = total_degree_problem([target], gamma)
    pb.note = f"dense quadratic n=10, seed {seed}, gamma {gamma:.6f}"
    return pb


def config5(seed=5, nsystems=64, max_total=16384):
    """The mixed-size workload: 64 sparse quadratic systems, n uniform in
    6..14, 3-6 monomials per polynomial plus a constant, unit-circle
    coefficients, total-degree homotopies.  Paths are capped at
    max_total // nsystems per system by a seeded uniform sample (the
    Bezout numbers 2^n exceed 16384 in total)."""
    rng = np.random.default_rng(seed)
    targets = [sparse_quadratic(rng, int(rng.integers(6, 15))) for _ in range(nsystems)]
    gamma = complex(unit(rng))
    pb = total_degree_problem(targets, gamma, max_paths_per_system=max_total // nsystems, rng=rng)
    pb.note = f"{nsystems} sparse quadratic systems, n in 6..14, seed {seed}, cap {max_total // nsystems}/system"
    return pb


def subset(pb: TrackProblem, paths) -> TrackProblem:
    """The same homotopies with a subset of the paths."""
    paths = np.asarray(paths)
    md = pb.maxdim
    x0 = pb.x0.reshape(-1, md * 2)[paths].reshape(-1)
    return TrackProblem(pb.nsys, pb.maxvar, pb.dim, pb.mono_off, pb.mono_nvr, pb.mono_idx, pb.mono_exp, pb.eq_off,
                        pb.term_off, pb.term_mono, pb.term_a, pb.term_b,
                        np.ascontiguousarray(pb.path_sys[paths]), np.ascontiguousarray(x0), pb.note)


@dataclass
class TrackResult:
    xend: np.ndarray    # npaths x maxdim x 2 x limbs (complex quad-double limbs; octo-double for rmode 8)
    status: np.ndarray
    steps: np.ndarray
    rejected: np.ndarray
    t: np.ndarray
    residual: np.ndarray
    limbs: int = 4
    nbpole: np.ndarray = None   # steps set by the pole step,
    nbhess: np.ndarray = None   # by the curvature step,
    nbmaxm: np.ndarray = None   # by maxsize

    def endpoints(self, maxdim):
        """complex128 end points (leading limbs)"""
        a = self.xend.reshape(-1, maxdim, 2 * self.limbs)
        L = self.limbs
        return (a[..., 0] + a[..., 1]) + 1j * (a[..., L] + a[..., L + 1])


def xend_limbs(rmode):
    """Limbs per part of an end point coordinate in xend."""
    return 8 if rmode == 8 else 4


def _result(xend, info, dinfo, limbs=4):
    info = info.reshape(-1, INFO_WORDS)
    dinfo = dinfo.reshape(-1, 2)
    return TrackResult(xend, info[:, 0].copy(), info[:, 1].copy(), info[:, 2].copy(), dinfo[:, 0].copy(),
                       dinfo[:, 1].copy(), limbs, info[:, 3].copy(), info[:, 4].copy(), info[:, 5].copy())


def track_host(pb: TrackProblem, pmode=1, rmode=2, step_mode=0, model=None, stream_ptr=0, **kw) -> TrackResult:
    """Track every path of pb on the GPU (host arrays in and out), the shape
    of gpumanypaths_dd: start solutions in, end points and per-path status
    out.  stream_ptr: a cudaStream_t as an int (0 = default stream)."""
    ipar, dpar = params(**kw)
    xend = np.zeros(pb.npaths * pb.maxdim * 2 * xend_limbs(rmode))
    info = np.zeros(pb.npaths * INFO_WORDS, np.int32)
    dinfo = np.zeros(pb.npaths * 2)
    m = np.ascontiguousarray(model) if model is not None else None
    _lib.call("phc_track_host", pb.nsys, _lib.ptr(pb.dim), pb.maxvar, _lib.ptr(pb.mono_off), _lib.ptr(pb.mono_nvr),
              _lib.ptr(pb.mono_idx), _lib.ptr(pb.mono_exp), _lib.ptr(pb.eq_off), _lib.ptr(pb.term_off),
              _lib.ptr(pb.term_mono), _lib.ptr(pb.term_a), _lib.ptr(pb.term_b), pb.npaths, _lib.ptr(pb.path_sys),
              _lib.ptr(pb.x0), _lib.ptr(ipar), _lib.ptr(dpar), pmode, rmode, step_mode, _lib.ptr(m),
              _lib.ptr(xend), _lib.ptr(info), _lib.ptr(dinfo), _lib.c_void_p(stream_ptr))
    return _result(xend, info, dinfo, xend_limbs(rmode))


def gather_lists(pb: TrackProblem):
    lib = _lib.lib()
    f = lib.phc_track_gather_count
    f.restype = _lib.ctypes.c_longlong
    njg = int(f(pb.nsys, _lib.ptr(pb.mono_off), _lib.ptr(pb.mono_nvr), _lib.ptr(pb.eq_off), _lib.ptr(pb.term_off),
                _lib.ptr(pb.term_mono)))
    neq = int(pb.eq_off[-1])
    jg_off = np.zeros(neq * pb.maxdim + 1, np.int32)
    jg_term = np.zeros(max(1, njg), np.int32)
    jg_slot = np.zeros(max(1, njg), np.int32)
    staged = _lib.call("phc_track_prepare", pb.nsys, _lib.ptr(pb.dim), pb.maxvar, _lib.ptr(pb.mono_off),
                       _lib.ptr(pb.mono_nvr), _lib.ptr(pb.mono_idx), _lib.ptr(pb.mono_exp), _lib.ptr(pb.eq_off),
                       _lib.ptr(pb.term_off), _lib.ptr(pb.term_mono), pb.maxdim, _lib.ptr(jg_off), _lib.ptr(jg_term),
                       _lib.ptr(jg_slot))
    return jg_off, jg_term, jg_slot, staged


class DeviceTracker:
    """A TrackProblem resident on the device (torch CUDA tensors as plain
    device buffers) for repeated batched runs."""

    def __init__(self, pb: TrackProblem, device="cuda", log_cap=0):
        import torch
        self.pb = pb
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)
        jg = gather_lists(pb)
        self.arr = {k: t(getattr(pb, k)) for k in ("dim", "mono_off", "mono_nvr", "mono_idx", "mono_exp", "eq_off",
                                                    "term_off", "term_mono", "term_a", "term_b", "path_sys", "x0")}
        self.arr["jg_off"], self.arr["jg_term"], self.arr["jg_slot"] = (t(a) for a in jg[:3])
        self.gstaged = int(jg[3])
        self.xend = torch.zeros(pb.npaths * pb.maxdim * 16, dtype=torch.float64, device=device)  # room for rmode 8
        self.rmode = 2
        self.info = torch.zeros(pb.npaths * INFO_WORDS, dtype=torch.int32, device=device)
        self.dinfo = torch.zeros(pb.npaths * 2, dtype=torch.float64, device=device)
        self.queue = torch.zeros(1, dtype=torch.int32, device=device)
        self.log_cap = log_cap
        self.log = torch.zeros(max(1, log_cap) * 32, dtype=torch.float32, device=device) if log_cap else None
        self.log_count = torch.zeros(1, dtype=torch.int32, device=device)
        self.model = None

    def set_model(self, model_bytes_array):
        import torch
        self.model = torch.from_numpy(np.ascontiguousarray(model_bytes_array)).to(self.xend.device)

    def run(self, pmode=1, rmode=2, step_mode=0, one_per_launch=False, stream=None, **kw):
        pb = self.pb
        ipar, dpar = params(**kw)
        a = self.arr
        s = 0 if stream is None else stream.cuda_stream
        if self.log is not None:
            self.log_count.zero_()
        self.rmode = rmode
        _lib.call("phc_track", pb.nsys, _lib.ptr(a["dim"]), pb.maxvar, pb.maxdim, pb.nmono_max, _lib.ptr(a["mono_off"]),
                  _lib.ptr(a["mono_nvr"]), _lib.ptr(a["mono_idx"]), _lib.ptr(a["mono_exp"]), _lib.ptr(a["eq_off"]),
                  _lib.ptr(a["term_off"]), _lib.ptr(a["term_mono"]), _lib.ptr(a["term_a"]), _lib.ptr(a["term_b"]),
                  _lib.ptr(a["jg_off"]), _lib.ptr(a["jg_term"]), _lib.ptr(a["jg_slot"]), self.gstaged, pb.npaths,
                  _lib.ptr(a["path_sys"]), _lib.ptr(a["x0"]), _lib.ptr(ipar), _lib.ptr(dpar), pmode, rmode, step_mode,
                  _lib.ptr(self.model) if ((step_mode & 1) and self.model is not None) else _lib.c_void_p(0),
                  _lib.ptr(self.xend), _lib.ptr(self.info), _lib.ptr(self.dinfo),
                  _lib.ptr(self.log) if self.log is not None else _lib.c_void_p(0), self.log_cap,
                  _lib.ptr(self.log_count), _lib.ptr(self.queue), int(one_per_launch), _lib.c_void_p(s))
        return pb.npaths if one_per_launch else 1

    def result(self) -> TrackResult:
        L = xend_limbs(self.rmode)
        xe = self.xend[:self.pb.npaths * self.pb.maxdim * 2 * L].cpu().numpy()
        return _result(xe, self.info.cpu().numpy(), self.dinfo.cpu().numpy(), L)
