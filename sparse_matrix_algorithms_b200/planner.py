"""Window planning for batched spectrum slicing: the plain rule and the learned planner.

For every window [emin, emax] the slicing solver needs an eigenvalue-count estimate, a
subspace width m0 and a filter degree K.  Both planners start from the same inputs: the
KPM moments of the matrix (``kpm_moments``, computed once per matrix on the GPU) and the
window's bounds mapped to [-1, 1].

Plain rule (the fallback, and the arbiter of every learned plan):
    N  = KPM count of the window
    m0 = 1.5 N + 16, rounded up to a multiple of 8
    K  = ceil(4 pi d / (emax - emin)),  d = (smax - smin) / 2
(the step filter's Jackson transition width is about pi d / K; a quarter of the window
separates its edge from the first eigenvalue outside a 1.5 N-wide subspace).

Learned planner: a three-layer perceptron (258 -> 256 -> 256 -> 3, BF16 weights, FP32
arithmetic, trained on the GPU by the library's own kernels) maps [mu_0..mu_255, a, b]
to (log s_K, log s_m, log s_N), and the plan is K = s_K K_plain, m0 = s_m m0_plain,
N = s_N N_kpm.  Its training targets come from runs of the plain solver: each training
window is solved at a grid of (s_K, s_m) scales and the cheapest converged run (fewest
column-steps, iterations x m0 x (K + 1)) is the target.

:func:`solve_windows` runs the learned plan and re-solves, with the plain rule, every
window that did not converge or returned clearly fewer eigenvalues than the KPM count
predicts.
"""
from __future__ import annotations

import ctypes
import math
import os
from typing import Iterable, List, Optional, Sequence, Tuple

import numpy as np

from . import _lib as L
from .api import _op_of, kpm_moments, kpm_count, slice_spectrum

N_MOMENTS = 256
IN_DIM = N_MOMENTS + 2
HIDDEN = 256
OUT_DIM = 3
SCALE_GRID_K = (0.25, 0.35, 0.5, 0.7, 1.0)
SCALE_GRID_M = (1.0, 1.5, 2.2)
_CLIP = (math.log(0.2), math.log(3.0))
WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "planner_data", "planner_weights.npz")


# ---------------------------------------------------------------------- features and rules
def mapped(smin: float, smax: float, e: float) -> float:
    c, d = 0.5 * (smin + smax), 0.5 * (smax - smin)
    return (e - c) / d


def window_features(mu: np.ndarray, smin: float, smax: float, emin: float, emax: float) -> np.ndarray:
    """The planner's input row: 256 KPM moments and the window's mapped bounds (float32)."""
    f = np.zeros(IN_DIM, dtype=np.float32)
    m = np.asarray(mu, dtype=np.float64)[:N_MOMENTS]
    f[:m.size] = m
    f[N_MOMENTS] = mapped(smin, smax, emin)
    f[N_MOMENTS + 1] = mapped(smin, smax, emax)
    return f


def plain_rule(count: float, smin: float, smax: float, emin: float, emax: float) -> Tuple[int, int]:
    """(degree, m0) of the plain rule for a window holding about ``count`` eigenvalues."""
    d = 0.5 * (smax - smin)
    K = int(math.ceil(4.0 * math.pi * d / (emax - emin)))
    m0 = int(8 * math.ceil((1.5 * max(count, 1.0) + 16.0) / 8.0))
    return K, m0


def scaled(K: int, m0: int, sK: float, sm: float, n: int) -> Tuple[int, int]:
    return max(1, int(round(K * sK))), min(n // 8 * 8, int(8 * math.ceil(m0 * sm / 8.0)))


# ---------------------------------------------------------------------- the network
class WindowPlanner:
    """The learned planner's network on the GPU (``sma_mlp_*``)."""

    def __init__(self, seed: int = 0, ctx=None, in_dim: int = IN_DIM, hidden: int = HIDDEN,
                 out_dim: int = OUT_DIM):
        from .api import context

        self.ctx = ctx or context()
        self.in_dim, self.hidden, self.out_dim = in_dim, hidden, out_dim
        h = ctypes.c_void_p()
        L.check(L.load().sma_mlp_create(self.ctx.handle, in_dim, hidden, out_dim, int(seed),
                                        ctypes.byref(h)))
        self.handle = h
        cnt = ctypes.c_int64()
        L.check(L.load().sma_mlp_num_params(h, ctypes.byref(cnt)))
        self.num_params = cnt.value

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                L.load().sma_mlp_destroy(h)
            except Exception:
                pass
            self.handle = None

    @property
    def params(self) -> np.ndarray:
        p = np.empty(self.num_params, dtype=np.float32)
        L.check(L.load().sma_mlp_get_params(self.handle, p.ctypes.data))
        return p

    @params.setter
    def params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != self.num_params:
            raise ValueError(f"expected {self.num_params} parameters, got {p.size}")
        L.check(L.load().sma_mlp_set_params(self.handle, p.ctypes.data))

    def forward(self, X: np.ndarray) -> np.ndarray:
        X = np.ascontiguousarray(X, dtype=np.float32).reshape(-1, self.in_dim)
        Y = np.empty((X.shape[0], self.out_dim), dtype=np.float32)
        L.check(L.load().sma_mlp_forward(self.handle, X.ctypes.data, X.shape[0], Y.ctypes.data))
        return Y

    def grad(self, X, T, w=None):
        X = np.ascontiguousarray(X, dtype=np.float32).reshape(-1, self.in_dim)
        T = np.ascontiguousarray(T, dtype=np.float32).reshape(-1, self.out_dim)
        wp = None if w is None else np.ascontiguousarray(w, dtype=np.float32).reshape(T.shape)
        g = np.empty(self.num_params, dtype=np.float32)
        loss = ctypes.c_float()
        L.check(L.load().sma_mlp_grad(self.handle, X.ctypes.data, T.ctypes.data,
                                      None if wp is None else wp.ctypes.data, X.shape[0],
                                      ctypes.byref(loss), g.ctypes.data))
        return loss.value, g

    def train(self, X, T, w=None, steps: int = 2000, lr: float = 1e-3, minibatch: int = 64,
              seed: int = 0, weight_decay: float = 1e-4) -> np.ndarray:
        X = np.ascontiguousarray(X, dtype=np.float32).reshape(-1, self.in_dim)
        T = np.ascontiguousarray(T, dtype=np.float32).reshape(-1, self.out_dim)
        wp = None if w is None else np.ascontiguousarray(w, dtype=np.float32).reshape(T.shape)
        hist = np.empty(max(int(steps), 1), dtype=np.float32)
        L.check(L.load().sma_mlp_train(self.handle, X.ctypes.data, T.ctypes.data,
                                       None if wp is None else wp.ctypes.data, X.shape[0],
                                       int(steps), float(lr), int(minibatch), int(seed),
                                       float(weight_decay), hist.ctypes.data))
        return hist[:int(steps)]

    def save(self, path: str) -> None:
        np.savez_compressed(path, params=self.params, in_dim=self.in_dim, hidden=self.hidden,
                            out_dim=self.out_dim)

    @classmethod
    def load(cls, path: str = WEIGHTS, ctx=None) -> "WindowPlanner":
        z = np.load(path)
        net = cls(ctx=ctx, in_dim=int(z["in_dim"]), hidden=int(z["hidden"]), out_dim=int(z["out_dim"]))
        net.params = z["params"]
        return net


# ---------------------------------------------------------------------- planning and solving
def plan_windows(A, windows: Sequence[Tuple[float, float]], planner: Optional[WindowPlanner] = None,
                 mu: Optional[np.ndarray] = None, smin=None, smax=None):
    """Per window: (count estimate, degree, m0), by the learned planner when given, else
    by the plain rule.  Returns the three lists and the plain rule's (degree, m0)."""
    op = _op_of(A)
    if smin is None or smax is None:
        smin, smax = op.gershgorin_bounds()
    if mu is None:
        mu = kpm_moments(op, N_MOMENTS, 16, smin=smin, smax=smax)
    counts, plain = [], []
    for a, b in windows:
        N = kpm_count(mu, op.n, smin, smax, a, b)
        counts.append(N)
        plain.append(plain_rule(N, smin, smax, a, b))
    if planner is None:
        return counts, [k for k, _ in plain], [m for _, m in plain], plain
    X = np.stack([window_features(mu, smin, smax, a, b) for a, b in windows])
    Y = np.clip(planner.forward(X), *_CLIP)
    deg, m0, cnt = [], [], []
    for (K, m), N, y in zip(plain, counts, Y):
        k2, m2 = scaled(K, m, math.exp(y[0]), math.exp(y[1]), op.n)
        deg.append(k2)
        m0.append(m2)
        cnt.append(N * math.exp(y[2]))
    return cnt, deg, m0, plain


def window_cost(iterations, m0, degree) -> np.ndarray:
    """Column-steps of a window's solve: iterations x m0 x (K + 1)."""
    return np.asarray(iterations) * np.asarray(m0) * (np.asarray(degree) + 1)


def solve_windows(A, windows, planner: Optional[WindowPlanner] = None, *, smin=None, smax=None,
                  mu=None, maxiter: int = 10, precision: str = "fp64", tol: float = 1e-10,
                  seed: int = 1, report: Optional[dict] = None):
    """Batched slicing with a planned (degree, m0) per window.  With a planner, windows
    that did not converge, or returned fewer than 0.85 N - 3 eigenvalues of the KPM count
    N, are solved again with the plain rule.  Returns ``(lam, X, res, win)`` like
    :func:`slice_spectrum`; ``report`` receives the plans, per-window column-steps and the
    windows redone."""
    op = _op_of(A)
    if smin is None or smax is None:
        smin, smax = op.gershgorin_bounds()
    if mu is None:
        mu = kpm_moments(op, N_MOMENTS, 16, smin=smin, smax=smax)
    counts, deg, m0, plain = plan_windows(op, windows, planner, mu, smin, smax)
    st = {}
    lam, X, res, win = slice_spectrum(op, windows, deg, m0, smin=smin, smax=smax, maxiter=maxiter,
                                      precision=precision, tol=tol, seed=seed, stats=st)
    cost = window_cost(st["window_iterations"], m0, deg)
    kpm_n = [kpm_count(mu, op.n, smin, smax, a, b) for a, b in windows]
    redo = []
    if planner is not None:
        for w in range(len(windows)):
            got = int(np.sum(win == w))
            if not st["window_converged"][w] or got < 0.85 * kpm_n[w] - 3:
                redo.append(w)
    if redo:
        st2 = {}
        sub = [windows[w] for w in redo]
        l2, X2, r2, w2 = slice_spectrum(op, sub, [plain[w][0] for w in redo],
                                        [plain[w][1] for w in redo], smin=smin, smax=smax,
                                        maxiter=maxiter, precision=precision, tol=tol, seed=seed,
                                        stats=st2)
        cost2 = window_cost(st2["window_iterations"], [plain[w][1] for w in redo],
                            [plain[w][0] for w in redo])
        keep = ~np.isin(win, redo)
        parts = [(lam[keep], X[:, keep], res[keep], win[keep])]
        for j, w in enumerate(redo):
            s = w2 == j
            parts.append((l2[s], X2[:, s], r2[s], np.full(int(s.sum()), w)))
            cost[w] += cost2[j]
        order_w = np.concatenate([p[3] for p in parts])
        lam_c = np.concatenate([p[0] for p in parts])
        perm = np.lexsort((lam_c, order_w))
        lam = lam_c[perm]
        X = np.concatenate([p[1] for p in parts], axis=1)[:, perm]
        res = np.concatenate([p[2] for p in parts])[perm]
        win = order_w[perm]
    if report is not None:
        report.update(dict(degree=deg, m0=m0, count_estimate=counts, plain=plain, cost=cost,
                           redone=redo, kpm_count=kpm_n, iterations=st["window_iterations"]))
    return lam, X, res, win


# ---------------------------------------------------------------------- training data
def training_rows(A, windows, *, smin=None, smax=None, mu=None, maxiter: int = 10, seed: int = 1,
                  grid_k: Iterable[float] = SCALE_GRID_K, grid_m: Iterable[float] = SCALE_GRID_M):
    """Rows (features, targets, weights) from runs of the plain solver on ``A``: every
    window is solved once per (s_K, s_m) of the grid, all in ONE batched slicing call; the
    target is the cheapest converged scale pair, and log(found / KPM count) where the most
    generous run converged.  Windows with no converged run get zero weight."""
    op = _op_of(A)
    if smin is None or smax is None:
        smin, smax = op.gershgorin_bounds()
    if mu is None:
        mu = kpm_moments(op, N_MOMENTS, 16, smin=smin, smax=smax)
    grid = [(sk, sm) for sk in grid_k for sm in grid_m]
    wins, deg, m0, owner = [], [], [], []
    plans = []
    for wi, (a, b) in enumerate(windows):
        N = kpm_count(mu, op.n, smin, smax, a, b)
        K, m = plain_rule(N, smin, smax, a, b)
        plans.append((N, K, m))
        for sk, sm in grid:
            k2, m2 = scaled(K, m, sk, sm, op.n)
            wins.append((a, b))
            deg.append(k2)
            m0.append(m2)
            owner.append(wi)
    st = {}
    lam, X, res, win = slice_spectrum(op, wins, deg, m0, smin=smin, smax=smax, maxiter=maxiter,
                                      seed=seed, stats=st)
    nrm = max(abs(smin), abs(smax))
    cost = window_cost(st["window_iterations"], m0, deg)
    F, T, W = [], [], []
    for wi, (a, b) in enumerate(windows):
        N, K, m = plans[wi]
        idx = [j for j in range(len(wins)) if owner[j] == wi]
        found = [int(np.sum((win == j) & (res <= 1e-10 * nrm))) for j in idx]
        ref = max(found)  # the most eigenvalues any converged run found
        ok = [j for jj, j in enumerate(idx) if st["window_converged"][j] and found[jj] == ref and ref > 0]
        f = window_features(mu, smin, smax, a, b)
        if not ok:
            F.append(f); T.append(np.zeros(OUT_DIM, np.float32)); W.append(np.zeros(OUT_DIM, np.float32))
            continue
        best = min(ok, key=lambda j: cost[j])
        g = grid[idx.index(best)]
        F.append(f)
        T.append(np.array([math.log(g[0]), math.log(g[1]), math.log(max(ref, 1) / max(N, 1.0))],
                          np.float32))
        W.append(np.ones(OUT_DIM, np.float32))
    return np.stack(F), np.stack(T), np.stack(W)


# ---------------------------------------------------------------------- window placement
def energy_at_count(mu, n: int, smin: float, smax: float, start: float, count: float,
                    hi: Optional[float] = None) -> float:
    """The energy e > start with ``count`` KPM-estimated eigenvalues in [start, e]
    (bisection; the estimate is monotone up to KPM ripple)."""
    lo_e, hi_e = start, smax if hi is None else hi
    for _ in range(80):
        mid = 0.5 * (lo_e + hi_e)
        if kpm_count(mu, n, smin, smax, start, mid) < count:
            lo_e = mid
        else:
            hi_e = mid
    return 0.5 * (lo_e + hi_e)


def windows_by_count(mu, n: int, smin: float, smax: float, center: float,
                     counts: Sequence[float]) -> List[Tuple[float, float]]:
    """Contiguous windows whose KPM-estimated counts are ``counts``, the whole run
    centred on ``center``."""
    total = float(sum(counts))
    # start so that about half of the total lies below the centre
    lo_e, hi_e = smin, center
    for _ in range(80):
        mid = 0.5 * (lo_e + hi_e)
        if kpm_count(mu, n, smin, smax, mid, center) > 0.5 * total:
            lo_e = mid
        else:
            hi_e = mid
    e = 0.5 * (lo_e + hi_e)
    out = []
    for c in counts:
        e2 = energy_at_count(mu, n, smin, smax, e, c)
        out.append((e, e2))
        e = e2
    return out


# ---------------------------------------------------------------------- POLFED windows
# The same network shape plans a POLFED solve of one window: its outputs are log-scales of
# the POLFED plain rule's degree and basis size (mmax blocks of s) and the count correction.
# POLFED plain rule (Jackson-damped delta filter centred on the window):
#     N = KPM count,  K = ceil(12 d / (emax - emin)),  mmax = ceil(2.8 N / s)
# (the reference's default mmax, polfed.jl:1131, and the degree that converged every
# configuration of this library's POLFED sweeps).
POLFED_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "planner_data",
                              "polfed_planner_weights.npz")
POLFED_GRID_K = (0.25, 0.33, 0.45, 0.6, 0.8, 1.0)
POLFED_GRID_M = (1.0, 1.5, 2.0, 2.7)


def polfed_plain_rule(count: float, smin: float, smax: float, emin: float, emax: float,
                      s: int) -> Tuple[int, int]:
    """(degree, mmax) of the POLFED plain rule for a window of about ``count`` eigenvalues."""
    d = 0.5 * (smax - smin)
    K = int(math.ceil(12.0 * d / (emax - emin)))
    mmax = max(2, int(math.ceil(2.8 * max(count, 1.0) / s)))
    return K, mmax


def polfed_cost(K: int, mmax: int, s: int) -> int:
    """Column-steps of a POLFED filter phase: mmax blocks of s columns, K steps each."""
    return int(K) * int(mmax) * int(s)


def polfed_nev(count: float) -> int:
    """The nev passed to POLFED for a window of about ``count`` eigenvalues: an upper bound,
    since POLFED returns at most nev pairs (the basis size still follows ``count``)."""
    return int(math.ceil(1.2 * max(count, 1.0))) + 2


def _polfed_good(lam, res, emin, emax, nrm):
    return int(np.sum((lam >= emin) & (lam <= emax) & (res <= 1e-10 * nrm)))


def solve_polfed_window(A, window, planner: Optional[WindowPlanner] = None, *, s: int = 8,
                        smin=None, smax=None, mu=None, seed: int = 1,
                        report: Optional[dict] = None, stats: Optional[dict] = None,
                        precision: str = "fp64", vectors: bool = True):
    """POLFED on one window with a planned (nev, degree, mmax): the learned plan when a
    planner is given, else the plain rule.  A learned plan that returns fewer than
    0.85 N - 3 converged in-window pairs (N the KPM count) is redone with the plain rule.
    Returns ``(lam, X, res)``; ``report`` receives the plans, the column-steps spent and
    whether the window was redone; ``stats`` the solver statistics of the last POLFED run.
    ``precision`` is the filter arithmetic of both runs (``"mixed"``: FP32 basis, FP64
    polish); ``vectors=False`` keeps the eigenvectors on the device (X is None)."""
    from .api import polfed

    op = _op_of(A)
    if smin is None or smax is None:
        smin, smax = op.gershgorin_bounds()
    if mu is None:
        mu = kpm_moments(op, N_MOMENTS, 16, smin=smin, smax=smax)
    a, b = window
    nrm = max(abs(smin), abs(smax))
    N = kpm_count(mu, op.n, smin, smax, a, b)
    K0, m0 = polfed_plain_rule(N, smin, smax, a, b, s)
    nev0 = polfed_nev(N)
    plan = (nev0, K0, m0)
    if planner is not None:
        y = np.clip(planner.forward(window_features(mu, smin, smax, a, b)[None, :])[0], *_CLIP)
        plan = (max(nev0, polfed_nev(N * math.exp(y[2]))), max(1, int(round(K0 * math.exp(y[0])))),
                max(2, int(math.ceil(m0 * math.exp(y[1])))))

    def run(nev, K, mmax):
        return polfed(op, nev, K, s=s, smin=smin, smax=smax, sigma=0.5 * (a + b), emin=a,
                      emax=b, window_type="delta", mmax=mmax, seed=seed, stats=stats,
                      precision=precision, vectors=vectors)

    lam, X, res = run(*plan)
    cost = polfed_cost(plan[1], plan[2], s)
    redone = False
    if planner is not None and _polfed_good(lam, res, a, b, nrm) < 0.85 * N - 3:
        lam, X, res = run(nev0, K0, m0)
        cost += polfed_cost(K0, m0, s)
        redone = True
    if report is not None:
        report.update(dict(plan=plan, plain=(nev0, K0, m0), cost=cost, redone=redone,
                           kpm_count=N, good=_polfed_good(lam, res, a, b, nrm)))
    return lam, X, res


def plan_polfed_windows(A, windows, planner: Optional[WindowPlanner], *, s: int, smin: float,
                        smax: float, mu: np.ndarray):
    """Per window: the KPM count N, the plain rule's (nev, degree, mmax) and the plan --
    the network's when a planner is given, else the plain rule."""
    op = _op_of(A)
    counts, plain, plans = [], [], []
    feats = []
    for a, b in windows:
        N = kpm_count(mu, op.n, smin, smax, a, b)
        K0, m0 = polfed_plain_rule(N, smin, smax, a, b, s)
        counts.append(N)
        plain.append((polfed_nev(N), K0, m0))
        feats.append(window_features(mu, smin, smax, a, b))
    if planner is None:
        return counts, plain, list(plain)
    Y = np.clip(planner.forward(np.stack(feats)), *_CLIP)
    for (nev0, K0, m0), N, y in zip(plain, counts, Y):
        plans.append((max(nev0, polfed_nev(N * math.exp(y[2]))),
                      max(1, int(round(K0 * math.exp(y[0])))),
                      max(2, int(math.ceil(m0 * math.exp(y[1]))))))
    return counts, plain, plans


def solve_polfed_windows(A, windows, planner: Optional[WindowPlanner] = None, *, s: int = 8,
                         smin=None, smax=None, mu=None, seed: int = 1,
                         precision: str = "fp64", tol: float = 1e-10,
                         report: Optional[dict] = None, stats: Optional[dict] = None,
                         vectors: bool = True):
    """Batched POLFED over ``windows`` with a planned (nev, degree, mmax) per window (the
    learned plan when a planner is given, else the plain rule), all windows in one
    :func:`polfed_windows` call.  Every window whose learned plan returns fewer than
    0.85 N - 3 converged in-window pairs (N its KPM count) is solved again with the plain
    rule (the redone windows batched together).  ``tol`` is polfed's residual tolerance
    (its return rule, and where a MIXED polish may stop).  Returns ``(lam, X, res, win)``;
    ``report`` receives the plans, the plain rule, the column-steps spent and the windows
    redone."""
    from .api import polfed_windows

    op = _op_of(A)
    if smin is None or smax is None:
        smin, smax = op.gershgorin_bounds()
    if mu is None:
        mu = kpm_moments(op, N_MOMENTS, 16, smin=smin, smax=smax)
    windows = [tuple(map(float, w)) for w in windows]
    nrm = max(abs(smin), abs(smax))
    counts, plain, plans = plan_polfed_windows(op, windows, planner, s=s, smin=smin, smax=smax,
                                               mu=mu)

    def run(ws, pl, st):
        return polfed_windows(op, [windows[w] for w in ws], [p[0] for p in pl], [p[1] for p in pl],
                              [p[2] for p in pl], s=s, smin=smin, smax=smax, window_type="delta",
                              seed=seed, precision=precision, tol=tol, stats=st, vectors=vectors)

    ids = list(range(len(windows)))
    lam, X, res, win = run(ids, plans, stats)
    cost = [polfed_cost(p[1], p[2], s) for p in plans]
    redo = []
    if planner is not None:
        for w in ids:
            a, b = windows[w]
            sel = win == w
            if _polfed_good(lam[sel], res[sel], a, b, nrm) < 0.85 * counts[w] - 3:
                redo.append(w)
    if redo:
        st2 = {}
        l2, X2, r2, w2 = run(redo, [plain[w] for w in redo], st2)
        keep = ~np.isin(win, redo)
        parts_l, parts_r, parts_w = [lam[keep]], [res[keep]], [win[keep]]
        parts_x = [X[:, keep]] if X is not None else []
        for j, w in enumerate(redo):
            sel = w2 == j
            parts_l.append(l2[sel])
            parts_r.append(r2[sel])
            parts_w.append(np.full(int(sel.sum()), w))
            if X2 is not None:
                parts_x.append(X2[:, sel])
            cost[w] += polfed_cost(plain[w][1], plain[w][2], s)
        order_w = np.concatenate(parts_w)
        perm = np.argsort(order_w, kind="stable")
        lam = np.concatenate(parts_l)[perm]
        res = np.concatenate(parts_r)[perm]
        win = order_w[perm]
        X = np.concatenate(parts_x, axis=1)[:, perm] if parts_x else None
        if stats is not None:
            for key in ("filter_ms", "orth_ms", "rr_ms", "filter_bytes", "polish_ms",
                        "polish_bytes", "spmm_steps", "spmm_columns", "kernel_launches",
                        "polish_iterations"):
                if key in st2:
                    stats[key] = stats.get(key, 0) + st2[key]
    if report is not None:
        report.update(dict(plan=plans, plain=plain, cost=cost, redone=redo, kpm_count=counts,
                           good=[_polfed_good(lam[win == w], res[win == w], *windows[w], nrm)
                                 for w in ids]))
    return lam, X, res, win


def polfed_training_rows_batched(A, windows, *, s: int = 32, smin: float, smax: float,
                                 mu: np.ndarray, grid_k: Iterable[float] = POLFED_GRID_K,
                                 grid_m: Iterable[float] = POLFED_GRID_M, seed: int = 1):
    """Training rows from plain-solver POLFED runs (FP64, Jackson-damped delta filter) at a
    grid of (degree, mmax) scales of the plain rule: every (window, scale) pair is one
    window of ONE batched POLFED call (sma_polfed_batch_solve), so the matrix is read once
    per step for all of them.  The target is the cheapest run (column-steps) that found as
    many converged in-window pairs as the best run, and log(found / KPM count)."""
    from .api import polfed_windows

    op = _op_of(A)
    nrm = max(abs(smin), abs(smax))
    grid = [(sk, sm) for sk in grid_k for sm in grid_m]
    wins, nevs, degs, mms, meta = [], [], [], [], []
    for wi, (a, b) in enumerate(windows):
        N = kpm_count(mu, op.n, smin, smax, a, b)
        K0, m0 = polfed_plain_rule(N, smin, smax, a, b, s)
        for sk, sm in grid:
            wins.append((a, b))
            nevs.append(polfed_nev(N))
            degs.append(max(1, int(round(K0 * sk))))
            mms.append(max(2, int(math.ceil(m0 * sm))))
            meta.append((wi, sk, sm, N))
    lam, _, res, win = polfed_windows(op, wins, nevs, degs, mms, s=s, smin=smin, smax=smax,
                                      window_type="delta", seed=seed, vectors=False)
    F, T, W = [], [], []
    for wi, (a, b) in enumerate(windows):
        runs = []
        for j, (wj, sk, sm, N) in enumerate(meta):
            if wj != wi:
                continue
            sel = win == j
            runs.append((sk, sm, polfed_cost(degs[j], mms[j], s),
                         _polfed_good(lam[sel], res[sel], a, b, nrm), N))
        ref = max(r[3] for r in runs)
        f = window_features(mu, smin, smax, a, b)
        ok = [r for r in runs if r[3] == ref and ref > 0]
        if not ok:
            F.append(f); T.append(np.zeros(OUT_DIM, np.float32)); W.append(np.zeros(OUT_DIM, np.float32))
            continue
        best = min(ok, key=lambda r: r[2])
        F.append(f)
        T.append(np.array([math.log(best[0]), math.log(best[1]), math.log(ref / max(best[4], 1.0))],
                          np.float32))
        W.append(np.ones(OUT_DIM, np.float32))
    return np.stack(F), np.stack(T), np.stack(W)


def polfed_training_rows(A, windows, *, s: int = 8, smin=None, smax=None, mu=None,
                         grid_k: Iterable[float] = POLFED_GRID_K,
                         grid_m: Iterable[float] = POLFED_GRID_M):
    """Rows (features, targets, weights) from POLFED runs of the plain rule at a grid of
    (degree, mmax) scales per window: the target is the cheapest run (column-steps) that
    found as many converged in-window pairs as the best run, and log(found / KPM count)."""
    from .api import polfed

    op = _op_of(A)
    if smin is None or smax is None:
        smin, smax = op.gershgorin_bounds()
    if mu is None:
        mu = kpm_moments(op, N_MOMENTS, 16, smin=smin, smax=smax)
    nrm = max(abs(smin), abs(smax))
    F, T, W = [], [], []
    for a, b in windows:
        N = kpm_count(mu, op.n, smin, smax, a, b)
        K0, m0 = polfed_plain_rule(N, smin, smax, a, b, s)
        nev = polfed_nev(N)
        runs = []
        for sk in grid_k:
            for sm in grid_m:
                K, mm = max(1, int(round(K0 * sk))), max(2, int(math.ceil(m0 * sm)))
                lam, _, res = polfed(op, nev, K, s=s, smin=smin, smax=smax, sigma=0.5 * (a + b),
                                     emin=a, emax=b, window_type="delta", mmax=mm)
                runs.append((sk, sm, polfed_cost(K, mm, s), _polfed_good(lam, res, a, b, nrm)))
        ref = max(r[3] for r in runs)
        f = window_features(mu, smin, smax, a, b)
        ok = [r for r in runs if r[3] == ref and ref > 0]
        if not ok:
            F.append(f); T.append(np.zeros(OUT_DIM, np.float32)); W.append(np.zeros(OUT_DIM, np.float32))
            continue
        best = min(ok, key=lambda r: r[2])
        F.append(f)
        T.append(np.array([math.log(best[0]), math.log(best[1]), math.log(ref / max(N, 1.0))],
                          np.float32))
        W.append(np.ones(OUT_DIM, np.float32))
    return np.stack(F), np.stack(T), np.stack(W)
