"""Benchmark: eigenpairs/s of POLFED on one B200 -- the untuned pipeline against the plain
FP64 GPU path -- plus the SpMM GB/s of the fused Clenshaw step.

Default workload (one "step" = one full solve of the window) -- the C3 configuration: the
3D Anderson model L=64 (n=262144, 7 nnz/row, periodic), W=16.5, seed 2; the 500-eigenvalue
window centred at E=0 placed by KPM (256 moments, 32 vectors, seed 11) and fixed (it holds
exactly 494 eigenvalues by Sylvester inertia, tests/golden/anderson_L64_inertia.json);
block size s=64.  ``--workload c2``: the random-field XXZ chain L=18 (n=48620), h=5, seed
1; the 200 eigenvalues nearest the spectral centre (exact, from the dense spectrum); s=32.

Arms, all POLFED through the library, the same window:
  pipeline  (value) nothing tuned for the workload: 100 GPU Lanczos steps for the spectral
            bounds, 256 KPM moments, then the GPU-trained planner's (nev, degree, mmax)
            for the window, the plain rule as fallback and judge -- all inside the timed
            step -- in the arithmetic given by --precision (default: mixed, an FP32 filter
            basis with FP64 orthogonalization, Rayleigh-Ritz, residuals and polish).
  plain     the plain FP64 GPU path: Gershgorin bounds, Jackson-damped delta window,
            degree 12 d / (emax - emin) (C3) or the smallest converging degree of a sweep
            (C2), mmax = ceil(2.8 nev / s) (polfed.jl:1132).
  tuned     FP64 with the (window, damping, degree, mmax) that a sweep ON THIS MATRIX found
            fastest -- reported for reference, not the value.

value      eigenpairs inside the window with relative residual ||Ax-lam x||/||A|| <= 1e-10,
           per second of device time (CUDA events on the library's stream); the matrix is
           resident in HBM, eigenvectors stay on the device; L2 flushed (256 MiB write)
           before every solve.  `steps` solves timed after `warmup` untimed ones; the plain
           and tuned arms run --arm-steps timed solves after one warm-up each.
e2e        the pipeline through the public API with host buffers: CSR upload, bounds, KPM,
           plan, solve and eigenvector download inside the timed region (host clock,
           device synchronized).
roofline   the fused Clenshaw-SpMM step of the pipeline's basis filter (one block shape,
           b = s): algorithmic bytes of all its launches (nnz (s_v + 4) + 4 (n+1) + 4 n b s_x
           per step) over the device time of the basis-filter phase, against the measured
           HBM copy bandwidth.  The MIXED polish (ragged per-column widths, residual forms,
           its own orthonormalization) is timed apart as polish_ms.
cpu_baseline  the plain arm's POLFED configuration run by the CPU restatement of the
           reference (oracle/, FP64, OpenMP over the block's columns, all host threads) on a
           bounded sample: every block column, a truncated recurrence (its time scaled by
           degree / steps run), one mid-run reorthogonalization + QR (times mmax), and the
           extraction (timed, matrix products scaled by the rows run).
With --gpus N under torchrun every rank runs an independent replica (the path has no data
exchange); value is the sum over ranks, timed as the max over ranks.
--impl reference prints the same CPU-restatement measurement as its own line.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "eigenpairs/s at residual<=1e-10: chosen vs plain FP64 on one B200; SpMM GB/s"
LANCZOS_STEPS = 100
# the C3 window: 500 eigenvalues by the KPM estimate (256 moments, 32 Rademacher vectors,
# seed 11, Gershgorin bounds) centred at E=0, fixed here
C3_WINDOW = (-0.016975627263859053, 0.016979915488252416)


def host_gershgorin(A):
    """Gershgorin interval of a sparse symmetric matrix, on the host (the plain degree must
    not depend on a GPU, since the CPU reference arm builds the same workload)."""
    import scipy.sparse as sp

    A = sp.csr_matrix(A)
    d = A.diagonal()
    r = np.asarray(abs(A).sum(axis=1)).ravel() - np.abs(d)
    return float(np.min(d - r)), float(np.max(d + r))


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


class Workload:
    """Matrix, window, POLFED sizes and the plain and tuned configurations of one
    benchmark workload."""

    def __init__(self, name):
        from sparse_matrix_algorithms_b200 import matrices as M

        self.name = name
        if name == "c2":
            self.A = M.config_matrix("xxz_L18")
            g = np.load(os.path.join(ROOT, "tests", "golden", "xxz_L18_spectrum.npz"))
            lam_min, lam_max = float(g["lam_min"]), float(g["lam_max"])
            central = g["central"]
            centre = 0.5 * (lam_min + lam_max)
            self.nev, self.s, self.mmax = 200, 32, 24
            order = np.argsort(np.abs(central - centre), kind="stable")[:self.nev]
            lo, hi = int(order.min()), int(order.max())
            self.emin = 0.5 * (central[lo - 1] + central[lo])
            self.emax = 0.5 * (central[hi] + central[hi + 1])
            self.exact = central[lo:hi + 1]
            self.exact_count = hi - lo + 1
            self.norm = max(abs(lam_min), abs(lam_max))
            self.norm_kind = "dense FP64 spectrum"
            # the smallest degree of the sweep {600..2200} x mmax {14, 18, 24} with which
            # every pair reaches residual <= 1e-10 ||A|| (the reference's rule: raise the
            # degree until converged, chebyshev_subspace_iteration.jl:1051)
            self.window_plain = "delta"
            self.degree_plain = 2200
            # Lanczos bounds, no Jackson damping; the sweep (degree, mmax) in
            # {700..1781} x {24..44}: the fewest filter steps with which all 200 converge
            self.tuned = dict(degree=700, mmax=44, jackson=False, window="delta")
            self.cpu_steps = 300
            self.text = ("C2 POLFED: XXZ L=18 Sz=0 periodic (n=48620), J=Delta=1, h~U[-5,5] "
                         "seed 1; 200 eigenvalues nearest the spectral centre; s=32")
        elif name == "c3":
            self.A = M.config_matrix("anderson_L64")
            self.nev, self.s, self.mmax = 500, 64, 22
            self.emin, self.emax = C3_WINDOW
            # exact count by Sylvester inertia at the two window ends
            # (tests/golden/make_inertia_counts.py -> anderson_L64_inertia.json)
            below = json.load(open(os.path.join(ROOT, "tests", "golden", "anderson_L64_inertia.json")))
            self.exact = None
            self.exact_count = below[repr(self.emax)] - below[repr(self.emin)]
            self.norm = None  # from the Lanczos bounds at set-up
            self.norm_kind = "Lanczos estimate"
            gl, gh = host_gershgorin(self.A)
            self.window_plain = "delta"
            self.degree_plain = int(12 * 0.5 * (gh - gl) / (self.emax - self.emin))
            # Lanczos bounds, no Jackson damping; sweep of (window, degree, mmax) over
            # delta/step x {1200..3857} x {22..50}: the fewest filter steps converging all
            # 494 pairs (step window 1200/44; the best delta point was 1600/44)
            self.tuned = dict(degree=1200, mmax=44, jackson=False, window="step")
            self.cpu_steps = 40
            self.text = ("C3 POLFED: 3D Anderson L=64 (n=262144), W=16.5, seed 2, periodic; "
                         "500 eigenvalues (KPM-placed window centred at E=0, 494 by inertia); s=64")
        else:
            raise ValueError(name)
        self.sigma = 0.5 * (self.emin + self.emax)

    def kwargs(self, smin, smax):
        return dict(s=self.s, smin=smin, smax=smax, sigma=self.sigma, emin=self.emin,
                    emax=self.emax, tol=1e-10, window_type=self.window_plain, mmax=self.mmax)

    def good_pairs(self, lam, res):
        inside = (lam >= self.emin) & (lam <= self.emax)
        return int(np.count_nonzero(inside & (res <= 1e-10 * self.norm)))

    def config(self, precision):
        return {"workload": self.text, "window": [self.emin, self.emax],
                "exact_count_in_window": self.exact_count, "norm": self.norm_kind,
                "pipeline": {"bounds": f"Lanczos ({LANCZOS_STEPS} steps)", "kpm": "256 moments, 16 vectors",
                             "plan": "GPU-trained POLFED planner, plain-rule fallback",
                             "precision": precision, "inside_timed_step": True},
                "plain": {"bounds": "Gershgorin", "window": self.window_plain, "jackson": True,
                          "degree": self.degree_plain, "mmax": self.mmax, "precision": "fp64"},
                "tuned": {"bounds": f"Lanczos ({LANCZOS_STEPS} steps)", **self.tuned,
                          "precision": "fp64"},
                "l2": "flushed before every solve (256 MiB write)", "parallelism": "replicas"}


# ---------------------------------------------------------------------- the arms
def arm_plain(wl, op, stats=None, vectors=False):
    """The plain FP64 GPU path: Gershgorin bounds, plain degree and mmax."""
    import sparse_matrix_algorithms_b200 as S

    gl, gh = op.gershgorin_bounds()
    if stats is not None:
        stats["plan"] = [wl.nev, wl.degree_plain, wl.mmax]
    return S.polfed(op, wl.nev, wl.degree_plain, stats=stats, vectors=vectors, **wl.kwargs(gl, gh))


def arm_tuned(wl, op, stats=None, vectors=False):
    """FP64 with the sweep-tuned configuration of this workload (Lanczos bounds inside)."""
    import sparse_matrix_algorithms_b200 as S

    lo, hi = S.lanczos_bounds(op, steps=LANCZOS_STEPS)
    kw = wl.kwargs(lo, hi)
    kw.update(mmax=wl.tuned["mmax"], jackson=wl.tuned["jackson"], window_type=wl.tuned["window"])
    if stats is not None:
        stats["plan"] = [wl.nev, wl.tuned["degree"], wl.tuned["mmax"]]
    return S.polfed(op, wl.nev, wl.tuned["degree"], stats=stats, vectors=vectors, **kw)


def arm_pipeline(wl, op, net, precision="mixed", stats=None, report=None, vectors=False):
    """The untuned pipeline: Lanczos bounds, KPM moments, the learned plan with the plain
    rule as fallback, batched POLFED (here over the workload's one window) in the given
    filter arithmetic."""
    import sparse_matrix_algorithms_b200 as S
    from sparse_matrix_algorithms_b200 import planner as P

    lo, hi = S.lanczos_bounds(op, steps=LANCZOS_STEPS)
    mu = S.kpm_moments(op, P.N_MOMENTS, 16, smin=lo, smax=hi)
    rep = {}
    # the acceptance criterion is relative: ||Ax - lam x|| <= 1e-10 ||A||, ||A|| from the bounds
    tol = 1e-10 * max(abs(lo), abs(hi))
    lam, X, res, _ = P.solve_polfed_windows(op, [(wl.emin, wl.emax)], net, s=wl.s, smin=lo,
                                            smax=hi, mu=mu, tol=tol, report=rep, stats=stats,
                                            precision=precision, vectors=vectors)
    if stats is not None:
        stats["plan"] = list(rep["plan"][0])
        stats["plain_rule"] = list(rep["plain"][0])
        stats["redone"] = bool(rep["redone"])
    if report is not None:
        report.update(rep)
    return lam, X, res


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    def __init__(self, device: int):
        self.proc = None
        self.device = device
        self.path = os.path.join(tempfile.gettempdir(), f"sma_bench_clocks_{os.getpid()}_{device}.csv")

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=index,clocks.sm,clocks.max.sm,"
                 "power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.3)
            self.proc.terminate()
            self.proc.wait()
            self.f.close()

    def summary(self):
        if self.proc is None:
            return None
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9 and parts[1].replace(".", "").isdigit():
                rows.append(parts)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]),
                "samples": len(rows), "reasons": reasons}


def measured_hbm_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        return float(json.load(open(path))["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------------- CPU baseline
def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import sma_oracle as O

    return O


_CPU_INPUTS = {}


def _cpu_inputs(wl: Workload):
    """The operands the CPU sample times its work on, made once per workload and reused by
    every sample (only the timed operations are repeated).  Their values do not change the
    work of any timed operation, so all but the start block are plain normal draws: an
    orthonormal mid-run basis or a true projected matrix would cost minutes to make and
    time the same."""
    if wl.name in _CPU_INPUTS:
        return _CPU_INPUTS[wl.name]
    O = _oracle()
    A = wl.A
    n, s, mmax = A.shape[0], wl.s, wl.mmax
    smin, smax = O.gershgorin_bounds(A)
    D = min(wl.cpu_steps, wl.degree_plain)
    rng = np.random.default_rng(0)
    inp = {
        "smin": smin, "smax": smax, "D": D,
        "coeffs": O.build_coeffs(D, smin, smax, wl.sigma, wl.emin, wl.emax, wl.window_plain, True),
        "Q": O.orth_block(rng.standard_normal((n, s))),
        "V": rng.standard_normal((n, s * mmax // 2)),
    }
    Mdim = s * mmax
    T = rng.standard_normal((Mdim, Mdim))
    inp["T"] = T + T.T
    inp["m"] = min(Mdim, max(2 * wl.nev, wl.nev + 8))
    inp["rows"] = max(1, n // 16)
    inp["Vs"] = np.ascontiguousarray(rng.standard_normal((inp["rows"], Mdim)))
    inp["mc"] = max(1, inp["m"] // 8)
    inp["Xs"] = np.asfortranarray(rng.standard_normal((n, inp["mc"])))
    _CPU_INPUTS[wl.name] = inp
    return inp


def cpu_plain_estimate(wl: Workload, threads: int) -> dict:
    """Seconds of one plain-arm POLFED solve by the CPU restatement (oracle, FP64), from a
    bounded sample on ``threads`` host threads:

    * filter: every one of the block's s columns through a recurrence truncated to
      ``wl.cpu_steps`` sparse products, timed and scaled by degree / cpu_steps (every step
      of the recurrence is the same work), times mmax blocks;
    * block dense work: the reorthogonalization of a block against a mid-run basis of
      mmax s / 2 columns and its rank-revealing QR, timed, times mmax;
    * extraction: eigen of the (mmax s)^2 projected matrix, timed in full; the Ritz-vector
      lift V U and the Rayleigh quotients (one sparse product) over the 2 nev candidates,
      timed on n / 16 rows and m / 8 columns and scaled; the refinement counted as a
      second Rayleigh pass.
    """
    O = _oracle()
    A = wl.A
    n, mmax = A.shape[0], wl.mmax
    inp = _cpu_inputs(wl)
    t0 = time.perf_counter()
    O.apply_poly_block(A, inp["Q"], inp["coeffs"], inp["smin"], inp["smax"], impl="c",
                       nthreads=threads)
    t_filter = (time.perf_counter() - t0) * wl.degree_plain / inp["D"]
    V = inp["V"]
    W = inp["Q"].copy()
    t1 = time.perf_counter()
    W -= V @ (V.T @ W)
    O.block_qr_factor(W)
    t_block = time.perf_counter() - t1
    t2 = time.perf_counter()
    _, U = np.linalg.eigh(inp["T"])
    t_eig = time.perf_counter() - t2
    t3 = time.perf_counter()
    inp["Vs"] @ U[:, :inp["m"]]
    t_lift = (time.perf_counter() - t3) * n / inp["rows"]
    t4 = time.perf_counter()
    O.rayleigh(A, inp["Xs"])
    t_ray = (time.perf_counter() - t4) * inp["m"] / inp["mc"]
    total = mmax * (t_filter + t_block) + t_eig + t_lift + 2 * t_ray
    return {"seconds": total, "filter_s": mmax * t_filter, "block_dense_s": mmax * t_block,
            "extract_s": t_eig + t_lift + 2 * t_ray}


def cpu_text(wl: Workload) -> str:
    return (f"the plain arm's configuration (Gershgorin bounds, Jackson-damped {wl.window_plain} "
            f"window, degree {wl.degree_plain}, mmax {wl.mmax}, s {wl.s}) in the CPU restatement "
            f"(oracle/, FP64): all {wl.s} block columns through {min(wl.cpu_steps, wl.degree_plain)} "
            f"recurrence steps, scaled to the degree, x {wl.mmax} blocks; one mid-run "
            f"reorthogonalization + QR x {wl.mmax}; extraction timed (products scaled from "
            f"row / column slices); credited with the exact count {wl.exact_count} in the window")


def cpu_full_solve(wl: Workload, threads: int) -> dict:
    """One complete plain-arm POLFED solve by the CPU restatement: wall time and the pairs
    it found inside the window at relative residual <= 1e-10 (the check of the sampled
    estimate; minutes of host time for C2)."""
    O = _oracle()
    smin, smax = O.gershgorin_bounds(wl.A)
    os.environ["OMP_NUM_THREADS"] = str(threads)
    t0 = time.perf_counter()
    lam, X, res = O.polfed(wl.A, wl.nev, wl.degree_plain, **wl.kwargs(smin, smax))
    dt = time.perf_counter() - t0
    norm = wl.norm if wl.norm is not None else max(abs(smin), abs(smax))
    good = int(np.sum((lam >= wl.emin) & (lam <= wl.emax) & (res <= 1e-10 * norm)))
    return {"seconds": dt, "pairs": good, "threads": threads}


def reduce_over_ranks(c_ms, p_ms, c_pairs, p_pairs, device=None):
    """Replicas: the job's time is the slowest rank's, its pairs the sum over ranks.  Every
    rank calls this, in the same order (two all-reduces)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([c_ms, p_ms, c_pairs, p_pairs], dtype=torch.float64, device=device)
    tmax = t.clone()
    dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(tmax[0]), float(tmax[1]), int(t[2]), int(t[3])


def run_reference(args, rank, world):
    if rank != 0:
        return
    wl = Workload(args.workload)
    threads = host_threads()
    if args.cpu_full_solve:
        est = cpu_plain_estimate(wl, threads)
        full = cpu_full_solve(wl, threads)
        print(json.dumps({"cpu_full_solve": wl.name, **full, "sampled_estimate_s": est["seconds"],
                          "estimate_over_full": est["seconds"] / full["seconds"]}), flush=True)
        return
    for _ in range(args.warmup):
        cpu_plain_estimate(wl, threads)
    t = [cpu_plain_estimate(wl, threads)["seconds"] for _ in range(args.steps)]
    t_solve = sum(t) / len(t)
    value = wl.exact_count / t_solve
    line = {
        "metric": METRIC, "impl": "reference", "value": value, "unit": "eigenpairs/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * t_solve, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": wl.config(args.precision),
        "cpu_baseline": {"value": value, "unit": "eigenpairs/s", "cores": threads, "kind": "port",
                         "sample": "per step, one estimated solve: " + cpu_text(wl)},
        "e2e": {"value": value, "unit": "eigenpairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, rank, world, device):
    import torch

    import sparse_matrix_algorithms_b200 as S
    from sparse_matrix_algorithms_b200 import _lib as L
    from sparse_matrix_algorithms_b200 import planner as P

    wl = Workload(args.workload)
    A = wl.A
    ctx = S.context(device)
    op = S.SparseOperator(A, ctx)
    if wl.norm is None:
        lo, hi = S.lanczos_bounds(op, steps=LANCZOS_STEPS)
        wl.norm = max(abs(lo), abs(hi))
    stream = torch.cuda.ExternalStream(ctx.stream, device=device)
    flush = torch.empty(256 * 2 ** 20 // 4, dtype=torch.float32, device=device)
    lib = L.load()
    net = P.WindowPlanner.load(P.POLFED_WEIGHTS)

    def pipeline(st):
        return arm_pipeline(wl, op, net, args.precision, stats=st)

    def plain(st):
        return arm_plain(wl, op, stats=st)

    def tuned(st):
        return arm_tuned(wl, op, stats=st)

    step_ms = {}
    plans = {}

    def timed(name, fn, steps):
        pairs, ms, launches = 0, [], 0
        agg = {"filter_bytes": 0.0, "filter_ms": 0.0, "orth_ms": 0.0, "rr_ms": 0.0,
               "polish_ms": 0.0}
        for _ in range(steps):
            flush.zero_()
            torch.cuda.synchronize(device)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            l0 = lib.sma_kernel_launch_count()
            e0.record(stream)
            st = {}
            lam, _, res = fn(st)
            e1.record(stream)
            e1.synchronize()
            launches += lib.sma_kernel_launch_count() - l0
            ms.append(e0.elapsed_time(e1))
            pairs += wl.good_pairs(lam, res)
            for k in agg:
                agg[k] += st.get(k, 0.0)
            plans[name] = {k: st[k] for k in ("plan", "plain_rule", "redone", "polish_iterations",
                                              "fp32_filter_calls", "basis_dim") if k in st}
        step_ms[name] = [round(m, 1) for m in ms]
        return pairs, sum(ms), agg, launches

    arm_steps = max(1, min(args.arm_steps, args.steps))
    # the clock sampler starts before the warm-up: starting nvidia-smi stalls the GPU's
    # work for about a second, which must not fall into a timed solve
    with ClockSampler(device) as clk:
        for _ in range(args.warmup):
            pipeline({})
        plain({})
        tuned({})
        torch.cuda.synchronize(device)
        if world > 1:
            torch.distributed.barrier()
        v_pairs, v_ms, v_agg, v_launch = timed("pipeline", pipeline, args.steps)
        torch.cuda.synchronize(device)
        p_pairs, p_ms, p_agg, _ = timed("plain", plain, arm_steps)
        t_pairs, t_ms, _, _ = timed("tuned", tuned, arm_steps)
    if world > 1:
        v_ms, p_ms, v_pairs, p_pairs = reduce_over_ranks(v_ms, p_ms, v_pairs, p_pairs, device)
        t_ms, _, t_pairs, _ = reduce_over_ranks(t_ms, 0.0, t_pairs, 0, device)
    value = v_pairs / (v_ms / 1e3)
    plain_value = p_pairs / (p_ms / 1e3)
    tuned_value = t_pairs / (t_ms / 1e3)

    # end to end through the public API with host buffers: upload, bounds, KPM, plan,
    # solve, eigenvector download
    e2e_ms, e2e_pairs = [], 0
    h2d = 8 * (A.shape[0] + 1) + 16 * A.nnz
    d2h = 0
    e2e_steps = max(1, min(args.steps, 2))
    for _ in range(e2e_steps):
        flush.zero_()
        torch.cuda.synchronize(device)
        t0 = time.perf_counter()
        hop = S.SparseOperator(A, ctx)
        lam, X, res = arm_pipeline(wl, hop, net, args.precision, vectors=True)
        e2e_ms.append(1e3 * (time.perf_counter() - t0))
        e2e_pairs += wl.good_pairs(lam, res)
        d2h = 8 * (X.size + lam.size + res.size)
        hop.close()
    e2e = {"value": e2e_pairs / (sum(e2e_ms) / 1e3), "unit": "eigenpairs/s",
           "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
           "timing": "host wall clock around the API calls, device synchronized"}

    if rank != 0:
        return
    peak, peak_kind = measured_hbm_peak()
    achieved = v_agg["filter_bytes"] / (v_agg["filter_ms"] / 1e3) / 1e9
    cpu = None
    if world == 1 and not args.no_cpu:
        threads = host_threads()
        est = cpu_plain_estimate(wl, threads)
        cpu_value = min(wl.exact_count, p_pairs / arm_steps) / est["seconds"]
        cpu = {"value": cpu_value, "unit": "eigenpairs/s", "cores": threads, "kind": "port",
               "sample": cpu_text(wl), "seconds_per_solve": est["seconds"],
               "gpu_plain_over_cpu_plain": plain_value / cpu_value,
               "value_over_cpu_plain": value / cpu_value}
    dtype = {"fp64": "f64", "fp32": "f32", "mixed": "f32 filter + f64 orth/RR/residual/polish"}
    line = {
        "metric": METRIC, "value": value, "unit": "eigenpairs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": v_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": dtype[args.precision], "data": "synthetic", "config": wl.config(args.precision),
        "pairs_per_step": v_pairs / args.steps / world,
        "pipeline_over_plain": value / plain_value if plain_value > 0 else None,
        "plain_fp64": {"value": plain_value, "unit": "eigenpairs/s", "ms_per_step": p_ms / arm_steps,
                       "pairs_per_step": p_pairs / arm_steps / world,
                       "spmm_gbs": p_agg["filter_bytes"] / (p_agg["filter_ms"] / 1e3) / 1e9},
        "tuned_fp64": {"value": tuned_value, "unit": "eigenpairs/s", "ms_per_step": t_ms / arm_steps,
                       "pairs_per_step": t_pairs / arm_steps / world,
                       "over_plain": tuned_value / plain_value if plain_value > 0 else None},
        "plans": plans,
        "phase_ms_per_step": {k: v_agg[k] / args.steps
                              for k in ("filter_ms", "orth_ms", "rr_ms", "polish_ms")},
        "step_ms": step_ms,
        "spmm_gbs": achieved,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": TRAFFIC.get((wl.name, args.precision)),
                     "kernel": "fused CSR Clenshaw step (SpMM + recurrence axpy), the basis filter's launches",
                     "peak_kind": f"{peak_kind} HBM copy bandwidth",
                     "note": ("working set (~56 MB) is L2-resident at this size"
                              if wl.name == "c2" else "blocks of 67-134 MB per step exceed L2")},
        "e2e": e2e,
        "gpu_launches": v_launch,
        "clocks": clk.summary(),
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


# dram__bytes_read.sum + dram__bytes_write.sum of one fused Clenshaw step of the arm's
# dominant block shape, per launch (ncu of `bench.py --profile-filter ...`); None when no
# capture of that shape exists
TRAFFIC = {
    ("c2", "fp64"): 43_698_688 + 242_944,
    ("c3", "fp64"): 429_926_656 + 117_963_264,
    # the MIXED pipeline's basis filter: the FP32 b=64 step (profiles/clenshaw_step_anderson_L64_b64_fp32.md)
    ("c3", "mixed"): 219_189_760 + 50_311_424,
    ("c3", "fp32"): 219_189_760 + 50_311_424,
}


def multi_workload(name):
    """C4 / C5: the matrix and its windows, placed from KPM moments (256 moments, 32
    Rademacher vectors, seed 11) on 100-step Lanczos bounds, computed at set-up.

    C4  XXZ L=20 Sz=0 (n=184756), h=3, seed 3: 16 contiguous windows centred at E=0 whose
        KPM counts are uneven, 50..400 (seeded); the 16 windows the configuration names as
        tiling [-2, 2] would each hold thousands of eigenvalues ([-2, 2] holds ~6e4), so the
        counts are kept and the windows placed contiguously around E=0 instead.
    C5  3D Anderson L=96 (n=884736), W=12, seed 4: one window of 1000 KPM-estimated
        eigenvalues centred at E=0."""
    import sparse_matrix_algorithms_b200 as S
    from sparse_matrix_algorithms_b200 import matrices as M
    from sparse_matrix_algorithms_b200 import planner as P

    if name == "c4":
        A = M.config_matrix("xxz_L20")
        counts = [float(np.round(50 + 350 * x)) for x in M.splitmix_uniform(3, 16)]
        s = 32
        text = ("C4 batched POLFED: XXZ L=20 Sz=0 (n=184756), h~U[-3,3] seed 3; 16 contiguous "
                "KPM-placed windows around E=0 with uneven counts 50..400; s=32")
    elif name == "c5":
        A = M.config_matrix("anderson_L96")
        counts = [1000.0]
        s = 64
        text = ("C5 POLFED: 3D Anderson L=96 (n=884736), W=12, seed 4; 1000 KPM-placed "
                "eigenvalues centred at E=0; s=64")
    else:
        raise ValueError(name)
    op = S.SparseOperator(A)
    lo, hi = S.lanczos_bounds(op, steps=LANCZOS_STEPS)
    mu = S.kpm_moments(op, P.N_MOMENTS, 32, smin=lo, smax=hi, seed=11)
    wins = P.windows_by_count(mu, A.shape[0], lo, hi, 0.0, counts)
    return A, op, wins, counts, s, (lo, hi), text


def run_multi(args):
    """C4 or C5 (one solve per arm, builder measurements): the pipeline -- Lanczos bounds,
    KPM moments, the learned plan per window, batched MIXED POLFED over all windows, the
    plain rule as fallback -- against the plain FP64 GPU path, one polfed call per window
    (Gershgorin bounds, Jackson-damped delta window, degree 12 d / width, mmax 2.8 N / s).
    Pairs count inside their windows at relative residual <= 1e-10; the two arms'
    eigenvalues are compared window by window."""
    import torch

    import sparse_matrix_algorithms_b200 as S
    from sparse_matrix_algorithms_b200 import planner as P

    torch.cuda.set_device(0)
    A, op, wins, counts, s, (lo, hi), text = multi_workload(args.workload)
    net = P.WindowPlanner.load(P.POLFED_WEIGHTS)
    stream = torch.cuda.ExternalStream(S.context(0).stream, device=0)
    norm = max(abs(lo), abs(hi))
    out = {"workload": text, "windows": wins, "kpm_counts": counts}

    def good(lam, res, win):
        return [int(np.sum((lam[win == w] >= a) & (lam[win == w] <= b) & (res[win == w] <= 1e-10 * norm)))
                for w, (a, b) in enumerate(wins)]

    def timed(fn):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = fn()
        e1.record(stream)
        e1.synchronize()
        return r, e0.elapsed_time(e1) / 1e3

    def pipeline():
        l2, h2 = S.lanczos_bounds(op, steps=LANCZOS_STEPS)
        mu = S.kpm_moments(op, P.N_MOMENTS, 16, smin=l2, smax=h2)
        rep, st = {}, {}
        r = P.solve_polfed_windows(op, wins, net, s=s, smin=l2, smax=h2, mu=mu,
                                   precision=args.precision, tol=1e-10 * max(abs(l2), abs(h2)),
                                   report=rep, stats=st, vectors=False)
        return r, rep, st

    ((lam, _, res, win), rep, st), t_pipe = timed(pipeline)
    g_pipe = good(lam, res, win)
    out["pipeline"] = {"seconds": t_pipe, "pairs": int(sum(g_pipe)), "per_window": g_pipe,
                       "eigenpairs_per_s": sum(g_pipe) / t_pipe, "plans": rep["plan"],
                       "plain_rule": rep["plain"], "redone": rep["redone"],
                       "filter_ms": st.get("filter_ms"), "orth_ms": st.get("orth_ms"),
                       "rr_ms": st.get("rr_ms"), "polish_ms": st.get("polish_ms"),
                       "polish_passes": st.get("polish_iterations"),
                       "spmm_gbs": st["filter_bytes"] / st["filter_ms"] / 1e6 if st.get("filter_ms") else None}
    print(json.dumps(out), flush=True)
    if args.no_plain:
        return
    gl, gh = op.gershgorin_bounds()
    mu_g = S.kpm_moments(op, P.N_MOMENTS, 16, smin=gl, smax=gh)

    def plain():
        res_all = []
        for (a, b) in wins:
            N = S.kpm_count(mu_g, op.n, gl, gh, a, b)
            K, mm = P.polfed_plain_rule(N, gl, gh, a, b, s)
            res_all.append(S.polfed(op, P.polfed_nev(N), K, s=s, smin=gl, smax=gh, sigma=0.5 * (a + b),
                                    emin=a, emax=b, window_type="delta", mmax=mm, vectors=False))
        return res_all

    res_plain, t_plain = timed(plain)
    g_plain, agree = [], []
    for w, ((a, b), (lp, _, rp)) in enumerate(zip(wins, res_plain)):
        okp = (lp >= a) & (lp <= b) & (rp <= 1e-10 * norm)
        g_plain.append(int(okp.sum()))
        sel = win == w
        okq = (lam[sel] >= a) & (lam[sel] <= b) & (res[sel] <= 1e-10 * norm)
        x, y = np.sort(lp[okp]), np.sort(lam[sel][okq])
        agree.append(float(np.abs(x - y).max() / norm) if x.size == y.size and x.size else None)
    out["plain_fp64"] = {"seconds": t_plain, "pairs": int(sum(g_plain)), "per_window": g_plain,
                         "eigenpairs_per_s": sum(g_plain) / t_plain}
    out["pipeline_over_plain"] = out["pipeline"]["eigenpairs_per_s"] / out["plain_fp64"]["eigenpairs_per_s"]
    out["max_dlambda_over_norm_per_window"] = agree
    print(json.dumps(out), flush=True)


def run_profile_filter(args):
    """Only the block Clenshaw filter of the workload on device blocks
    (sma_apply_poly_block_dev), `calls` times: the small case for ncu captures of the
    fused step.  Prints the per-step time it measured with CUDA events."""
    import torch

    import sparse_matrix_algorithms_b200 as S
    from sparse_matrix_algorithms_b200 import _lib as L

    wl = Workload(args.workload)
    ctx = S.context(0)
    op = S.SparseOperator(wl.A, ctx)
    smin, smax = op.gershgorin_bounds()
    dt = torch.float64 if args.precision == "fp64" else torch.float32
    width = args.width or wl.s
    Q = torch.randn(wl.A.shape[0], width, dtype=dt, device="cuda")
    Y = torch.empty_like(Q)
    c = np.ascontiguousarray(S.build_coeffs(args.degree, smin, smax, wl.sigma, wl.emin, wl.emax,
                                            wl.window_plain))
    stream = torch.cuda.ExternalStream(ctx.stream)
    torch.cuda.synchronize()
    times = []
    prec = "fp64" if args.precision == "fp64" else "fp32"
    for _ in range(args.calls):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        L.check(L.load().sma_apply_poly_block_dev(op.handle, c.ctypes.data, args.degree, smin, smax,
                                                  Q.data_ptr(), width, Y.data_ptr(), width, width,
                                                  L.PRECISIONS[prec]))
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1) / args.degree)
    print(json.dumps({"profile_filter": prec, "workload": wl.name, "width": width,
                      "degree": args.degree, "us_per_step_last": 1e3 * times[-1]}), flush=True)


def run_profile_orth(args):
    """A short POLFED solve on the C3 matrix (s=64, mmax=8, degree 60): its block
    orthogonalization and reorthogonalization GEMMs have the shapes of the C3 solve
    (n=262144, basis up to 512 columns, block 64) -- the small case for ncu captures of the
    dense part.  Prints the phase times."""
    import sparse_matrix_algorithms_b200 as S

    wl = Workload("c3")
    op = S.SparseOperator(wl.A, S.context(0))
    gl, gh = op.gershgorin_bounds()
    st = {}
    kw = wl.kwargs(gl, gh)
    kw["mmax"] = 8
    S.polfed(op, 100, 60, stats=st, vectors=False, **kw)
    print(json.dumps({"profile_orth": "c3", "orth_ms": st["orth_ms"], "rr_ms": st["rr_ms"],
                      "filter_ms": st["filter_ms"], "basis_dim": st["basis_dim"]}), flush=True)


def run_profile_pipeline(args):
    """One solve of the value arm (the pipeline) on the workload after its set-up (matrix
    upload, Lanczos bounds for the norm): the command for ncu launch lists of a whole
    pipeline solve.  Prints the solve's phase times and pairs."""
    import torch

    import sparse_matrix_algorithms_b200 as S
    from sparse_matrix_algorithms_b200 import planner as P

    wl = Workload(args.workload)
    ctx = S.context(0)
    op = S.SparseOperator(wl.A, ctx)
    if wl.norm is None:
        lo, hi = S.lanczos_bounds(op, steps=LANCZOS_STEPS)
        wl.norm = max(abs(lo), abs(hi))
    net = P.WindowPlanner.load(P.POLFED_WEIGHTS)
    st = {}
    lam, _, res = arm_pipeline(wl, op, net, args.precision, stats=st)
    torch.cuda.synchronize()
    print(json.dumps({"profile_pipeline": wl.name, "precision": args.precision,
                      "pairs": wl.good_pairs(lam, res),
                      **{k: st[k] for k in ("filter_ms", "orth_ms", "rr_ms", "polish_ms", "plan",
                                            "kernel_launches") if k in st}}), flush=True)


def run_profile_dense(args):
    """This library's DMMA products (sma_dense_gram_dev, sma_dense_update_dev) against
    torch.matmul in float64 (cuBLAS) at the tall-skinny shapes of a C3 POLFED solve
    (n = 262144): the CholQR2 products (64 x 64), the reorthogonalization against a basis
    of 2048 columns, the polish's Rayleigh-Ritz (1976 x 1976) and the Ritz-vector lift
    (3904 -> 3000).  Best of 4 timed runs after one warm-up, CUDA events."""
    import torch

    import sparse_matrix_algorithms_b200 as S
    from sparse_matrix_algorithms_b200 import _lib as L

    ctx = S.context(0)
    lib = L.load()
    stream = torch.cuda.ExternalStream(ctx.stream)
    n = 262144
    shapes = [("gram", 64, 64), ("update", 64, 64), ("gram", 2048, 64), ("update", 2048, 64),
              ("gram", 1976, 1976), ("update", 1976, 1976), ("update", 3904, 3000)]

    def timeit(fn, s=None):
        ts = []
        for _ in range(5):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            fn()
            e1.record(s)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        return min(ts[1:])

    for kind, m, k in shapes:
        X = torch.randn(n, m, dtype=torch.float64, device="cuda")
        if kind == "gram":  # C (m x k, column-major) = X^T Y
            Y = torch.randn(n, k, dtype=torch.float64, device="cuda")
            C = torch.empty(k, m, dtype=torch.float64, device="cuda")

            def ours():
                L.check(lib.sma_dense_gram_dev(ctx.handle, n, m, k, X.data_ptr(), m, Y.data_ptr(),
                                               k, C.data_ptr(), m, 1.0, 0.0))

            def ref():
                torch.matmul(X.T, Y)
        else:  # Y (n x k) = X B, B column-major m x k
            B = torch.randn(k, m, dtype=torch.float64, device="cuda")
            Y = torch.empty(n, k, dtype=torch.float64, device="cuda")

            def ours():
                L.check(lib.sma_dense_update_dev(ctx.handle, n, m, k, X.data_ptr(), m, B.data_ptr(),
                                                 m, 0, Y.data_ptr(), k, 1.0, 0.0))

            def ref():
                torch.matmul(X, B.T)
        flops = 2.0 * n * m * k
        t_ours, t_ref = timeit(ours, stream), timeit(ref)
        print(json.dumps({"profile_dense": kind, "n": n, "m": m, "k": k, "ms": round(t_ours, 3),
                          "tflops": round(flops / t_ours / 1e9, 1), "cublas_ms": round(t_ref, 3),
                          "cublas_tflops": round(flops / t_ref / 1e9, 1)}), flush=True)
        del X, Y
        torch.cuda.empty_cache()


def run_profile_stream(args):
    """The HBM rate of plain streams with the fused step's traffic mix, as a practical
    ceiling beside the copy peak: torch elementwise kernels over FP32 blocks of the C3
    step's size (n = 262144 rows x 64 columns = 67 MB each, and x 768 = 805 MB):
    copy (1 read + 1 write), add (2 + 1) and addcmul (3 reads + 1 write, the step's Q, B1,
    B2 -> out).  Best of 10 after warm-up, CUDA events."""
    import torch

    n = 262144
    for cols in (64, 768):
        a, b, c, d = (torch.randn(n, cols, device="cuda") for _ in range(4))
        blk = a.numel() * 4
        for name, fn, nbytes in (("copy", lambda: d.copy_(a), 2 * blk),
                                 ("add", lambda: torch.add(a, b, out=d), 3 * blk),
                                 ("addcmul", lambda: torch.addcmul(a, b, c, out=d), 4 * blk)):
            for _ in range(3):
                fn()
            ts = []
            for _ in range(10):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                fn()
                e1.record()
                e1.synchronize()
                ts.append(e0.elapsed_time(e1))
            t = min(ts)
            print(json.dumps({"profile_stream": name, "block_mb": round(blk / 1e6, 1),
                              "us": round(1e3 * t, 1), "gbs": round(nbytes / t / 1e6, 1)}), flush=True)
        del a, b, c, d
        torch.cuda.empty_cache()


def run_profile_slice(args):
    """One iteration of batched slicing on the C3 matrix: four windows around E=0 with
    degrees 400/300/200/100 and widths 256/192/192/128 (768 columns at the top degree),
    FP32 -- the segmented Clenshaw step for ncu captures."""
    import sparse_matrix_algorithms_b200 as S

    wl = Workload("c3")
    op = S.SparseOperator(wl.A, S.context(0))
    wins = [(-0.08, -0.04), (-0.04, 0.0), (0.0, 0.04), (0.04, 0.08)]
    st = {}
    S.slice_spectrum(op, wins, [400, 300, 200, 100], [256, 192, 192, 128], maxiter=1,
                     two_hit=False, precision="fp32", graph=False, stats=st)
    print(json.dumps({"profile_slice": "c3", "filter_ms": st["filter_ms"],
                      "spmm_steps": st["spmm_steps"], "spmm_columns": st["spmm_columns"],
                      "gbs": st["filter_bytes"] / st["filter_ms"] / 1e6}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--arm-steps", type=int, default=2,
                    help="timed solves of the plain and tuned arms (each after one warm-up)")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c3", choices=["c2", "c3", "c4", "c5"],
                    help="c4 / c5: one solve per arm of the batched pipeline and the plain path")
    ap.add_argument("--no-plain", action="store_true", help="c4 / c5: pipeline arm only")
    ap.add_argument("--precision", default="mixed", choices=["fp64", "fp32", "mixed"],
                    help="filter arithmetic of the pipeline arm (and of --profile-filter)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--cpu-full-solve", action="store_true",
                    help="with --impl reference: one complete CPU solve plus the sampled estimate")
    ap.add_argument("--profile-filter", action="store_true",
                    help="run only the Clenshaw filter of the workload (for ncu captures)")
    ap.add_argument("--profile-orth", action="store_true",
                    help="a short C3 POLFED solve for ncu captures of its GEMMs")
    ap.add_argument("--profile-pipeline", action="store_true",
                    help="one pipeline solve of the workload (for ncu launch lists)")
    ap.add_argument("--profile-dense", action="store_true",
                    help="this library's DMMA products against cuBLAS at the solver's shapes")
    ap.add_argument("--profile-stream", action="store_true",
                    help="HBM rate of plain elementwise streams with the step's traffic mix")
    ap.add_argument("--profile-slice", action="store_true",
                    help="one batched slicing iteration on the C3 matrix for ncu captures")
    ap.add_argument("--width", type=int, default=0, help="block width (default: the workload's s)")
    ap.add_argument("--degree", type=int, default=60)
    ap.add_argument("--calls", type=int, default=3)
    args = ap.parse_args()
    if args.profile_filter:
        run_profile_filter(args)
        return
    if args.profile_orth:
        run_profile_orth(args)
        return
    if args.profile_pipeline:
        run_profile_pipeline(args)
        return
    if args.profile_dense:
        run_profile_dense(args)
        return
    if args.profile_stream:
        run_profile_stream(args)
        return
    if args.profile_slice:
        run_profile_slice(args)
        return
    if args.workload in ("c4", "c5"):
        run_multi(args)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    import datetime

    import torch

    torch.cuda.set_device(local)
    if world > 1:
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                             device_id=torch.device("cuda", local))
    try:
        run_ours(args, rank, world, local)
    finally:
        if world > 1:
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
