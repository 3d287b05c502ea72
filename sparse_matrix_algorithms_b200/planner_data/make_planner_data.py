"""Training data and weights of the learned window planner.

    python -m sparse_matrix_algorithms_b200.planner_data.make_planner_data gen   # -> planner_train.npz
    python -m sparse_matrix_algorithms_b200.planner_data.make_planner_data train # -> planner_weights.npz
    ... gen-polfed / train-polfed / eval-polfed: the same for the POLFED planner

``gen`` draws matrices from the two model families -- 3D Anderson (L in 12..20, W uniform
in [2, 20]) and the XXZ chain (L in 12..16, h uniform in [0.5, 8]) -- places windows of
12..64 KPM-estimated eigenvalues in the bulk of each spectrum, and solves every window at
the grid of (degree, width) scales of the plain rule in one batched slicing call per
matrix (``planner.training_rows``).  ``gen-polfed`` does the same for POLFED on matrices
of the target distribution -- Anderson L in 16..48 (W in [2, 20]), XXZ L in 14..18 (h in
[0.5, 8]) -- with windows of 40..400 eigenvalues, Lanczos bounds as the pipeline uses them,
and every window's scale grid run as ONE batched POLFED call
(``planner.polfed_training_rows_batched``).  ``train`` fits the network on the GPU with
the library's own kernels.  Needs a GPU.  The features (KPM moments and mapped window
bounds) do not depend on n.
"""
import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from sparse_matrix_algorithms_b200 import api as S  # noqa: E402
from sparse_matrix_algorithms_b200 import matrices as M  # noqa: E402
from sparse_matrix_algorithms_b200 import planner as P  # noqa: E402


def sample_matrix(rng):
    if rng.uniform() < 0.6:
        L = int(rng.choice([12, 14, 16, 18, 20]))
        W = float(rng.uniform(2.0, 20.0))
        seed = int(rng.integers(1 << 30))
        return f"anderson L={L} W={W:.3f} seed={seed}", M.anderson3d(L, W, seed)
    L = int(rng.choice([12, 14, 16]))
    h = float(rng.uniform(0.5, 8.0))
    seed = int(rng.integers(1 << 30))
    return f"xxz L={L} h={h:.3f} seed={seed}", M.xxz_sz0(L, h, seed)


def sample_windows(rng, mu, n, smin, smax, k):
    # window centres between the 15% and 85% points of the KPM cumulative count
    lo = P.energy_at_count(mu, n, smin, smax, smin, 0.15 * n)
    hi = P.energy_at_count(mu, n, smin, smax, smin, 0.85 * n)
    out = []
    for _ in range(k):
        c = float(rng.uniform(lo, hi))
        N = float(rng.uniform(12, 64))
        w = P.windows_by_count(mu, n, smin, smax, c, [N])[0]
        out.append(w)
    return out


def gen(args):
    rng = np.random.default_rng(args.seed)
    F, T, W, names = [], [], [], []
    t0 = time.time()
    for i in range(args.matrices):
        name, A = sample_matrix(rng)
        op = S.SparseOperator(A)
        smin, smax = op.gershgorin_bounds()
        mu = S.kpm_moments(op, P.N_MOMENTS, 16, smin=smin, smax=smax)
        wins = sample_windows(rng, mu, A.shape[0], smin, smax, args.windows)
        f, t, w = P.training_rows(op, wins, smin=smin, smax=smax, mu=mu)
        F.append(f); T.append(t); W.append(w); names += [name] * len(wins)
        print(f"{i + 1}/{args.matrices} {name}: {int(w[:, 0].sum())}/{len(wins)} windows usable, "
              f"{time.time() - t0:.1f} s", flush=True)
    np.savez_compressed(args.out, X=np.concatenate(F), T=np.concatenate(T), W=np.concatenate(W),
                        names=np.array(names))


def train(args):
    z = np.load(args.data)
    net = P.WindowPlanner(seed=args.seed)
    hist = net.train(z["X"], z["T"], z["W"], steps=args.steps, lr=args.lr,
                     minibatch=args.minibatch, seed=args.seed, weight_decay=args.weight_decay)
    print(f"loss {hist[:20].mean():.4f} -> {hist[-20:].mean():.4f}")
    net.save(args.out)


HELD_OUT = [("anderson", 14, 12.0, 77), ("anderson", 18, 4.0, 78), ("xxz", 14, 3.0, 79),
            ("xxz", 12, 6.5, 80)]


def held_out_problem(kind, L, p, seed):
    return M.anderson3d(L, p, seed) if kind == "anderson" else M.xxz_sz0(L, p, seed)


def evaluate(weights=P.WEIGHTS, problems=HELD_OUT, counts=(20, 45, 30), verbose=True):
    """Column-steps of the plain rule and of the learned plan (fallback re-solves
    included) on held-out matrices; also whether both found the same eigenvalues."""
    net = P.WindowPlanner.load(weights)
    rows = []
    for kind, L, p, seed in problems:
        A = held_out_problem(kind, L, p, seed)
        op = S.SparseOperator(A)
        smin, smax = op.gershgorin_bounds()
        nrm = max(abs(smin), abs(smax))
        mu = S.kpm_moments(op, P.N_MOMENTS, 16, smin=smin, smax=smax)
        centre = P.energy_at_count(mu, A.shape[0], smin, smax, smin, 0.5 * A.shape[0])
        wins = P.windows_by_count(mu, A.shape[0], smin, smax, centre, counts)
        rp, rl = {}, {}
        lp, _, resp, wp = P.solve_windows(op, wins, None, smin=smin, smax=smax, mu=mu, report=rp)
        ll, _, resl, wl = P.solve_windows(op, wins, net, smin=smin, smax=smax, mu=mu, report=rl)
        same = lp.size == ll.size and bool(np.all(wp == wl)) and (
            lp.size == 0 or float(np.abs(lp - ll).max()) <= 1e-12 * nrm)
        row = dict(problem=f"{kind} L={L} p={p} seed={seed}", plain=int(np.sum(rp["cost"])),
                   learned=int(np.sum(rl["cost"])), redone=len(rl["redone"]), same=same,
                   found=int(lp.size), maxres=float(max(resp.max(), resl.max()) / nrm) if lp.size else None,
                   plain_deg=rp["degree"], learned_deg=rl["degree"], plain_m0=rp["m0"],
                   learned_m0=rl["m0"])
        rows.append(row)
        if verbose:
            print(row, flush=True)
    return rows


def sample_polfed_matrix(rng):
    """The POLFED planner's training distribution: 3D Anderson, L in 16..48, W uniform in
    [2, 20]; XXZ chain, L in 14..18, h uniform in [0.5, 8]."""
    if rng.uniform() < 0.6:
        L = int(rng.choice([16, 20, 24, 28, 32, 40, 48]))
        W = float(rng.uniform(2.0, 20.0))
        seed = int(rng.integers(1 << 30))
        return f"anderson L={L} W={W:.3f} seed={seed}", M.anderson3d(L, W, seed)
    L = int(rng.choice([14, 16, 18]))
    h = float(rng.uniform(0.5, 8.0))
    seed = int(rng.integers(1 << 30))
    return f"xxz L={L} h={h:.3f} seed={seed}", M.xxz_sz0(L, h, seed)


def sample_polfed_windows(rng, mu, n, smin, smax, k, lo_count, hi_count):
    lo = P.energy_at_count(mu, n, smin, smax, smin, 0.2 * n)
    hi = P.energy_at_count(mu, n, smin, smax, smin, 0.8 * n)
    out = []
    for _ in range(k):
        c = float(rng.uniform(lo, hi))
        N = float(np.exp(rng.uniform(np.log(lo_count), np.log(min(hi_count, 0.02 * n)))))
        out.append(P.windows_by_count(mu, n, smin, smax, c, [N])[0])
    return out


def gen_polfed(args):
    """Lanczos bounds (100 steps) and KPM moments on them, as the pipeline computes them;
    every window's scale grid of the plain rule solved in one batched POLFED call."""
    rng = np.random.default_rng(args.seed)
    F, T, W, names = [], [], [], []
    t0 = time.time()
    for i in range(args.matrices):
        name, A = sample_polfed_matrix(rng)
        op = S.SparseOperator(A)
        smin, smax = S.lanczos_bounds(op, steps=100)
        mu = S.kpm_moments(op, P.N_MOMENTS, 16, smin=smin, smax=smax)
        wins = sample_polfed_windows(rng, mu, A.shape[0], smin, smax, args.windows, args.min_count,
                                     args.max_count)
        rows = [P.polfed_training_rows_batched(op, [win], s=args.s, smin=smin, smax=smax, mu=mu)
                for win in wins]  # one window (its whole scale grid) per batched call
        f, t, w = (np.concatenate([r[i] for r in rows]) for i in range(3))
        F.append(f); T.append(t); W.append(w); names += [name] * len(wins)
        print(f"{i + 1}/{args.matrices} {name}: {int(w[:, 0].sum())}/{len(wins)} windows usable, "
              f"targets {np.round(np.exp(t[:, :2]), 2).tolist()}, {time.time() - t0:.1f} s", flush=True)
        op.close()
        np.savez_compressed(args.out, X=np.concatenate(F), T=np.concatenate(T),
                            W=np.concatenate(W), names=np.array(names))


HELD_OUT_POLFED = [("anderson", 24, 12.0, 77), ("anderson", 32, 4.0, 78), ("xxz", 16, 3.0, 79),
                   ("xxz", 18, 6.5, 80)]


def evaluate_polfed(weights=P.POLFED_WEIGHTS, problems=HELD_OUT_POLFED, counts=(60, 150),
                    verbose=True, s=32):
    """Column-steps of POLFED's plain rule and of the learned plan (fallback included) on
    held-out matrices of the training distribution -- both windows of a matrix in one
    batched call per planner -- and whether both found the same converged eigenvalues."""
    net = P.WindowPlanner.load(weights)
    rows = []
    for kind, L, p, seed in problems:
        A = held_out_problem(kind, L, p, seed)
        op = S.SparseOperator(A)
        smin, smax = S.lanczos_bounds(op, steps=100)
        nrm = max(abs(smin), abs(smax))
        mu = S.kpm_moments(op, P.N_MOMENTS, 16, smin=smin, smax=smax)
        centre = P.energy_at_count(mu, A.shape[0], smin, smax, smin, 0.5 * A.shape[0])
        wins = P.windows_by_count(mu, A.shape[0], smin, smax, centre, counts)
        rp, rl = {}, {}
        lp, _, resp, wp = P.solve_polfed_windows(op, wins, None, s=s, smin=smin, smax=smax, mu=mu,
                                                 report=rp, vectors=False)
        ll, _, resl, wl = P.solve_polfed_windows(op, wins, net, s=s, smin=smin, smax=smax, mu=mu,
                                                 report=rl, vectors=False)
        for w, win in enumerate(wins):
            sp, sl = wp == w, wl == w
            gp = np.sort(lp[sp][(lp[sp] >= win[0]) & (lp[sp] <= win[1]) & (resp[sp] <= 1e-10 * nrm)])
            gl = np.sort(ll[sl][(ll[sl] >= win[0]) & (ll[sl] <= win[1]) & (resl[sl] <= 1e-10 * nrm)])
            same = gp.size == gl.size and (gp.size == 0 or float(np.abs(gp - gl).max()) <= 1e-12 * nrm)
            # every pair the plain rule converged, the learned plan converged too (to 1e-12 ||A||)
            covers = all(gl.size and float(np.abs(gl - x).min()) <= 1e-12 * nrm for x in gp)
            row = dict(problem=f"{kind} L={L} p={p} seed={seed}", window=win, plain=rp["cost"][w],
                       learned=rl["cost"][w], redone=w in rl["redone"], same=same, covers=covers,
                       found=int(gp.size), found_learned=int(gl.size),
                       plain_plan=rp["plan"][w], learned_plan=rl["plan"][w])
            rows.append(row)
            if verbose:
                print(row, flush=True)
        op.close()
    return rows


def main():
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    g = sub.add_parser("gen")
    g.add_argument("--matrices", type=int, default=32)
    g.add_argument("--windows", type=int, default=4)
    g.add_argument("--seed", type=int, default=2024)
    g.add_argument("--out", default=os.path.join(HERE, "planner_train.npz"))
    t = sub.add_parser("train")
    t.add_argument("--data", default=os.path.join(HERE, "planner_train.npz"))
    t.add_argument("--steps", type=int, default=3000)
    t.add_argument("--lr", type=float, default=1e-3)
    t.add_argument("--minibatch", type=int, default=32)
    t.add_argument("--weight-decay", type=float, default=1e-3)
    t.add_argument("--seed", type=int, default=7)
    t.add_argument("--out", default=P.WEIGHTS)
    e = sub.add_parser("eval")
    e.add_argument("--weights", default=P.WEIGHTS)
    gp = sub.add_parser("gen-polfed")
    gp.add_argument("--matrices", type=int, default=24)
    gp.add_argument("--windows", type=int, default=2)
    gp.add_argument("--s", type=int, default=32)
    gp.add_argument("--min-count", type=float, default=40)
    gp.add_argument("--max-count", type=float, default=400)
    gp.add_argument("--seed", type=int, default=4049)
    gp.add_argument("--out", default=os.path.join(HERE, "polfed_planner_train.npz"))
    tp_ = sub.add_parser("train-polfed")
    tp_.add_argument("--data", default=os.path.join(HERE, "polfed_planner_train.npz"))
    tp_.add_argument("--steps", type=int, default=3000)
    tp_.add_argument("--lr", type=float, default=1e-3)
    tp_.add_argument("--minibatch", type=int, default=32)
    tp_.add_argument("--weight-decay", type=float, default=1e-3)
    tp_.add_argument("--seed", type=int, default=7)
    tp_.add_argument("--out", default=P.POLFED_WEIGHTS)
    ep = sub.add_parser("eval-polfed")
    ep.add_argument("--weights", default=P.POLFED_WEIGHTS)
    a = ap.parse_args()
    if a.cmd == "gen":
        gen(a)
    elif a.cmd in ("train", "train-polfed"):
        train(a)
    elif a.cmd == "gen-polfed":
        gen_polfed(a)
    else:
        rows = evaluate(a.weights) if a.cmd == "eval" else evaluate_polfed(a.weights)
        tp, tl = sum(r["plain"] for r in rows), sum(r["learned"] for r in rows)
        print(f"column-steps: plain {tp}, learned {tl}, ratio {tp / tl:.2f}")


if __name__ == "__main__":
    main()
