"""The learned window planner's CUDA kernels against the CPU oracle, and its training."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import mlp_ref as R  # noqa: E402

pytestmark = pytest.mark.gpu


def _random_net(P, in_dim, hid, out, seed):
    net = P.WindowPlanner(seed=seed, in_dim=in_dim, hidden=hid, out_dim=out)
    rng = np.random.default_rng(seed)
    p = rng.normal(0, 1, net.num_params).astype(np.float32)
    # He-scaled weights, small biases
    o = 0
    for rows, cols in [(hid, in_dim), (hid, 1), (hid, hid), (hid, 1), (out, hid), (out, 1)]:
        p[o:o + rows * cols] *= (np.sqrt(2.0 / cols) if cols > 1 else 0.1)
        o += rows * cols
    net.params = p
    return net, p


@pytest.mark.parametrize("dims", [(258, 256, 3), (13, 40, 5)])
def test_forward_and_gradient_match_oracle(lib_built, dims):
    from sparse_matrix_algorithms_b200 import planner as P

    i, h, o = dims
    net, p = _random_net(P, i, h, o, 3)
    rng = np.random.default_rng(5)
    B = 77
    X = rng.normal(0, 1, (B, i)).astype(np.float32)
    T = rng.normal(0, 1, (B, o)).astype(np.float32)
    w = rng.uniform(0.2, 1.0, (B, o)).astype(np.float32)
    Y = net.forward(X)
    _, _, Yo, _ = R.forward(p, X, i, h, o, bf16=True)
    np.testing.assert_allclose(Y, Yo, rtol=1e-4, atol=1e-4 * np.abs(Yo).max())
    loss, g = net.grad(X, T, w)
    lo, go = R.loss_and_grad(p, X, T, w, i, h, o, bf16=True)
    assert abs(loss - lo) <= 1e-4 * lo
    scale = np.abs(go).max()
    np.testing.assert_allclose(g, go, rtol=1e-3, atol=1e-4 * scale)
    # the BF16 rounding matters: the FP64 network's gradient differs measurably
    _, g64 = R.loss_and_grad64(p, X, T, w, i, h, o)
    assert np.abs(g64 - go).max() > 1e-6 * scale


def test_training_fits_a_smooth_map(lib_built):
    from sparse_matrix_algorithms_b200 import planner as P

    rng = np.random.default_rng(1)
    N, i = 512, 258
    X = rng.uniform(-1, 1, (N, i)).astype(np.float32)
    T = np.stack([np.sin(X[:, 0] * 2) + 0.5 * X[:, 256], X[:, 1] * X[:, 2], 0.3 * X[:, 257]],
                 axis=1).astype(np.float32)
    net = P.WindowPlanner(seed=2)
    l0, _ = net.grad(X, T)
    hist = net.train(X, T, steps=600, lr=2e-3, minibatch=64, seed=3)
    l1, _ = net.grad(X, T)
    assert hist.shape == (600,) and np.isfinite(hist).all()
    assert l1 < 0.1 * l0, (l0, l1)
    assert np.isfinite(net.params).all()
    # a second network trained with the same seeds reproduces the run exactly
    net2 = P.WindowPlanner(seed=2)
    hist2 = net2.train(X, T, steps=600, lr=2e-3, minibatch=64, seed=3)
    np.testing.assert_array_equal(hist, hist2)


def test_learned_plan_beats_plain_rule(lib_built):
    """What the trained network gains: on matrices it never saw, the learned (degree,
    width) plans need fewer column-steps than the plain rule -- fallback re-solves
    included -- and return the same eigenvalues, all at residual <= 1e-10 ||A||."""
    from sparse_matrix_algorithms_b200.planner_data import make_planner_data as D

    rows = D.evaluate(problems=[("anderson", 14, 12.0, 77), ("xxz", 12, 6.5, 80)], verbose=False)
    for r in rows:
        assert r["same"], r
        assert r["found"] >= 80 and r["maxres"] <= 1e-10, r
    plain = sum(r["plain"] for r in rows)
    learned = sum(r["learned"] for r in rows)
    assert learned <= 0.85 * plain, (plain, learned)


def test_plain_rule_fallback_redoes_failed_windows(lib_built):
    """A planner whose degree output is forced far too low: the windows do not converge,
    the plain rule re-solves them, and the result equals the plain rule's."""
    import sparse_matrix_algorithms_b200 as S
    from sparse_matrix_algorithms_b200 import matrices as M
    from sparse_matrix_algorithms_b200 import planner as P

    A = M.anderson3d(12, 12.0, 5)
    op = S.SparseOperator(A)
    smin, smax = op.gershgorin_bounds()
    mu = S.kpm_moments(op, P.N_MOMENTS, 16, smin=smin, smax=smax)
    centre = P.energy_at_count(mu, A.shape[0], smin, smax, smin, 0.5 * A.shape[0])
    wins = P.windows_by_count(mu, A.shape[0], smin, smax, centre, [40, 30])
    net = P.WindowPlanner(seed=1)
    p = net.params
    # output layer: weights 0, biases = degree and width scales 0.01 (clipped to 0.2), so
    # each window's subspace (16 columns) is narrower than 0.85 N - 3 of its KPM count N
    p[-3:] = [np.log(0.01), np.log(0.01), 0.0]
    p[-3 - 3 * 256:-3] = 0.0
    net.params = p
    rep, rep0 = {}, {}
    lam, _, res, win = P.solve_windows(op, wins, net, smin=smin, smax=smax, mu=mu, maxiter=8, report=rep)
    lam0, _, res0, win0 = P.solve_windows(op, wins, None, smin=smin, smax=smax, mu=mu, maxiter=8, report=rep0)
    assert rep["m0"] == [16, 16]
    assert rep["redone"] == [0, 1]
    np.testing.assert_array_equal(win, win0)
    np.testing.assert_allclose(lam, lam0, rtol=0, atol=1e-12 * max(abs(smin), abs(smax)))


def test_learned_polfed_plan_beats_plain_rule(lib_built):
    """The POLFED planner (same network, trained on POLFED runs): on matrices it never saw,
    its (degree, mmax) plans need fewer filter column-steps than POLFED's plain rule --
    fallback re-solves included -- and find every converged in-window eigenvalue the plain
    rule finds (held-out matrices of its training distribution, Lanczos bounds)."""
    from sparse_matrix_algorithms_b200.planner_data import make_planner_data as D

    rows = D.evaluate_polfed(problems=[("anderson", 24, 12.0, 77), ("xxz", 16, 3.0, 79)],
                             verbose=False)
    for r in rows:  # the learned plan finds every pair the plain rule converged, and more
        assert r["covers"] and r["found_learned"] >= r["found"] >= 15, r
    plain = sum(r["plain"] for r in rows)
    learned = sum(r["learned"] for r in rows)
    assert learned <= 0.85 * plain, (plain, learned)
