"""The MMA oracle (oracle/mma_oracle.c) against optimality conditions.

The reference ships no MMA outputs, so the restatement of mmaOpt.cu is pinned by
what a converged MMA run must satisfy: the KKT conditions of small problems whose
optimum is known in closed form or checkable directly."""
import numpy as np

import oracle.oracle as O


def toy_problem(mma, x, iters):
    """min |x|^2 s.t. |x - c1|^2 <= 9, |x - c2|^2 <= 9, 0 <= x <= 5 (Svanberg's toy problem)"""
    c1, c2 = np.array([5.0, 2.0, 1.0]), np.array([3.0, 4.0, 3.0])
    for it in range(1, iters + 1):
        g = np.array([((x - c1) ** 2).sum() - 9, ((x - c2) ** 2).sum() - 9])
        dg = np.stack([2 * (x - c1), 2 * (x - c2)])
        x = mma.update(it, x, 2 * x, g, dg)
    return x, c1, c2


def test_toy_problem_reaches_a_kkt_point():
    mma = O.MMA(2, 3)
    mma.set_bound(0.0, 5.0)
    x, c1, c2 = toy_problem(mma, np.array([4.0, 3.0, 2.0]), 30)
    g = np.array([((x - c1) ** 2).sum() - 9, ((x - c2) ** 2).sum() - 9])
    assert np.all(np.abs(g) < 1e-5)  # both constraints active
    A = np.stack([2 * (x - c1), 2 * (x - c2)], axis=1)
    lam, *_ = np.linalg.lstsq(A, -2 * x, rcond=None)
    assert np.all(lam > 0)
    assert np.linalg.norm(2 * x + A @ lam) < 1e-5
    assert np.all((x > 0) & (x < 5))


def test_volume_constrained_compliance_has_the_closed_form_optimum():
    """min sum_j w_j / x_j s.t. mean(x) <= V, 0.001 <= x <= 1: the optimum is
    x_j = clamp(sqrt(w_j / mu)) with mu set by the active volume constraint."""
    rng = np.random.default_rng(3)
    n, V = 400, 0.3
    w = rng.uniform(0.2, 1.0, n)
    mma = O.MMA(1, n)
    mma.set_bound(0.001, 1.0)
    x = np.full(n, V)
    for it in range(60):
        g = np.array([x.mean() / V - 1.0])
        x = mma.update(it, x, -w / x ** 2, g, np.full((1, n), 1.0 / (n * V)))
    lo, hi = 1e-8, 1e8
    for _ in range(200):
        mu = np.sqrt(lo * hi)
        if np.clip(np.sqrt(w / mu), 0.001, 1.0).mean() > V:
            lo = mu
        else:
            hi = mu
    xs = np.clip(np.sqrt(w / mu), 0.001, 1.0)
    assert abs(x.mean() - V) < 1e-4
    assert np.abs(x - xs).max() < 2e-3


def test_first_iterations_use_the_initial_asymptotes():
    """itn <= 2 places the asymptotes at x -/+ 0.5 (xmax - xmin) (mmaOpt.cu:848-851)"""
    mma = O.MMA(1, 5)
    mma.set_bound(0.0, 2.0)
    x = np.linspace(0.5, 1.5, 5)
    mma.update(1, x, np.ones(5), np.array([-1.0]), np.ones((1, 5)))
    assert np.allclose(mma.low, x - 1.0) and np.allclose(mma.upp, x + 1.0)
    assert np.allclose(mma.xold1, x)
