"""The fit driver's optimiser on the host: trust-region L-BFGS on smooth and on noisy
objectives (a stand-in for the Monte Carlo likelihood)."""
import numpy as np

from ppc_b200.fit import lbfgs_direction, minimize_trust_lbfgs


def test_lbfgs_direction_is_newton_step_on_a_quadratic():
    """With A-conjugate pairs spanning the space the two-loop recursion applies A^-1 exactly."""
    rng = np.random.default_rng(0)
    A = np.diag(rng.uniform(1, 100, 6))
    S = [np.eye(6)[i] * rng.uniform(0.5, 2) for i in range(6)]
    Y = [A @ s for s in S]
    g = rng.normal(size=6)
    d = lbfgs_direction(g, S, Y)
    assert np.allclose(d, -np.linalg.solve(A, g), rtol=1e-6)


def test_trust_lbfgs_converges_on_a_quadratic():
    rng = np.random.default_rng(1)
    a = np.exp(rng.uniform(0, np.log(1e2), 40))
    xs = rng.uniform(-0.3, 0.3, 40)

    def fg(x):
        return 0.5 * float(np.sum(a * (x - xs) ** 2)), a * (x - xs)

    x, f, evals, acc = minimize_trust_lbfgs(fg, np.zeros(40), 60, -1.0, 1.0, radius=0.05)
    assert evals == 61 and acc > 30
    assert np.abs(x - xs).max() < 1e-3


def test_trust_lbfgs_makes_progress_under_noise():
    """Gradient noise of 5% and a jumpy objective, as the Monte Carlo likelihood has."""
    rng = np.random.default_rng(2)
    a = np.exp(rng.uniform(0, np.log(100), 30))
    xs = rng.uniform(-0.2, 0.2, 30)

    def fg(x):
        f = 0.5 * float(np.sum(a * (x - xs) ** 2)) + 1e-4 * rng.normal()
        g = a * (x - xs) * (1 + 0.05 * rng.normal(size=30))
        return f, g

    x, f, evals, acc = minimize_trust_lbfgs(fg, np.zeros(30), 40, -0.5, 0.5)
    assert np.sqrt(np.mean((x - xs) ** 2)) < 0.2 * np.sqrt(np.mean(xs ** 2))


def test_penalty_gradient_matches_differences():
    from ppc_b200.fit import penalty
    rng = np.random.default_rng(3)
    u = rng.normal(size=20)
    p, g = penalty(u, 10, 3.0, 0.5)
    e = 1e-6
    num = np.array([(penalty(u + e * np.eye(20)[i], 10, 3.0, 0.5)[0] - penalty(u - e * np.eye(20)[i], 10, 3.0, 0.5)[0])
                    / (2 * e) for i in range(20)])
    assert np.allclose(g, num, rtol=1e-6, atol=1e-6)
