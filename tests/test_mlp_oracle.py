"""The CPU FP64 oracle of the learned Riemann guess checks itself: its
analytic gradient against central finite differences, and its random state
generator against the stated distributions."""
import numpy as np


def test_oracle_gradient_matches_finite_differences():
    import mlp_oracle as M
    rng = np.random.default_rng(0)
    p = rng.normal(0, 0.2, M.NPARAM)
    st = M.random_states(64, seed=3)
    x = M.features(st)
    t = rng.normal(0, 1, 64)
    _, g = M.loss_and_grad(p, x, t)
    for k in [0, 100, 319, 330, 383, 500, 4479, 4500, 8639, 8700, 8767, 8768]:
        e = np.zeros_like(p)
        e[k] = 1e-6
        num = (M.loss_and_grad(p + e, x, t)[0] - M.loss_and_grad(p - e, x, t)[0]) / 2e-6
        assert abs(num - g[k]) <= 1e-6 * max(1.0, abs(g[k])), k


def test_random_states_distribution():
    import mlp_oracle as M
    s = M.random_states(100_000, seed=12345)
    lr = np.log10(s[:, 4] / s[:, 1])
    lp = np.log10(s[:, 5] / s[:, 2])
    du = (s[:, 3] - s[:, 0]) / np.sqrt(s[:, 6] * s[:, 2] / s[:, 1])
    assert -3 <= lr.min() and lr.max() <= 3 and abs(lr.mean()) < 0.05
    assert -4 <= lp.min() and lp.max() <= 4 and abs(lp.mean()) < 0.05
    assert np.abs(du).max() <= 5.0 + 1e-12
    assert set(np.unique(s[:, 6])) == {1.4, 5.0 / 3.0}
    np.testing.assert_array_equal(s, M.random_states(100_000, seed=12345))
