"""The perceptron oracle's gradient against central finite differences of
its exact (FP64, no BF16 rounding) loss (CPU only)."""
import numpy as np

from oracle import mlp as M


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    shapes = [(16, 5), (16, 16), (3, 16)]
    n = sum(a * b + a for a, b in shapes)
    p = rng.normal(0, 0.4, n)
    x = rng.normal(0, 1, (9, 5))
    t = rng.normal(0, 1, (9, 3))
    _, g = M.loss_grad(p, shapes, x, t, bf=False)
    eps = 1e-6
    for i in rng.choice(n, 40, replace=False):
        pp, pm = p.copy(), p.copy()
        pp[i] += eps
        pm[i] -= eps
        fd = (M.loss_grad(pp, shapes, x, t, bf=False)[0] - M.loss_grad(pm, shapes, x, t, bf=False)[0]) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-7 + 1e-5 * abs(fd), (i, fd, g[i])


def test_bf16_rounding():
    a = np.array([1.0, 1.00390625, 1.005859375, -3.14159265, 1e-30], np.float32)
    r = M.bf16(a)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: rounds to even (1.0)
    np.testing.assert_array_equal(r[:3], [1.0, 1.0, 1.0078125])
    assert abs(r[3] + 3.140625) < 1e-12


def test_gelu_tanh_form_is_within_1e3_of_erf_gelu():
    """The tanh GELU (Hendrycks & Gimpel 2016) against x Phi(x) with erf."""
    from scipy.special import erf
    x = np.linspace(-10.0, 10.0, 200001)
    exact = 0.5 * x * (1.0 + erf(x / np.sqrt(2.0)))
    assert np.max(np.abs(M.gelu(x) - exact)) <= 1e-3
