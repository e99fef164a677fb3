"""The float64 reference MLP (oracle/mlp_ref.py) used to check the GPU
training kernel: analytic gradient against central finite differences, the
bf16 rounding helper, and the generator replica's distribution."""
import numpy as np

from oracle import mlp_ref


def test_analytic_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    w = rng.normal(size=mlp_ref.NPARAM) * 0.2
    X = rng.normal(size=(64, 8))
    T = rng.normal(size=64)
    _, g = mlp_ref.loss_and_grad(w, X, T)
    idx = np.concatenate([rng.choice(mlp_ref.NPARAM, 60, replace=False), [mlp_ref.OFF_B3]])
    fd = mlp_ref.fd_grad(w, X, T, idx)
    assert np.max(np.abs(g[idx] - fd)) <= 1e-6 * max(1.0, np.abs(fd).max())


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -3.14159, 1e-20], np.float32)
    y = mlp_ref.bf16(x)
    assert y[0] == 1.0 and y[1] == 1.0          # ties to even
    assert y[2] == np.float32(1.0 + 2 ** -7)
    assert abs(y[3] + 3.140625) < 1e-6


def test_generator_replica_ranges():
    S = mlp_ref.generate(7, range(2000))
    dl, ul, pl, dr, ur, pr, g = S
    assert np.all((pr >= 1e-4) & (pr <= 1e4)) and np.all((dr >= 1e-3) & (dr <= 1e3))
    assert set(np.unique(g)) <= {1.4, 5.0 / 3.0}
    cl, cr = np.sqrt(g), np.sqrt(g * pr / dr)
    assert np.all(np.abs(ul) <= 5 * cl) and np.all(np.abs(ur) <= 5 * cr)
