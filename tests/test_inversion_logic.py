"""The UKI restatement (fastiso_b200.inversion, Huang, Schneider & Stuart 2022 as in
EnsembleKalmanProcesses.jl) on problems with known answers, on the CPU: a linear
forward model (alpha = 1 converges to the weighted least-squares solution) and a
nonlinear scalar model."""
import numpy as np

from fastiso_b200 import inversion as I


def test_uki_linear_converges_to_least_squares():
    rng = np.random.default_rng(0)
    A = rng.standard_normal((12, 3))
    theta_true = np.array([1.0, -2.0, 0.5])
    Gam = np.diag(0.01 * (1 + rng.random(12)))
    y = A @ theta_true + rng.multivariate_normal(np.zeros(12), Gam)
    uki = I.UnscentedKalman(np.zeros(3), 4.0 * np.eye(3), y, Gam, alpha_reg=1.0, update_freq=1)
    for _ in range(30):
        uki.step(lambda th: A @ th)
    W = np.linalg.inv(Gam)
    ls = np.linalg.solve(A.T @ W @ A, A.T @ W @ y)
    assert np.abs(uki.m - ls).max() < 1e-6
    # the error decreases and the covariance stays symmetric positive definite
    assert uki.errors[-1] <= uki.errors[0]
    assert np.all(np.linalg.eigvalsh(uki.C) > 0)


def test_uki_nonlinear_scalar():
    truth = 0.7
    f = lambda th: np.vstack([np.exp(th[0]), th[0] ** 3])  # noqa: E731
    y = f(np.array([truth]))[:, 0]
    uki = I.UnscentedKalman([0.0], [[1.0]], y, 1e-6 * np.eye(2))
    for _ in range(25):
        uki.step(lambda th: f(th))
    assert abs(uki.m[0] - truth) < 1e-3


def test_inversion_problem_and_regions():
    regions = [np.zeros((4, 4), bool), np.zeros((4, 4), bool)]
    regions[0][:2] = True
    regions[1][2:] = True
    red = I.ViscosityRegions(regions, make_sim=lambda f: f)
    np.testing.assert_array_equal(red.reconstruct([20.0, 21.0])[:2], 20.0)
    data = I.InversionData(t=[1.0, 2.0], Y=[np.ones((4, 4)), 2 * np.ones((4, 4))], mask=regions[0])
    assert data.nY == 2 and data.countmask == 8 and data.y.size == 16
    cfg = I.InversionConfig(N_iter=3, n_samples=50, scale_obscov=1.0)
    p = I.inversion_problem(cfg, data, red, [20.0, 21.0], np.eye(2))
    assert np.allclose(np.diag(p.uki.Gam), 0.5)  # scale / (1 + 1)
    # a forward model that returns the data exactly at theta = (20.5, 20.5)
    target = np.array([20.5, 20.5])
    fwd = lambda th: np.vstack([data.y[:, None] + 0.1 * (th[0] - target[0]) + 0.05 * (th[1] - target[1])] * 1)  # noqa
    I.solve(p, forward=fwd)
    assert len(p.out) == 4 and p.forward_launches == 3
    params, Gx, abserr = I.extract_inversion(p)
    assert params.shape == (2,) and Gx.shape == data.y.shape
