"""The surrogate end to end at a reduced size: trajectories from the GPU solver, training
with the FNO's own CUDA kernels, held-out accuracy, and screening in which the plain
solver checks the surrogate's proposals -- against the same screening without it."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N, W, T_END = 64, 1.5e6, 3000.0


@pytest.fixture(scope="module")
def trained():
    pytest.importorskip("torch")
    from fastiso_b200 import surrogate as S
    from fastiso_b200.fno import FNO

    train_specs = [S.member_spec(s, N, W) for s in range(512)]
    test_specs = [S.member_spec(5000 + s, N, W) for s in range(16)]
    data = S.Dataset(train_specs, S.generate_trajectories(train_specs, T_END, device="cuda"))
    test = S.Dataset(test_specs, S.generate_trajectories(test_specs, T_END))
    net = FNO(S=N, max_batch=16, seed=0)
    hist = S.train(net, data, steps=8000, batch=16, lr=1e-3)
    return S, net, data, test, hist


def test_training_reduces_loss(trained):
    _, _, _, _, hist = trained
    first, last = np.mean(hist["loss"][:50]), np.mean(hist["loss"][-200:])
    assert last < 0.1 * first, (first, last)


def test_held_out_rollout(trained):
    S, net, _, test, _ = trained
    ev = S.evaluate(net, test)
    # one macro-step from the solver's state, and a 30-step rollout from rest
    assert ev["one_step_relL2_du_pooled"] < 0.45, ev
    assert ev["rollout_relL2_final_mean"] < 0.3, ev


def test_screening_gain(trained):
    S, net, _, _, _ = trained
    truth, pool = S.calibration_pool(96, N, W, seed=777)
    obs = S.solve_final([truth], T_END)[0]
    tol, bound = 0.06, 0.15
    with_s = S.screen(net, pool, obs, n_accept=3, tol_obs=tol, bound=bound, t_end=T_END, solve_batch=3)
    without = S.screen_without_surrogate(pool, obs, n_accept=3, tol_obs=tol, t_end=T_END, seed=1, solve_batch=3)
    assert len(with_s.accepted) == 3 and len(without.accepted) == 3
    for _, u in with_s.accepted:     # accepted members carry the solver's own states
        assert S._misfit(u, obs) <= tol
    assert with_s.solver_runs < without.solver_runs, (with_s.solver_runs, without.solver_runs, with_s.checked)
