"""The screening loop (surrogate.screen / screen_without_surrogate) on the CPU with a
stand-in network and solver: both follow per-cell relaxation u -> u_eq (1 - exp(-t/tau))
with u_eq = -0.27 H and tau set by the viscosity channel; the stand-in solver uses a 2x
longer tau for every third candidate, where the surrogate may then be out of bound.  Checks:
every accepted member fits the observation and was within the bound, out-of-bound
proposals are replaced, and screening needs fewer solver runs than the solver alone."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from fastiso_b200 import surrogate as S  # noqa: E402

N, W, T_END = 16, 1.5e6, 3000.0


def tau_of(log10eta):
    return 1500.0 * 10.0 ** (0.8 * (log10eta - 21.0))


class RelaxNet:
    """predict(x): the macro-step increment of the relaxation model, in the surrogate's units."""
    max_batch = 64

    def predict(self, x):
        u = x[:, 0] * S.U_SCALE
        H = x[:, 1] * S.H_SCALE
        eta = x[:, 2] * S.ETA_SCALE + S.ETA_MEAN
        a = 1.0 - torch.exp(-S.MACRO_DT / tau_of(eta))
        return ((-0.27 * H - u) * a) / S.DU_SCALE


def solver(specs, t_end):
    out = []
    for sp in specs:
        tau = tau_of(sp.log10eta) * (2.0 if sp.meta.get("slow") else 1.0)
        u = -0.27 * sp.H * (1.0 - np.exp(-t_end / tau))
        out.append(u.T.astype(np.float32))          # solver (nx, ny) -> [j, i]
    return np.stack(out)


def test_screening_accepts_within_bounds_and_replaces():
    truth, pool = S.calibration_pool(60, N, W, seed=5)
    for i, sp in enumerate(pool):
        sp.meta["slow"] = (i % 3 == 0)
    obs = solver([truth], T_END)[0]
    misfit = np.array([S._misfit(u, obs) for u in solver(pool, T_END)])
    tol, bound = float(np.sort(misfit)[5]), 0.05      # six qualifying candidates
    rep = S.screen(RelaxNet(), pool, obs, n_accept=3, tol_obs=tol, bound=bound, t_end=T_END, solve_batch=2,
                   solver=solver, device="cpu")
    assert len(rep.accepted) == 3
    accepted = {i for i, _ in rep.accepted}
    for i, u in rep.accepted:
        assert S._misfit(u, obs) <= tol
    for i, e, m, ok in rep.checked:
        assert ok == (m <= tol and e <= bound)      # accepted iff it fits and the surrogate was in bound
        assert ok == (i in accepted)
        if not pool[i].meta["slow"]:
            assert e < 1e-5                          # the stand-ins agree where the solver is not perturbed
    assert rep.out_of_bound == sum(1 for i, e, m, ok in rep.checked if e > bound) >= 1  # a replacement ran
    assert rep.solver_runs == len(rep.checked)
    base = S.screen_without_surrogate(pool, obs, n_accept=3, tol_obs=tol, t_end=T_END, seed=1, solve_batch=2,
                                      solver=solver)
    assert len(base.accepted) == 3
    assert rep.solver_runs < base.solver_runs
