"""Batched ensembles (fi_ensemble_*): members of different grids stepped together give
bitwise the results of stepping each member alone (with the persistent ensemble kernel
and with one CUDA graph per member on its own stream), and a failing member is flagged
without stopping the others."""
import numpy as np
import pytest

import fastiso_b200 as F
from fastiso_b200 import abi
from helpers import F_, RUN_TOL, oracle_for, rel_l2

pytestmark = pytest.mark.gpu


TILES = F.Ensemble.DEFAULT_TILES


def member(N, mean_log10eta, seed, t_end=400.0, t_ice_end=None, tiles=TILES):
    W_ = 15e3 * N
    domain = F.RegionalDomain(W_, W_, N, N)
    rng = np.random.default_rng(seed)
    log10eta = mean_log10eta + 0.3 * rng.standard_normal((N, N))
    se = F.SolidEarth(domain, layer_boundaries=[100e3], layer_viscosities=(10**log10eta).reshape(N, N, 1))
    H1 = 1e3 * (domain.R < 0.4 * W_)
    te = t_ice_end or t_end
    it = F.TimeInterpolatedIceThickness([0.0, 1.0, te], [domain.zeros(), H1, 1.2 * H1], domain)
    bcs = F.BoundaryConditions(domain, ice_thickness=it)
    sl = F.RegionalSeaLevel(surface=F.LaterallyVariableSeaSurface())
    return F.Simulation(domain, bcs, sl, se, (0.0, t_end), form="fp32", tiles=tiles)


SPECS = [(32, 21.0, 1), (48, 20.5, 2), (40, 21.5, 3)]


@pytest.mark.parametrize("executor", ["persist", "streams"])
def test_ensemble_bitwise_equals_members_alone(monkeypatch, executor):
    monkeypatch.setenv("FI_ENS_EXECUTOR", executor)
    alone = []
    for N, mu, seed in SPECS:
        sim = member(N, mu, seed)
        integ = F.init_integrator(sim)
        F.step(integ, 150.0, True)
        F.step(integ, 150.0, True)
        alone.append((F_(sim.get_field("u")), F_(sim.get_field("ue")), sim.stats()))
        sim.close()
    sims = [member(N, mu, seed) for N, mu, seed in SPECS]
    ens = F.Ensemble(sims, tiles=TILES)
    assert ens.step(150.0) == [abi.FI_OK] * len(SPECS)
    assert ens.step(150.0) == [abi.FI_OK] * len(SPECS)
    assert ens.last_gpu_ms > 0
    for sim, (u, ue, st) in zip(sims, alone):
        s2 = sim.stats()
        assert s2["t"] == 300.0
        for k in ("naccept", "nreject", "nf", "nsparse"):
            assert s2[k] == st[k], k
        assert np.array_equal(F_(sim.get_field("u")), u)
        assert np.array_equal(F_(sim.get_field("ue")), ue)
    ens.close()


def test_ensemble_member_parity_with_oracle():
    N, mu, seed = SPECS[1]
    sim = member(N, mu, seed)
    sim.nout.t = [300.0]
    ref = oracle_for(sim)
    ref.init()
    ens = F.Ensemble([sim, member(32, 21.0, 7)], tiles=TILES)
    ref.init_integrator(np.asarray([300.0]))
    ens.step(300.0)
    ref.step(300.0)
    assert rel_l2(F_(sim.get_field("u")), ref.get_field(abi.FIELDS["u"])) < RUN_TOL["fp32"]


def test_ensemble_failing_member_is_isolated():
    # the middle member's ice history ends at 200 yr: stepping to 300 yr leaves its
    # forcing range (TimeInterpolation2D out of range); the others are unaffected
    sims = [member(32, 21.0, 1), member(48, 20.5, 2, t_ice_end=200.0), member(40, 21.5, 3)]
    ens = F.Ensemble(sims, tiles=TILES)
    st = ens.step(300.0)
    assert st[0] == abi.FI_OK and st[2] == abi.FI_OK
    assert st[1] == abi.FI_ERR_FORCING_RANGE
    assert sims[0].stats()["t"] == 300.0 and sims[2].stats()["t"] == 300.0
    ref = member(40, 21.5, 3)
    F.step(F.init_integrator(ref), 300.0, True)
    assert np.array_equal(F_(sims[2].get_field("u")), F_(ref.get_field("u")))
    ens.close()
