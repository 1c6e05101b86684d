"""GPU parity of the other rheologies on the plain FP64 form's FFT engine (src/deformation.jl:21-89):
ELRA (RelaxedMantle with a laterally constant lithosphere), RigidMantle, and the
laterally-constant Maxwell scheme stepped by fixed-step Euler (dt_min).  Against the
FP64 oracle: 1e-10 per right-hand side, 1e-8 per run."""
import numpy as np
import pytest

import fastiso_b200 as F
from fastiso_b200 import abi
from helpers import F_, lib_outputs, oracle_for, oracle_outputs, rel_l2

pytestmark = pytest.mark.gpu


def _sim(kind, form="fp64", N=40, t_end=600.0):
    domain = F.RegionalDomain(1.2e6, 1.2e6, N, N)
    rng = np.random.default_rng(5)
    H1 = 1.5e3 * (domain.R < 4e5)
    it = F.TimeInterpolatedIceThickness([0.0, 1.0, 2e3], [domain.zeros(), H1, 1.2 * H1], domain)
    bcs = F.BoundaryConditions(domain, ice_thickness=it)
    opts = None
    if kind == "elra":
        tau = 500.0 + 200.0 * rng.random((N, N))  # laterally variable relaxation time
        se = F.SolidEarth(domain, layer_boundaries=[100e3], layer_viscosities=[1e21], mantle=F.RelaxedMantle(),
                          lithosphere=F.LaterallyConstantLithosphere(), tau=tau)
    elif kind == "rigid":
        se = F.SolidEarth(domain, layer_boundaries=[100e3], layer_viscosities=[1e21], mantle=F.RigidMantle())
    else:
        se = F.SolidEarth(domain, layer_boundaries=[100e3], layer_viscosities=[1e21],
                          lithosphere=F.LaterallyConstantLithosphere())
        opts = F.SolverOptions(diffeq=F.DiffEqOptions(alg="Euler", dt_min=5.0))
    sl = F.RegionalSeaLevel(surface=F.LaterallyVariableSeaSurface())
    return F.Simulation(domain, bcs, sl, se, (0.0, t_end), form=form, opts=opts,
                        nout=F.NativeOutput(t=[100.0, 350.0, t_end]))


@pytest.mark.parametrize("kind", ["elra", "rigid", "lc_maxwell"])
def test_rheology_rhs_parity(kind):
    sim = _sim(kind)
    ref = oracle_for(sim)
    ref.init()
    sim.init_problem()
    rng = np.random.default_rng(2)
    u = -30 * np.exp(-sim.domain.R**2 / (2 * 3e5**2)) + 0.2 * rng.standard_normal((sim.domain.nx, sim.domain.ny))
    for t in (0.5, 12.5, 31.0):
        ug, dg = u.copy(), np.zeros_like(u)
        F.update_diagnostics(dg, ug, sim, t)
        ur, dr = ref.rhs(t, F_(u))
        assert rel_l2(F_(ug), ur) < 1e-10, (t, rel_l2(F_(ug), ur))  # LC Maxwell: u is the implicit step
        if kind != "lc_maxwell":
            assert rel_l2(F_(dg), dr) < 1e-10, (t, rel_l2(F_(dg), dr))
        if kind == "elra":
            assert rel_l2(F_(sim.get_field("u_eq")), ref.get_field(abi.FIELDS["u_eq"])) < 1e-10
    ref.close()
    sim.close()


@pytest.mark.parametrize("kind", ["elra", "lc_maxwell"])
def test_rheology_run_parity(kind):
    """The library replays the oracle's attempt sequence (identical stage times)."""
    sim = _sim(kind)
    t_outs = list(sim.nout.t)
    ref = oracle_for(sim)
    ref.init()
    fields = ("u", "ue", "dz_ss")
    out_r, rec = oracle_outputs(ref, t_outs, fields=fields, record=1 << 20)
    ref.close()
    out_g, _ = lib_outputs(sim, t_outs, fields=fields, replay=rec)
    sim.close()
    for name in fields:
        for k in range(len(t_outs)):
            e = rel_l2(out_g[name][k], out_r[name][k])
            assert e < 1e-8, (name, k, e)
    assert np.abs(out_r["u"][-1]).max() > 1.0


def test_fp32_form_rejects_other_rheologies():
    with pytest.raises(F.UnsupportedError):
        _sim("elra", form="fp32")
