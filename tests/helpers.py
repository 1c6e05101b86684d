"""Test helpers: build a library simulation and the oracle (the checker) from the same
host-side inputs, and compare fields."""
from __future__ import annotations

import numpy as np

import fastiso_b200 as F
from fastiso_b200 import abi
from oracle import oracle as O


def F_(a):
    """numpy (nx, ny) -> flat x-fastest buffer"""
    return np.asarray(a, dtype=np.float64).ravel(order="F")


oracle_for = O.oracle_for


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


#: one right-hand side on identical inputs (dudt, ue, dz_ss): kernel-level parity
TOL = {"fp64": 1e-10, "fp32": 1e-6}
#: displacement over a run at the reference tolerance (reltol = Float64(1f-5)); the
#: adaptive step sequence amplifies round-off, so two correct runs differ by up to the
#: integrator's own error (about 6e-4 against a tight-tolerance solution here)
RUN_TOL = {"fp64": 1e-6, "fp32": 2e-3}
#: sparse diagnostics (ue, dz_ss) are sampled at stage times every 10 yr and are more
#: sensitive to the step sequence
RUN_TOL_SPARSE = {"fp64": 2e-3, "fp32": 5e-3}


# ---- cases of the committed golden fixtures (tests/golden/make_golden.py) ----------
def golden_sim(form, nx=24, ny=20, t_end=600.0, seed=11):
    """A small LV-ELVA case with every channel on (elastic, viscous, sea surface),
    seeded viscosity and lithosphere maps and a ramped disc load."""
    W_ = 0.6e6
    domain = F.RegionalDomain(W_, W_ * ny / nx, nx, ny)
    rng = np.random.default_rng(seed)
    log10eta = 21 + 0.4 * np.exp(-domain.R**2 / (2 * (W_ / 3) ** 2)) + 0.1 * rng.standard_normal((nx, ny))
    T = 90e3 + 30e3 * rng.random((nx, ny))
    se = F.SolidEarth(domain, layer_boundaries=T.reshape(nx, ny, 1),
                      layer_viscosities=(10**log10eta).reshape(nx, ny, 1))
    H1 = 1.2e3 * (domain.R < 0.45 * W_)
    it = F.TimeInterpolatedIceThickness([0.0, 1.0, t_end], [domain.zeros(), H1, 1.1 * H1], domain)
    bcs = F.BoundaryConditions(domain, ice_thickness=it)
    sl = F.RegionalSeaLevel(surface=F.LaterallyVariableSeaSurface())
    return F.Simulation(domain, bcs, sl, se, (0.0, t_end), form=form)


def golden_u(sim, seed=12):
    rng = np.random.default_rng(seed)
    d = sim.domain
    return -40 * np.exp(-d.R**2 / (2 * (0.35 * d.Wx) ** 2)) + 0.3 * rng.standard_normal((d.nx, d.ny))


GOLDEN_RHS_TIMES = (0.5, 12.5)
GOLDEN_RUN_TIMES = (300.0, 600.0, 1000.0)
GOLDEN_RUN_T_END = 1000.0


def lib_outputs(sim, t_outs, fields=("u", "dudt", "dz_ss"), record=0, replay=None):
    """Integrate a library Simulation with init_integrator (output times as tstops) and
    step! to each output time; returns ({field: [flat x-fastest arrays]}, record).
    record > 0 stores the attempt sequence (fi_record_steps); replay installs one.
    The output times are the run's tstops with the output callback (nout.t), as the
    oracle's init_integrator(t_outs) has them."""
    sim.nout.t = [float(t) for t in t_outs]
    integ = F.init_integrator(sim)
    if record:
        sim.record_steps(record)
    if replay is not None:
        sim.set_step_replay(replay)
    out = {f: [] for f in fields}
    for t in t_outs:
        F.step(integ, t - integ.t, True)
        for f in fields:
            out[f].append(F_(sim.get_field(f)))
    return out, (sim.step_record() if record else None)


def oracle_outputs(ref, t_outs, fields=("u", "dudt", "dz_ss"), record=0, replay=None):
    """The same for the oracle (already initialised with ref.init())."""
    ref.init_integrator(np.asarray(t_outs, dtype=np.float64))
    if record:
        ref.record_steps(record)
    if replay is not None:
        ref.set_step_replay(replay)
    out = {f: [] for f in fields}
    for t in t_outs:
        ref.step(t - ref.stats()["t"])
        for f in fields:
            out[f].append(ref.get_field(abi.FIELDS[f]))
    return out, (ref.step_record() if record else None)


def sealevel_sim(form, bsl=None, interactive=True, nx=40, ny=36, t_end=400.0, seed=21, adjustment=False):
    """A coastal case for the sea-level rows: bedrock from +600 m at the centre to
    -1400 m at the edges (an ocean all around), a disc of ice thick enough to ground
    on the shelf, active-load mask on the inner 40 % of the width (under the 60 % limit
    of interactive sea levels) reaching into the ocean beyond 0.3 of the width, elastic,
    viscous and sea-surface convolutions on."""
    W_ = 0.8e6
    domain = F.RegionalDomain(W_, W_ * ny / nx, nx, ny)
    rng = np.random.default_rng(seed)
    log10eta = 21 + 0.3 * np.exp(-domain.R**2 / (2 * (W_ / 3) ** 2)) + 0.05 * rng.standard_normal((nx, ny))
    T = 100e3 + 20e3 * rng.random((nx, ny))
    mask = domain.R < 0.45 * W_
    se = F.SolidEarth(domain, layer_boundaries=T.reshape(nx, ny, 1),
                      layer_viscosities=(10**log10eta).reshape(nx, ny, 1), maskactive=mask)
    z_b_ref = 600.0 - 2000.0 * domain.R / W_
    H1 = 2.5e3 * (domain.R < 0.25 * W_)
    it = F.TimeInterpolatedIceThickness([0.0, 1.0, 200.0, max(t_end, 400.0)], [domain.zeros(), H1, 0.4 * H1, 0.2 * H1],
                                        domain)
    bcs = F.BoundaryConditions(domain, ice_thickness=it)
    sl = F.RegionalSeaLevel(surface=F.LaterallyVariableSeaSurface(),
                            load=F.InteractiveSealevelLoad() if interactive else F.NoSealevelLoad(),
                            bsl=bsl if bsl is not None else F.ConstantBSL(),
                            adjustment_contribution=(F.GoelzerAdjustmentContribution() if adjustment
                                                     else F.NoAdjustmentContribution()))
    return F.Simulation(domain, bcs, sl, se, (0.0, t_end), z_b_ref=z_b_ref, form=form)


def ocean_surface_table():
    """A synthetic ocean-area table A(z) for PiecewiseConstantBSL (the reference downloads
    one): +-200 m around the present level, A(0) = A_OCEAN_PD, 3 % area change per 100 m."""
    z = np.linspace(-200.0, 200.0, 41)
    return z, abi.A_OCEAN_PD * (1.0 + 3e-4 * z)
