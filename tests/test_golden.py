"""The committed golden fixtures (tests/golden, written by make_golden.py after the
oracle passed the reference's known-answer tests): the oracle still reproduces them
(CPU), and the CUDA path matches them within the stated tolerances (GPU)."""
import pathlib

import numpy as np
import pytest

import fastiso_b200 as F
from fastiso_b200 import abi
from helpers import (F_, GOLDEN_RHS_TIMES, GOLDEN_RUN_T_END, GOLDEN_RUN_TIMES, RUN_TOL, RUN_TOL_SPARSE, TOL, golden_sim, golden_u,
                     oracle_for, rel_l2)
from oracle import oracle as O

G = pathlib.Path(__file__).resolve().parent / "golden"


def load(name):
    return np.load(G / name)


def test_oracle_reproduces_rhs_fixture():
    g = load("rhs_n24.npz")
    ref = oracle_for(golden_sim("fp64"))
    ref.init()
    for i, t in enumerate(GOLDEN_RHS_TIMES):
        uo, du = ref.rhs(t, g["u_in"])
        assert rel_l2(uo, g[f"u_out{i}"]) < 1e-13
        assert rel_l2(du, g[f"dudt{i}"]) < 1e-12
        assert rel_l2(ref.get_field(abi.FIELDS["ue"]), g[f"ue{i}"]) < 1e-12
        assert rel_l2(ref.get_field(abi.FIELDS["dz_ss"]), g[f"dz_ss{i}"]) < 1e-12


def test_oracle_reproduces_run_fixture():
    g = load("run_n32.npz")
    ref = oracle_for(golden_sim("fp64", 32, 32, t_end=GOLDEN_RUN_T_END))
    ref.init()
    out = ref.run(np.asarray(GOLDEN_RUN_TIMES))
    for var in ("u", "ue", "dudt", "dz_ss"):
        assert rel_l2(out[var], g[var]) < 1e-10, var


def test_oracle_convolution_fixture():
    g = load("conv_32.npz")
    got = O.conv_full(g["k"], g["x"])
    assert np.abs(got - g["full"]).max() <= 1e-12 * np.abs(g["full"]).max()


def test_analytic_fixture_matches_formula():
    import test_oracle_kats as K

    g = load("analytic.npz")
    domain = F.RegionalDomain(3e6, 7)
    se = F.SolidEarth(domain, layer_boundaries=[88e3], layer_viscosities=[1e21], rho_litho=0.0)
    c = F.PhysicalConstants()
    D, eta = float(np.mean(se.litho_rigidity)), float(np.mean(se.effective_viscosity))
    xs = g["x"][::16]
    ana = [K.analytic_solution(abs(x), g["t"][1] * c.seconds_per_year, c.rho_ice, c.g, se.rho_uppermantle, D, eta)
           for x in xs]
    assert np.allclose(ana, g["u"][1][::16], rtol=1e-10, atol=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["fp64", "fp32"])
def test_cuda_rhs_matches_fixture(form):
    g = load("rhs_n24.npz")
    sim = golden_sim(form)
    sim.init_problem()
    nx, ny = sim.domain.nx, sim.domain.ny
    u0 = g["u_in"].reshape(ny, nx).T
    for i, t in enumerate(GOLDEN_RHS_TIMES):
        u, du = u0.copy(), np.zeros_like(u0)
        F.update_diagnostics(du, u, sim, t)
        assert rel_l2(F_(u), g[f"u_out{i}"]) < 1e-12
        assert rel_l2(F_(du), g[f"dudt{i}"]) < TOL[form]
        assert rel_l2(F_(sim.get_field("ue")), g[f"ue{i}"]) < TOL[form]
        assert rel_l2(F_(sim.get_field("dz_ss")), g[f"dz_ss{i}"]) < TOL[form]


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["fp64", "fp32"])
def test_cuda_run_matches_fixture(form):
    g = load("run_n32.npz")
    sim = golden_sim(form, 32, 32, t_end=GOLDEN_RUN_T_END)
    sim.nout.t = list(GOLDEN_RUN_TIMES)
    F.run(sim)
    for k in range(len(GOLDEN_RUN_TIMES)):
        assert rel_l2(F_(sim.nout.out["u"][k]), g["u"][k]) < RUN_TOL[form], (form, k)
        for var in ("ue", "dz_ss"):
            assert rel_l2(F_(sim.nout.out[var][k]), g[var][k]) < RUN_TOL_SPARSE[form], (form, k, var)
