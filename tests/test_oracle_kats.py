"""The oracle against the reference's known-answer tests and independent maths
(numpy / scipy), CPU only.

* test/test_derivatives.jl: u = X^2 Y^2 on 128^2 (W = 3e6): interior second
  derivatives match 2Y^2, 2X^2, 4XY.
* test/test_convolution.jl: conv! of a random 64x64 kernel and input equals the full
  linear convolution (DSP.conv there, scipy's direct convolution here).
* src/integrators.jl:205-217: BS3 on u' = -0.5 u matches exp(-0.5 t).
* src/analytic_solutions.jl:11-65 (Bueler et al. 2007): disc load on an elastic plate
  over a viscous half-space (docs/src/examples/benchmark_analytic.jl set-up).
"""
import numpy as np
import pytest
import scipy.signal
import scipy.special

import fastiso_b200 as F
from oracle import oracle as O
from helpers import oracle_for, rel_l2


@pytest.mark.parametrize("n", [8, 12, 15, 17, 64, 71, 96, 128, 350, 700])
def test_fft_matches_numpy(n):
    rng = np.random.default_rng(n)
    a = rng.standard_normal((n, n + 2)) + 1j * rng.standard_normal((n, n + 2))
    assert np.abs(O.fft2(a) - np.fft.fft2(a)).max() < 1e-12 * np.abs(np.fft.fft2(a)).max()
    assert np.abs(O.fft2(a, inverse=True) - np.fft.ifft2(a)).max() < 1e-12 * np.abs(np.fft.ifft2(a)).max()


def test_nextfastfft():
    for n, m in [(127, 128), (191, 192), (255, 256), (383, 384), (511, 512), (699, 700), (2047, 2048), (33, 35)]:
        assert O.nextfastfft(n) == m == F.nextfastfft(n)


def test_derivative_polynomial_kat():
    domain = F.RegionalDomain(3e6, 7)
    X, Y = domain.X, domain.Y
    u = X**2 * Y**2
    uxx, uyy, ux, uxy = O.second_derivatives(u, domain.dx, domain.dy)
    inn = (slice(1, -1), slice(1, -1))
    for got, want in [(uxx, 2 * Y**2), (uyy, 2 * X**2), (uxy, 4 * X * Y)]:
        assert np.linalg.norm(got[inn] - want[inn]) <= 1.5e-8 * np.linalg.norm(want[inn])


def test_derivative_edge_rules():
    """CPU edge rules (derivatives.jl:66-76, 171-191): copy-of-neighbour for the second
    differences, one-sided first differences."""
    rng = np.random.default_rng(0)
    u = rng.standard_normal((9, 7))
    dx, dy = 2.0, 3.0
    uxx, uyy, ux, uxy = O.second_derivatives(u, dx, dy)
    assert np.allclose(uxx[0], (u[2] - 2 * u[1] + u[0]) / dx**2)
    assert np.allclose(uxx[-1], (u[-1] - 2 * u[-2] + u[-3]) / dx**2)
    assert np.allclose(ux[0], (u[1] - u[0]) / dx)
    assert np.allclose(ux[4], (u[5] - u[3]) / (2 * dx))
    assert np.allclose(uyy[:, 0], (u[:, 2] - 2 * u[:, 1] + u[:, 0]) / dy**2)
    assert np.allclose(uxy[:, -1], (ux[:, -1] - ux[:, -2]) / dy)


def test_convolution_vs_direct():
    rng = np.random.default_rng(64)
    k = rng.random((64, 64)).astype(np.float32).astype(np.float64)
    x = rng.random((64, 64)).astype(np.float32).astype(np.float64)
    got = O.conv_full(k, x)
    want = scipy.signal.convolve2d(k, x, mode="full")
    assert got.shape == (127, 127)
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()


def test_bs3_exponential_decay():
    t_out = np.arange(0, 6, 1.0)
    u, _ = O.bs3_decay(-0.5, 1.0, 5.0, t_out, reltol=1e-3, abstol=1e-6)
    assert np.allclose(u, np.exp(-0.5 * t_out), atol=1e-3)
    u2, _ = O.bs3_decay(-0.5, 1.0, 5.0, t_out, reltol=1e-9, abstol=1e-12)
    assert np.allclose(u2, np.exp(-0.5 * t_out), atol=1e-7)


def _looped_quadrature(f, support, n=5):
    x, w = np.polynomial.legendre.leggauss(n)
    total = 0.0
    for a, b in zip(support[:-1], support[1:]):
        m = 2.0 / (b - a)
        p = -1.0 - m * a
        total += np.sum(f((x - p) / m) * w / m)
    return total


def analytic_solution(r, t_sec, rho_ice, g, rho_um, D, eta, H0=1e3, R0=1e6):
    """src/analytic_solutions.jl:11-65 (transient branch)."""
    support = np.concatenate([[1e-14], 10.0 ** np.arange(-10, -3 + 1e-9, 0.05), [1.0]])
    scaling = rho_ice * g * H0 * R0

    def integrand(kappa):
        beta = rho_um * g + D * kappa**4
        return (np.exp(-beta * t_sec / (2 * eta * kappa)) - 1) * scipy.special.j0(kappa * r) * \
            scipy.special.j1(kappa * R0) / beta

    return scaling * _looped_quadrature(integrand, support)


def test_analytic_disc_load():
    """Laterally constant Earth, elastic term off (rho_litho = 0), as in
    docs/src/examples/benchmark_analytic.jl; the viscous solve must follow the
    Hankel-transform solution along the x transect."""
    domain = F.RegionalDomain(3e6, 7)
    H1 = 1e3 * (domain.R < 1e6)
    it = F.TimeInterpolatedIceThickness([0.0, 1.0, 50e3], [domain.zeros(), H1, H1], domain)
    bcs = F.BoundaryConditions(domain, ice_thickness=it)
    se = F.SolidEarth(domain, layer_boundaries=[88e3], layer_viscosities=[1e21], rho_litho=0.0)
    t_check = [5e3, 10e3]
    sim = F.Simulation(domain, bcs, F.RegionalSeaLevel(), se, (0.0, 10e3), nout=F.NativeOutput(t=t_check),
                       form="fp64")
    ref = oracle_for(sim)
    ref.init()
    out = ref.run(np.asarray(t_check), want=("u",))
    j = domain.my - 1  # y ~ 0 row
    xs = domain.x[domain.mx - 1:]
    c = F.PhysicalConstants()
    D = float(np.mean(se.litho_rigidity))
    eta = float(np.mean(se.effective_viscosity))
    for k, t in enumerate(t_check):
        u = out["u"][k].reshape(domain.ny, domain.nx).T  # [i, j]
        num = u[domain.mx - 1:, j]
        ana = np.array([analytic_solution(abs(x), t * c.seconds_per_year, c.rho_ice, c.g, se.rho_uppermantle, D,
                                          eta) for x in xs])
        # the corner BC fixes the far field at 0 while the half-space solution does not vanish there
        err = rel_l2(num - num[-1], ana - ana[-1])
        assert err < 0.02, (t, err)


def test_oracle_replay_reproduces_its_run():
    """The attempt record (accepted dt > 0, rejected dt < 0) replayed on a fresh oracle
    visits the same stage times, rejected attempts and sparse updates included, and
    reproduces the run bit for bit (the basis of the FP32-vs-Float64 replay tests)."""
    import fastiso_b200.workloads as W

    t_outs = np.array([100.0, 300.0])

    def fresh():
        sim = W.config2(form="fp64", N=32, t_end=300.0, out_every=300.0, n_snap=2)
        r = O.oracle_for(sim)
        r.init()
        r.init_integrator(t_outs)
        return r

    a = fresh()
    a.record_steps(1 << 16)
    ua = []
    for t in t_outs:
        a.step(t - a.stats()["t"])
        ua.append(a.get_field(8))
    rec = a.step_record()
    st_a = a.stats()
    assert (rec < 0).sum() == st_a["nreject"] and (rec > 0).sum() == st_a["naccept"]
    b = fresh()
    b.set_step_replay(rec)
    for t, u in zip(t_outs, ua):
        b.step(t - b.stats()["t"])
        np.testing.assert_array_equal(b.get_field(8), u)
    st_b = b.stats()
    assert (st_b["naccept"], st_b["nreject"], st_b["nsparse"]) == (st_a["naccept"], st_a["nreject"], st_a["nsparse"])


def test_oracle_resume_continues_the_run():
    """or_resume at t from a state taken at t continues the same solution: it differs
    from the uninterrupted run only by the restarted step sequence (new initial dt),
    i.e. by the integrator's own error."""
    import fastiso_b200.workloads as W

    def fresh():
        sim = W.config2(form="fp64", N=32, t_end=600.0, out_every=600.0, n_snap=2)
        r = O.oracle_for(sim)
        r.init()
        return r

    a = fresh()
    a.init_integrator([300.0, 600.0])
    a.step(300.0)
    st = a.stats()
    state = [a.get_field(i) for i in (8, 9, 11)]  # u, ue, dz_ss
    b = fresh()
    b.resume(st["t"], st["nsparse"], *state, tstops=[600.0])
    assert b.stats()["t"] == 300.0
    a.step(300.0)
    b.step(300.0)
    assert rel_l2(b.get_field(8), a.get_field(8)) < 2e-3
    assert b.stats()["nsparse"] >= st["nsparse"] + 29


def test_kei_matches_scipy():
    """The Kelvin function of the ELRA Green's function, imag(besselk(0, x e^{i pi/4}))
    as src/material.jl:370-373 defines it, against scipy's complex K_0 (AMOS) to 1e-13
    of |K_0|, and against scipy.special.kei (a separate algorithm, ~1e-11 here) to 1e-9."""
    for x in (1e-5, 1e-3, 0.1, 0.5, 1.0, 2.0, 5.0, 7.9, 8.1, 12.0, 20.0, 40.0):
        k0 = scipy.special.kv(0, x * np.exp(1j * np.pi / 4))
        assert abs(O.kei(x) - k0.imag) <= 1e-13 * abs(k0), (x, O.kei(x), k0)
        assert abs(O.kei(x) - scipy.special.kei(x)) <= 1e-9 * abs(k0), x


def test_analytic_disc_load_laterally_constant_maxwell():
    """The laterally-constant Maxwell scheme (src/deformation.jl:52-89, Bueler et al.
    2007) with Euler steps of dt_min = 10 yr follows the same analytic disc-load
    solution as the LV-ELVA solve."""
    domain = F.RegionalDomain(3e6, 7)
    H1 = 1e3 * (domain.R < 1e6)
    it = F.TimeInterpolatedIceThickness([0.0, 1.0, 50e3], [domain.zeros(), H1, H1], domain)
    bcs = F.BoundaryConditions(domain, ice_thickness=it)
    se = F.SolidEarth(domain, layer_boundaries=[88e3], layer_viscosities=[1e21], rho_litho=0.0,
                      lithosphere=F.LaterallyConstantLithosphere())
    t_check = [5e3, 10e3]
    opts = F.SolverOptions(diffeq=F.DiffEqOptions(alg="Euler", dt_min=10.0))
    sim = F.Simulation(domain, bcs, F.RegionalSeaLevel(), se, (0.0, 10e3), nout=F.NativeOutput(t=t_check),
                       form="fp64", opts=opts)
    ref = oracle_for(sim)
    ref.init()
    out = ref.run(np.asarray(t_check), want=("u",))
    j = domain.my - 1
    xs = domain.x[domain.mx - 1:]
    c = F.PhysicalConstants()
    D = float(np.mean(se.litho_rigidity))
    eta = float(np.mean(se.effective_viscosity))
    for k, t in enumerate(t_check):
        u = out["u"][k].reshape(domain.ny, domain.nx).T
        num = u[domain.mx - 1:, j]
        ana = np.array([analytic_solution(abs(x), t * c.seconds_per_year, c.rho_ice, c.g, se.rho_uppermantle, D,
                                          eta) for x in xs])
        assert rel_l2(num, ana) < 0.03, (t, rel_l2(num, ana))


def test_elra_relaxes_to_equilibrium():
    """ELRA (src/deformation.jl:29-45): with a constant load the displacement relaxes to
    the equilibrium u_eq = Kelvin-function convolution of the load, dudt = (u_eq - u)/tau."""
    domain = F.RegionalDomain(1.5e6, 1.5e6, 48, 48)
    H1 = 1e3 * (domain.R < 5e5)
    it = F.TimeInterpolatedIceThickness([0.0, 1.0, 20e3], [domain.zeros(), H1, H1], domain)
    bcs = F.BoundaryConditions(domain, ice_thickness=it)
    se = F.SolidEarth(domain, layer_boundaries=[100e3], layer_viscosities=[1e21], mantle=F.RelaxedMantle(),
                      lithosphere=F.LaterallyConstantLithosphere(), tau=300.0)
    sim = F.Simulation(domain, bcs, F.RegionalSeaLevel(), se, (0.0, 6e3), nout=F.NativeOutput(t=[6e3]),
                       form="fp64")
    ref = oracle_for(sim)
    ref.init()
    out = ref.run(np.asarray([6e3]), want=("u", "dudt"))
    u_eq = ref.get_field(F.abi.FIELDS["u_eq"])
    assert u_eq.min() < -100.0
    assert rel_l2(out["u"][0], u_eq) < 1e-4
    np.testing.assert_allclose(ref.get_field(F.abi.FIELDS["dudt"]), (u_eq - ref.get_field(8)) / 300.0, rtol=1e-10,
                               atol=1e-12)
