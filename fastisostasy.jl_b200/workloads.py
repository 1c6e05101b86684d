"""Seeded synthetic inputs with the shapes of the benchmark configurations.

No dataset is read: every field is generated here from fixed seeds.

* ``config1``  -- N=64 over 3000 km, one Gaussian log10-viscosity bump (+0.5,
  sigma=400 km), lithosphere 100 km, 1000 km / 1000 m ice disc switched on over
  the first year, 10 kyr, outputs every kyr (the layout of
  docs/src/examples/benchmark_3D.jl:17-43 with the disc of benchmark_analytic.jl).
* ``config2``  -- N=350 over 6000 km, Gaussian random fields for log10 viscosity
  (mean 21, std 0.5, l=500 km, clip [19,23]) and lithosphere thickness (mean
  120 km, std 40 km, l=500 km, clip [50,250] km), random ice (0-4000 m, l=800 km)
  times a 100-kyr sawtooth sampled every kyr, elastic and sea-surface on, 120 kyr.
* ``config3``  -- 128-member mixed-N ensemble (N in {64,96,128,192,256}, 30 km
  cells), per-member log10-viscosity fields (mean ~ U[20,22]), 100 km lithosphere,
  shared disc-plus-random-field ice history, 20 kyr.
* ``config5``  -- N=1024 over 6000 km with the config2 generators, 30-kyr segment.

Random fields: PCG64 white noise, spectral filter exp(-|k|^2 l^2 / 4), normalised
to zero mean and unit sample standard deviation.
"""
from __future__ import annotations

import numpy as np

from . import model as M

SEED_VISC, SEED_LITHO, SEED_ICE = 1001, 1002, 1003


def gaussian_random_field(nx, ny, Wx, Wy, corr_len, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    w = rng.standard_normal((nx, ny))
    kx = 2 * np.pi * np.fft.fftfreq(nx, d=2 * Wx / nx)
    ky = 2 * np.pi * np.fft.fftfreq(ny, d=2 * Wy / ny)
    KX, KY = np.meshgrid(kx, ky, indexing="ij")
    filt = np.exp(-(KX**2 + KY**2) * corr_len**2 / 4)
    g = np.real(np.fft.ifft2(np.fft.fft2(w) * filt))
    g = g - g.mean()
    return g / g.std()


def sawtooth(t, period=100e3, rise=90e3):
    """Glacial-cycle modulation: 0 -> 1 linearly over `rise`, back to 0 over the rest."""
    tau = np.mod(np.asarray(t, dtype=np.float64), period)
    return np.where(tau <= rise, tau / rise, 1.0 - (tau - rise) / (period - rise))


def _disc(domain, R=1e6, H=1e3):
    return H * (domain.R < R).astype(np.float64)


def config1(form="fp32", N=64, W=1.5e6, t_end=10e3, sea_surface=False):
    domain = M.RegionalDomain(W, W, N, N)
    log10eta = 21 + 0.5 * np.exp(-domain.R**2 / (2 * 400e3**2))
    solidearth = M.SolidEarth(domain, layer_boundaries=[100e3],
                              layer_viscosities=(10**log10eta).reshape(N, N, 1))
    H1 = _disc(domain)
    it = M.TimeInterpolatedIceThickness([0.0, 1.0, t_end], [domain.zeros(), H1, H1], domain)
    bcs = M.BoundaryConditions(domain, ice_thickness=it)
    sl = M.RegionalSeaLevel(surface=M.LaterallyVariableSeaSurface() if sea_surface else M.LaterallyConstantSeaSurface())
    nout = M.NativeOutput(t=list(np.arange(0.0, t_end + 1, 1e3)))
    return M.Simulation(domain, bcs, sl, solidearth, (0.0, t_end), nout=nout, form=form)


def config2_fields(N=350, W=3e6):
    domain = M.RegionalDomain(W, W, N, N)
    g_eta = gaussian_random_field(N, N, W, W, 500e3, SEED_VISC)
    log10eta = np.clip(21 + 0.5 * g_eta, 19, 23)
    g_T = gaussian_random_field(N, N, W, W, 500e3, SEED_LITHO)
    T = np.clip(120e3 + 40e3 * g_T, 50e3, 250e3)
    g_H = gaussian_random_field(N, N, W, W, 800e3, SEED_ICE)
    H = np.clip(4000 * np.maximum(g_H, 0), 0, 4000)
    return domain, log10eta, T, H


def config2(form="fp32", N=350, W=3e6, t_end=120e3, out_every=10e3, n_snap=None):
    domain, log10eta, T, H = config2_fields(N, W)
    solidearth = M.SolidEarth(domain, layer_boundaries=T.reshape(N, N, 1),
                              layer_viscosities=(10**log10eta).reshape(N, N, 1))
    n_snap = n_snap or int(round(t_end / 1e3)) + 1
    t_ice = np.arange(n_snap) * 1e3
    it = M.TimeInterpolatedIceThickness(list(t_ice), [H * m for m in sawtooth(t_ice)], domain)
    bcs = M.BoundaryConditions(domain, ice_thickness=it)
    sl = M.RegionalSeaLevel(surface=M.LaterallyVariableSeaSurface())
    nout = M.NativeOutput(t=list(np.arange(out_every, t_end + 1, out_every)))
    return M.Simulation(domain, bcs, sl, solidearth, (0.0, t_end), nout=nout, form=form)


def config3_members(n_members=128, seed=2024, t_end=20e3):
    rng = np.random.Generator(np.random.PCG64(seed))
    Ns = rng.choice([64, 96, 128, 192, 256], size=n_members)
    means = rng.uniform(20.0, 22.0, size=n_members)
    big_domain, _, _, H_rand = config2_fields(350, 3e6)
    members = []
    for m in range(n_members):
        N = int(Ns[m])
        W = 15e3 * N
        domain = M.RegionalDomain(W, W, N, N)
        g = gaussian_random_field(N, N, W, W, 500e3, 5000 + m)
        log10eta = np.clip(means[m] + 0.5 * g, 19, 23)
        # shared ice: disc + the config2 random field sampled at this grid's cells
        xi = np.clip(np.searchsorted(big_domain.x, domain.x), 0, 349)
        yi = np.clip(np.searchsorted(big_domain.y, domain.y), 0, 349)
        Hr = H_rand[np.ix_(xi, yi)]
        H = np.clip(_disc(domain) + Hr, 0, 4000)
        members.append({"N": N, "W": W, "log10eta": log10eta, "H": H, "domain": domain})
    t_ice = np.arange(int(round(t_end / 1e3)) + 1) * 1e3
    return members, t_ice, sawtooth(t_ice)


def config3_simulation(member, t_ice, mod, form="fp32", t_end=20e3):
    domain = member["domain"]
    N = member["N"]
    solidearth = M.SolidEarth(domain, layer_boundaries=[100e3],
                              layer_viscosities=(10**member["log10eta"]).reshape(N, N, 1))
    it = M.TimeInterpolatedIceThickness(list(t_ice), [member["H"] * m for m in mod], domain)
    bcs = M.BoundaryConditions(domain, ice_thickness=it)
    nout = M.NativeOutput(t=[t_end])
    return M.Simulation(domain, bcs, M.RegionalSeaLevel(), solidearth, (0.0, t_end), nout=nout, form=form)


def config5(form="fp32", N=1024, W=3e6, t_end=30e3, out_every=5e3):
    return config2(form=form, N=N, W=W, t_end=t_end, out_every=out_every)
