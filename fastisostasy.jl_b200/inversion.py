"""Unscented Kalman inversion (UKI) of solid-Earth parameters over the batched engine.

The reference's inversion layer (src/inversion.jl: InversionConfig, InversionData,
InversionProblem, ParameterReduction with reconstruct!/extract_output, and the
EnsembleKalmanProcesses extension ext/FastIsostasyEnsembleKalmanProcessesExt.jl:47-141:
inversion_problem, solve!, extract_inversion) runs one forward simulation per sigma
point on host threads.  Here every iteration's sigma points are the members of one
batched ensemble (fi_ensemble_*: all members advance in one persistent launch per
segment), and the Kalman update runs on the host in FP64.

UKI itself lives in the third-party package EnsembleKalmanProcesses.jl (compat "2.0",
Project.toml:49), which is not part of the reference tree.  It is restated from its
published form (Huang, Schneider & Stuart 2022, "Iterated Kalman methodology for inverse
problems", J. Comput. Phys. 463, the "modified unscented transform" that the package uses
by default):

  prediction   m^ = r + alpha (m - r),  C^ = alpha^2 C + Sigma_w,  Sigma_w = (2 - alpha^2) Lambda
               (r, the prior mean; Lambda, the prior covariance, replaced by the current
               covariance every `update_freq` iterations when update_freq > 0)
  sigma points th_0 = m^,  th_{j, j+N} = m^ +- c [sqrt C^]_j,  c = a sqrt(N),
               a = min(sqrt(4 / N), 1)
  analysis     y^ = G(th_0),  C_tp = sum_j w (th_j - m^)(G(th_j) - y^)^T,
               C_pp = sum_j w (G(th_j) - y^)(G(th_j) - y^)^T + Sigma_v,  w = 1 / (2 a^2 N),
               Sigma_v = 2 Sigma_eta,  K = C_tp C_pp^-1,
               m = m^ + K (y - y^),  C = C^ - K C_tp^T.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import model as M


@dataclass
class InversionConfig:
    """InversionConfig(method, N_ens, N_iter, n_samples; alpha_reg, update_freq,
    scale_obscov) (src/inversion.jl:26-42)."""

    method: str = "UKI"
    N_ens: int = 0          # the UKI ensemble is 2 N_params + 1 sigma points
    N_iter: int = 10
    n_samples: int = 100    # noisy realisations of the data whose mean is observed
    alpha_reg: float = 1.0
    update_freq: int = 1
    scale_obscov: float = 1000.0


@dataclass
class InversionData:
    """InversionData(t, Y, mask) (src/inversion.jl:57-71): observation times, the
    observed fields at those times and the region of interest."""

    t: list
    Y: list
    mask: np.ndarray
    nY: int = field(init=False)
    countmask: int = field(init=False)

    def __post_init__(self):
        self.mask = np.asarray(self.mask, bool)
        self.nY = len(self.Y)
        self.countmask = int(self.mask.sum())

    @property
    def y(self):
        return np.concatenate([np.asarray(Yk)[self.mask] for Yk in self.Y])


class ParameterReduction:
    """ParameterReduction (src/inversion.jl:1-8): maps a parameter vector to a
    Simulation (`reconstruct`) and a Simulation's outputs to the observed vector
    (`extract_output`)."""

    nparams = 0

    def reconstruct(self, theta) -> M.Simulation:
        raise NotImplementedError

    def extract_output(self, outputs, data: InversionData) -> np.ndarray:
        return np.concatenate([np.asarray(o)[data.mask] for o in outputs])


class ViscosityRegions(ParameterReduction):
    """The upper-mantle log10 viscosity of each region of a partition of the domain:
    theta_i is log10 eta on region i.  `make_sim(log10eta)` builds the Simulation
    of a viscosity map (the rest of its inputs fixed)."""

    def __init__(self, regions, make_sim):
        self.regions = [np.asarray(r, bool) for r in regions]
        self.nparams = len(self.regions)
        self.make_sim = make_sim

    def field(self, theta):
        theta = np.asarray(theta, float)
        out = np.zeros(self.regions[0].shape)
        for r, v in zip(self.regions, theta):
            out[r] = v
        return out

    def reconstruct(self, theta):
        return self.make_sim(self.field(theta))


class UnscentedKalman:
    """The UKI iteration (module docstring) on a parameter vector of size N."""

    def __init__(self, prior_mean, prior_cov, obs_mean, obs_cov, alpha_reg=1.0, update_freq=1):
        self.r = np.asarray(prior_mean, float).copy()
        self.m = self.r.copy()
        self.C = np.asarray(prior_cov, float).copy()
        self.Lam = self.C.copy()
        self.y = np.asarray(obs_mean, float)
        self.Gam = np.asarray(obs_cov, float)
        self.alpha = float(alpha_reg)
        self.update_freq = int(update_freq)
        self.N = self.r.size
        self.a = min(np.sqrt(4.0 / self.N), 1.0)
        self.c = self.a * np.sqrt(self.N)
        self.w = 1.0 / (2.0 * self.a**2 * self.N)
        self.iter = 0
        self.errors = []
        self.m_hat = None
        self.C_hat = None

    def sigma_points(self):
        """Prediction step, then the 2N + 1 sigma points (columns)."""
        a = self.alpha
        self.m_hat = self.r + a * (self.m - self.r)
        self.C_hat = a**2 * self.C + (2.0 - a**2) * self.Lam
        L = np.linalg.cholesky(0.5 * (self.C_hat + self.C_hat.T))
        pts = np.empty((self.N, 2 * self.N + 1))
        pts[:, 0] = self.m_hat
        for j in range(self.N):
            pts[:, 1 + j] = self.m_hat + self.c * L[:, j]
            pts[:, 1 + self.N + j] = self.m_hat - self.c * L[:, j]
        self._pts = pts
        return pts

    def update(self, G):
        """Analysis step with the forward outputs G (one column per sigma point of the
        last sigma_points() call)."""
        G = np.asarray(G, float)
        yh = G[:, 0]
        dth = self._pts - self.m_hat[:, None]
        dG = G[:, 1:] - yh[:, None]
        C_tp = self.w * dth[:, 1:] @ dG.T
        C_pp = self.w * dG @ dG.T + 2.0 * self.Gam
        K = np.linalg.solve(C_pp.T, C_tp.T).T
        self.m = self.m_hat + K @ (self.y - yh)
        self.C = self.C_hat - K @ C_tp.T
        self.C = 0.5 * (self.C + self.C.T)
        self.iter += 1
        if self.update_freq > 0 and self.iter % self.update_freq == 0:
            self.Lam = self.C.copy()
        r = self.y - yh
        self.errors.append(float(r @ np.linalg.solve(self.Gam, r)))
        return self.m

    def step(self, forward):
        """One iteration: sigma points -> forward(points) -> analysis."""
        return self.update(forward(self.sigma_points()))


def uncorrelated_obs_covariance(scale_obscov, loadscaling):
    """diag(scale / (loadscaling + 1)) (ext/FastIsostasyEnsembleKalmanProcessesExt.jl:95-98)."""
    return np.diag(scale_obscov / (np.asarray(loadscaling, float) + 1.0))


@dataclass
class InversionProblem:
    """InversionProblem (src/inversion.jl:90-103)."""

    config: InversionConfig
    data: InversionData
    reduction: ParameterReduction
    prior_mean: np.ndarray
    prior_cov: np.ndarray
    uki: UnscentedKalman
    error: list
    out: list
    G_ens: np.ndarray | None = None
    forward_launches: int = 0


def inversion_problem(config, data, reduction, prior_mean, prior_cov, seed=0):
    """inversion_problem (ext/FastIsostasyEnsembleKalmanProcessesExt.jl:47-93): noisy
    realisations of the observed vector with covariance Sigma_y, their mean as the
    observation, and the UKI process on the priors."""
    y = data.y
    Sigma_y = uncorrelated_obs_covariance(config.scale_obscov, np.ones(y.size))
    rng = np.random.default_rng(seed)
    # MvNormal(0, Sigma_y) with a diagonal Sigma_y: independent normal components
    yn = y[:, None] + np.sqrt(np.diag(Sigma_y))[:, None] * rng.standard_normal((y.size, config.n_samples))
    uki = UnscentedKalman(prior_mean, prior_cov, yn.mean(axis=1), Sigma_y, config.alpha_reg, config.update_freq)
    return InversionProblem(config, data, reduction, np.asarray(prior_mean, float), np.asarray(prior_cov, float),
                            uki, [], [uki.m.copy()])


def forward_ensemble(reduction, data, thetas):
    """The forward model of every sigma point at once: one FP32 Simulation per column
    of thetas, all advanced together by the batched ensemble engine; the observed
    vector of each member at the data times."""
    sims = [reduction.reconstruct(thetas[:, j]) for j in range(thetas.shape[1])]
    ens = M.Ensemble(sims)
    outs = [[] for _ in sims]
    t_prev = sims[0].t_span[0]
    for t in data.t:
        if t > t_prev:
            st = ens.step(t - t_prev)
            if any(s != 0 for s in st):
                raise RuntimeError(f"ensemble members failed: {st}")
            t_prev = t
        for j, s in enumerate(sims):
            outs[j].append(s.get_field("u"))
    G = np.stack([reduction.extract_output(o, data) for o in outs], axis=1)
    ens.close()
    for s in sims:
        s.close()
    return G


def solve(paraminv: InversionProblem, forward=None, verbose=False):
    """solve!(paraminv) (ext/FastIsostasyEnsembleKalmanProcessesExt.jl:103-141):
    N_iter UKI iterations, the sigma points of each run as one batched ensemble."""
    fwd = forward or (lambda th: forward_ensemble(paraminv.reduction, paraminv.data, th))
    for n in range(paraminv.config.N_iter):
        def wrapped(th):
            G = fwd(th)
            paraminv.G_ens = G
            paraminv.forward_launches += 1
            return G
        paraminv.uki.step(wrapped)
        paraminv.error.append(paraminv.uki.errors[-1])
        paraminv.out.append(paraminv.uki.m.copy())
        if verbose:
            print(f"UKI iteration {n + 1}: error {paraminv.error[-1]:.4g}, mean {paraminv.uki.m}")
    return paraminv


def extract_inversion(paraminv: InversionProblem):
    """extract_inversion (ext/FastIsostasyEnsembleKalmanProcessesExt.jl:158-163): the
    parameter mean, the forward output at it (the central sigma point of the last
    iteration) and the absolute misfit."""
    p = paraminv.uki.m.copy()
    Gx = paraminv.G_ens[:, 0] if paraminv.G_ens is not None else None
    abserror = np.abs(paraminv.data.y - Gx) if Gx is not None else None
    return p, Gx, abserror
