"""UKI over the batched ensemble engine (fastiso_b200.inversion; the reference's
ext/FastIsostasyEnsembleKalmanProcessesExt.jl:47-163): recover the log10 viscosity of
two regions from synthetic displacement data; every iteration's five sigma points run
as one ensemble on the GPU."""
import numpy as np
import pytest

import fastiso_b200 as F
from fastiso_b200 import inversion as I

pytestmark = pytest.mark.gpu

N, W_ = 40, 1.2e6


def _make_sim(log10eta):
    domain = F.RegionalDomain(W_, W_, N, N)
    se = F.SolidEarth(domain, layer_boundaries=[100e3], layer_viscosities=(10**log10eta).reshape(N, N, 1))
    H1 = 1.5e3 * (domain.R < 5e5)
    it = F.TimeInterpolatedIceThickness([0.0, 1.0, 1e3], [domain.zeros(), H1, H1], domain)
    bcs = F.BoundaryConditions(domain, ice_thickness=it)
    return F.Simulation(domain, bcs, F.RegionalSeaLevel(), se, (0.0, 600.0), nout=F.NativeOutput(t=[600.0]))


def test_uki_recovers_two_region_viscosity():
    domain = F.RegionalDomain(W_, W_, N, N)
    regions = [domain.X < 0, domain.X >= 0]
    red = I.ViscosityRegions(regions, _make_sim)
    truth = np.array([20.6, 21.3])
    t_obs = [200.0, 600.0]
    G_true = I.forward_ensemble(red, I.InversionData(t=t_obs, Y=[domain.zeros()] * 2, mask=domain.R < 8e5),
                                truth[:, None])
    mask = domain.R < 8e5
    k = int(mask.sum())
    Y = [np.zeros((N, N)), np.zeros((N, N))]
    Y[0][mask] = G_true[:k, 0]
    Y[1][mask] = G_true[k:, 0]
    data = I.InversionData(t=t_obs, Y=Y, mask=mask)
    cfg = I.InversionConfig(N_iter=6, n_samples=20, scale_obscov=1e-4)
    p = I.inversion_problem(cfg, data, red, prior_mean=[21.0, 21.0], prior_cov=0.25 * np.eye(2))
    I.solve(p)
    params, Gx, abserr = I.extract_inversion(p)
    assert np.abs(params - truth).max() < 0.05, params
    assert p.error[-1] < p.error[0]
    assert p.forward_launches == 6 and p.G_ens.shape == (2 * k, 5)
