"""fi_rhs_noalloc (device buffers, result scratch in a static device array, no
allocation) against fi_rhs on two handles fed the same inputs.  The file name puts it
last in collection; it also passes when run alone."""
import ctypes as C

import numpy as np
import pytest

import fastiso_b200 as F
from fastiso_b200 import abi
from helpers import F_, TOL, rel_l2

pytestmark = pytest.mark.gpu


def _sim(nx, ny, form="fp32", seed=3):
    W_ = 0.75e6
    domain = F.RegionalDomain(W_, W_ * ny / nx, nx, ny)
    rng = np.random.default_rng(seed)
    log10eta = 21 + 0.5 * np.exp(-domain.R**2 / (2 * (W_ / 4) ** 2)) + 0.1 * rng.standard_normal((nx, ny))
    T = 100e3 + 20e3 * rng.random((nx, ny))
    se = F.SolidEarth(domain, layer_boundaries=T.reshape(nx, ny, 1),
                      layer_viscosities=(10**log10eta).reshape(nx, ny, 1))
    H1 = 1e3 * (domain.R < 0.4 * W_)
    it = F.TimeInterpolatedIceThickness([0.0, 1.0, 100.0], [domain.zeros(), H1, 1.3 * H1], domain)
    bcs = F.BoundaryConditions(domain, ice_thickness=it)
    sl = F.RegionalSeaLevel(surface=F.LaterallyVariableSeaSurface())
    return F.Simulation(domain, bcs, sl, se, (0.0, 100.0), form=form)


def _noalloc(sim, t, u_dev, dudt_dev):
    return sim.lib.fi_rhs_noalloc(sim._handle, float(t), C.c_void_p(u_dev.data_ptr()),
                                  C.c_void_p(dudt_dev.data_ptr()))


def test_rhs_noalloc_matches_fi_rhs():
    torch = pytest.importorskip("torch")
    nx, ny = 48, 40
    a, b = _sim(nx, ny), _sim(nx, ny)
    a.init_problem()
    b.init_problem()
    rng = np.random.default_rng(7)
    u = -50 * np.exp(-a.domain.R**2 / (2 * (0.3 * a.domain.Wx) ** 2)) + 0.5 * rng.standard_normal((nx, ny))
    # two calls in a row; the second one (t - t0 >= 10 yr) also runs the sparse update
    for t in (0.5, 12.5):
        ua, da = u.copy(), np.zeros_like(u)
        F.update_diagnostics(da, ua, a, t)
        u_dev = torch.from_numpy(F_(u)).to("cuda:0")
        dudt_dev = torch.full_like(u_dev, float("nan"))
        torch.cuda.synchronize()
        rc = _noalloc(b, t, u_dev, dudt_dev)
        assert rc == abi.FI_OK, b.lib.fi_last_error(b._handle)
        assert rel_l2(u_dev.cpu().numpy(), F_(ua)) < 1e-12
        assert rel_l2(dudt_dev.cpu().numpy(), F_(da)) < TOL["fp32"]
        for name in ("ue", "dz_ss"):
            assert rel_l2(F_(b.get_field(name)), F_(a.get_field(name))) < TOL["fp32"], name


def test_rhs_noalloc_rejects_oversized_grid_and_fp64_form():
    torch = pytest.importorskip("torch")
    big = _sim(1040, 1032)
    big._ensure_handle()  # created, not initialised: the size check comes first
    buf = torch.zeros(1040 * 1032, dtype=torch.float64, device="cuda:0")
    assert _noalloc(big, 0.0, buf, buf) == abi.FI_ERR_ARG
    assert b"static scratch limit" in big.lib.fi_last_error(big._handle)
    big.close()
    s64 = _sim(16, 16, form="fp64")
    s64.init_problem()
    buf = torch.zeros(16 * 16, dtype=torch.float64, device="cuda:0")
    assert _noalloc(s64, 0.0, buf, buf) == abi.FI_ERR_ARG


def test_rhs_noalloc_leaves_device_memory_unchanged():
    """After a first call on the device (which looks up the scratch address), 100 more
    calls change neither the device's free memory (cudaMemGetInfo) nor torch's
    reserved pool: the entry point allocates nothing per call."""
    torch = pytest.importorskip("torch")
    nx, ny = 48, 40
    b = _sim(nx, ny)
    b.init_problem()
    rng = np.random.default_rng(5)
    u = -50 * np.exp(-b.domain.R**2 / (2 * (0.3 * b.domain.Wx) ** 2)) + 0.5 * rng.standard_normal((nx, ny))
    u_dev = torch.from_numpy(F_(u)).to("cuda:0")
    dudt_dev = torch.empty_like(u_dev)
    assert _noalloc(b, 0.5, u_dev, dudt_dev) == abi.FI_OK
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    reserved0 = torch.cuda.memory_reserved(0)
    for k in range(100):
        assert _noalloc(b, 0.5 + 0.25 * k, u_dev, dudt_dev) == abi.FI_OK
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0, (free0, free1)
    assert torch.cuda.memory_reserved(0) == reserved0
    assert torch.isfinite(dudt_dev).all()
    b.close()
