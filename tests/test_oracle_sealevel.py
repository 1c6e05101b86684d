"""The oracle's sea-level rows (interactive sea-level load, barystatic sea level,
masks, water column, volume terms), checked on the CPU against identities the
reference's own definitions imply (src/loads.jl:56-85, src/sealevel.jl:242-332,
src/barystatic_sealevel.jl:215-235, src/topography.jl:1-28)."""
import numpy as np
import pytest

import fastiso_b200 as F
from fastiso_b200 import abi
from helpers import ocean_surface_table, oracle_for, sealevel_sim

RHO_SW, RHO_I, RHO_W = 1023.0, 910.0, 1000.0


def _run(sim, t_outs):
    ref = oracle_for(sim)
    ref.init()
    sl0 = ref.sealevel()
    ref.init_integrator(np.asarray(t_outs, float))
    for t in t_outs:
        ref.step(t - ref.stats()["t"])
    return ref, sl0


def _field(ref, name):
    return ref.get_field(abi.FIELDS[name])


def test_masks_water_column_and_seawater_anomaly():
    sim = sealevel_sim("fp64", t_end=100.0)
    ref, _ = _run(sim, [60.0])
    # one more right-hand side past the next 10-yr mark runs the sparse update: every
    # field below then belongs to that call
    n0 = ref.stats()["nsparse"]
    ref.rhs(85.0, _field(ref, "u"))
    assert ref.stats()["nsparse"] == n0 + 1
    H, Haf = _field(ref, "H_ice"), _field(ref, "H_af")
    zss, zb = _field(ref, "z_ss"), _field(ref, "z_b")
    gr, oc = _field(ref, "maskgrounded"), _field(ref, "maskocean")
    sw, hw = _field(ref, "columnanom_seawater"), _field(ref, "H_water")
    np.testing.assert_array_equal(gr, (Haf > 0).astype(float))
    assert oc.sum() > 0 and gr.sum() > 0, "the case needs both ocean and grounded ice"
    np.testing.assert_array_equal(oc, ((zss - zb > 0) & (gr == 0)).astype(float))
    wc = np.maximum(zss - zb, 0)
    np.testing.assert_allclose(hw, np.where(H <= 1, wc, 0) + np.where((gr == 0) & (H > 1), wc - H * RHO_I / RHO_SW, 0),
                               rtol=0, atol=1e-9)
    zss_ref = 0.0 + sim.dz_ss_ref.ravel(order="F")
    mask = sim.solidearth.maskactive.ravel(order="F").astype(float)
    np.testing.assert_allclose(sw, RHO_SW * (zss - zss_ref) * oc * mask, rtol=1e-12, atol=1e-9)
    assert np.abs(sw).max() > 0
    # ConstantBSL keeps the level; the volumes are the Goelzer sums of the last update
    sl = ref.sealevel()
    assert sl["z_bsl"] == 0.0 and sl["tracked"] == 1
    assert sl["V_pov"] == 0.0 and sl["V_af"] > 0 and sl["V_den"] > 0
    ref.close()
    sim.close()


def test_constant_ocean_surface_bsl_telescopes():
    """z_bsl = ref.z - (V(t_last) - V(0)) / ref.A: each sparse update adds -delta_V / A."""
    sim = sealevel_sim("fp64", bsl=F.ConstantOceanSurfaceBSL(), adjustment=True, t_end=300.0)
    ref, sl0 = _run(sim, [100.0, 300.0])
    sl = ref.sealevel()
    V0 = sl0["V_af"] + sl0["V_den"] + sl0["V_pov"]
    V1 = sl["V_af"] + sl["V_den"] + sl["V_pov"]
    assert V0 > 0 and sl["V_pov"] > 0
    assert abs(sl["z_bsl"] - (0.0 - (V1 - V0) / abi.A_OCEAN_PD)) < 1e-12 * max(1.0, abs(sl["z_bsl"]))
    assert sl["z_bsl"] != 0.0
    ref.close()
    sim.close()


def test_piecewise_constant_and_imposed_bsl():
    z, A = ocean_surface_table()
    sim = sealevel_sim("fp64", bsl=F.PiecewiseConstantBSL(ref=F.ReferenceBSL(z_vec=list(z), A_vec=list(A))),
                       t_end=120.0)
    ref, _ = _run(sim, [120.0])
    sl = ref.sealevel()
    assert sl["z_bsl"] != 0.0
    np.testing.assert_allclose(sl["A_bsl"], np.interp(sl["z_bsl"], z, A), rtol=1e-13)
    ref.close()
    sim.close()
    th, zh = [0.0, 50.0, 400.0], [0.0, -10.0, -40.0]
    sim = sealevel_sim("fp64", bsl=F.ImposedBSL(t_vec=th, z_vec=zh), t_end=120.0)
    ref, _ = _run(sim, [120.0])
    # the last sparse update ran at the first stage time t >= 120 - 10 crossing a 10-yr mark
    zss = _field(ref, "z_ss")
    assert -40.0 < ref.sealevel()["z_bsl"] < -10.0
    assert np.isfinite(zss).all()
    ref.close()
    sim.close()


def test_interactive_load_mask_limit():
    sim = sealevel_sim("fp64", t_end=60.0)
    sim.solidearth.maskactive[:] = True
    ref = oracle_for(sim)
    with pytest.raises(RuntimeError, match="60%"):
        ref.init()
    ref.close()
    sim.close()
