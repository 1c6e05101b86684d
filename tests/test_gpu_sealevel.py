"""GPU parity of the sea-level rows (interactive sea-level load, barystatic sea level,
masks, water column, volume terms; src/loads.jl:56-85, src/sealevel.jl:242-332,
src/barystatic_sealevel.jl:215-235, src/topography.jl:1-28) against the FP64 oracle.
Tolerances as the other parity tests: per right-hand side 1e-10 (plain FP64 form) and
1e-6 (FP32 form); runs replay the oracle's attempt sequence (1e-9 FP64, 1e-4 FP32)."""
import numpy as np
import pytest

import fastiso_b200 as F
from fastiso_b200 import abi
from helpers import F_, TOL, lib_outputs, ocean_surface_table, oracle_for, oracle_outputs, rel_l2, sealevel_sim

pytestmark = pytest.mark.gpu

RUN_GATE = {"fp64": 1e-9, "fp32": 1e-4}


def _bsl(kind):
    if kind == "constant":
        return F.ConstantBSL()
    if kind == "ocean_surface":
        return F.ConstantOceanSurfaceBSL()
    if kind == "piecewise":
        z, A = ocean_surface_table()
        return F.PiecewiseConstantBSL(ref=F.ReferenceBSL(z_vec=list(z), A_vec=list(A)))
    return F.ImposedBSL(t_vec=[0.0, 50.0, 400.0], z_vec=[0.0, -10.0, -40.0])


CASES = [("fp64", "constant"), ("fp64", "ocean_surface"), ("fp64", "piecewise"), ("fp64", "imposed"),
         ("fp32", "constant"), ("fp32", "imposed")]


def _u0(sim, seed=4):
    rng = np.random.default_rng(seed)
    d = sim.domain
    return -60 * np.exp(-d.R**2 / (2 * (0.25 * d.Wx) ** 2)) + 0.5 * rng.standard_normal((d.nx, d.ny))


@pytest.mark.parametrize("form,bsl", CASES)
def test_sealevel_rhs_parity(form, bsl):
    sim = sealevel_sim(form, bsl=_bsl(bsl), adjustment=(bsl == "ocean_surface"), t_end=400.0)
    ref = oracle_for(sim)
    ref.init()
    sim.init_problem()
    u = _u0(sim)

    def surfaces():
        # the masks change only in a sparse update: keep the surfaces they were made from
        return (ref.get_field(abi.FIELDS["z_ss"]) - ref.get_field(abi.FIELDS["z_b"]),
                ref.get_field(abi.FIELDS["H_af"]).copy())

    w_gate, haf_gate = surfaces()
    for t in (0.5, 12.5, 12.7, 31.0):
        ug, dg = u.copy(), np.zeros_like(u)
        F.update_diagnostics(dg, ug, sim, t)
        ns0 = ref.stats()["nsparse"]
        ur, dr = ref.rhs(t, F_(u))
        if ref.stats()["nsparse"] > ns0:
            w_gate, haf_gate = surfaces()
        assert rel_l2(F_(dg), dr) < TOL[form], (t, rel_l2(F_(dg), dr))
        for name in ("dz_ss", "columnanom_seawater", "H_water"):
            # the water column and its anomaly are differences of O(km) surfaces
            # (sea surface minus bedrock, minus the reference column): in FP64 they
            # carry ~1e-10 of cancellation, hence 10x the right-hand-side tolerance
            e = rel_l2(F_(sim.get_field(name)), ref.get_field(abi.FIELDS[name]))
            assert e < TOL[form] * (1 if name == "dz_ss" and form == "fp64" else 10), (t, name, e)
        for name in ("maskgrounded", "maskocean"):
            a, b = F_(sim.get_field(name)), ref.get_field(abi.FIELDS[name])
            # a mask is a sign test of a difference of surfaces: in FP64 only cells within
            # rounding of the threshold may flip
            if form == "fp64":
                # maskocean flips at w = z_ss - z_b = 0, maskgrounded where H_af leaves 0, both
                # taken at the last sparse update; FP64 may differ only within rounding of them
                bad = np.nonzero(a != b)[0]
                edge = np.abs(w_gate[bad]) if name == "maskocean" else np.abs(haf_gate[bad])
                assert bad.size == 0 or edge.max() < 1e-6, (t, name, bad.tolist(), edge.tolist())
            else:
                assert np.mean(a != b) <= 0.01, (t, name, int(np.sum(a != b)))
        sg, sr = sim.sealevel_state(), ref.sealevel()
        assert abs(sg["z_bsl"] - sr["z_bsl"]) <= 1e-9 * max(1.0, abs(sr["z_bsl"])), (t, sg, sr)
        if form == "fp64":
            vol = abs(sr["V_af"]) + abs(sr["V_den"]) + abs(sr["V_pov"])
            for k in ("V_af", "V_den", "V_pov", "delta_V", "A_bsl"):
                # delta_V is a difference of volume sums (~1e15 m^3): rounding of the sums
                scale = max(1.0, vol) if k == "delta_V" else max(1.0, abs(sr[k]))
                assert abs(sg[k] - sr[k]) <= 1e-9 * scale, (t, k, sg[k], sr[k])
    assert np.abs(ref.get_field(abi.FIELDS["columnanom_seawater"])).max() > 0
    ref.close()
    sim.close()


@pytest.mark.parametrize("form,bsl", CASES)
def test_sealevel_run_parity_replayed(form, bsl):
    t_outs = [50.0, 150.0, 300.0]
    sim = sealevel_sim(form, bsl=_bsl(bsl), adjustment=(bsl == "ocean_surface"), t_end=300.0)
    ref = oracle_for(sim)
    ref.init()
    fields = ("u", "dudt", "dz_ss", "columnanom_seawater")
    out_r, rec = oracle_outputs(ref, t_outs, fields=fields, record=1 << 20)
    sl_r = ref.sealevel()
    ref.close()
    out_g, _ = lib_outputs(sim, t_outs, fields=fields, replay=rec)
    sl_g = sim.sealevel_state()
    sim.close()
    for f in fields:
        errs = [rel_l2(a, b) for a, b in zip(out_g[f], out_r[f])]
        assert max(errs) < RUN_GATE[form] * (10 if f == "columnanom_seawater" else 1), (f, errs)
    assert abs(sl_g["z_bsl"] - sl_r["z_bsl"]) <= 1e-8 * max(1.0, abs(sl_r["z_bsl"]))


def test_fp32_rejects_volume_driven_bsl():
    sim = sealevel_sim("fp32", bsl=F.ConstantOceanSurfaceBSL())
    with pytest.raises(abi.FiError) as e:
        sim.init_problem()
    assert e.value.code == abi.FI_ERR_UNSUPPORTED
    sim.close()
