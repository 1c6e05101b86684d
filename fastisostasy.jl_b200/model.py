"""Host-side mirror of the FastIsostasy.jl user API for the LV-ELVA path.

The types keep the reference's names and argument meaning (Julia ``!`` dropped):

  RegionalDomain            src/domain.jl:35-169
  PhysicalConstants         src/constants.jl:16-28
  SolidEarth + tags         src/solidearth.jl:13-234, src/material.jl:10-278
  BoundaryConditions        src/boundary_conditions.jl:1-325
  RegionalSeaLevel + tags   src/sealevel.jl:103-166, src/barystatic_sealevel.jl:88-110
  SolverOptions             src/simulation.jl:11-26
  NativeOutput              src/io.jl:336-353
  Simulation, run, init_integrator, step, update_diagnostics
                            src/simulation.jl:77-393

Everything here is set-up and marshalling: the time loop, the right-hand side and
all per-step arithmetic run in ``libfastiso_b200.so`` on the GPU.  Element
``a[i, j]`` of every numpy field is cell (x_i, y_j), as in the reference's
column-major matrices; it crosses the C ABI with x fastest.
"""
from __future__ import annotations

import ctypes as C
import math
import pathlib
from dataclasses import dataclass, field

import numpy as np

from . import abi

# ---------------------------------------------------------------------------
# tags (src/solidearth.jl:13-109, src/material.jl:29-118, src/sealevel.jl:114-166)
# ---------------------------------------------------------------------------


class _Tag:
    def __repr__(self):
        return f"{type(self).__name__}()"

    def __eq__(self, other):
        return type(self) is type(other)

    def __hash__(self):
        return hash(type(self).__name__)


class LaterallyVariableLithosphere(_Tag): pass
class LaterallyConstantLithosphere(_Tag): pass
class RigidLithosphere(_Tag): pass
class MaxwellMantle(_Tag): pass
class RelaxedMantle(_Tag): pass
class RigidMantle(_Tag): pass
class CompressibleMantle(_Tag): pass
class IncompressibleMantle(_Tag): pass
class NoCalibration(_Tag): pass
class FreqDomainViscosityLumping(_Tag): pass
class TimeDomainViscosityLumping(_Tag): pass
class MeanViscosityLumping(_Tag): pass
class MeanLogViscosityLumping(_Tag): pass
class IncompressibleLithosphereColumn(_Tag): pass
class CompressibleLithosphereColumn(_Tag): pass
class LaterallyConstantSeaSurface(_Tag): pass
class LaterallyVariableSeaSurface(_Tag): pass
class NoSealevelLoad(_Tag): pass
class InteractiveSealevelLoad(_Tag): pass
class InternalBSLUpdate(_Tag): pass
class ExternalBSLUpdate(_Tag): pass
class NoVolumeContribution(_Tag): pass
class GoelzerVolumeContribution(_Tag): pass
class NoDensityContribution(_Tag): pass
class GoelzerDensityContribution(_Tag): pass
class NoAdjustmentContribution(_Tag): pass
class GoelzerAdjustmentContribution(_Tag): pass
class RegularBCSpace(_Tag): pass
class ExtendedBCSpace(_Tag): pass


@dataclass
class SeakonCalibration:
    ref_viscosity: float = float(np.float32(1e21))


@dataclass
class ReferenceBSL:
    """ReferenceBSL(z) (src/barystatic_sealevel.jl:3-42): the reference level z, its
    ocean area A and the table A(z) of PiecewiseConstantBSL.  The reference downloads
    the ocean-surface table; here the caller supplies it (z_vec, A_vec, already
    unbiased so that A(0) = A_OCEAN_PD) when a BSL needs it, and A defaults to
    A_OCEAN_PD, its value at z = 0."""

    z: float = 0.0
    A: float = 3.625e14
    z_vec: list | None = None
    A_vec: list | None = None


@dataclass
class ConstantBSL:
    """ConstantBSL(; ref): z = ref.z for ever (src/barystatic_sealevel.jl:100-110, 215-218)."""

    ref: ReferenceBSL = field(default_factory=ReferenceBSL)

    @property
    def z(self):
        return self.ref.z

    @property
    def A(self):
        return self.ref.A


@dataclass
class ConstantOceanSurfaceBSL(ConstantBSL):
    """z += delta_V / ref.A at every sparse update (src/barystatic_sealevel.jl:220-224)."""


@dataclass
class PiecewiseConstantBSL(ConstantBSL):
    """z += delta_V / A, then A = A(z) from ref's table (src/barystatic_sealevel.jl:226-230)."""


@dataclass
class ImposedBSL(ConstantBSL):
    """z = z(t) linear in the given history (src/barystatic_sealevel.jl:172-181, 232-235)."""

    t_vec: list = field(default_factory=list)
    z_vec: list = field(default_factory=list)


class UnsupportedError(NotImplementedError):
    """Raised for options outside the LV-ELVA hot path."""


# ---------------------------------------------------------------------------
# RegionalDomain (src/domain.jl:70-169)
# ---------------------------------------------------------------------------


def fftint(N: int) -> np.ndarray:
    """src/derivatives.jl:216-223"""
    N2 = N // 2
    if N % 2 == 0:
        return np.concatenate([np.arange(0, N2 + 1), np.arange(N2 - 1, 0, -1)]).astype(np.float64)
    return np.concatenate([np.arange(0, N2 + 1), np.arange(N2, 0, -1)]).astype(np.float64)


def samesize_conv_indices(N: int, M: int):
    """src/convolutions.jl:196-204 (1-based)"""
    j1 = M if N % 2 == 0 else M + 1
    return j1, 2 * N - 1 - M


def nextfastfft(n: int) -> int:
    """nextprod((2, 3, 5, 7), n), src/convolutions.jl:17-19"""
    m = max(int(n), 1)
    while True:
        r = m
        for p in (2, 3, 5, 7):
            while r % p == 0:
                r //= p
        if r == 1:
            return m
        m += 1


class RegionalDomain:
    """RegionalDomain(W, n) or RegionalDomain(Wx, Wy, nx, ny).

    ``correct_distortion=True`` (stereographic scale factor K != 1) is outside the
    path: K is identically one here, as in the reference default."""

    def __init__(self, Wx, Wy_or_n=None, nx=None, ny=None, *, correct_distortion=False, use_cuda=True):
        if correct_distortion:
            raise UnsupportedError("correct_distortion=True (K != 1) is outside the LV-ELVA path")
        if nx is None:
            n = int(Wy_or_n)
            Wx, Wy, nx, ny = float(Wx), float(Wx), 2**n, 2**n
        else:
            Wy = float(Wy_or_n)
        self.Wx, self.Wy, self.nx, self.ny = float(Wx), float(Wy), int(nx), int(ny)
        self.mx, self.my = self.nx // 2, self.ny // 2
        self.dx = 2 * self.Wx / self.nx
        self.dy = 2 * self.Wy / self.ny
        self.x = np.linspace(-self.Wx + self.dx, self.Wx, self.nx)
        self.y = np.linspace(-self.Wy + self.dy, self.Wy, self.ny)
        self.X, self.Y = np.meshgrid(self.x, self.y, indexing="ij")
        self.R = np.sqrt(self.X**2 + self.Y**2)
        self.K = np.ones((self.nx, self.ny))
        self.Dx, self.Dy = self.K * self.dx, self.K * self.dy
        self.A = (self.dx * self.dy) * self.K**2
        self.i1, self.i2 = samesize_conv_indices(self.nx, self.mx)
        self.j1, self.j2 = samesize_conv_indices(self.ny, self.my)
        self.convo_offset = 0
        self.correct_distortion = False
        self.use_cuda = use_cuda
        mux, muy = math.pi / self.Wx, math.pi / self.Wy
        Xc, Yc = np.meshgrid(mux * fftint(self.nx), muy * fftint(self.ny), indexing="ij")
        self.pseudodiff = np.sqrt(Xc**2 + Yc**2)
        self.pseudodiff[0, 0] = 1e-3 * ((self.pseudodiff[0, 1] + self.pseudodiff[1, 0]) / 2)

    def zeros(self):
        return np.zeros((self.nx, self.ny))

    def fill(self, v):
        return np.full((self.nx, self.ny), float(v))


# ---------------------------------------------------------------------------
# PhysicalConstants (src/constants.jl:16-28)
# ---------------------------------------------------------------------------


@dataclass
class PhysicalConstants:
    mE: float = 5.972e24
    r_equator: float = 6371e3
    r_pole: float = 6357e3
    A_ocean_pd: float = 3.625e14
    g: float = 9.8
    G: float = 6.674e-11
    seconds_per_year: float = abi.SECONDS_PER_YEAR
    rho_ice: float = 0.910e3
    rho_water: float = 1e3
    rho_seawater: float = 1.023e3

    @property
    def rho_sw_ice(self):
        return self.rho_seawater / self.rho_ice


# ---------------------------------------------------------------------------
# SolidEarth (src/solidearth.jl:175-234; material laws src/material.jl)
# ---------------------------------------------------------------------------


def get_rigidity(t, E, nu):
    """src/material.jl:10"""
    return (E * t**3) / (12 * (1 - nu**2))


def _matrify(v, nx, ny):
    v = np.asarray(v, dtype=np.float64)
    if v.ndim == 1:
        return np.broadcast_to(v[None, None, :], (nx, ny, v.size)).copy()
    if v.ndim == 2:
        return v[:, :, None].copy()
    return v.copy()


class SolidEarth:
    """SolidEarth(domain; layer_boundaries, layer_viscosities, ...).

    Only the LaterallyVariableLithosphere + MaxwellMantle branch of update_dudt!
    (src/deformation.jl:91-103) is the hot path; RigidLithosphere is accepted for
    the elastic response (ue = 0).  The channel-scaling factor R(|k|) of the
    frequency-domain lumping is evaluated in FP64 on the GPU from the per-channel
    means computed here (src/material.jl:154-179, 264-278)."""

    def __init__(self, domain: RegionalDomain, *, lithosphere=None, mantle=None, calibration=None,
                 compressibility=None, lumping=None, lithosphere_column=None, maskactive=None,
                 layer_boundaries=(88e3, 400e3), layer_viscosities=(1e19, 1e21), litho_youngmodulus=6.6e10,
                 litho_poissonratio=0.28, mantle_poissonratio=0.28, tau=855.0, scale_elralength=1.0,
                 rho_uppermantle=3.4e3, rho_litho=3.2e3):
        self.lithosphere = lithosphere or LaterallyVariableLithosphere()
        self.mantle = mantle or MaxwellMantle()
        self.calibration = calibration or NoCalibration()
        self.compressibility = compressibility or CompressibleMantle()
        self.lumping = lumping or FreqDomainViscosityLumping()
        self.lithosphere_column = lithosphere_column or IncompressibleLithosphereColumn()
        if self.mantle not in (MaxwellMantle(), RelaxedMantle(), RigidMantle()):
            raise UnsupportedError(f"mantle {self.mantle!r}")
        if self.lithosphere not in (LaterallyVariableLithosphere(), LaterallyConstantLithosphere(),
                                    RigidLithosphere()):
            raise UnsupportedError(f"lithosphere {self.lithosphere!r}")
        if self.mantle == RelaxedMantle() and self.lithosphere == LaterallyVariableLithosphere():
            # src/deformation.jl:47-50
            raise UnsupportedError("Relaxed rheology is not implemented for laterally variable lithosphere.")
        if self.lumping != FreqDomainViscosityLumping():
            raise UnsupportedError(f"{self.lumping!r}: only FreqDomainViscosityLumping is supported")
        nx, ny = domain.nx, domain.ny
        self.maskactive = np.ones((nx, ny), dtype=bool) if maskactive is None else np.asarray(maskactive, bool)
        lb = _matrify(layer_boundaries, nx, ny)
        lv = _matrify(layer_viscosities, nx, ny)
        self.litho_thickness = lb[:, :, 0].copy()
        self.litho_youngmodulus = float(litho_youngmodulus)
        self.litho_poissonratio = float(litho_poissonratio)
        self.mantle_poissonratio = float(mantle_poissonratio)
        self.rho_uppermantle = float(rho_uppermantle)
        self.rho_litho = float(rho_litho)
        self.tau = np.full((nx, ny), float(tau)) if np.isscalar(tau) else np.asarray(tau, float)
        self.scale_elralength = float(scale_elralength)
        self.litho_rigidity = get_rigidity(self.litho_thickness, self.litho_youngmodulus, self.litho_poissonratio)
        # get_effective_viscosity_and_scaling(.., ::FreqDomainViscosityLumping), material.jl:154-179
        eta = lv[:, :, -1].copy()
        self.channel_ratio_means = []
        self.channel_thickness_means = []
        L = lv.shape[2]
        for l in range(1, L):
            thick = lb[:, :, L - l] - lb[:, :, L - l - 1]
            ratio = lv[:, :, L - l - 1] / eta
            self.channel_ratio_means.append(float(np.mean(ratio[self.maskactive])))
            self.channel_thickness_means.append(float(np.mean(thick)))
        # apply_compressibility!, apply_calibration! (material.jl:46-52, 81-87)
        if self.compressibility == CompressibleMantle():
            eta = eta * ((1 + 0.5) / (1 + self.mantle_poissonratio))
        if isinstance(self.calibration, SeakonCalibration):
            eta = eta * np.exp(np.log10(self.calibration.ref_viscosity / eta))
        self.effective_viscosity = eta
        self.litho_shearmodulus = self.litho_youngmodulus / (2 * (1 + self.litho_poissonratio))


# ---------------------------------------------------------------------------
# Boundary conditions and ice forcing (src/boundary_conditions.jl)
# ---------------------------------------------------------------------------


@dataclass
class CornerBC:
    space: object
    x_border: float = 0.0


@dataclass
class TimeInterpolatedIceThickness:
    """TimeInterpolatedIceThickness(t_vec, H_vec, domain), boundary_conditions.jl:25-40"""

    t_vec: list
    H_vec: list
    domain: RegionalDomain = None
    flat_bc: bool = False


class ExternallyUpdatedIceThickness(_Tag):
    pass


class BoundaryConditions:
    def __init__(self, domain, *, ice_thickness=None, viscous_displacement=None, elastic_displacement=None,
                 sea_surface_perturbation=None):
        self.ice_thickness = ice_thickness if ice_thickness is not None else ExternallyUpdatedIceThickness()
        self.viscous_displacement = viscous_displacement or CornerBC(RegularBCSpace(), 0.0)
        self.elastic_displacement = elastic_displacement or CornerBC(ExtendedBCSpace(), 0.0)
        self.sea_surface_perturbation = sea_surface_perturbation or CornerBC(ExtendedBCSpace(), 0.0)
        if not isinstance(self.viscous_displacement.space, RegularBCSpace):
            raise AssertionError("viscous_displacement must be defined on a regular grid")
        for name in ("viscous_displacement", "elastic_displacement", "sea_surface_perturbation"):
            bc = getattr(self, name)
            if not isinstance(bc, CornerBC):
                raise UnsupportedError(f"{name}: only CornerBC is on the hot path")
        for name in ("elastic_displacement", "sea_surface_perturbation"):
            if not isinstance(getattr(self, name).space, ExtendedBCSpace):
                raise UnsupportedError(f"{name}: only the ExtendedBCSpace default is supported")


# ---------------------------------------------------------------------------
# Sea level and solver options
# ---------------------------------------------------------------------------


@dataclass
class RegionalSeaLevel:
    """RegionalSeaLevel (src/sealevel.jl:114-130) with the same keyword defaults."""

    surface: object = field(default_factory=LaterallyConstantSeaSurface)
    load: object = field(default_factory=NoSealevelLoad)
    bsl: ConstantBSL = field(default_factory=ConstantBSL)
    update_bsl: object = field(default_factory=InternalBSLUpdate)
    volume_contribution: object = field(default_factory=GoelzerVolumeContribution)
    density_contribution: object = field(default_factory=GoelzerDensityContribution)
    adjustment_contribution: object = field(default_factory=NoAdjustmentContribution)

    def __post_init__(self):
        if self.load not in (NoSealevelLoad(), InteractiveSealevelLoad()):
            raise UnsupportedError(f"sea-level load {self.load!r}")
        if not isinstance(self.bsl, ConstantBSL):
            raise UnsupportedError(f"BSL {type(self.bsl).__name__} (PiecewiseLinearOceanSurfaceBSL needs NLsolve "
                                   "and is not on the device path)")
        if isinstance(self.bsl, PiecewiseConstantBSL) and self.bsl.ref.z_vec is None:
            raise UnsupportedError("PiecewiseConstantBSL needs ReferenceBSL(z_vec, A_vec), the ocean-surface table")

    @property
    def bsl_mode(self):
        for cls, mode in ((ImposedBSL, abi.FI_BSL_IMPOSED), (PiecewiseConstantBSL, abi.FI_BSL_PIECEWISE_CONSTANT),
                          (ConstantOceanSurfaceBSL, abi.FI_BSL_CONSTANT_OCEAN_SURFACE)):
            if isinstance(self.bsl, cls):
                return mode
        return abi.FI_BSL_CONSTANT


@dataclass
class DiffEqOptions:
    alg: str = "BS3"
    reltol: float = abi.RELTOL_DEFAULT
    dt_min: float | None = None


@dataclass
class SolverOptions:
    diffeq: DiffEqOptions = field(default_factory=DiffEqOptions)
    dt_sparse_diagnostics: float = 10.0
    verbose: bool = False


@dataclass
class NativeOutput:
    vars: list = field(default_factory=lambda: ["u", "ue", "dudt", "dz_ss"])
    t: list = field(default_factory=list)
    k: int = 0
    out: dict = field(default_factory=dict)
    t_written: list = field(default_factory=list)


def get_greenintegrand_coeffs():
    """(distance rm, GE) of the Farrell (1972) table (src/dataloaders.jl:257-273),
    from the copy extracted by data/make_farrell_table.py."""
    path = pathlib.Path(__file__).resolve().parent / "data" / "elasticgreencoeffs_farrell1972.txt"
    data = np.loadtxt(path)
    return np.ascontiguousarray(data[:, 1]), np.ascontiguousarray(data[:, 2])


# ---------------------------------------------------------------------------
# Simulation
# ---------------------------------------------------------------------------


def to_c(a):
    return abi.to_julia_layout(a)


def from_c(buf, nx, ny):
    return abi.from_julia_layout(buf, nx, ny)


class Simulation:
    """Simulation(domain, bcs, sealevel, solidearth, t_span; opts, u_ref, ue_ref,
    dz_ss_ref, z_b_ref, nout, c) -- src/simulation.jl:105-156.

    ``form`` picks the compute form: "fp32" (fused FP32 kernels with FP64 state,
    the default) or "fp64" (the plain FP64 form).  ``tiles`` = (rows per row task,
    spectral columns per column task) of the FP32 kernels; None takes the tuned value
    for square grids from fastiso_b200.autotune's table, else the library's default."""

    def __init__(self, domain, bcs, sealevel, solidearth, t_span, *, opts=None, u_ref=None, ue_ref=None,
                 dz_ss_ref=None, z_b_ref=None, nout=None, c=None, form="fp32", max_steps=1_000_000, device=0,
                 tiles=None):
        self.domain, self.bcs, self.sealevel, self.solidearth = domain, bcs, sealevel, solidearth
        self.opts = opts or SolverOptions()
        self.c = c or PhysicalConstants()
        self.nout = nout or NativeOutput()
        self.t_span = (float(t_span[0]), float(t_span[1]))
        dq = self.opts.diffeq
        if dq.alg not in ("BS3", "Euler"):
            raise UnsupportedError(f"integrator {dq.alg!r}: BS3 (adaptive) or Euler (fixed dt_min)")
        if (dq.dt_min is not None) != (dq.alg == "Euler"):
            # src/simulation.jl:244-256
            raise UnsupportedError("The `dt_min` option is only compatible with the Euler algorithm.")
        if form == "fp32" and (dq.alg != "BS3" or solidearth.mantle != MaxwellMantle()
                               or solidearth.lithosphere == LaterallyConstantLithosphere()):
            raise UnsupportedError("the FP32 form runs the LV-ELVA path (MaxwellMantle, laterally variable or rigid "
                                   "lithosphere, BS3); other rheologies run in the plain FP64 form (form='fp64')")
        nx, ny = domain.nx, domain.ny
        z = domain.zeros
        self.u_ref = z() if u_ref is None else np.asarray(u_ref, float)
        self.ue_ref = z() if ue_ref is None else np.asarray(ue_ref, float)
        self.dz_ss_ref = z() if dz_ss_ref is None else np.asarray(dz_ss_ref, float)
        self.z_b_ref = domain.fill(float(np.float32(1e6))) if z_b_ref is None else np.asarray(z_b_ref, float)
        if sealevel.load != NoSealevelLoad():
            pass  # rejected by RegionalSeaLevel
        cfg = abi.default_config(nx, ny, domain.Wx, domain.Wy)
        c_ = self.c
        cfg.mE, cfg.r_pole, cfg.g, cfg.seconds_per_year = c_.mE, c_.r_pole, c_.g, c_.seconds_per_year
        cfg.rho_ice, cfg.rho_water, cfg.rho_seawater = c_.rho_ice, c_.rho_water, c_.rho_seawater
        cfg.rho_litho, cfg.rho_uppermantle = solidearth.rho_litho, solidearth.rho_uppermantle
        cfg.litho_poissonratio = solidearth.litho_poissonratio
        cfg.lithosphere = {RigidLithosphere(): abi.FI_LITHO_RIGID,
                           LaterallyConstantLithosphere(): abi.FI_LITHO_LATERALLY_CONSTANT}.get(
            solidearth.lithosphere, abi.FI_LITHO_LATERALLY_VARIABLE)
        cfg.mantle = {RelaxedMantle(): abi.FI_MANTLE_RELAXED, RigidMantle(): abi.FI_MANTLE_RIGID}.get(
            solidearth.mantle, abi.FI_MANTLE_MAXWELL)
        cfg.alg = abi.FI_ALG_EULER if dq.alg == "Euler" else abi.FI_ALG_BS3
        cfg.dt_min = float(dq.dt_min) if dq.dt_min is not None else 0.0
        cfg.lithosphere_column = (abi.FI_COLUMN_COMPRESSIBLE
                                  if solidearth.lithosphere_column == CompressibleLithosphereColumn()
                                  else abi.FI_COLUMN_INCOMPRESSIBLE)
        cfg.sea_surface = (abi.FI_SEA_SURFACE_LATERALLY_VARIABLE
                           if sealevel.surface == LaterallyVariableSeaSurface()
                           else abi.FI_SEA_SURFACE_LATERALLY_CONSTANT)
        cfg.z_bsl = sealevel.bsl.z
        cfg.bsl_ref_A = sealevel.bsl.A
        cfg.sealevel_load = (abi.FI_SEALEVEL_LOAD_INTERACTIVE if sealevel.load == InteractiveSealevelLoad()
                             else abi.FI_SEALEVEL_LOAD_NONE)
        cfg.bsl_mode = sealevel.bsl_mode
        cfg.bsl_update = (abi.FI_BSL_UPDATE_EXTERNAL if sealevel.update_bsl == ExternalBSLUpdate()
                          else abi.FI_BSL_UPDATE_INTERNAL)
        cfg.volume_contribution = (abi.FI_CONTRIB_NONE if sealevel.volume_contribution == NoVolumeContribution()
                                   else abi.FI_CONTRIB_GOELZER)
        cfg.density_contribution = (abi.FI_CONTRIB_NONE if sealevel.density_contribution == NoDensityContribution()
                                    else abi.FI_CONTRIB_GOELZER)
        cfg.adjustment_contribution = (abi.FI_CONTRIB_GOELZER
                                       if sealevel.adjustment_contribution == GoelzerAdjustmentContribution()
                                       else abi.FI_CONTRIB_NONE)
        cfg.bc_viscous_border = bcs.viscous_displacement.x_border
        cfg.bc_elastic_border = bcs.elastic_displacement.x_border
        cfg.bc_sea_surface_border = bcs.sea_surface_perturbation.x_border
        it = bcs.ice_thickness
        if isinstance(it, TimeInterpolatedIceThickness):
            cfg.ice_mode = abi.FI_ICE_TIME_INTERPOLATED
            cfg.ice_flat_bc = int(bool(it.flat_bc))
            self.ice_t = np.asarray(it.t_vec, dtype=np.float64)
            self.ice_H = np.stack([np.asarray(h, dtype=np.float64) for h in it.H_vec])
        else:
            cfg.ice_mode = abi.FI_ICE_EXTERNAL
            self.ice_t = None
            self.ice_H = None
        cfg.t0, cfg.t1 = self.t_span
        cfg.reltol = float(self.opts.diffeq.reltol)
        cfg.abstol = 1e-6
        cfg.dt_sparse_diagnostics = float(self.opts.dt_sparse_diagnostics)
        cfg.max_steps = int(max_steps)
        cfg.form = {"fp32": abi.FI_FORM_FP32, "fp64": abi.FI_FORM_FP64}[form]
        cfg.device = int(device)
        self.form = form
        self.cfg = cfg
        self.tiles = tiles
        #: {transform length: [radix, ...]} applied at handle creation (FP32 and FP64
        #: forms); lengths without an entry take the tuned table's schedule, if any
        self.fft_schedules = {}
        self.elastic_table = get_greenintegrand_coeffs()
        self._handle = None
        self._initialized = False
        self._integrator_started = False

    # -- inputs handed to the native library (also used by tests to drive the oracle)
    def prepared_inputs(self):
        se = self.solidearth
        fields = {
            "litho_rigidity": se.litho_rigidity,
            "effective_viscosity": se.effective_viscosity,
            "maskactive": se.maskactive.astype(np.float64),
            "tau": se.tau,
            "u_ref": self.u_ref,
            "ue_ref": self.ue_ref,
            "dz_ss_ref": self.dz_ss_ref,
            "z_b_ref": self.z_b_ref,
        }
        return {
            "cfg": self.cfg,
            "fields": fields,
            "ice_t": self.ice_t,
            "ice_H": self.ice_H,
            "elastic_table": self.elastic_table,
            "channels": (np.asarray(se.channel_ratio_means, float), np.asarray(se.channel_thickness_means, float)),
            "ocean_surface": ((np.asarray(self.sealevel.bsl.ref.z_vec, float), np.asarray(self.sealevel.bsl.ref.A_vec,
                                                                                         float))
                              if self.sealevel.bsl.ref.z_vec is not None else None),
            "bsl_history": ((np.asarray(self.sealevel.bsl.t_vec, float), np.asarray(self.sealevel.bsl.z_vec, float))
                            if isinstance(self.sealevel.bsl, ImposedBSL) else None),
        }

    # -- native handle
    @property
    def lib(self):
        return abi.load_library()

    def _check(self, rc, what):
        if rc != abi.FI_OK:
            msg = self.lib.fi_last_error(self._handle)
            raise abi.FiError(rc, f"{what}: {msg.decode() if msg else ''}")

    def _ensure_handle(self):
        if self._handle is not None:
            return
        lib = self.lib
        h = C.c_void_p()
        rc = lib.fi_create(C.byref(self.cfg), C.byref(h))
        if rc != abi.FI_OK:
            raise abi.FiError(rc, "fi_create failed")
        self._handle = h
        if self.tiles is None and self.cfg.form == abi.FI_FORM_FP32 and self.domain.nx == self.domain.ny:
            from .autotune import tiles_for  # noqa: WPS433 (the tuner imports this module)

            self.tiles = tiles_for(f"single:{self.domain.nx}")
        if self.tiles is not None and self.cfg.form == abi.FI_FORM_FP32:
            self._check(lib.fi_set_tiles(h, int(self.tiles[0]), int(self.tiles[1])), "fi_set_tiles")
        from .autotune import fft_schedule_for  # noqa: WPS433

        lengths = {self.domain.nx, self.domain.ny, nextfastfft(2 * self.domain.nx - 1),
                   nextfastfft(2 * self.domain.ny - 1)}
        for L in sorted(lengths):
            sched = self.fft_schedules.get(L)
            if sched is None and self.cfg.form == abi.FI_FORM_FP32:
                sched = fft_schedule_for(L)
            if sched:
                self.set_fft_schedule(L, sched)
        inp = self.prepared_inputs()
        for name, arr in inp["fields"].items():
            self.set_field(name, arr)
        if self.ice_t is not None:
            H = np.ascontiguousarray(np.stack([to_c(h) for h in self.ice_H]))
            t = abi.as_f64(self.ice_t)
            self._check(lib.fi_set_ice_history(h, t.size, abi.dptr(t), abi.dptr(H.reshape(-1))), "fi_set_ice_history")
        rm, GE = self.elastic_table
        self._check(lib.fi_set_elastic_table(h, rm.size, abi.dptr(rm), abi.dptr(GE)), "fi_set_elastic_table")
        ratio, thick = inp["channels"]
        if ratio.size:
            self._check(lib.fi_set_channel_scaling(h, ratio.size, abi.dptr(ratio), abi.dptr(thick)),
                        "fi_set_channel_scaling")
        if inp["ocean_surface"] is not None:
            z, A = (abi.as_f64(a) for a in inp["ocean_surface"])
            self._check(lib.fi_set_ocean_surface_table(h, z.size, abi.dptr(z), abi.dptr(A)),
                        "fi_set_ocean_surface_table")
        if inp["bsl_history"] is not None:
            t, z = (abi.as_f64(a) for a in inp["bsl_history"])
            self._check(lib.fi_set_bsl_history(h, t.size, abi.dptr(t), abi.dptr(z)), "fi_set_bsl_history")

    def set_fft_schedule(self, L, radices):
        """Radix order of the length-L transforms (before init_problem)."""
        r = (C.c_int32 * len(radices))(*[int(x) for x in radices])
        self._check(self.lib.fi_set_fft_schedule(self._handle, int(L), len(radices), r), "fi_set_fft_schedule")

    def get_fft_schedule(self, L):
        self._ensure_handle()
        n = C.c_int32(0)
        r = (C.c_int32 * 20)()
        self._check(self.lib.fi_get_fft_schedule(self._handle, int(L), C.byref(n), r), "fi_get_fft_schedule")
        return list(r[:n.value])

    def set_field(self, name, arr):
        self._ensure_handle()
        buf = to_c(arr)
        self._check(self.lib.fi_set_field(self._handle, abi.FIELDS[name], abi.dptr(buf), buf.size), f"set {name}")

    def get_field(self, name):
        self._ensure_handle()
        buf = np.empty(self.domain.nx * self.domain.ny)
        self._check(self.lib.fi_get_field(self._handle, abi.FIELDS[name], abi.dptr(buf), buf.size), f"get {name}")
        return from_c(buf, self.domain.nx, self.domain.ny)

    def init_problem(self):
        """Reference state + init_problem! (src/simulation.jl:305-312)."""
        self._ensure_handle()
        if not self._initialized:
            self._check(self.lib.fi_init(self._handle), "fi_init")
            self._initialized = True

    def sealevel_state(self):
        """sim.now.z_bsl, bsl.A and the volume terms (fi_get_sealevel)."""
        out = abi.FiSealevel()
        self._check(self.lib.fi_get_sealevel(self._handle, C.byref(out)), "fi_get_sealevel")
        return {k: getattr(out, k) for k, _ in abi.FiSealevel._fields_ if k != "pad"}

    def stats(self):
        st = abi.FiStats()
        self._check(self.lib.fi_get_stats(self._handle, C.byref(st)), "fi_get_stats")
        return {k: getattr(st, k) for k, _ in abi.FiStats._fields_}

    # -- no reference counterpart: checkpoints and step-sequence record / replay
    def checkpoint(self) -> bytes:
        """fi_checkpoint: the integrator and diagnostic state as bytes."""
        size = C.c_size_t(0)
        self._check(self.lib.fi_checkpoint(self._handle, None, C.byref(size)), "fi_checkpoint")
        buf = C.create_string_buffer(size.value)
        self._check(self.lib.fi_checkpoint(self._handle, buf, C.byref(size)), "fi_checkpoint")
        return buf.raw[:size.value]

    def restore(self, blob: bytes):
        """fi_restore of a checkpoint taken from a handle of the same form and grid."""
        buf = C.create_string_buffer(bytes(blob), len(blob))
        self._check(self.lib.fi_restore(self._handle, buf, len(blob)), "fi_restore")

    def record_steps(self, cap: int):
        """fi_record_steps: store the dt of the next `cap` accepted steps."""
        self._check(self.lib.fi_record_steps(self._handle, int(cap)), "fi_record_steps")

    def step_record(self) -> np.ndarray:
        """The recorded accepted step sizes (fi_get_step_record)."""
        n = C.c_int64(0)
        self._check(self.lib.fi_get_step_record(self._handle, None, 0, C.byref(n)), "fi_get_step_record")
        out = np.empty(max(1, n.value))
        self._check(self.lib.fi_get_step_record(self._handle, abi.dptr(out), n.value, C.byref(n)),
                    "fi_get_step_record")
        return out[:n.value].copy()

    def set_step_replay(self, dts):
        """fi_set_step_replay: the next len(dts) attempts take these step sizes and are accepted."""
        d = abi.as_f64(dts)
        self._check(self.lib.fi_set_step_replay(self._handle, d.size, abi.dptr(d) if d.size else None),
                    "fi_set_step_replay")

    @property
    def now(self):
        return _NowView(self)

    def close(self):
        if self._handle is not None:
            self.lib.fi_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _NowView:
    """sim.now.<field> reads the device state."""

    def __init__(self, sim):
        object.__setattr__(self, "_sim", sim)

    def __getattr__(self, name):
        return self._sim.get_field(name)

    def __setattr__(self, name, value):
        self._sim.set_field(name, value)


def update_diagnostics(dudt, u, sim: Simulation, t):
    """update_diagnostics!(dudt, u, sim, t): one RHS evaluation; u and dudt are
    (nx, ny) float64 arrays updated in place."""
    sim.init_problem()
    ub = to_c(u)
    db = np.empty_like(ub)
    sim._check(sim.lib.fi_rhs(sim._handle, float(t), abi.dptr(ub), abi.dptr(db)), "fi_rhs")
    u[...] = from_c(ub, sim.domain.nx, sim.domain.ny)
    dudt[...] = from_c(db, sim.domain.nx, sim.domain.ny)


def run(sim: Simulation):
    """run!(sim), src/simulation.jl:236-262: integrates t_span with BS3 and stores
    the NativeOutput fields at nout.t."""
    sim.init_problem()
    nx, ny = sim.domain.nx, sim.domain.ny
    n = nx * ny
    t_out = abi.as_f64(sim.nout.t)
    k = t_out.size
    wanted = set(sim.nout.vars)
    bufs = {v: (np.zeros(k * n) if v in wanted else None) for v in ("u", "ue", "dudt", "dz_ss")}
    ot = np.zeros(max(k, 1))
    ptr = lambda a: abi.dptr(a) if a is not None else None  # noqa: E731
    sim._check(sim.lib.fi_run(sim._handle, k, abi.dptr(t_out) if k else None, abi.dptr(ot), ptr(bufs["u"]),
                              ptr(bufs["ue"]), ptr(bufs["dudt"]), ptr(bufs["dz_ss"])), "fi_run")
    sim.nout.out = {v: [from_c(b[i * n:(i + 1) * n], nx, ny) for i in range(k)] for v, b in bufs.items()
                    if b is not None}
    sim.nout.t_written = list(ot[:k])
    sim.nout.k = k
    return None


class Integrator:
    def __init__(self, sim):
        self.sim = sim

    @property
    def t(self):
        return self.sim.stats()["t"]


def init_integrator(sim: Simulation):
    """init_integrator(sim), src/simulation.jl:293-303"""
    sim.init_problem()
    ts = abi.as_f64(sim.nout.t)
    sim._check(sim.lib.fi_init_integrator(sim._handle, ts.size, abi.dptr(ts) if ts.size else None),
               "fi_init_integrator")
    return Integrator(sim)


def step(integrator: Integrator, dt, force_dt=True):
    """step!(integrator, dt, true), src/simulation.jl:319-322"""
    if not force_dt:
        raise UnsupportedError("step! is always used with force_dt = true")
    sim = integrator.sim
    sim._check(sim.lib.fi_step(sim._handle, float(dt)), "fi_step")


class Ensemble:
    """Batched ensemble of FP32 simulations stepped together (no counterpart in the
    reference; its only batching is the host-threaded ensemble of
    ext/FastIsostasyEnsembleKalmanProcessesExt.jl:107-122).  Each member keeps its own
    grid, fields and integrator; ``step(dt)`` is ``step!(integrator_m, dt, true)`` for
    every member, the members' step loops running concurrently on the GPU.  A member
    that fails is reported in the returned status list and does not stop the others."""

    #: tile shape of members whose handles do not exist yet when the tuning table has
    #: neither a per-member rule ("ensemble:per_n": h = B = c / N) nor an entry for this
    #: ensemble size: tall tiles, since the ensemble is throughput-bound
    DEFAULT_TILES = (8, 8)

    def __init__(self, sims, tiles="auto"):
        self.sims = list(sims)
        if not self.sims:
            raise ValueError("an ensemble needs at least one member")
        rule = None
        if isinstance(tiles, str):
            from .autotune import ensemble_rule_for, tiles_for  # noqa: WPS433

            rule = ensemble_rule_for()
            tiles = tiles_for(f"ensemble:{len(self.sims)}") or self.DEFAULT_TILES
        self.integrators = []
        for s in self.sims:
            if s.cfg.form != abi.FI_FORM_FP32:
                raise UnsupportedError("ensemble members use the FP32 form")
            if s._handle is None and s.tiles is None:
                if rule is not None:
                    from .autotune import rule_tiles  # noqa: WPS433

                    s.tiles = rule_tiles(rule, max(s.domain.nx, s.domain.ny))
                elif tiles is not None:
                    s.tiles = tuple(tiles)
            self.integrators.append(init_integrator(s))
        self.lib = self.sims[0].lib
        arr = (C.c_void_p * len(self.sims))(*[s._handle.value for s in self.sims])
        h = C.c_void_p()
        rc = self.lib.fi_ensemble_create(arr, len(self.sims), C.byref(h))
        if rc != abi.FI_OK:
            raise abi.FiError(rc, "fi_ensemble_create failed")
        self._h = h

    def step(self, dt):
        st = (C.c_int32 * len(self.sims))()
        rc = self.lib.fi_ensemble_step(self._h, float(dt), st)
        if rc != abi.FI_OK:
            raise abi.FiError(rc, "fi_ensemble_step failed")
        return list(st)

    @property
    def last_gpu_ms(self):
        return float(self.lib.fi_ensemble_last_gpu_ms(self._h))

    def trace(self, on=None):
        """Phase timeline of the persistent ensemble executor: ``trace(True)`` starts
        recording, ``trace()`` returns {phase: (ms, count)}, ``trace(False)`` stops."""
        ms = (C.c_double * abi.FI_NUM_PHASES)()
        cnt = (C.c_int64 * abi.FI_NUM_PHASES)()
        rc = self.lib.fi_ensemble_trace(self._h, -1 if on is None else int(bool(on)), ms, cnt)
        if rc != abi.FI_OK:
            raise abi.FiError(rc, "fi_ensemble_trace failed")
        return {name: (m, c) for name, m, c in zip(abi.PHASE_NAMES, ms, cnt)}

    def close(self):
        if getattr(self, "_h", None):
            self.lib.fi_ensemble_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
