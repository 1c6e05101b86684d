"""fastiso_b200 -- B200-native LV-ELVA hot path of FastIsostasy.jl.

The package mirrors the reference's Julia API (RegionalDomain, SolidEarth,
BoundaryConditions, RegionalSeaLevel, Simulation, run!, init_integrator, step!,
update_diagnostics!) over the C ABI of libfastiso_b200.so (include/fastiso_b200.h).
"""
from . import abi  # noqa: F401
from .fno import FNO  # noqa: F401  (the surrogate network; its workflow is fastiso_b200.surrogate)
from .model import (  # noqa: F401
    BoundaryConditions, CompressibleLithosphereColumn, CompressibleMantle, ConstantBSL, CornerBC, DiffEqOptions, Ensemble,
    ExtendedBCSpace, ExternallyUpdatedIceThickness, FreqDomainViscosityLumping, IncompressibleLithosphereColumn,
    IncompressibleMantle, Integrator, LaterallyConstantSeaSurface, LaterallyVariableLithosphere,
    LaterallyVariableSeaSurface, MaxwellMantle, NativeOutput, NoCalibration, NoSealevelLoad, PhysicalConstants,
    RegionalDomain, RegionalSeaLevel, RegularBCSpace, RigidLithosphere, SeakonCalibration, Simulation, SolidEarth,
    SolverOptions, TimeInterpolatedIceThickness, UnsupportedError, get_greenintegrand_coeffs, get_rigidity,
    init_integrator, nextfastfft, run, samesize_conv_indices, step, update_diagnostics,
)
from .model import (  # noqa: F401
    ConstantOceanSurfaceBSL, ExternalBSLUpdate, GoelzerAdjustmentContribution, GoelzerDensityContribution,
    GoelzerVolumeContribution, ImposedBSL, InteractiveSealevelLoad, InternalBSLUpdate, NoAdjustmentContribution,
    NoDensityContribution, NoVolumeContribution, PiecewiseConstantBSL, ReferenceBSL,
)
from .model import LaterallyConstantLithosphere, RelaxedMantle, RigidMantle  # noqa: F401
