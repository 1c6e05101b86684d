"""ctypes description of the C ABI in include/fastiso_b200.h and the loader of the
native library ``libfastiso_b200.so``.

The library is the only compute path: ``load_library()`` raises if the shared
object is missing instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes as C
import os
import pathlib

import numpy as np

PKG_DIR = pathlib.Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "lib" / "libfastiso_b200.so"

# ---- status codes -------------------------------------------------------
FI_OK = 0
FI_ERR_ARG = 1
FI_ERR_CUDA = 2
FI_ERR_NONFINITE = 3
FI_ERR_DT_UNDERFLOW = 4
FI_ERR_FORCING_RANGE = 5
FI_ERR_TIMEOUT = 6
FI_ERR_STATE = 7
FI_ERR_UNSUPPORTED = 8
FI_ERR_MAXITERS = 9

# ---- enums ----------------------------------------------------------------
FI_FORM_FP32 = 0
FI_FORM_FP64 = 1
FI_LITHO_LATERALLY_VARIABLE = 0
FI_LITHO_RIGID = 1
FI_SEA_SURFACE_LATERALLY_CONSTANT = 0
FI_SEA_SURFACE_LATERALLY_VARIABLE = 1
FI_COLUMN_INCOMPRESSIBLE = 0
FI_COLUMN_COMPRESSIBLE = 1
FI_ICE_TIME_INTERPOLATED = 0
FI_ICE_EXTERNAL = 1
FI_SEALEVEL_LOAD_NONE = 0
FI_SEALEVEL_LOAD_INTERACTIVE = 1
FI_BSL_CONSTANT = 0
FI_BSL_CONSTANT_OCEAN_SURFACE = 1
FI_BSL_PIECEWISE_CONSTANT = 2
FI_BSL_IMPOSED = 3
FI_BSL_UPDATE_INTERNAL = 0
FI_BSL_UPDATE_EXTERNAL = 1
FI_CONTRIB_NONE = 0
FI_CONTRIB_GOELZER = 1
#: A_OCEAN_PD, present-day ocean surface (m^2), src/barystatic_sealevel.jl:1
A_OCEAN_PD = 3.625e14
FI_LITHO_LATERALLY_CONSTANT = 2
FI_MANTLE_MAXWELL = 0
FI_MANTLE_RELAXED = 1
FI_MANTLE_RIGID = 2
FI_ALG_BS3 = 0
FI_ALG_EULER = 1
FI_EXEC_PERSIST = 0
FI_EXEC_GRAPH = 1
FI_EXEC_LOOP = 2
FI_WAIT_GRID_POLLS = 0
FI_WAIT_GRID_EXTRA_ARRIVALS = 1
FI_WAIT_TC_POLLS = 2
FI_NUM_PHASES = 11
PHASE_NAMES = ("conv_rows", "conv_cols", "conv_rows_inv", "rows_fwd2", "cols2", "rows_fwd3", "cols3", "rows_fwd4",
               "cols4", "rows_inv4", "controller")

FIELDS = {
    "litho_rigidity": 0,
    "effective_viscosity": 1,
    "pseudodiff_scaling": 2,
    "maskactive": 3,
    "u_ref": 4,
    "ue_ref": 5,
    "dz_ss_ref": 6,
    "z_b_ref": 7,
    "u": 8,
    "ue": 9,
    "dudt": 10,
    "dz_ss": 11,
    "H_ice": 12,
    "z_ss": 13,
    "z_b": 14,
    "elastic_green": 15,
    "dz_ss_green": 16,
    "pseudodiff": 17,
    "scaled_pseudodiff_inv": 18,
    "columnanom_load": 19,
    "columnanom_full": 20,
    "H_af": 21,
    "maskgrounded": 22,
    "maskocean": 23,
    "H_water": 24,
    "columnanom_seawater": 25,
    "tau": 26,
    "u_eq": 27,
}

#: Float64(1f-5): the reference passes reltol as a Float32 literal (src/simulation.jl:13)
RELTOL_DEFAULT = float(np.float32(1e-5))
#: SECONDS_PER_YEAR = 60^2 * 24 * 365.25 (src/utils.jl:7)
SECONDS_PER_YEAR = 60.0**2 * 24 * 365.25


class FiConfig(C.Structure):
    """``fi_config`` (include/fastiso_b200.h)."""

    _fields_ = [
        ("nx", C.c_int32),
        ("ny", C.c_int32),
        ("Wx", C.c_double),
        ("Wy", C.c_double),
        ("mE", C.c_double),
        ("r_pole", C.c_double),
        ("g", C.c_double),
        ("seconds_per_year", C.c_double),
        ("rho_ice", C.c_double),
        ("rho_water", C.c_double),
        ("rho_seawater", C.c_double),
        ("rho_litho", C.c_double),
        ("rho_uppermantle", C.c_double),
        ("litho_poissonratio", C.c_double),
        ("lithosphere", C.c_int32),
        ("lithosphere_column", C.c_int32),
        ("sea_surface", C.c_int32),
        ("z_bsl", C.c_double),
        ("bc_viscous_border", C.c_double),
        ("bc_elastic_border", C.c_double),
        ("bc_sea_surface_border", C.c_double),
        ("ice_mode", C.c_int32),
        ("ice_flat_bc", C.c_int32),
        ("t0", C.c_double),
        ("t1", C.c_double),
        ("reltol", C.c_double),
        ("abstol", C.c_double),
        ("dt_sparse_diagnostics", C.c_double),
        ("max_steps", C.c_int64),
        ("form", C.c_int32),
        ("device", C.c_int32),
        ("sealevel_load", C.c_int32),
        ("bsl_mode", C.c_int32),
        ("bsl_update", C.c_int32),
        ("volume_contribution", C.c_int32),
        ("density_contribution", C.c_int32),
        ("adjustment_contribution", C.c_int32),
        ("bsl_ref_A", C.c_double),
        ("mantle", C.c_int32),
        ("alg", C.c_int32),
        ("dt_min", C.c_double),
    ]


class FiSealevel(C.Structure):
    """``fi_sealevel`` (include/fastiso_b200.h)."""

    _fields_ = [
        ("z_bsl", C.c_double),
        ("A_bsl", C.c_double),
        ("V_af", C.c_double),
        ("V_den", C.c_double),
        ("V_pov", C.c_double),
        ("delta_V", C.c_double),
        ("tracked", C.c_int32),
        ("pad", C.c_int32),
    ]


class FiStats(C.Structure):
    """``fi_stats`` (include/fastiso_b200.h)."""

    _fields_ = [
        ("t", C.c_double),
        ("dt", C.c_double),
        ("nf", C.c_int64),
        ("naccept", C.c_int64),
        ("nreject", C.c_int64),
        ("nsparse", C.c_int64),
        ("status", C.c_int32),
        ("form", C.c_int32),
        ("gpu_ms", C.c_double),
        ("last_gpu_ms", C.c_double),
        ("segments", C.c_int64),
        ("executor", C.c_int32),
        ("grid", C.c_int32),
    ]


def default_config(nx: int, ny: int, Wx: float, Wy: float) -> FiConfig:
    """Reference defaults (src/constants.jl:16-28, src/solidearth.jl:115-121,
    src/simulation.jl:11-26, src/boundary_conditions.jl:308-313); the same values
    ``fi_config_default`` writes."""
    c = FiConfig()
    c.nx, c.ny, c.Wx, c.Wy = int(nx), int(ny), float(Wx), float(Wy)
    c.mE = 5.972e24
    c.r_pole = 6357e3
    c.g = 9.8
    c.seconds_per_year = SECONDS_PER_YEAR
    c.rho_ice = 0.910e3
    c.rho_water = 1e3
    c.rho_seawater = 1.023e3
    c.rho_litho = 3.2e3
    c.rho_uppermantle = 3.4e3
    c.litho_poissonratio = 0.28
    c.lithosphere = FI_LITHO_LATERALLY_VARIABLE
    c.lithosphere_column = FI_COLUMN_INCOMPRESSIBLE
    c.sea_surface = FI_SEA_SURFACE_LATERALLY_CONSTANT
    c.z_bsl = 0.0
    c.bc_viscous_border = 0.0
    c.bc_elastic_border = 0.0
    c.bc_sea_surface_border = 0.0
    c.ice_mode = FI_ICE_TIME_INTERPOLATED
    c.ice_flat_bc = 0
    c.t0, c.t1 = 0.0, 1.0
    c.reltol = RELTOL_DEFAULT
    c.abstol = 1e-6
    c.dt_sparse_diagnostics = 10.0
    c.max_steps = 1_000_000
    c.form = FI_FORM_FP32
    c.device = 0
    c.sealevel_load = FI_SEALEVEL_LOAD_NONE
    c.bsl_mode = FI_BSL_CONSTANT
    c.bsl_update = FI_BSL_UPDATE_INTERNAL
    c.volume_contribution = FI_CONTRIB_GOELZER
    c.density_contribution = FI_CONTRIB_GOELZER
    c.adjustment_contribution = FI_CONTRIB_NONE
    c.bsl_ref_A = A_OCEAN_PD
    c.mantle = FI_MANTLE_MAXWELL
    c.alg = FI_ALG_BS3
    c.dt_min = 0.0
    return c


def dptr(a: np.ndarray):
    """Pointer to a C-contiguous float64 array."""
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_double))


def as_f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def to_julia_layout(a: np.ndarray) -> np.ndarray:
    """A numpy (nx, ny) array indexed [i, j] -> flat buffer with x fastest (column-major)."""
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).T).reshape(-1)


def from_julia_layout(buf: np.ndarray, nx: int, ny: int) -> np.ndarray:
    """Flat x-fastest buffer -> numpy (nx, ny) array indexed [i, j]."""
    return np.asarray(buf).reshape(ny, nx).T.copy()


_LIB = None

_SIGS = {
    "fi_config_default": (None, [C.POINTER(FiConfig), C.c_int32, C.c_int32, C.c_double, C.c_double]),
    "fi_create": (C.c_int, [C.POINTER(FiConfig), C.POINTER(C.c_void_p)]),
    "fi_set_field": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_double), C.c_size_t]),
    "fi_get_field": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_double), C.c_size_t]),
    "fi_set_ice_history": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "fi_set_elastic_table": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "fi_set_channel_scaling": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "fi_set_tiles": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32]),
    "fi_set_fft_schedule": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_int32)]),
    "fi_get_fft_schedule": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "fi_init": (C.c_int, [C.c_void_p]),
    "fi_rhs": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "fi_rhs_noalloc": (C.c_int, [C.c_void_p, C.c_double, C.c_void_p, C.c_void_p]),
    "fi_run": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double),
                         C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double),
                         C.POINTER(C.c_double)]),
    "fi_init_integrator": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_double)]),
    "fi_step": (C.c_int, [C.c_void_p, C.c_double]),
    "fi_record_steps": (C.c_int, [C.c_void_p, C.c_int64]),
    "fi_get_step_record": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.c_int64, C.POINTER(C.c_int64)]),
    "fi_set_step_replay": (C.c_int, [C.c_void_p, C.c_int64, C.POINTER(C.c_double)]),
    "fi_get_stats": (C.c_int, [C.c_void_p, C.POINTER(FiStats)]),
    "fi_get_sealevel": (C.c_int, [C.c_void_p, C.POINTER(FiSealevel)]),
    "fi_set_ocean_surface_table": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_double),
                                             C.POINTER(C.c_double)]),
    "fi_set_bsl_history": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "fi_checkpoint": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_size_t)]),
    "fi_restore": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t]),
    "fi_time_kernels": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_double)]),
    "fi_trace_phases": (C.c_int, [C.c_void_p, C.c_int32]),
    "fi_get_phase_trace": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int64)]),
    "fi_ensemble_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int32, C.POINTER(C.c_void_p)]),
    "fi_ensemble_step": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(C.c_int32)]),
    "fi_ensemble_last_gpu_ms": (C.c_double, [C.c_void_p]),
    "fi_ensemble_trace": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_int64)]),
    "fi_ensemble_destroy": (None, [C.c_void_p]),
    "fi_fno_gemm": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_int32, C.c_void_p, C.c_int32,
                             C.c_void_p, C.c_int32, C.c_int32, C.c_int64, C.c_int64, C.c_int64, C.c_int32]),
    "fi_fno_create": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_uint64, C.POINTER(C.c_void_p)]),
    "fi_fno_num_params": (C.c_int64, [C.c_void_p]),
    "fi_fno_get_params": (C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.c_int64]),
    "fi_fno_set_params": (C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.c_int64]),
    "fi_fno_get_grads": (C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.c_int64]),
    "fi_fno_forward": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]),
    "fi_fno_backward": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p]),
    "fi_fno_train_step": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_float,
                                    C.POINTER(C.c_float)]),
    "fi_fno_train_step_weighted": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                             C.c_float, C.POINTER(C.c_float)]),
    "fi_fno_adam": (C.c_int, [C.c_void_p, C.c_float]),
    "fi_fno_loss_backward": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.POINTER(C.c_float)]),
    "fi_fno_grads_device": (C.c_void_p, [C.c_void_p]),
    "fi_fno_set_adam": (C.c_int, [C.c_void_p, C.c_float, C.c_float, C.c_float]),
    "fi_fno_last_error": (C.c_char_p, [C.c_void_p]),
    "fi_fno_destroy": (None, [C.c_void_p]),
    "fi_debug_set_wait_limit": (C.c_int, [C.c_int32, C.c_int64]),
    "fi_last_error": (C.c_char_p, [C.c_void_p]),
    "fi_status_string": (C.c_char_p, [C.c_int32]),
    "fi_destroy": (None, [C.c_void_p]),
}


def exported_symbols():
    """Entry points declared in include/fastiso_b200.h (checked by the CPU tests)."""
    return list(_SIGS)


def load_library(path: os.PathLike | str | None = None):
    """Load libfastiso_b200.so (built in-tree).  Raises if it is missing: there is
    no CPU fallback for the hot path."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = pathlib.Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(
            f"native library {p} is missing; build it with `python -c 'import __graft_entry__ as g; g.build()'`"
        )
    lib = C.CDLL(str(p))
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _LIB = lib
    return lib


class FiError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code
