"""TEST INFRASTRUCTURE ONLY: ctypes driver of the FP64 CPU oracle (oracle/fi_oracle.c).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import this
module, always as the checker of the CUDA library, never as a compute path.
"""
from __future__ import annotations

import ctypes as C
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "build" / "libfi_oracle.so"

_lib = None


def build() -> pathlib.Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        build()
    from fastiso_b200.abi import FiConfig, FiStats  # noqa: WPS433 (shared ABI structs)

    L = C.CDLL(str(LIB_PATH))
    dp = C.POINTER(C.c_double)
    sig = {
        "or_create": (C.c_int, [C.POINTER(FiConfig), C.POINTER(C.c_void_p)]),
        "or_set_field": (C.c_int, [C.c_void_p, C.c_int32, dp, C.c_size_t]),
        "or_get_field": (C.c_int, [C.c_void_p, C.c_int32, dp, C.c_size_t]),
        "or_set_ice_history": (C.c_int, [C.c_void_p, C.c_int32, dp, dp]),
        "or_set_elastic_table": (C.c_int, [C.c_void_p, C.c_int32, dp, dp]),
        "or_set_channel_scaling": (C.c_int, [C.c_void_p, C.c_int32, dp, dp]),
        "or_init": (C.c_int, [C.c_void_p]),
        "or_rhs": (C.c_int, [C.c_void_p, C.c_double, dp, dp]),
        "or_run": (C.c_int, [C.c_void_p, C.c_int32, dp, dp, dp, dp, dp, dp]),
        "or_init_integrator": (C.c_int, [C.c_void_p, C.c_int32, dp]),
        "or_step": (C.c_int, [C.c_void_p, C.c_double]),
        "or_get_stats": (C.c_int, [C.c_void_p, C.POINTER(FiStats)]),
        "or_record_steps": (C.c_int, [C.c_void_p, C.c_int64]),
        "or_get_sealevel": (C.c_int, [C.c_void_p, C.c_void_p]),
        "or_set_ocean_surface_table": (C.c_int, [C.c_void_p, C.c_int32, dp, dp]),
        "or_set_bsl_history": (C.c_int, [C.c_void_p, C.c_int32, dp, dp]),
        "or_resume": (C.c_int, [C.c_void_p, C.c_double, C.c_int64, dp, dp, dp, C.c_int32, dp]),
        "or_get_step_record": (C.c_int, [C.c_void_p, dp, C.c_int64, C.POINTER(C.c_int64)]),
        "or_set_step_replay": (C.c_int, [C.c_void_p, C.c_int64, dp]),
        "or_last_error": (C.c_char_p, [C.c_void_p]),
        "or_destroy": (None, [C.c_void_p]),
        "or_set_threads": (None, [C.c_int32]),
        "or_nextfastfft": (C.c_int32, [C.c_int32]),
        "or_kei": (C.c_double, [C.c_double]),
        "or_second_derivatives": (None, [C.c_int32, C.c_int32, C.c_double, C.c_double, dp, dp, dp, dp, dp]),
        "or_fft2": (C.c_int, [C.c_int32, C.c_int32, dp, dp, dp, dp, C.c_int32]),
        "or_conv_full": (C.c_int, [C.c_int32, C.c_int32, dp, dp, dp]),
        "or_bs3_decay": (C.c_int, [C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int32, dp,
                                   dp, C.POINTER(C.c_int64)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _p(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_double))


def set_threads(n: int) -> None:
    lib().or_set_threads(int(n))


class OracleSim:
    """Oracle simulation, driven with the same fi_config / field ids as the library."""

    def __init__(self, cfg):
        self.cfg = cfg
        self.n = cfg.nx * cfg.ny
        h = C.c_void_p()
        rc = lib().or_create(C.byref(cfg), C.byref(h))
        if rc:
            raise RuntimeError(f"or_create failed ({rc})")
        self.h = h

    def _check(self, rc, what):
        if rc:
            raise RuntimeError(f"oracle {what} failed ({rc}): {lib().or_last_error(self.h).decode()}")

    def set_field(self, fid: int, a):
        a = np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
        self._check(lib().or_set_field(self.h, fid, _p(a), a.size), "set_field")

    def get_field(self, fid: int):
        a = np.empty(self.n)
        self._check(lib().or_get_field(self.h, fid, _p(a), a.size), "get_field")
        return a

    def set_ice_history(self, t, H):
        t = np.ascontiguousarray(t, dtype=np.float64)
        H = np.ascontiguousarray(H, dtype=np.float64).reshape(-1)
        self._check(lib().or_set_ice_history(self.h, t.size, _p(t), _p(H)), "set_ice_history")

    def set_elastic_table(self, rm, GE):
        rm = np.ascontiguousarray(rm, dtype=np.float64)
        GE = np.ascontiguousarray(GE, dtype=np.float64)
        self._check(lib().or_set_elastic_table(self.h, rm.size, _p(rm), _p(GE)), "set_elastic_table")

    def set_channel_scaling(self, ratio, thick):
        ratio = np.ascontiguousarray(ratio, dtype=np.float64)
        thick = np.ascontiguousarray(thick, dtype=np.float64)
        self._check(lib().or_set_channel_scaling(self.h, ratio.size, _p(ratio), _p(thick)), "set_channel_scaling")

    def init(self):
        self._check(lib().or_init(self.h), "init")

    def rhs(self, t, u):
        u = np.array(u, dtype=np.float64).reshape(-1)
        du = np.empty_like(u)
        self._check(lib().or_rhs(self.h, float(t), _p(u), _p(du)), "rhs")
        return u, du

    def run(self, t_out, want=("u", "ue", "dudt", "dz_ss")):
        t_out = np.ascontiguousarray(t_out, dtype=np.float64)
        k = t_out.size
        outs = {name: (np.zeros(k * self.n) if name in want else None) for name in ("u", "ue", "dudt", "dz_ss")}
        ot = np.zeros(k)
        self._check(lib().or_run(self.h, k, _p(t_out), _p(ot), _p(outs["u"]), _p(outs["ue"]), _p(outs["dudt"]),
                                 _p(outs["dz_ss"])), "run")
        res = {name: v.reshape(k, self.n) for name, v in outs.items() if v is not None}
        res["t"] = ot
        return res

    def init_integrator(self, tstops=()):
        ts = np.ascontiguousarray(tstops, dtype=np.float64)
        self._check(lib().or_init_integrator(self.h, ts.size, _p(ts) if ts.size else None), "init_integrator")

    def step(self, dt):
        self._check(lib().or_step(self.h, float(dt)), "step")

    def sealevel(self):
        from fastiso_b200.abi import FiSealevel

        out = FiSealevel()
        self._check(lib().or_get_sealevel(self.h, C.byref(out)), "get_sealevel")
        return {k: getattr(out, k) for k, _ in FiSealevel._fields_ if k != "pad"}

    def set_ocean_surface_table(self, z, A):
        z = np.ascontiguousarray(z, dtype=np.float64)
        A = np.ascontiguousarray(A, dtype=np.float64)
        self._check(lib().or_set_ocean_surface_table(self.h, z.size, _p(z), _p(A)), "set_ocean_surface_table")

    def set_bsl_history(self, t, z):
        t = np.ascontiguousarray(t, dtype=np.float64)
        z = np.ascontiguousarray(z, dtype=np.float64)
        self._check(lib().or_set_bsl_history(self.h, t.size, _p(t), _p(z)), "set_bsl_history")

    def resume(self, t, count_sparse, u, ue, dz_ss, tstops=()):
        """Start the integrator at t from a state computed elsewhere (flat x-fastest
        u, ue, dz_ss and the sparse-update count at t)."""
        arrs = [np.ascontiguousarray(a, dtype=np.float64).reshape(-1) for a in (u, ue, dz_ss)]
        ts = np.ascontiguousarray(tstops, dtype=np.float64)
        self._check(lib().or_resume(self.h, float(t), int(count_sparse), *[_p(a) for a in arrs], ts.size,
                                    _p(ts) if ts.size else None), "resume")

    def record_steps(self, cap):
        self._check(lib().or_record_steps(self.h, int(cap)), "record_steps")

    def step_record(self, cap=None):
        n = C.c_int64()
        self._check(lib().or_get_step_record(self.h, None, 0, C.byref(n)), "get_step_record")
        k = n.value if cap is None else min(n.value, cap)
        out = np.empty(max(k, 1))
        self._check(lib().or_get_step_record(self.h, _p(out), k, C.byref(n)), "get_step_record")
        return out[:min(k, n.value)]

    def set_step_replay(self, dts):
        dts = np.ascontiguousarray(dts, dtype=np.float64)
        self._check(lib().or_set_step_replay(self.h, dts.size, _p(dts) if dts.size else None), "set_step_replay")

    def stats(self):
        from fastiso_b200.abi import FiStats

        st = FiStats()
        self._check(lib().or_get_stats(self.h, C.byref(st)), "get_stats")
        return {k: getattr(st, k) for k, _ in FiStats._fields_}

    def close(self):
        if self.h:
            lib().or_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def second_derivatives(u2d, Dx, Dy):
    """Reference CPU stencils on a numpy (nx, ny) array [i, j]; returns uxx, uyy, ux, uxy."""
    nx, ny = u2d.shape
    u = np.ascontiguousarray(u2d.T).reshape(-1)
    outs = [np.empty_like(u) for _ in range(4)]
    lib().or_second_derivatives(nx, ny, float(Dx), float(Dy), _p(u), *[_p(o) for o in outs])
    return [o.reshape(ny, nx).T for o in outs]


def fft2(a2d, inverse=False):
    nx, ny = a2d.shape
    a = np.ascontiguousarray(a2d.T)
    re = np.ascontiguousarray(a.real, dtype=np.float64).reshape(-1)
    im = np.ascontiguousarray(a.imag, dtype=np.float64).reshape(-1)
    ore, oim = np.empty_like(re), np.empty_like(im)
    lib().or_fft2(nx, ny, _p(re), _p(im), _p(ore), _p(oim), 1 if inverse else 0)
    return (ore + 1j * oim).reshape(ny, nx).T


def conv_full(kernel2d, input2d):
    nx, ny = kernel2d.shape
    k = np.ascontiguousarray(kernel2d.T, dtype=np.float64).reshape(-1)
    x = np.ascontiguousarray(input2d.T, dtype=np.float64).reshape(-1)
    out = np.empty((2 * ny - 1) * (2 * nx - 1))
    lib().or_conv_full(nx, ny, _p(k), _p(x), _p(out))
    return out.reshape(2 * ny - 1, 2 * nx - 1).T


def kei(x: float) -> float:
    """The Kelvin function kei of the oracle's ELRA Green's function."""
    return float(lib().or_kei(float(x)))


def nextfastfft(n: int) -> int:
    return int(lib().or_nextfastfft(int(n)))


def bs3_decay(lam, u0, t1, t_out, reltol=1e-3, abstol=1e-6):
    t_out = np.ascontiguousarray(t_out, dtype=np.float64)
    u = np.empty_like(t_out)
    ns = C.c_int64()
    rc = lib().or_bs3_decay(float(lam), float(u0), float(t1), float(reltol), float(abstol), t_out.size, _p(t_out),
                            _p(u), C.byref(ns))
    if rc:
        raise RuntimeError(f"bs3_decay failed {rc}")
    return u, ns.value


def oracle_for(sim):
    """An OracleSim fed the same host inputs as a library Simulation (fields, ice
    history, Farrell table, channel scaling)."""
    from fastiso_b200 import abi

    inp = sim.prepared_inputs()
    ref = OracleSim(inp["cfg"])
    for name, arr in inp["fields"].items():
        ref.set_field(abi.FIELDS[name], np.asarray(arr, dtype=np.float64).ravel(order="F"))
    if inp["ice_t"] is not None:
        ref.set_ice_history(inp["ice_t"], np.stack([np.asarray(h, dtype=np.float64).ravel(order="F")
                                                    for h in inp["ice_H"]]))
    ref.set_elastic_table(*inp["elastic_table"])
    ratio, thick = inp["channels"]
    if ratio.size:
        ref.set_channel_scaling(ratio, thick)
    if inp.get("ocean_surface") is not None:
        ref.set_ocean_surface_table(*inp["ocean_surface"])
    if inp.get("bsl_history") is not None:
        ref.set_bsl_history(*inp["bsl_history"])
    return ref
