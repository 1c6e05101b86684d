"""Writes the golden fixtures of this directory from the FP64 oracle (the checker of
the CUDA path), after checking the oracle against the reference's known-answer tests
(test/test_derivatives.jl, test/test_convolution.jl, src/analytic_solutions.jl,
src/integrators.jl:205-217).  Run from the repository root, on CPU:

    python tests/golden/make_golden.py

Fixtures (x fastest, as the C ABI):
  rhs_n24.npz   two update_diagnostics! calls on golden_sim (24 x 20): u in/out, dudt,
                ue, dz_ss after each call
  run_n32.npz   run! of golden_sim(32 x 32) to 1000 yr, outputs at 300, 600, 1000 yr
  conv_32.npz   full linear convolution of seeded 32 x 32 float32 arrays (scipy direct)
  analytic.npz  the Bueler disc-load solution along the x transect at 5 and 10 kyr
"""
import pathlib
import sys

import numpy as np
import scipy.signal

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))
import __graft_entry__  # noqa: E402

__graft_entry__.load_package()
import fastiso_b200 as F  # noqa: E402
from fastiso_b200 import abi  # noqa: E402
from helpers import (F_, GOLDEN_RHS_TIMES, GOLDEN_RUN_T_END, GOLDEN_RUN_TIMES, golden_sim, golden_u,  # noqa: E402
                     oracle_for)
from oracle import oracle as O  # noqa: E402
import test_oracle_kats as K  # noqa: E402


def main():
    # the oracle must pass the reference's known-answer tests first
    K.test_derivative_polynomial_kat()
    K.test_convolution_vs_direct()
    K.test_bs3_exponential_decay()
    K.test_analytic_disc_load()

    sim = golden_sim("fp64")
    ref = oracle_for(sim)
    ref.init()
    u = F_(golden_u(sim))
    rec = {"u_in": u}
    for i, t in enumerate(GOLDEN_RHS_TIMES):
        uo, du = ref.rhs(t, u)
        rec[f"u_out{i}"] = uo
        rec[f"dudt{i}"] = du
        rec[f"ue{i}"] = ref.get_field(abi.FIELDS["ue"])
        rec[f"dz_ss{i}"] = ref.get_field(abi.FIELDS["dz_ss"])
    np.savez_compressed(HERE / "rhs_n24.npz", t=np.asarray(GOLDEN_RHS_TIMES), **rec)

    sim = golden_sim("fp64", 32, 32, t_end=GOLDEN_RUN_T_END)
    ref = oracle_for(sim)
    ref.init()
    out = ref.run(np.asarray(GOLDEN_RUN_TIMES))
    np.savez_compressed(HERE / "run_n32.npz", t=out["t"], u=out["u"], ue=out["ue"], dudt=out["dudt"],
                        dz_ss=out["dz_ss"])

    rng = np.random.default_rng(32)
    k = rng.random((32, 32)).astype(np.float32).astype(np.float64)
    x = rng.random((32, 32)).astype(np.float32).astype(np.float64)
    np.savez_compressed(HERE / "conv_32.npz", k=k, x=x, full=scipy.signal.convolve2d(k, x, mode="full"))

    domain = F.RegionalDomain(3e6, 7)
    se = F.SolidEarth(domain, layer_boundaries=[88e3], layer_viscosities=[1e21], rho_litho=0.0)
    c = F.PhysicalConstants()
    xs = domain.x[domain.mx - 1:]
    D = float(np.mean(se.litho_rigidity))
    eta = float(np.mean(se.effective_viscosity))
    ana = np.array([[K.analytic_solution(abs(xv), t * c.seconds_per_year, c.rho_ice, c.g, se.rho_uppermantle, D,
                                         eta) for xv in xs] for t in (5e3, 10e3)])
    np.savez_compressed(HERE / "analytic.npz", t=np.array([5e3, 10e3]), x=xs, u=ana)
    for f in sorted(HERE.glob("*.npz")):
        print(f.name, f.stat().st_size, "bytes")


if __name__ == "__main__":
    main()
