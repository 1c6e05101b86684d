"""FFT radix schedules (fi_set_fft_schedule): right-hand-side parity with the FP64 oracle
under non-default radix orders, the radix-16 butterfly included, and the API's checks."""
import numpy as np
import pytest

import fastiso_b200 as F
from fastiso_b200 import abi
from helpers import F_, TOL, rel_l2
from test_gpu_parity import pair, small_sim

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("form", ["fp32", "fp64"])
@pytest.mark.parametrize("N,sched,Msched", [
    (64, [16, 4], [16, 8]), (64, [4, 16], [8, 16]), (64, [2, 2, 16], [2, 4, 16]),
    (96, [3, 2, 16], [16, 3, 4]), (35, [7, 5], [7, 2, 5]), (50, [10, 5], [4, 25]),
])
def test_schedule_rhs_parity(form, N, sched, Msched):
    sim = small_sim(form, N, N, t_end=100.0)
    M = F.nextfastfft(2 * N - 1)
    assert int(np.prod(Msched)) == M
    sim._ensure_handle()
    sim.set_fft_schedule(N, sched)
    sim.set_fft_schedule(M, Msched)
    assert sim.get_fft_schedule(N) == sched and sim.get_fft_schedule(M) == Msched
    ref = pair(sim)
    rng = np.random.default_rng(N)
    u = -40 * np.exp(-sim.domain.R**2 / (2 * (0.3 * sim.domain.Wx) ** 2)) + 0.3 * rng.standard_normal((N, N))
    for t in (0.5, 12.5, 31.0):
        ug, dg = u.copy(), np.zeros_like(u)
        F.update_diagnostics(dg, ug, sim, t)
        _, dr = ref.rhs(t, F_(u))
        assert rel_l2(F_(dg), dr) < TOL[form], (sched, t, rel_l2(F_(dg), dr))
        assert rel_l2(F_(sim.get_field("ue")), ref.get_field(abi.FIELDS["ue"])) < TOL[form]
        assert rel_l2(F_(sim.get_field("dz_ss")), ref.get_field(abi.FIELDS["dz_ss"])) < TOL[form]
        u = u + 0.1 * dg
    sim.close()
    ref.close()


def test_schedule_checks():
    sim = small_sim("fp32", 64, 64, t_end=100.0)
    sim._ensure_handle()
    with pytest.raises(abi.FiError) as e:
        sim.set_fft_schedule(64, [8, 4])          # product 32
    assert e.value.code == abi.FI_ERR_ARG
    with pytest.raises(abi.FiError) as e:
        sim.set_fft_schedule(60, [4, 3, 5])       # not a transform length of a 64 x 64 grid
    assert e.value.code == abi.FI_ERR_ARG
    with pytest.raises(abi.FiError) as e:
        sim.set_fft_schedule(64, [64, 1])         # radix 1
    assert e.value.code == abi.FI_ERR_ARG
    sim.init_problem()
    with pytest.raises(abi.FiError) as e:
        sim.set_fft_schedule(64, [16, 4])         # after fi_init
    assert e.value.code == abi.FI_ERR_STATE
    sim.close()
