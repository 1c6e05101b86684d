"""The persistent kernels with the radix sequences of the benchmark grids compiled in
(350 = 5*5*2*7, 1024 = 8*4*8*4) against the kernel that runs the plans' passes at run
time: the same butterflies in the same order, so the trajectories are bitwise equal."""
import hashlib

import numpy as np
import pytest

import fastiso_b200 as F
import fastiso_b200.workloads as W

pytestmark = pytest.mark.gpu


def _trajectory(monkeypatch, seq, N, years, outs):
    if seq:
        monkeypatch.delenv("FI_PERSIST_SEQ", raising=False)
    else:
        monkeypatch.setenv("FI_PERSIST_SEQ", "0")
    sim = W.config2(form="fp32", N=N, t_end=2e3, n_snap=3)
    sim.cfg.max_steps = 10**8
    it = F.init_integrator(sim)
    fields = []
    for k in range(outs):
        F.step(it, years, True)
        fields.append({f: sim.get_field(f) for f in ("u", "ue", "dz_ss")})
    st = sim.stats()
    sched = sim.get_fft_schedule(N)
    sim.close()
    return fields, st, sched


@pytest.mark.parametrize("N,years,outs", [(350, 12.0, 3), (1024, 1.0, 2)])
def test_compiled_sequence_bitwise(monkeypatch, N, years, outs):
    a, sa, sched = _trajectory(monkeypatch, True, N, years, outs)
    b, sb, _ = _trajectory(monkeypatch, False, N, years, outs)
    assert list(sched) == ([5, 5, 2, 7] if N == 350 else [8, 4, 8, 4])
    for k in ("naccept", "nreject", "nf", "nsparse"):
        assert sa[k] == sb[k], (k, sa[k], sb[k])
    assert sa["nsparse"] >= 1
    for fa, fb in zip(a, b):
        for f in fa:
            assert np.array_equal(fa[f], fb[f]), (N, f, hashlib.sha1(fa[f].tobytes()).hexdigest()[:8])
