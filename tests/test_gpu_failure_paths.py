"""Failure paths on the GPU without a GPU fault: bounded device waits that run out
(the kernel returns FI_ERR_TIMEOUT, the context and the handle stay usable) and
checkpoints that do not fit the handle (rejected before any state changes)."""
import ctypes as C

import numpy as np
import pytest

import fastiso_b200 as F
import fastiso_b200.workloads as W
from fastiso_b200 import abi
from helpers import F_

pytestmark = pytest.mark.gpu


def _small(form="fp32", N=48):
    s = W.config2(form=form, N=N, t_end=2000.0, out_every=1000.0)
    s.cfg.max_steps = 10_000_000
    return s


@pytest.fixture
def wait_limits():
    lib = abi.load_library()
    yield lib
    for which in (abi.FI_WAIT_GRID_POLLS, abi.FI_WAIT_GRID_EXTRA_ARRIVALS, abi.FI_WAIT_TC_POLLS):
        assert lib.fi_debug_set_wait_limit(which, -1) == abi.FI_OK


def test_grid_barrier_timeout_returns_and_handle_recovers(wait_limits):
    """Every grid barrier of the persistent step kernel expects one block more than the
    launch has, with a bound of 4096 polls: each wait runs out, the kernel returns, the
    call reports FI_ERR_TIMEOUT; restoring the checkpoint taken before, the same handle
    then steps bitwise like a handle that never timed out."""
    lib = wait_limits
    a, b = _small(), _small()
    ia, ib = F.init_integrator(a), F.init_integrator(b)
    if a.stats()["executor"] != abi.FI_EXEC_PERSIST:
        pytest.skip("persistent executor not selected on this device")
    F.step(ia, 5.0, True)
    F.step(ib, 5.0, True)
    ck = a.checkpoint()
    assert lib.fi_debug_set_wait_limit(abi.FI_WAIT_GRID_EXTRA_ARRIVALS, 1) == abi.FI_OK
    assert lib.fi_debug_set_wait_limit(abi.FI_WAIT_GRID_POLLS, 4096) == abi.FI_OK
    rc = lib.fi_step(a._handle, 5.0)
    assert rc == abi.FI_ERR_TIMEOUT, (rc, lib.fi_last_error(a._handle))
    assert b"grid barrier" in lib.fi_last_error(a._handle)
    assert lib.fi_debug_set_wait_limit(abi.FI_WAIT_GRID_EXTRA_ARRIVALS, -1) == abi.FI_OK
    assert lib.fi_debug_set_wait_limit(abi.FI_WAIT_GRID_POLLS, -1) == abi.FI_OK
    a.restore(ck)
    F.step(ia, 5.0, True)
    F.step(ib, 5.0, True)
    np.testing.assert_array_equal(F_(a.get_field("u")), F_(b.get_field("u")))
    assert a.stats()["status"] == abi.FI_OK
    a.close()
    b.close()


def test_tensor_core_wait_timeout_returns(wait_limits):
    """A commit wait bound of 0 polls makes the GEMM's first wait give up at once: the
    block lets its issued MMAs finish, frees its tensor memory and the call reports
    FI_ERR_TIMEOUT; with the default bound the next call is exact again."""
    torch = pytest.importorskip("torch")
    lib = wait_limits
    M, N, K = 256, 64, 128
    g = torch.Generator(device="cpu").manual_seed(3)
    A = torch.randn(M, K, generator=g).to(torch.bfloat16).cuda()
    B = torch.randn(N, K, generator=g).to(torch.bfloat16).cuda()
    Cm = torch.zeros(M, N, dtype=torch.float32, device="cuda")

    def gemm():
        return lib.fi_fno_gemm(M, N, K, C.c_void_p(A.data_ptr()), K, C.c_void_p(B.data_ptr()), K,
                               C.c_void_p(Cm.data_ptr()), N, 1, 0, 0, 0, 0)

    assert lib.fi_debug_set_wait_limit(abi.FI_WAIT_TC_POLLS, 0) == abi.FI_OK
    assert gemm() == abi.FI_ERR_TIMEOUT
    assert lib.fi_debug_set_wait_limit(abi.FI_WAIT_TC_POLLS, -1) == abi.FI_OK
    Cm.zero_()
    assert gemm() == abi.FI_OK
    ref = A.float() @ B.float().T
    assert float((Cm - ref).norm() / ref.norm()) < 1e-5


def _restore_rc(sim, blob):
    buf = C.create_string_buffer(bytes(blob), len(blob))
    return sim.lib.fi_restore(sim._handle, buf, len(blob))


def test_restore_rejects_foreign_or_corrupt_checkpoints():
    a32, b32 = _small("fp32"), _small("fp32")
    a64 = _small("fp64")
    other = _small("fp32", N=40)
    for s in (a32, b32, a64, other):
        F.step(F.init_integrator(s), 2.0, True)
    ck32, ck64, ck_other = a32.checkpoint(), a64.checkpoint(), other.checkpoint()
    u_before = F_(b32.get_field("u"))
    st_before = b32.stats()
    # another form, another grid
    assert _restore_rc(b32, ck64) == abi.FI_ERR_ARG
    assert _restore_rc(b32, ck_other) == abi.FI_ERR_ARG
    # truncated: inside the header, inside the tstops, inside the state
    for cut in (8, 200, len(ck32) // 2, len(ck32) - 1):
        assert _restore_rc(b32, ck32[:cut]) == abi.FI_ERR_ARG, cut
    # a corrupt tstop count (header field at byte 32) and a corrupt magic
    bad = bytearray(ck32)
    bad[32:40] = (1 << 60).to_bytes(8, "little")
    assert _restore_rc(b32, bytes(bad)) == abi.FI_ERR_ARG
    bad = bytearray(ck32)
    bad[0] = ord("X")
    assert _restore_rc(b32, bytes(bad)) == abi.FI_ERR_ARG
    # nothing changed on the rejected handle
    np.testing.assert_array_equal(F_(b32.get_field("u")), u_before)
    st = b32.stats()
    assert (st["t"], st["naccept"], st["nreject"]) == (st_before["t"], st_before["naccept"], st_before["nreject"])
    # the matching checkpoint restores
    assert _restore_rc(b32, ck32) == abi.FI_OK
    np.testing.assert_array_equal(F_(b32.get_field("u")), F_(a32.get_field("u")))
    for s in (a32, b32, a64, other):
        s.close()
