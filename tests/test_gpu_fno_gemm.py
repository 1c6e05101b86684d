"""tcgen05 BF16 GEMM of the surrogate (fi_fno_gemm) against an FP32 matmul of the
same BF16-rounded operands."""
import ctypes as C

import pytest

import fastiso_b200 as F  # noqa: F401
from fastiso_b200 import abi

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("M,N,K,batch", [(128, 32, 64, 1), (300, 64, 200, 1), (1000, 128, 512, 3),
                                         (256, 50, 32, 2), (129, 17, 8, 1)])
def test_tc_gemm_matches_fp32(M, N, K, batch):
    torch = pytest.importorskip("torch")
    g = torch.Generator(device="cpu").manual_seed(M * 7 + N)
    A = torch.randn(batch, M, K, generator=g).to(torch.bfloat16).cuda()
    B = torch.randn(batch, N, K, generator=g).to(torch.bfloat16).cuda()
    Cm = torch.full((batch, M, N), float("nan"), dtype=torch.float32, device="cuda")
    lib = abi.load_library()
    rc = lib.fi_fno_gemm(M, N, K, C.c_void_p(A.data_ptr()), K, C.c_void_p(B.data_ptr()), K,
                         C.c_void_p(Cm.data_ptr()), N, batch, M * K, N * K, M * N)
    assert rc == 0
    want = torch.bmm(A.float(), B.float().transpose(1, 2))
    err = (Cm - want).abs().max().item() / want.abs().max().item()
    assert err < 1e-5, err
