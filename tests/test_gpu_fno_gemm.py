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
                         C.c_void_p(Cm.data_ptr()), N, batch, M * K, N * K, M * N, 0)
    assert rc == 0
    want = torch.bmm(A.float(), B.float().transpose(1, 2))
    err = (Cm - want).abs().max().item() / want.abs().max().item()
    assert err < 1e-5, err


@pytest.mark.parametrize("M,N,K,batch,flags", [(128, 32, 64, 1, 1), (256, 64, 32, 2, 1), (136, 48, 96, 1, 2),
                                               (128, 128, 64, 1, 3), (64, 32, 8, 3, 1)])
def test_tc_gemm_mn_major_operands(M, N, K, batch, flags):
    """MN-major A (stored K x M, e.g. an NCHW activation read as pixels x channels) and B."""
    torch = pytest.importorskip("torch")
    g = torch.Generator(device="cpu").manual_seed(M + 3 * N + K)
    A = torch.randn(batch, M, K, generator=g).to(torch.bfloat16)
    B = torch.randn(batch, N, K, generator=g).to(torch.bfloat16)
    Ad = (A.transpose(1, 2).contiguous() if flags & 1 else A).cuda()
    Bd = (B.transpose(1, 2).contiguous() if flags & 2 else B).cuda()
    lda = M if flags & 1 else K
    ldb = N if flags & 2 else K
    Cm = torch.full((batch, M, N), float("nan"), dtype=torch.float32, device="cuda")
    lib = abi.load_library()
    rc = lib.fi_fno_gemm(M, N, K, C.c_void_p(Ad.data_ptr()), lda, C.c_void_p(Bd.data_ptr()), ldb,
                         C.c_void_p(Cm.data_ptr()), N, batch, M * K, N * K, M * N, flags)
    assert rc == 0
    want = torch.bmm(A.float(), B.float().transpose(1, 2)).cuda()
    err = (Cm - want).abs().max().item() / want.abs().max().item()
    assert err < 1e-5, err
