"""Argument checks of the surrogate's entry points that run on the host before any CUDA
call, so they are exercised without a GPU: invalid sizes, layouts and alignments return
FI_ERR_ARG."""
import ctypes as C

from fastiso_b200 import abi

ALIGNED = C.c_void_p(1 << 20)       # never dereferenced: the checks reject before any use
MISALIGNED = C.c_void_p((1 << 20) + 2)


def _gemm(lib, M=128, N=32, K=64, A=ALIGNED, lda=64, B=ALIGNED, ldb=64, batch=1, sA=0, sB=0, flags=0):
    return lib.fi_fno_gemm(M, N, K, A, lda, B, ldb, ALIGNED, N, batch, sA, sB, 0, flags)


def test_fno_gemm_rejects_bad_shapes_and_layouts():
    lib = abi.load_library()
    assert _gemm(lib, K=60, lda=60, ldb=60) == abi.FI_ERR_ARG        # K not a multiple of 8
    assert _gemm(lib, lda=63) == abi.FI_ERR_ARG                      # row pitch
    assert _gemm(lib, sA=12) == abi.FI_ERR_ARG                       # batch stride
    assert _gemm(lib, A=MISALIGNED) == abi.FI_ERR_ARG                # 16-byte alignment
    assert _gemm(lib, M=100, lda=104, flags=1) == abi.FI_ERR_ARG     # MN-major A needs M % 8 == 0
    assert _gemm(lib, N=20, ldb=24, flags=2) == abi.FI_ERR_ARG       # MN-major B needs N % 8 == 0
    assert _gemm(lib, M=0) == abi.FI_ERR_ARG
    assert _gemm(lib, batch=0) == abi.FI_ERR_ARG
    assert lib.fi_fno_gemm(128, 32, 64, None, 64, ALIGNED, 64, ALIGNED, 32, 1, 0, 0, 0, 0) == abi.FI_ERR_ARG


def test_fno_create_rejects_bad_sizes():
    lib = abi.load_library()
    h = C.c_void_p()
    for S, B in ((48, 4), (16, 4), (512, 4), (128, 0), (128, 257)):
        assert lib.fi_fno_create(S, B, 0, 0, C.byref(h)) == abi.FI_ERR_ARG, (S, B)
        assert not h.value
    assert lib.fi_fno_create(128, 4, 0, 0, None) == abi.FI_ERR_ARG
    assert lib.fi_fno_num_params(None) == -1
