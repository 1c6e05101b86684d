// fno_gemm.cu -- tcgen05 GEMM kernels of the Fourier-neural-operator surrogate (see
// fno_gemm.cuh for the data layout and the pipeline).
#include "../../include/fastiso_b200.h"
#include "fno_gemm.cuh"

using namespace fi;

// C[z] = A[z] * B[z]^T, BF16 inputs, FP32 output; device pointers.  flags bit 0: A is
// MN-major (element (m, k) at A[k * lda + m]), bit 1: B is MN-major.
extern "C" int fi_fno_gemm(int32_t M, int32_t N, int32_t K, const void* A, int32_t lda, const void* B, int32_t ldb,
                           float* C, int32_t ldc, int32_t batch, int64_t sA, int64_t sB, int64_t sC, int32_t flags) {
    if (M < 1 || N < 1 || K < 1 || batch < 1 || !A || !B || !C) return FI_ERR_ARG;
    const int amn = flags & 1, bmn = (flags >> 1) & 1;
    if (lda % 8 || ldb % 8 || sA % 8 || sB % 8 || ((uintptr_t)A & 15) || ((uintptr_t)B & 15))
        return FI_ERR_ARG;  // 16-byte vector copies
    if ((amn ? M : K) % 8 || (bmn ? N : K) % 8 || K % 8) return FI_ERR_ARG;
    int* d_err = nullptr;
    if (cudaMalloc(&d_err, sizeof(int)) != cudaSuccess) return FI_ERR_CUDA;
    cudaMemset(d_err, 0, sizeof(int));
    TcGemmArgs g;
    g.M = M;
    g.N = N;
    g.K = K;
    g.A.p = (const __nv_bfloat16*)A;
    g.A.ld = lda;
    g.A.s = sA;
    g.A.mn = amn;
    g.B.p = (const __nv_bfloat16*)B;
    g.B.ld = ldb;
    g.B.s = sB;
    g.B.mn = bmn;
    g.err = d_err;
    EpiStoreF32 epi{C, ldc, sC};
    cudaError_t e = N <= 32 ? launch_gemm_tc<32>(g, batch, epi, 0)
                  : N <= 64 ? launch_gemm_tc<64>(g, batch, epi, 0)
                            : launch_gemm_tc<128>(g, batch, epi, 0);
    int herr = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(d_err);
    if (e != cudaSuccess) return FI_ERR_CUDA;
    return herr ? herr : FI_OK;
}
