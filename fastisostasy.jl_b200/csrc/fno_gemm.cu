// fno_gemm.cu -- tcgen05 GEMM kernels of the Fourier-neural-operator surrogate (see
// fno_gemm.cuh for the data layout and the pipeline).
#include "../../include/fastiso_b200.h"
#include "fno_gemm.cuh"

using namespace fi;

// C[z] = A[z] * B[z]^T, BF16 inputs (K-contiguous rows), FP32 output; device pointers.
extern "C" int fi_fno_gemm(int32_t M, int32_t N, int32_t K, const void* A, int32_t lda, const void* B, int32_t ldb,
                           float* C, int32_t ldc, int32_t batch, int64_t sA, int64_t sB, int64_t sC) {
    if (M < 1 || N < 1 || K < 1 || batch < 1 || !A || !B || !C) return FI_ERR_ARG;
    if (K % 8 || lda % 8 || ldb % 8 || sA % 8 || sB % 8 || ((uintptr_t)A & 15) || ((uintptr_t)B & 15))
        return FI_ERR_ARG;  // 16-byte vector copies of the operand rows
    int* d_err = nullptr;
    if (cudaMalloc(&d_err, sizeof(int)) != cudaSuccess) return FI_ERR_CUDA;
    cudaMemset(d_err, 0, sizeof(int));
    TcGemmArgs g{M, N, K, (const __nv_bfloat16*)A, (const __nv_bfloat16*)B, lda, ldb, sA, sB, d_err, 1, 0, 0};
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
