// fno_gemm.cu -- tcgen05 GEMM kernels of the Fourier-neural-operator surrogate (see
// fno_gemm.cuh for the data layout and the pipeline).
#include "../../include/fastiso_b200.h"
#include "fno_gemm.cuh"

#include <atomic>
#include <mutex>

using namespace fi;

namespace fi {

static std::atomic<long long> g_tc_polls{TC_SPIN_LIMIT};
long long tc_wait_polls() { return g_tc_polls.load(); }
void tc_set_wait_polls(long long polls) { g_tc_polls.store(polls < 0 ? TC_SPIN_LIMIT : polls); }

// The status word of fi_fno_gemm: one static device int.  Its address on each device is
// looked up once (cudaGetSymbolAddress with that device current) and cached.
static __device__ int g_gemm_err;

namespace {
constexpr int GEMM_MAX_DEVICES = 64;
std::mutex g_err_mu;
int* g_err_ptr[GEMM_MAX_DEVICES] = {};

cudaError_t gemm_err_word(int** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= GEMM_MAX_DEVICES) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_err_mu);
    if (!g_err_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_gemm_err);
        if (e != cudaSuccess) return e;
        g_err_ptr[dev] = (int*)p;
    }
    *out = g_err_ptr[dev];
    return cudaSuccess;
}
}  // namespace

}  // namespace fi

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
    if (gemm_err_word(&d_err) != cudaSuccess) return FI_ERR_CUDA;
    // stream 0 (legacy) orders the clear, the GEMM and the read-back; calls from several
    // host threads share the word and are serialised by that stream
    if (cudaMemsetAsync(d_err, 0, sizeof(int), 0) != cudaSuccess) return FI_ERR_CUDA;
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
    if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    if (e != cudaSuccess) return FI_ERR_CUDA;
    return herr ? herr : FI_OK;
}
