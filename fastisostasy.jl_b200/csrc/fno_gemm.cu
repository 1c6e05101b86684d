// fno_gemm.cu -- tcgen05 GEMM kernels of the Fourier-neural-operator surrogate (see
// fno_gemm.cuh for the data layout and the pipeline).
#include "../../include/fastiso_b200.h"
#include "fno_gemm.cuh"

namespace fi {

// ---------------------------------------------------------------------------
// PTX wrappers (sm_100a)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// true when the phase with the given parity has completed
__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// bounded wait; false when the limit ran out
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    for (long long i = 0; i < TC_SPIN_LIMIT; i++)
        if (mbar_test(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tc_alloc(uint32_t* dst_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)),
                 "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tc_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tc_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void tc_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// ---------------------------------------------------------------------------
// the GEMM
// ---------------------------------------------------------------------------
struct TcGemmArgs {
    int M, N, K;
    const __nv_bfloat16* A;  // M x K, row pitch lda (elements)
    const __nv_bfloat16* B;  // N x K, row pitch ldb
    int lda, ldb;
    long long sA, sB;        // batch strides (elements)
    int* err;                // set to FI_ERR_TIMEOUT when a wait gives up
};

// rows x 64 chunk of a K-contiguous operand into the canonical layout (zero outside)
template <int ROWS>
__device__ __forceinline__ void tc_stage(unsigned char* dst, const __nv_bfloat16* src, int ld, int row0, int nrows,
                                         int k0, int K) {
    for (int v = threadIdx.x; v < ROWS * 8; v += TC_THREADS) {
        const int r = v >> 3, kv = v & 7;
        const int gr = row0 + r, gk = k0 + kv * 8;
        uint4 val = make_uint4(0u, 0u, 0u, 0u);
        if (gr < nrows && gk < K) val = *reinterpret_cast<const uint4*>(src + (size_t)gr * ld + gk);
        *reinterpret_cast<uint4*>(dst + tc_operand_offset(ROWS, r, kv * 8)) = val;
    }
}

template <int BN, class Epi>
__global__ void __launch_bounds__(TC_THREADS) k_gemm_tc(TcGemmArgs g, Epi epi) {
    constexpr int A_BYTES = TC_BM * TC_BK * 2, B_BYTES = BN * TC_BK * 2, STAGE = A_BYTES + B_BYTES;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ uint32_t tmem_base;
    __shared__ int s_fail;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * TC_BM, n0 = blockIdx.y * BN;
    const __nv_bfloat16* A = g.A + (size_t)blockIdx.z * g.sA;
    const __nv_bfloat16* B = g.B + (size_t)blockIdx.z * g.sB;
    if (warp == 0) {
        tc_alloc(&tmem_base, BN < 32 ? 32 : BN);
        tc_relinquish();
    }
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_fail = 0;
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base;
    const uint32_t idesc = tc_instr_desc(TC_BM, BN);
    const int nchunks = (g.K + TC_BK - 1) / TC_BK;
    for (int c = 0; c < nchunks; c++) {
        const int s = c & 1;
        unsigned char* sa = smem + s * STAGE;
        unsigned char* sb = sa + A_BYTES;
        if (c >= 2 && tid == 0 && !mbar_wait(&bars[s], ((c - 2) >> 1) & 1)) s_fail = 1;
        __syncthreads();
        if (s_fail) break;
        tc_stage<TC_BM>(sa, A, g.lda, m0, g.M, c * TC_BK, g.K);
        tc_stage<BN>(sb, B, g.ldb, n0, g.N, c * TC_BK, g.K);
        fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t a0 = smem_u32(sa), b0 = smem_u32(sb);
#pragma unroll
            for (int ks = 0; ks < TC_BK / 16; ks++) {
                // K step ks covers core-matrix columns 2ks and 2ks + 1
                const uint64_t da = tc_smem_desc(a0 + 2 * ks * (TC_BM * 16), TC_BM * 16, 128);
                const uint64_t db = tc_smem_desc(b0 + 2 * ks * (BN * 16), BN * 16, 128);
                tc_mma(tmem, da, db, idesc, (c > 0 || ks > 0) ? 1u : 0u);
            }
            tc_commit(&bars[s]);
        }
    }
    if (tid == 0 && !s_fail && nchunks > 0 && !mbar_wait(&bars[(nchunks - 1) & 1], ((nchunks - 1) >> 1) & 1))
        s_fail = 1;
    __syncthreads();
    tc_fence_after();
    if (!s_fail) {
        const int row = m0 + warp * 32 + lane;
        for (int c0 = 0; c0 < BN; c0 += 16) {
            float v[16];
            tc_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
            if (row < g.M) epi(blockIdx.z, row, n0 + c0, v, g.N - (n0 + c0));
        }
    } else if (tid == 0 && g.err) {
        atomicExch(g.err, FI_ERR_TIMEOUT);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tc_dealloc(tmem, BN < 32 ? 32 : BN);
}

// plain FP32 store: C[z][row][col], pitch ldc
struct EpiStoreF32 {
    float* C;
    int ldc;
    long long sC;
    __device__ __forceinline__ void operator()(int z, int row, int col0, const float* v, int nvalid) const {
        float* c = C + (size_t)z * sC + (size_t)row * ldc + col0;
        const int n = nvalid < 16 ? nvalid : 16;
        for (int i = 0; i < n; i++) c[i] = v[i];
    }
};

template <int BN, class Epi>
static cudaError_t launch_gemm_tc(const TcGemmArgs& g, int batch, const Epi& epi, cudaStream_t st) {
    constexpr int STAGE = (TC_BM + BN) * TC_BK * 2;
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k_gemm_tc<BN, Epi>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             2 * STAGE);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    dim3 grid((g.M + TC_BM - 1) / TC_BM, (g.N + BN - 1) / BN, batch);
    k_gemm_tc<BN, Epi><<<grid, TC_THREADS, 2 * STAGE, st>>>(g, epi);
    return cudaGetLastError();
}

}  // namespace fi

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
    TcGemmArgs g{M, N, K, (const __nv_bfloat16*)A, (const __nv_bfloat16*)B, lda, ldb, sA, sB, d_err};
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
