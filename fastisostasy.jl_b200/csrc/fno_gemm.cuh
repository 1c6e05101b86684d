// fno_gemm.cuh -- BF16 x BF16 -> FP32 GEMM on the 5th-generation tensor cores (tcgen05)
// for the Fourier-neural-operator surrogate.
//
//   C[m][n] = sum_k A[m][k] * B[n][k]      (A: M x K, B: N x K, both K-contiguous rows)
//
// One block of 128 threads computes a 128 x BN tile.  Per K chunk of 64 the block copies
// its A and B rows into shared memory in the K-major, no-swizzle canonical layout of the
// UMMA operand descriptors (8-row x 16-byte core matrices; the core matrices of one
// 8-row group follow each other along K at LBO bytes, the 8-row groups at SBO bytes),
// one elected thread issues four tcgen05.mma (K = 16 each, kind::f16, BF16 inputs, FP32
// accumulation in tensor memory) and commits them to an mbarrier; the chunks are double
// buffered so the copy of chunk i+1 overlaps the MMAs of chunk i.  The epilogue reads the
// accumulator with tcgen05.ld (warp w owns TMEM lanes 32w..32w+31, i.e. tile rows) and
// hands each row's BN values to an epilogue functor.  Every mbarrier wait is bounded: on
// expiry the block raises an error word, frees its tensor memory and returns.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/fastiso_b200.h"

namespace fi {

constexpr int TC_BM = 128;       // tile rows (UMMA M)
constexpr int TC_BK = 64;        // K per chunk (4 UMMA of K = 16)
constexpr int TC_THREADS = 128;  // one warpgroup
constexpr long long TC_SPIN_LIMIT = 1LL << 26;

// K-major no-swizzle operand layout of `rows` rows x 64 K elements (BF16): byte offset of
// element (r, k).  Core matrix (8 rows x 8 elements = 128 B) of row group g, K group c
// at c * (rows * 16) + g * 128; inside it row r % 8 at 16 B steps.
__host__ __device__ inline uint32_t tc_operand_offset(int rows, int r, int k) {
    return (uint32_t)((k >> 3) * (rows * 16) + (r >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// UMMA shared-memory descriptor (sm_100): start >> 4 in bits [0,14), LBO >> 4 in [16,30),
// SBO >> 4 in [32,46), version 1 in [46,48), layout type 0 (no swizzle) in [61,64).
__host__ __device__ inline uint64_t tc_smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// UMMA instruction descriptor, kind::f16: FP32 accumulator, BF16 A and B, both K-major,
// N >> 3 in bits [17,23), M >> 4 in bits [24,29).
__host__ __device__ inline uint32_t tc_instr_desc(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}


// ---------------------------------------------------------------------------
// PTX wrappers (sm_100a)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t tc_smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(tc_smem_u32(bar)), "r"(count) : "memory");
}

// true when the phase with the given parity has completed
__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(tc_smem_u32(bar)), "r"(parity)
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
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem_u32(dst_smem)),
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
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(tc_smem_u32(bar))
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
    // Two-level batch (split-K reductions): with zdiv > 1 batch z reads
    // A + (z / zdiv) * sA + (z % zdiv) * sA2, and likewise for B.
    int zdiv;
    long long sA2, sB2;
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
    const int z1 = g.zdiv > 1 ? (int)blockIdx.z / g.zdiv : (int)blockIdx.z;
    const int z2 = g.zdiv > 1 ? (int)blockIdx.z % g.zdiv : 0;
    const __nv_bfloat16* A = g.A + (size_t)z1 * g.sA + (size_t)z2 * g.sA2;
    const __nv_bfloat16* B = g.B + (size_t)z1 * g.sB + (size_t)z2 * g.sB2;
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
            const uint32_t a0 = tc_smem_u32(sa), b0 = tc_smem_u32(sb);
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
        // the epilogue is copied so that it may carry per-row state across its column chunks
        Epi e = epi;
        const int row = m0 + warp * 32 + lane;
        for (int c0 = 0; c0 < BN; c0 += 16) {
            float v[16];
            tc_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
            if (row < g.M && n0 + c0 < g.N) e(blockIdx.z, row, n0 + c0, v, g.N - (n0 + c0));
        }
        if (row < g.M) e.row_done(blockIdx.z, row);
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
    __device__ __forceinline__ void row_done(int, int) const {}
};

template <int BN, class Epi>
inline cudaError_t launch_gemm_tc(const TcGemmArgs& g, int batch, const Epi& epi, cudaStream_t st) {
    constexpr int STAGE = (TC_BM + BN) * TC_BK * 2;
    static unsigned attr_set = 0;  // one bit per device
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev >= 32 || !(attr_set & (1u << dev))) {
        e = cudaFuncSetAttribute(k_gemm_tc<BN, Epi>, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * STAGE);
        if (e != cudaSuccess) return e;
        if (dev < 32) attr_set |= 1u << dev;
    }
    dim3 grid((g.M + TC_BM - 1) / TC_BM, (g.N + BN - 1) / BN, batch);
    k_gemm_tc<BN, Epi><<<grid, TC_THREADS, 2 * STAGE, st>>>(g, epi);
    return cudaGetLastError();
}

}  // namespace fi
