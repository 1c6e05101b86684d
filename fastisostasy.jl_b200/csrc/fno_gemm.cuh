// fno_gemm.cuh -- BF16 x BF16 -> FP32 GEMM on the 5th-generation tensor cores (tcgen05)
// for the Fourier-neural-operator surrogate.
//
//   C[z][m][n] = sum_k A[z][m][k] * B[z][n][k]
//
// Each 128-thread block computes 128 x BN output tiles (one per block as launched below).
// Per K chunk of 64 the block copies its A and B rows into shared memory with cp.async
// (16-byte copies, zero-filled outside the matrix) in the no-swizzle canonical layout of
// the UMMA operand descriptors (8-row x 16-byte core matrices; the core matrices of one
// 8-row group follow each other along K at LBO bytes, the 8-row groups at SBO bytes);
// one elected thread issues four tcgen05.mma (K = 16 each, kind::f16, BF16 inputs, FP32
// accumulation in tensor memory) and commits them to an mbarrier.  Two stage buffers:
// the copy of the next chunk -- of this tile or of the block's next tile -- is in flight
// while the tensor cores run the current one and while the epilogue reads the finished
// accumulator with tcgen05.ld (warp w owns TMEM lanes 32w..32w+31, i.e. tile rows) and
// hands each row's BN values to an epilogue functor.  Every mbarrier wait is bounded: on
// expiry the block raises an error word, waits for its copies, frees its tensor memory and
// returns.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <atomic>

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

// bounded wait of at most `polls` tests; false when the limit ran out
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long long polls = TC_SPIN_LIMIT) {
    for (long long i = 0; i < polls; i++)
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
// One GEMM operand.  K-major (mn = 0): element (r, k) of batch (z1, z2) at
// p[z1 * s + z2 * s2 + r * ld + k], rows K-contiguous.  MN-major (mn = 1): at
// p[z1 * s + z2 * s2 + k * ld + r], each K column contiguous along the rows (an NCHW
// activation read as pixels x channels).  The tensor cores take either form: the shared
// memory image keeps the same core-matrix grid and only the inside of each 128-byte
// core matrix is transposed, which bit 15 (A) / 16 (B) of the instruction descriptor
// announces.
struct TcOperand {
    const __nv_bfloat16* p = nullptr;
    int ld = 0;
    long long s = 0, s2 = 0;
    int mn = 0;
};

struct TcGemmArgs {
    int M = 0, N = 0, K = 0;
    TcOperand A, B;    // product columns [0, K1)
    TcOperand A2, B2;  // product columns [K1, K) read at column k - K1 (unused when K1 == K)
    int K1 = 0;        // multiple of 16; 0 means K
    int batch = 1;
    // two-level batch: with zdiv > 1 batch z is (z / zdiv, z % zdiv), else (z, 0)
    int zdiv = 1;
    int* err = nullptr;  // set to FI_ERR_TIMEOUT when a wait gives up
    long long polls = TC_SPIN_LIMIT;  // bound of each commit wait (tc_wait_polls())
};

// Poll bound of the commit waits for the next launches: TC_SPIN_LIMIT unless a test
// lowered it with fi_debug_set_wait_limit (fno_gemm.cu).
long long tc_wait_polls();

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, bool valid) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(valid ? 16 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// rows x 64 chunk (product columns k0 .. k0 + 63) of one side (A or B) of the product
// into the canonical layout at shared address dst, zero outside [0, nrows) x [0, K).
// Column groups of 8 below K1 come from o1, the rest from o2 at column k - K1.  `safe`
// is any valid global address (the source operand of a zero-filled copy, never read).
template <int ROWS>
__device__ __forceinline__ void tc_stage(uint32_t dst, const TcOperand& o1, const TcOperand& o2, int z1, int z2,
                                         int row0, int nrows, int k0, int K, int K1, const void* safe) {
    static_assert(TC_THREADS % 8 == 0, "a thread keeps one K group of the K-major copies");
    // K-major groups: one 16-byte copy = 8 consecutive K elements of one row; thread t
    // always copies K group t % 8, so its operand and column are fixed
    if (!(o1.mn && o2.mn)) {
        const int kv = threadIdx.x & 7, gk = k0 + kv * 8;
        const bool second = gk >= K1;
        const TcOperand& o = second ? o2 : o1;
        if (!o.mn) {
            const bool kok = gk < K;
            const __nv_bfloat16* base =
                kok ? o.p + (size_t)z1 * o.s + (size_t)z2 * o.s2 + (second ? gk - K1 : gk) : nullptr;
            for (int r = threadIdx.x >> 3; r < ROWS; r += TC_THREADS / 8) {
                const int gr = row0 + r;
                const bool ok = kok && gr < nrows;
                cp_async16(dst + tc_operand_offset(ROWS, r, kv * 8),
                           ok ? (const void*)(base + (size_t)gr * o.ld) : safe, ok);
            }
        }
    }
    // MN-major groups: one 16-byte copy = 8 consecutive rows of one K column, stored as
    // row (k % 8) of core matrix (k / 8, r / 8)
    if (o1.mn || o2.mn) {
        constexpr int RV = ROWS / 8;
        for (int v = threadIdx.x; v < RV * 64; v += TC_THREADS) {
            const int kc = v / RV, rv = v - kc * RV;
            const int gk = k0 + kc;
            const bool second = gk >= K1;
            const TcOperand& o = second ? o2 : o1;
            if (!o.mn) continue;
            const int gr = row0 + rv * 8, ck = second ? gk - K1 : gk;
            const bool ok = gr < nrows && gk < K;
            const void* src =
                ok ? (const void*)(o.p + (size_t)z1 * o.s + (size_t)z2 * o.s2 + (size_t)ck * o.ld + gr) : safe;
            cp_async16(dst + (kc >> 3) * (ROWS * 16) + rv * 128 + (kc & 7) * 16, src, ok);
        }
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
    const int mt = (g.M + TC_BM - 1) / TC_BM, nt = (g.N + BN - 1) / BN;
    const int nch = (g.K + TC_BK - 1) / TC_BK;
    const int K1 = g.K1 > 0 ? g.K1 : g.K;
    const long long ntiles = (long long)mt * nt * g.batch;
    const long long my_tiles = ntiles > blockIdx.x ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    const long long njobs = my_tiles * nch;  // (tile, chunk) pairs of this block, chunk fastest
    const uint32_t sbase = tc_smem_u32(smem);
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
    // output tile and chunk of job j, in 32-bit arithmetic (the launch checks that tiles x
    // chunks fit; 64-bit divisions cost ~10x more instructions in every thread)
    const unsigned umnt = (unsigned)mt * (unsigned)nt, unch = (unsigned)nch, umt = (unsigned)mt;
    auto job = [&](long long j, int& m0, int& n0, int& z, int& c) {
        const unsigned jj = (unsigned)j;
        const unsigned jq = jj / unch;
        const unsigned tile = blockIdx.x + jq * gridDim.x;
        c = (int)(jj - jq * unch);
        const unsigned zt = tile / umnt;
        const unsigned mn = tile - zt * umnt;
        z = (int)zt;
        const unsigned nq = mn / umt;
        m0 = (int)(mn - nq * umt) * TC_BM;
        n0 = (int)nq * BN;
    };
    auto stage = [&](long long j) {
        int m0, n0, z, c;
        job(j, m0, n0, z, c);
        const int z1 = g.zdiv > 1 ? z / g.zdiv : z, z2 = g.zdiv > 1 ? z % g.zdiv : 0;
        const uint32_t sa = sbase + (uint32_t)(j & 1) * STAGE;
        tc_stage<TC_BM>(sa, g.A, g.A2, z1, z2, m0, g.M, c * TC_BK, g.K, K1, g.A.p);
        tc_stage<BN>(sa + A_BYTES, g.B, g.B2, z1, z2, n0, g.N, c * TC_BK, g.K, K1, g.A.p);
        cp_async_commit();
    };
    long long last_commit = -1;  // thread 0: the last job whose MMAs were committed
    if (njobs > 0) stage(0);
    for (long long j = 0; j < njobs; j++) {
        const int s = (int)(j & 1);
        if (j + 1 < njobs) {
            // the other stage buffer was last read by the MMAs of job j - 1
            if (j >= 1 && tid == 0 && !mbar_wait(&bars[(j - 1) & 1], (uint32_t)(((j - 1) >> 1) & 1), g.polls))
                s_fail = 1;
            __syncthreads();
            if (s_fail) break;
            stage(j + 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        fence_async_smem();
        __syncthreads();
        int m0, n0, z, c;
        job(j, m0, n0, z, c);
        if (tid == 0) {
            tc_fence_after();
            const uint32_t a0 = sbase + (uint32_t)s * STAGE, b0 = a0 + A_BYTES;
#pragma unroll
            for (int ks = 0; ks < TC_BK / 16; ks++) {
                // K step ks covers core-matrix columns 2ks and 2ks + 1
                const uint64_t da = tc_smem_desc(a0 + 2 * ks * (TC_BM * 16), TC_BM * 16, 128);
                const uint64_t db = tc_smem_desc(b0 + 2 * ks * (BN * 16), BN * 16, 128);
                const bool second = c * TC_BK + ks * 16 >= K1;
                const uint32_t amn = second ? g.A2.mn : g.A.mn, bmn = second ? g.B2.mn : g.B.mn;
                tc_mma(tmem, da, db, idesc | (amn << 15) | (bmn << 16), (c > 0 || ks > 0) ? 1u : 0u);
            }
            tc_commit(&bars[s]);
            last_commit = j;
        }
        if (c == nch - 1) {
            // tile complete: wait for its MMAs, read the accumulator, hand rows to the epilogue
            if (tid == 0 && !mbar_wait(&bars[s], (uint32_t)((j >> 1) & 1), g.polls)) s_fail = 1;
            __syncthreads();
            if (s_fail) break;
            tc_fence_after();
            Epi e = epi;  // per tile: the epilogue may carry per-row state across its column chunks
            const int row = m0 + warp * 32 + lane;
            for (int c0 = 0; c0 < BN; c0 += 16) {
                float v[16];
                tc_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
                if (row < g.M && n0 + c0 < g.N) e(z, row, n0 + c0, v, g.N - (n0 + c0));
            }
            if (row < g.M) e.row_done(z, row);
            tc_fence_before();
            __syncthreads();  // the next tile's MMAs overwrite the accumulator
        }
    }
    cp_async_wait<0>();
    if (s_fail && tid == 0) {
        if (g.err) atomicExch(g.err, FI_ERR_TIMEOUT);
        // before the tensor memory is released, let the MMAs already issued finish
        // (their commit completes every earlier tcgen05 operation of this thread);
        // bounded again, with the full limit
        if (last_commit >= 0) mbar_wait(&bars[last_commit & 1], (uint32_t)((last_commit >> 1) & 1));
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
        if (nvalid >= 16 && ((uintptr_t)c & 15) == 0) {
            float4* c4 = reinterpret_cast<float4*>(c);
#pragma unroll
            for (int q = 0; q < 4; q++) c4[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
            return;
        }
#pragma unroll
        for (int i = 0; i < 16; i++)
            if (i < nvalid) c[i] = v[i];
    }
    __device__ __forceinline__ void row_done(int, int) const {}
};

// One block per output tile (the kernel also walks several tiles per block when the grid
// is smaller; measured slower here, where most products have a single K chunk: separate
// blocks overlap one tile's epilogue with another's MMAs through their own tensor memory).
template <int BN, class Epi>
inline cudaError_t launch_gemm_tc(const TcGemmArgs& g, int batch, const Epi& epi, cudaStream_t st) {
    constexpr int STAGE = (TC_BM + BN) * TC_BK * 2;
    static std::atomic<unsigned> attr_set{0};  // one bit per device (handles may run on several threads)
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev >= 32) return cudaErrorInvalidDevice;
    if (!(attr_set.load() & (1u << dev))) {
        e = cudaFuncSetAttribute(k_gemm_tc<BN, Epi>, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * STAGE);
        if (e != cudaSuccess) return e;
        attr_set.fetch_or(1u << dev);
    }
    TcGemmArgs a = g;
    a.batch = batch;
    a.polls = tc_wait_polls();
    const long long ntiles =
        (long long)((g.M + TC_BM - 1) / TC_BM) * ((g.N + BN - 1) / BN) * (long long)batch;
    if (ntiles <= 0) return cudaSuccess;
    if (ntiles > 0x7fffffffLL || ntiles * (long long)((g.K + TC_BK - 1) / TC_BK) > 0x7fffffffLL)
        return cudaErrorInvalidValue;
    k_gemm_tc<BN, Epi><<<(unsigned)ntiles, TC_THREADS, 2 * STAGE, st>>>(a, epi);
    return cudaGetLastError();
}

}  // namespace fi
