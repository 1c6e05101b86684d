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

}  // namespace fi
