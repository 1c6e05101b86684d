// fno.cu -- Fourier neural operator (FNO) surrogate of the LV-ELVA solver: forward pass,
// its adjoint (backward pass), Adam, all on the device.
//
// Network (fixed shape, S x S grid, S a multiple of 32 in [32, 256]):
//   input 6 channels -> lift (pointwise 6 -> 32) -> 4 Fourier layers of width 32
//   -> projection (pointwise 32 -> 128, GELU, 128 -> 1).
//   Fourier layer: z = SpectralConv(v) + Wloc v + b;  v' = GELU(z) (identity after the last).
//   SpectralConv keeps kx in [0, 16) (half axis, x) and ky in {0..15, S-16..S-1} (full axis,
//   y): 512 complex modes, one complex 32 x 32 channel matrix per mode; the inverse is the
//   real inverse DFT of that truncated half spectrum (weight 1 at kx = 0, 2 otherwise, 1/S^2).
//
// Every contraction but the per-mode weight gradient runs on the tcgen05 GEMM of
// fno_gemm.cuh (BF16 operands, FP32 accumulators in tensor memory):
//   DFT along x:   v[(b,c,y)][x]            x F1[(part,kx)][x]            -> T
//   DFT along y:   T[(kx,b,c)][(part,y)]    x F2[(kyi,part')][(part,y)]   -> Z (per mode)
//   channel mix:   Z[mode][b][(part,ci)]    x Wmat[mode][(part',co)][(part,ci)]  (512 batches)
//   inverse y:     Y[(b,co,kx)][(kyi,part)] x G2[(part',y)][(kyi,part)]   -> G[(b,y)][co][(kx,part)]
//   inverse x + pointwise path, one GEMM per row (b, y) of pixels x channels with K = 32 + 32:
//                  [G1[x][(kx,part)] | v[b][ci][y][x]]  x  [G[(b,y)][co][(kx,part)] | Wloc[co][ci]]
//                  (the activation v read in place from NCHW as an MN-major operand)
// The backward pass runs the same GEMMs against the transposed matrices, and the weight
// gradients of the pointwise layers are split-K GEMMs over pixels whose B operand carries a
// row of ones (bias gradient) and, for the projection, the loss gradient (dQ2).
//
// Activations live in NCHW ([b][c][y*S+x]) only: the pointwise layers and the projection
// read them as MN-major operands (pixels x channels).  All parameters are FP32 masters
// (Adam), packed to BF16 operand copies after each update.
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/fastiso_b200.h"
#include "fno_gemm.cuh"

namespace fi {
namespace fno {

typedef __nv_bfloat16 bf16;

constexpr int C = 32;         // width
constexpr int KX = 16;        // kept kx
constexpr int KY = 32;        // kept ky (kyi < 16: ky = kyi; else ky = S - 32 + kyi)
constexpr int NM = KX * KY;   // complex modes per layer
constexpr int NIN = 6;        // input channels
constexpr int XC = 8;         // padded input channels (6 inputs, ones, zero)
constexpr int VC = 34;        // channels of an NCHW activation buffer: 32, ones, loss gradient
constexpr int PW = 128;       // projection width
constexpr int NLAYER = 4;
constexpr long long SPEC = (long long)NM * 2 * C * C;  // [mode][re, im][ci][co]
constexpr long long LAYER = SPEC + C * C + C;          // spectral, Wloc[co][ci], bloc[co]

// offsets into the flat FP32 parameter (and gradient) vector
struct Offsets {
    long long P, bP, layer[NLAYER], Q1, b1, Q2, b2, total;
};

inline Offsets offsets() {
    Offsets o;
    o.P = 0;                // [32][6]
    o.bP = C * NIN;         // [32]
    long long p = o.bP + C;
    for (int l = 0; l < NLAYER; l++) {
        o.layer[l] = p;
        p += LAYER;
    }
    o.Q1 = p;               // [128][32]
    o.b1 = o.Q1 + PW * C;   // [128]
    o.Q2 = o.b1 + PW;       // [128]
    o.b2 = o.Q2 + PW;       // [1]
    o.total = o.b2 + 1;
    return o;
}

// ---------------------------------------------------------------------------
// device helpers
// ---------------------------------------------------------------------------
// GELU(a) = a Phi(a), Phi the standard normal distribution function
__device__ __forceinline__ float gelu(float a) { return 0.5f * a * (1.f + erff(a * 0.70710678118654752f)); }
// GELU and GELU'(a) = Phi(a) + a phi(a), Phi evaluated once
__device__ __forceinline__ void gelu_both(float a, float& g, float& gp) {
    const float Phi = 0.5f * (1.f + erff(a * 0.70710678118654752f));
    g = a * Phi;
    gp = Phi + a * 0.39894228040143268f * expf(-0.5f * a * a);
}
__device__ __forceinline__ float gelu_grad(float a) {
    float g, gp;
    gelu_both(a, g, gp);
    return gp;
}
__device__ __forceinline__ uint32_t pack2(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&h);
}
// 16 values as BF16 to a 32-byte aligned address
__device__ __forceinline__ void store16(bf16* dst, const float* v) {
    uint4* d = reinterpret_cast<uint4*>(dst);
    d[0] = make_uint4(pack2(v[0], v[1]), pack2(v[2], v[3]), pack2(v[4], v[5]), pack2(v[6], v[7]));
    d[1] = make_uint4(pack2(v[8], v[9]), pack2(v[10], v[11]), pack2(v[12], v[13]), pack2(v[14], v[15]));
}

// ---------------------------------------------------------------------------
// GEMM epilogues (called per row and 16-column chunk; every N below is a multiple of 16)
// ---------------------------------------------------------------------------

// lift: batch z = b, row p, col c -> v0 in NCHW
struct EpiLift {
    bf16* vext;
    const float* bias;
    int S2;
    __device__ __forceinline__ void operator()(int z, int p, int c0, const float* v, int) const {
        bf16* o = vext + ((size_t)z * VC + c0) * S2 + p;
#pragma unroll
        for (int i = 0; i < 16; i++) o[(size_t)i * S2] = __float2bfloat16_rn(v[i] + bias[c0 + i]);
    }
    __device__ __forceinline__ void row_done(int, int) const {}
};

// DFT along x and the adjoint of the inverse along x: col n = part*16 + kx,
// out T[kx][b][c][part][y].  per_sample: batch z = b and row = (c, y); else row = (b, c, y).
struct EpiDftX {
    bf16* T;
    int B, S, per_sample;
    __device__ __forceinline__ void operator()(int z, int row, int n0, const float* v, int) const {
        int b, c, y;
        if (per_sample) {
            b = z;
            c = row / S;
            y = row - c * S;
        } else {
            const int bc = row / S;
            y = row - bc * S;
            b = bc / C;
            c = bc - b * C;
        }
        const int part = n0 >> 4;
#pragma unroll
        for (int i = 0; i < 16; i++)
            T[(((size_t)i * B + b) * C + c) * 2 * S + part * S + y] = __float2bfloat16_rn(v[i]);
    }
    __device__ __forceinline__ void row_done(int, int) const {}
};

// DFT along y (and the adjoint of the inverse along y): row (kx, b, c), col n = kyi*2 + part,
// out Z[kx*KY + kyi][b][part*32 + c]
struct EpiModes {
    bf16* Z;
    int B;
    __device__ __forceinline__ void operator()(int, int row, int n0, const float* v, int) const {
        const int c = row % C, t = row / C, b = t % B, kx = t / B;
#pragma unroll
        for (int i = 0; i < 16; i++) {
            const int n = n0 + i, kyi = n >> 1, part = n & 1;
            Z[((size_t)(kx * KY + kyi) * B + b) * 64 + part * 32 + c] = __float2bfloat16_rn(v[i]);
        }
    }
    __device__ __forceinline__ void row_done(int, int) const {}
};

// channel mixing (forward and adjoint): batch z = mode, row b, col n = part*32 + c,
// out Y[b][c][kx][kyi*2 + part]
struct EpiMix {
    bf16* Y;
    __device__ __forceinline__ void operator()(int z, int row, int n0, const float* v, int) const {
        const int kx = z / KY, kyi = z - kx * KY;
#pragma unroll
        for (int i = 0; i < 16; i++) {
            const int n = n0 + i, part = n >> 5, c = n & 31;
            Y[(((size_t)row * C + c) * KX + kx) * 64 + kyi * 2 + part] = __float2bfloat16_rn(v[i]);
        }
    }
    __device__ __forceinline__ void row_done(int, int) const {}
};

// inverse DFT along y (and the adjoint of the DFT along y): row (b, c, kx), col n = part*S + y,
// out G[(b, y)][c][kx*2 + part]
struct EpiIdftY {
    bf16* G;
    int S;
    __device__ __forceinline__ void operator()(int, int row, int n0, const float* v, int) const {
        const int bc = row / KX, kx = row - bc * KX, b = bc / C, c = bc - b * C;
        const int part = n0 / S, y0 = n0 - part * S;
#pragma unroll
        for (int i = 0; i < 16; i++)
            G[(((size_t)b * S + y0 + i) * C + c) * 32 + kx * 2 + part] = __float2bfloat16_rn(v[i]);
    }
    __device__ __forceinline__ void row_done(int, int) const {}
};

// row (b, p), col c -> out[b][c][p] in FP32, stored or accumulated
struct EpiNchw {
    float* out;
    int S2, accumulate;
    __device__ __forceinline__ void operator()(int, int row, int c0, const float* v, int) const {
        const int b = row / S2, p = row - b * S2;
        float* o = out + ((size_t)b * C + c0) * S2 + p;
        if (accumulate) {
#pragma unroll
            for (int i = 0; i < 16; i++) o[(size_t)i * S2] += v[i];
        } else {
#pragma unroll
            for (int i = 0; i < 16; i++) o[(size_t)i * S2] = v[i];
        }
    }
    __device__ __forceinline__ void row_done(int, int) const {}
};

// inverse DFT along x + pointwise path + bias: batch z = (b, y), row x, col c.  Saves z
// (FP32) and writes the activation, both NCHW.
struct EpiPixAct {
    const float* bias;
    float* zs;
    bf16* vext;
    int S, S2, act;
    __device__ __forceinline__ void operator()(int z, int x, int c0, const float* v, int) const {
        const int b = z / S, y = z - b * S;
        const size_t p = (size_t)y * S + x;
        float* zo = zs + ((size_t)b * C + c0) * S2 + p;
        bf16* vo = vext + ((size_t)b * VC + c0) * S2 + p;
#pragma unroll
        for (int i = 0; i < 16; i++) {
            const float zz = v[i] + bias[c0 + i];
            zo[(size_t)i * S2] = zz;
            vo[(size_t)i * S2] = __float2bfloat16_rn(act ? gelu(zz) : zz);
        }
    }
    __device__ __forceinline__ void row_done(int, int) const {}
};

// batch z = (b, y), row x, col c -> out[b][c][y*S + x] (FP32)
struct EpiPixStore {
    float* out;
    int S, S2;
    __device__ __forceinline__ void operator()(int z, int x, int c0, const float* v, int) const {
        const int b = z / S, y = z - b * S;
        float* o = out + ((size_t)b * C + c0) * S2 + (size_t)y * S + x;
#pragma unroll
        for (int i = 0; i < 16; i++) o[(size_t)i * S2] = v[i];
    }
    __device__ __forceinline__ void row_done(int, int) const {}
};

// projection: batch z = b, row p, col j (all 128 in one tile): q = sum_j GELU(a_j + b1_j) Q2_j + b2
struct EpiProj {
    const float* b1;
    const float* Q2;
    const float* b2;
    float* q;
    int S2;
    float acc;
    __device__ __forceinline__ void operator()(int, int, int j0, const float* v, int) {
#pragma unroll
        for (int i = 0; i < 16; i++) acc += gelu(v[i] + b1[j0 + i]) * Q2[j0 + i];
    }
    __device__ __forceinline__ void row_done(int z, int p) { q[(size_t)z * S2 + p] = acc + b2[0]; }
};

// projection adjoint (recomputes the hidden pre-activation a; batch z = b, row p):
// da = dq Q2 GELU'(a) in [(b,p)][j] and [b][j][p], the hidden GELU(a) in [b][128 + j][p]
struct EpiProjBwd {
    const float* b1;
    const float* Q2;
    const float* dq;
    bf16* da_rows;
    bf16* daT;
    int S2;
    __device__ __forceinline__ void operator()(int b, int p, int j0, const float* v, int) const {
        const size_t row = (size_t)b * S2 + p;
        const float g = dq[row];
        float d[16];
        bf16* t = daT + ((size_t)b * 2 * PW + j0) * S2 + p;
#pragma unroll
        for (int i = 0; i < 16; i++) {
            const float a = v[i] + b1[j0 + i];
            float ga, gpa;
            gelu_both(a, ga, gpa);
            d[i] = g * Q2[j0 + i] * gpa;
            t[(size_t)i * S2] = __float2bfloat16_rn(d[i]);
            t[(size_t)(PW + i) * S2] = __float2bfloat16_rn(ga);
        }
        store16(da_rows + (size_t)row * PW + j0, d);
    }
    __device__ __forceinline__ void row_done(int, int) const {}
};

// ---------------------------------------------------------------------------
// element-wise and reduction kernels
// ---------------------------------------------------------------------------

// x [B][6][S2] FP32 -> NCHW [b][8][S2] BF16 (channel 6 = 1 for the lift's bias gradient)
__global__ void k_prep_input(const float* __restrict__ x, bf16* xe, int B, int S2) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)B * S2) return;
    const int b = (int)(i / S2), p = (int)(i - (size_t)b * S2);
#pragma unroll
    for (int c = 0; c < NIN; c++)
        xe[((size_t)b * XC + c) * S2 + p] = __float2bfloat16_rn(x[((size_t)b * NIN + c) * S2 + p]);
    xe[((size_t)b * XC + 6) * S2 + p] = __float2bfloat16_rn(1.f);
    xe[((size_t)b * XC + 7) * S2 + p] = __float2bfloat16_rn(0.f);
}

// channel `ch` of every sample of an NCHW activation buffer := value
__global__ void k_fill_channel(bf16* v, int B, int S2, int ch, float value) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)B * S2) return;
    const int b = (int)(i / S2), p = (int)(i - (size_t)b * S2);
    v[((size_t)b * VC + ch) * S2 + p] = __float2bfloat16_rn(value);
}

// dz = dv * GELU'(z) (identity when z is null) -> BF16 NCHW and, if dzh, NHWC.
// One block per (sample, 64 pixels).
__global__ void __launch_bounds__(256) k_act_bwd(const float* __restrict__ dv, const float* __restrict__ z,
                                                 bf16* dz, bf16* dzh, int S2) {
    __shared__ float tile[C][65];
    const int tiles = S2 / 64;
    const int b = blockIdx.x / tiles, p0 = (blockIdx.x - b * tiles) * 64;
    for (int i = threadIdx.x; i < C * 64; i += 256) {
        const int c = i >> 6, px = i & 63;
        const size_t idx = ((size_t)b * C + c) * S2 + p0 + px;
        float d = dv[idx];
        if (z) d *= gelu_grad(z[idx]);
        dz[idx] = __float2bfloat16_rn(d);
        tile[c][px] = d;
    }
    if (!dzh) return;
    __syncthreads();
    for (int i = threadIdx.x; i < 64 * C; i += 256) {
        const int px = i >> 5, c = i & 31;
        dzh[((size_t)b * S2 + p0 + px) * C + c] = __float2bfloat16_rn(tile[c][px]);
    }
}

// loss gradient: weighted MSE against target, loss = (1/n) sum_i w_b(i) (q_i - t_i)^2 with
// per-sample weights w (1 when null), dq = 2 w (q - t) / n; or a given dy.
// Writes dq (FP32), its BF16 copy into channel 33 of the last activation buffer, and
// accumulates sum(dq) (gradient of b2).
__global__ void __launch_bounds__(256) k_loss(const float* __restrict__ q, const float* __restrict__ target,
                                              const float* __restrict__ w, const float* __restrict__ dy, int n,
                                              int S2, float inv_n, float* dq, bf16* vext4, float* part) {
    const int i = blockIdx.x * 256 + threadIdx.x;
    float l = 0.f, d = 0.f;
    if (i < n) {
        const int b = i / S2, p = i - b * S2;
        if (target) {
            const float e = q[i] - target[i], wb = w ? w[b] : 1.f;
            l = wb * e * e * inv_n;
            d = 2.f * wb * e * inv_n;
        } else {
            d = dy[i];
        }
        dq[i] = d;
        vext4[((size_t)b * VC + 33) * S2 + p] = __float2bfloat16_rn(d);
    }
    for (int o = 16; o > 0; o >>= 1) {
        l += __shfl_xor_sync(0xffffffffu, l, o);
        d += __shfl_xor_sync(0xffffffffu, d, o);
    }
    __shared__ float sl[8], sd[8];
    if ((threadIdx.x & 31) == 0) {
        sl[threadIdx.x >> 5] = l;
        sd[threadIdx.x >> 5] = d;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        float a = 0.f, c = 0.f;
        for (int w = 0; w < 8; w++) {
            a += sl[w];
            c += sd[w];
        }
        part[blockIdx.x] = a;
        part[gridDim.x + blockIdx.x] = c;
    }
}

// the per-block partials of k_loss summed in a fixed order (one block): the loss and the
// output-bias gradient come out the same on every run
__global__ void __launch_bounds__(256) k_loss_sum(const float* __restrict__ part, int nblk, float* loss, float* gb2) {
    __shared__ float sl[256], sd[256];
    float a = 0.f, c = 0.f;
    for (int i = threadIdx.x; i < nblk; i += 256) {
        a += part[i];
        c += part[nblk + i];
    }
    sl[threadIdx.x] = a;
    sd[threadIdx.x] = c;
    for (int o = 128; o > 0; o >>= 1) {
        __syncthreads();
        if (threadIdx.x < o) {
            sl[threadIdx.x] += sl[threadIdx.x + o];
            sd[threadIdx.x] += sd[threadIdx.x + o];
        }
    }
    if (threadIdx.x == 0) {
        *loss = sl[0];
        *gb2 += sd[0];
    }
}

// spectral weight gradient of one mode (block = mode):
//   dWr[ci][co] = sum_b dYr[co] Zr[ci] + dYi[co] Zi[ci]
//   dWi[ci][co] = sum_b dYi[co] Zr[ci] - dYr[co] Zi[ci]
__global__ void __launch_bounds__(256) k_spec_wgrad(const bf16* __restrict__ Z, const bf16* __restrict__ dY,
                                                    float* gW, int B) {
    __shared__ float zs[64][64], ds[64][64];
    const int mode = blockIdx.x, tid = threadIdx.x;
    float sr[4] = {0.f, 0.f, 0.f, 0.f}, si[4] = {0.f, 0.f, 0.f, 0.f};
    for (int b0 = 0; b0 < B; b0 += 64) {
        const int nb = min(64, B - b0);
        __syncthreads();
        for (int i = tid; i < nb * 64; i += 256) {
            const size_t g = ((size_t)mode * B + b0) * 64 + i;
            zs[i >> 6][i & 63] = __bfloat162float(Z[g]);
            ds[i >> 6][i & 63] = __bfloat162float(dY[g]);
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int idx = tid + 256 * k, ci = idx >> 5, co = idx & 31;
            for (int bb = 0; bb < nb; bb++) {
                const float zr = zs[bb][ci], zi = zs[bb][32 + ci], dr = ds[bb][co], di = ds[bb][32 + co];
                sr[k] += dr * zr + di * zi;
                si[k] += di * zr - dr * zi;
            }
        }
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int idx = tid + 256 * k;
        gW[(size_t)mode * 2 * C * C + idx] = sr[k];
        gW[((size_t)mode * 2 + 1) * C * C + idx] = si[k];
    }
}

// split-K partials [z][MN] summed over z and added to grad[base + map[i]] (map < 0: not a
// parameter; grad is zeroed before the backward pass; map is one-to-one), in two passes
// with a fixed summation order, so that gradients are the same on every run.  Pass 1:
// block (x, y) sums the z range y of gridDim.y for 256 consecutive i and leaves the sum
// in row z0 of its own range.  Pass 2 (k_reduce_map_fin) adds the ranges in order.
__global__ void k_reduce_map(float* part, int nz, int MN, const int* __restrict__ map) {
    const int i = blockIdx.x * 256 + threadIdx.x;
    if (i >= MN) return;
    if (map[i] < 0) return;
    const int per = (nz + gridDim.y - 1) / gridDim.y, z0 = blockIdx.y * per, z1 = min(nz, z0 + per);
    if (z1 <= z0) return;
    float s = 0.f;
    for (int z = z0; z < z1; z++) s += part[(size_t)z * MN + i];
    part[(size_t)z0 * MN + i] = s;
}

__global__ void k_reduce_map_fin(const float* __restrict__ part, int nz, int MN, int ny,
                                 const int* __restrict__ map, float* grad, long long base) {
    const int i = blockIdx.x * 256 + threadIdx.x;
    if (i >= MN) return;
    const int t = map[i];
    if (t < 0) return;
    const int per = (nz + ny - 1) / ny;
    float s = 0.f;
    for (int z0 = 0; z0 < nz; z0 += per) s += part[(size_t)z0 * MN + i];
    grad[base + t] += s;
}

static cudaError_t reduce_map(float* part, cudaStream_t st, int nz, int MN, int ny, const int* map, float* grad,
                              long long base) {
    const unsigned gx = (unsigned)((MN + 255) / 256);
    k_reduce_map<<<dim3(gx, ny), 256, 0, st>>>(part, nz, MN, map);
    k_reduce_map_fin<<<gx, 256, 0, st>>>(part, nz, MN, ny, map, grad, base);
    return cudaGetLastError();
}

__global__ void k_adam(float* p, const float* __restrict__ g, float* m, float* v, long long n, float lr, float b1,
                       float b2, float eps, float c1, float c2) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
    }
}

// spectral weights -> real 64 x 64 block matrices [[Wr, -Wi], [Wi, Wr]] (rows part'*32 + co,
// cols part*32 + ci) and their transposes; grid (mode, layer).  The weights are read and
// both matrices written along their rows, through a shared-memory copy of the mode.
__global__ void __launch_bounds__(256) k_pack_spec(const float* __restrict__ params, long long off0, bf16* Wm,
                                                   bf16* WmT) {
    __shared__ float w[2][C][C + 1];  // [re, im][ci][co]
    const int mode = blockIdx.x, l = blockIdx.y;
    const float* W = params + off0 + (long long)l * LAYER + (size_t)mode * 2 * C * C;
    for (int i = threadIdx.x; i < 2 * C * C; i += 256) w[i >> 10][(i >> 5) & 31][i & 31] = W[i];
    __syncthreads();
    const size_t o = ((size_t)l * NM + mode) * 4096;
    for (int i = threadIdx.x; i < 4096; i += 256) {
        // Wm row n = (pO, co), col k = (pI, ci)
        const int n = i >> 6, k = i & 63, pO = n >> 5, co = n & 31, pI = k >> 5, ci = k & 31;
        const float wr = w[0][ci][co], wi = w[1][ci][co];
        Wm[o + i] = __float2bfloat16_rn(pO == pI ? wr : (pO == 0 ? -wi : wi));
        // WmT row k' = (pI, ci), col n' = (pO, co): WmT[k'][n'] = Wm[n'][k']
        const int kk = i >> 6, nn = i & 63, pI2 = kk >> 5, ci2 = kk & 31, pO2 = nn >> 5, co2 = nn & 31;
        const float wr2 = w[0][ci2][co2], wi2 = w[1][ci2][co2];
        WmT[o + i] = __float2bfloat16_rn(pO2 == pI2 ? wr2 : (pO2 == 0 ? -wi2 : wi2));
    }
}

// pointwise weights -> BF16 operands: P [32][8], Wloc [l][co][ci] and [l][ci][co], Q1 [128][32], [32][128]
__global__ void k_pack_small(const float* __restrict__ params, Offsets o, bf16* Pb, bf16* Wl, bf16* WlT, bf16* Q1b,
                             bf16* Q1Tb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < C * XC) {
        const int c = i / XC, k = i - c * XC;
        Pb[i] = __float2bfloat16_rn(k < NIN ? params[o.P + c * NIN + k] : 0.f);
    }
    if (i < NLAYER * C * C) {
        const int l = i / (C * C), r = i - l * C * C, co = r / C, ci = r - co * C;
        const float w = params[o.layer[0] + (long long)l * LAYER + SPEC + r];
        Wl[i] = __float2bfloat16_rn(w);
        WlT[(size_t)l * C * C + ci * C + co] = __float2bfloat16_rn(w);
    }
    if (i < PW * C) {
        const int j = i / C, c = i - j * C;
        const float w = params[o.Q1 + i];
        Q1b[i] = __float2bfloat16_rn(w);
        Q1Tb[c * PW + j] = __float2bfloat16_rn(w);
    }
}

}  // namespace fno
}  // namespace fi

using namespace fi;
using namespace fi::fno;

struct fi_fno {
    int S = 0, S2 = 0, maxB = 0, device = 0, SL = 0, ns = 0;
    Offsets o{};
    cudaStream_t st = nullptr;
    float *params = nullptr, *grads = nullptr, *m = nullptr, *v = nullptr;
    long long adam_t = 0;
    float beta1 = 0.9f, beta2 = 0.999f, eps = 1e-8f;
    // BF16 operand copies of the parameters and the DFT matrices
    bf16 *Pb = nullptr, *Wm = nullptr, *WmT = nullptr, *Wl = nullptr, *WlT = nullptr, *Q1b = nullptr,
         *Q1Tb = nullptr;
    bf16 *F1 = nullptr, *F2 = nullptr, *G2 = nullptr, *G1 = nullptr, *F1T = nullptr, *F2T = nullptr,
         *G2T = nullptr, *G1T = nullptr;
    // activations (saved for the backward pass) and scratch
    bf16 *xe = nullptr, *vext[NLAYER + 1] = {}, *Tb = nullptr, *Zm[NLAYER] = {}, *Yb = nullptr, *Gt = nullptr,
         *dz = nullptr, *dYm = nullptr, *da_rows = nullptr, *daT = nullptr;
    float *zs[NLAYER] = {}, *q = nullptr, *dq = nullptr, *dvf = nullptr, *part = nullptr, *scal = nullptr;
    int *map_loc = nullptr, *map_proj = nullptr, *map_lift = nullptr, *err = nullptr;
    int fwdB = 0;  // batch of the last forward pass (0: none)
    std::vector<void*> allocs;
    std::string msg;
};

namespace {

int fail(fi_fno* h, int code, const std::string& m) {
    if (h) h->msg = m;
    return code;
}

#define FNO_CK(expr)                                                                         \
    do {                                                                                     \
        cudaError_t e_ = (expr);                                                             \
        if (e_ != cudaSuccess)                                                               \
            return fail(h, FI_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
    } while (0)

template <class T>
cudaError_t dalloc(fi_fno* h, T** p, size_t count) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, count * sizeof(T) + 16);
    if (e != cudaSuccess) return e;
    h->allocs.push_back(q);
    *p = (T*)q;
    return cudaMemset(q, 0, count * sizeof(T) + 16);
}

// operands: K-major (rows K-contiguous) and MN-major (NCHW read as pixels x channels)
TcOperand opK(const bf16* p, int ld, long long s = 0, long long s2 = 0) {
    TcOperand o;
    o.p = p;
    o.ld = ld;
    o.s = s;
    o.s2 = s2;
    o.mn = 0;
    return o;
}
TcOperand opMN(const bf16* p, int ld, long long s = 0, long long s2 = 0) {
    TcOperand o = opK(p, ld, s, s2);
    o.mn = 1;
    return o;
}

// C[z] = A[z] B[z]^T over K columns (columns [K1, K) from A2, B2 when K1 > 0)
template <class Epi>
cudaError_t gemm(fi_fno* h, int M, int N, int K, TcOperand A, TcOperand B, int batch, const Epi& epi, int zdiv = 1,
                 TcOperand A2 = TcOperand(), TcOperand B2 = TcOperand(), int K1 = 0) {
    TcGemmArgs g;
    g.M = M;
    g.N = N;
    g.K = K;
    g.A = A;
    g.B = B;
    g.A2 = A2;
    g.B2 = B2;
    g.K1 = K1;
    g.zdiv = zdiv;
    g.err = h->err;
    if (N <= 32) return launch_gemm_tc<32>(g, batch, epi, h->st);
    if (N <= 64) return launch_gemm_tc<64>(g, batch, epi, h->st);
    return launch_gemm_tc<128>(g, batch, epi, h->st);
}

uint64_t splitmix64(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
double unif(uint64_t& s) { return (double)(splitmix64(s) >> 11) * (1.0 / 9007199254740992.0); }

// default initialisation: pointwise layers U(-1/sqrt(fan_in), 1/sqrt(fan_in)); spectral
// weights U(0, 1/(C*C)) for the real and imaginary parts
std::vector<float> init_params(const Offsets& o, uint64_t seed) {
    std::vector<float> p(o.total);
    uint64_t s = seed;
    auto fill = [&](long long off, long long n, double lo, double hi) {
        for (long long i = 0; i < n; i++) p[off + i] = (float)(lo + (hi - lo) * unif(s));
    };
    const double a_in = 1.0 / std::sqrt((double)NIN), a_c = 1.0 / std::sqrt((double)C),
                 a_pw = 1.0 / std::sqrt((double)PW);
    fill(o.P, C * NIN, -a_in, a_in);
    fill(o.bP, C, -a_in, a_in);
    for (int l = 0; l < NLAYER; l++) {
        fill(o.layer[l], SPEC, 0.0, 1.0 / (C * C));
        fill(o.layer[l] + SPEC, C * C, -a_c, a_c);
        fill(o.layer[l] + SPEC + C * C, C, -a_c, a_c);
    }
    fill(o.Q1, PW * C, -a_c, a_c);
    fill(o.b1, PW, -a_c, a_c);
    fill(o.Q2, PW, -a_pw, a_pw);
    fill(o.b2, 1, -a_pw, a_pw);
    return p;
}

// truncated DFT matrices (FP64, rounded once to BF16); angles reduced exactly mod S
void build_dft(int S, std::vector<bf16> (&mats)[8]) {
    const double tw = 2.0 * M_PI / S, inv = 1.0 / ((double)S * S);
    auto ky_of = [S](int kyi) { return kyi < 16 ? kyi : S - KY + kyi; };
    std::vector<double> F1(32 * S), F2(64 * 2 * S), G2(2 * S * 64), G1(S * 32);
    for (int part = 0; part < 2; part++)
        for (int kx = 0; kx < KX; kx++)
            for (int x = 0; x < S; x++) {
                const double a = tw * ((kx * x) % S);
                F1[(part * 16 + kx) * S + x] = part ? -std::sin(a) : std::cos(a);
                const double w = (kx == 0 ? 1.0 : 2.0) * inv;
                G1[x * 32 + kx * 2 + part] = part ? -w * std::sin(a) : w * std::cos(a);
            }
    for (int kyi = 0; kyi < KY; kyi++)
        for (int y = 0; y < S; y++) {
            const double a = tw * (((long long)ky_of(kyi) * y) % S), c = std::cos(a), s = std::sin(a);
            // Z = sum_y (Tr + i Ti)(c - i s):  Zr = Tr c + Ti s,  Zi = -Tr s + Ti c
            F2[(kyi * 2 + 0) * 2 * S + 0 * S + y] = c;
            F2[(kyi * 2 + 0) * 2 * S + 1 * S + y] = s;
            F2[(kyi * 2 + 1) * 2 * S + 0 * S + y] = -s;
            F2[(kyi * 2 + 1) * 2 * S + 1 * S + y] = c;
            // G = sum_ky (Yr + i Yi)(c + i s):  Gr = Yr c - Yi s,  Gi = Yr s + Yi c
            G2[(0 * S + y) * 64 + kyi * 2 + 0] = c;
            G2[(0 * S + y) * 64 + kyi * 2 + 1] = -s;
            G2[(1 * S + y) * 64 + kyi * 2 + 0] = s;
            G2[(1 * S + y) * 64 + kyi * 2 + 1] = c;
        }
    auto bf = [](double d) { return __float2bfloat16_rn((float)d); };
    for (auto& m : mats) m.clear();
    mats[0].resize(32 * S);      // F1  [part*16+kx][x]
    mats[1].resize(64 * 2 * S);  // F2  [kyi*2+part'][part*S+y]
    mats[2].resize(2 * S * 64);  // G2  [part'*S+y][kyi*2+part]
    mats[3].resize(S * 32);      // G1  [x][kx*2+part]
    mats[4].resize(S * 32);      // F1T [x][kx*2+part]
    mats[5].resize(2 * S * 64);  // F2T [part*S+y][kyi*2+part']
    mats[6].resize(64 * 2 * S);  // G2T [kyi*2+part][part'*S+y]
    mats[7].resize(32 * S);      // G1T [part*16+kx][x]
    for (size_t i = 0; i < F1.size(); i++) mats[0][i] = bf(F1[i]);
    for (size_t i = 0; i < F2.size(); i++) mats[1][i] = bf(F2[i]);
    for (size_t i = 0; i < G2.size(); i++) mats[2][i] = bf(G2[i]);
    for (size_t i = 0; i < G1.size(); i++) mats[3][i] = bf(G1[i]);
    for (int x = 0; x < S; x++)
        for (int kx = 0; kx < KX; kx++)
            for (int part = 0; part < 2; part++) {
                mats[4][x * 32 + kx * 2 + part] = bf(F1[(part * 16 + kx) * S + x]);
                mats[7][(part * 16 + kx) * S + x] = bf(G1[x * 32 + kx * 2 + part]);
            }
    for (int r = 0; r < 2 * S; r++)
        for (int n = 0; n < 64; n++) {
            mats[5][r * 64 + n] = bf(F2[n * 2 * S + r]);
            mats[6][n * 2 * S + r] = bf(G2[r * 64 + n]);
        }
}

int pack(fi_fno* h) {
    k_pack_spec<<<dim3(NM, NLAYER), 256, 0, h->st>>>(h->params, h->o.layer[0], h->Wm, h->WmT);
    k_pack_small<<<(PW * C + 255) / 256, 256, 0, h->st>>>(h->params, h->o, h->Pb, h->Wl, h->WlT, h->Q1b, h->Q1Tb);
    FNO_CK(cudaGetLastError());
    return FI_OK;
}

// wait for the stream and read the GEMMs' timeout flag
int finish(fi_fno* h) {
    FNO_CK(cudaStreamSynchronize(h->st));
    int e = 0;
    FNO_CK(cudaMemcpy(&e, h->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) return fail(h, e, "a tensor-core GEMM wait gave up");
    return FI_OK;
}

int forward(fi_fno* h, int B, const float* x, float* y) {
    const int S = h->S, S2 = h->S2;
    const Offsets& o = h->o;
    const long long nb = (long long)B * S2, vs = (long long)VC * S2;
    k_prep_input<<<(unsigned)((nb + 255) / 256), 256, 0, h->st>>>(x, h->xe, B, S2);
    FNO_CK(cudaGetLastError());
    // lift: per sample, pixels x inputs (MN-major) times P
    FNO_CK(gemm(h, S2, C, XC, opMN(h->xe, S2, (long long)XC * S2), opK(h->Pb, XC), B,
                EpiLift{h->vext[0], h->params + o.bP, S2}));
    for (int l = 0; l < NLAYER; l++) {
        const float* lp = h->params + o.layer[l];
        // DFT along x: per sample, rows (c, y)
        FNO_CK(gemm(h, C * S, 2 * KX, S, opK(h->vext[l], S, vs), opK(h->F1, S), B, EpiDftX{h->Tb, B, S, 1}));
        // DFT along y: rows (kx, b, c)
        FNO_CK(gemm(h, KX * B * C, 2 * KY, 2 * S, opK(h->Tb, 2 * S), opK(h->F2, 2 * S), 1, EpiModes{h->Zm[l], B}));
        // channel mixing, one batch per mode
        FNO_CK(gemm(h, B, 64, 64, opK(h->Zm[l], 64, (long long)B * 64), opK(h->Wm + (size_t)l * NM * 4096, 64, 4096),
                    NM, EpiMix{h->Yb}));
        // inverse along y: rows (b, c, kx) -> G[(b, y)][c][(kx, part)]
        FNO_CK(gemm(h, B * C * KX, 2 * S, 64, opK(h->Yb, 64), opK(h->G2, 64), 1, EpiIdftY{h->Gt, S}));
        // inverse along x + pointwise path: batch (b, y), rows x, K = (kx, part) | ci
        FNO_CK(gemm(h, S, C, 64, opK(h->G1, 2 * KX), opK(h->Gt, 2 * KX, (long long)S * C * 32, (long long)C * 32),
                    B * S, EpiPixAct{lp + SPEC + C * C, h->zs[l], h->vext[l + 1], S, S2, l < NLAYER - 1 ? 1 : 0}, S,
                    opMN(h->vext[l], S2, vs, S), opK(h->Wl + (size_t)l * C * C, C), 2 * KX));
    }
    FNO_CK(gemm(h, S2, PW, C, opMN(h->vext[NLAYER], S2, vs), opK(h->Q1b, C), B,
                EpiProj{h->params + o.b1, h->params + o.Q2, h->params + o.b2, y, S2, 0.f}));
    h->fwdB = B;
    return FI_OK;
}

// gradients of all parameters from dq (and its BF16 copy) set by k_loss
int backward(fi_fno* h, int B) {
    const int S = h->S, S2 = h->S2, SL = h->SL, ns = h->ns;
    const Offsets& o = h->o;
    const long long vs = (long long)VC * S2, cs = (long long)C * S2;
    float* gr = h->grads;
    bf16* v4 = h->vext[NLAYER];
    // projection: recompute the hidden layer, da and GELU(a); weights by split-K over pixels
    FNO_CK(gemm(h, S2, PW, C, opMN(v4, S2, vs), opK(h->Q1b, C), B,
                EpiProjBwd{h->params + o.b1, h->params + o.Q2, h->dq, h->da_rows, h->daT, S2}));
    FNO_CK(gemm(h, 2 * PW, VC, SL, opK(h->daT, S2, (long long)2 * PW * S2, SL), opK(v4, S2, vs, SL), B * ns,
                EpiStoreF32{h->part, VC, (long long)2 * PW * VC}, ns));
    FNO_CK(reduce_map(h->part, h->st, B * ns, 2 * PW * VC, 16, h->map_proj, gr, 0));
    FNO_CK(gemm(h, B * S2, C, PW, opK(h->da_rows, PW), opK(h->Q1Tb, PW), 1, EpiNchw{h->dvf, S2, 0}));
    for (int l = NLAYER - 1; l >= 0; l--) {
        k_act_bwd<<<B * (S2 / 64), 256, 0, h->st>>>(h->dvf, l < NLAYER - 1 ? h->zs[l] : nullptr, h->dz, nullptr, S2);
        FNO_CK(cudaGetLastError());
        // pointwise path weights and bias: [co][ci | ones]
        FNO_CK(gemm(h, C, C + 1, SL, opK(h->dz, S2, cs, SL), opK(h->vext[l], S2, vs, SL), B * ns,
                    EpiStoreF32{h->part, C + 1, (long long)C * (C + 1)}, ns));
        FNO_CK(reduce_map(h->part, h->st, B * ns, C * (C + 1), 32, h->map_loc, gr, o.layer[l]));
        // spectral path: adjoint of the inverse DFT along x, then along y
        FNO_CK(gemm(h, B * C * S, 2 * KX, S, opK(h->dz, S), opK(h->G1T, S), 1, EpiDftX{h->Tb, B, S, 0}));
        FNO_CK(gemm(h, KX * B * C, 2 * KY, 2 * S, opK(h->Tb, 2 * S), opK(h->G2T, 2 * S), 1, EpiModes{h->dYm, B}));
        k_spec_wgrad<<<NM, 256, 0, h->st>>>(h->Zm[l], h->dYm, gr + o.layer[l], B);
        FNO_CK(cudaGetLastError());
        // adjoint of the channel mixing and of the DFT along y
        FNO_CK(gemm(h, B, 64, 64, opK(h->dYm, 64, (long long)B * 64), opK(h->WmT + (size_t)l * NM * 4096, 64, 4096),
                    NM, EpiMix{h->Yb}));
        FNO_CK(gemm(h, B * C * KX, 2 * S, 64, opK(h->Yb, 64), opK(h->F2T, 64), 1, EpiIdftY{h->Gt, S}));
        // adjoint of the DFT along x + the pointwise path: batch (b, y), rows x, K = (kx, part) | co
        FNO_CK(gemm(h, S, C, 64, opK(h->F1T, 2 * KX), opK(h->Gt, 2 * KX, (long long)S * C * 32, (long long)C * 32),
                    B * S, EpiPixStore{h->dvf, S, S2}, S, opMN(h->dz, S2, cs, S), opK(h->WlT + (size_t)l * C * C, C),
                    2 * KX));
    }
    // lift weights and bias: [c][inputs | ones | zero]
    k_act_bwd<<<B * (S2 / 64), 256, 0, h->st>>>(h->dvf, nullptr, h->dz, nullptr, S2);
    FNO_CK(cudaGetLastError());
    FNO_CK(gemm(h, C, XC, SL, opK(h->dz, S2, cs, SL), opK(h->xe, S2, (long long)XC * S2, SL), B * ns,
                EpiStoreF32{h->part, XC, (long long)C * XC}, ns));
    FNO_CK(reduce_map(h->part, h->st, B * ns, C * XC, 64, h->map_lift, gr, 0));
    return FI_OK;
}

int set_loss(fi_fno* h, int B, const float* target, const float* w, const float* dy) {
    const int n = B * h->S2;
    FNO_CK(cudaMemsetAsync(h->grads, 0, sizeof(float) * h->o.total, h->st));
    FNO_CK(cudaMemsetAsync(h->scal, 0, sizeof(float) * 4, h->st));
    // per-block partials in the split-K scratch (free until the backward pass)
    const int nblk = (n + 255) / 256;
    k_loss<<<nblk, 256, 0, h->st>>>(h->q, target, w, dy, n, h->S2, 1.f / n, h->dq, h->vext[NLAYER], h->part);
    k_loss_sum<<<1, 256, 0, h->st>>>(h->part, nblk, h->scal, h->grads + h->o.b2);
    FNO_CK(cudaGetLastError());
    return FI_OK;
}

int adam(fi_fno* h, float lr) {
    h->adam_t++;
    const float c1 = (float)(1.0 / (1.0 - std::pow((double)h->beta1, (double)h->adam_t)));
    const float c2 = (float)(1.0 / (1.0 - std::pow((double)h->beta2, (double)h->adam_t)));
    k_adam<<<148 * 8, 256, 0, h->st>>>(h->params, h->grads, h->m, h->v, h->o.total, lr, h->beta1, h->beta2, h->eps,
                                       c1, c2);
    FNO_CK(cudaGetLastError());
    return pack(h);
}

int check_batch(fi_fno* h, int B) {
    if (B < 1 || B > h->maxB) return fail(h, FI_ERR_ARG, "batch outside [1, max_batch]");
    return FI_OK;
}

}  // namespace

extern "C" {

int fi_fno_create(int32_t S, int32_t max_batch, int32_t device, uint64_t seed, fi_fno** out) {
    if (!out) return FI_ERR_ARG;
    *out = nullptr;
    if (S < 32 || S > 256 || S % 32 || max_batch < 1 || max_batch > 256) return FI_ERR_ARG;
    fi_fno* h = new fi_fno();
    h->S = S;
    h->S2 = S * S;
    h->maxB = max_batch;
    h->device = device;
    h->o = offsets();
    h->SL = 512;  // pixels per split-K slice of the weight gradients (S2 is a multiple of 1024)
    h->ns = h->S2 / h->SL;
    auto bad = [&](int rc) {
        fi_fno_destroy(h);
        return rc;
    };
    if (cudaSetDevice(device) != cudaSuccess) return bad(FI_ERR_CUDA);
    if (cudaStreamCreateWithFlags(&h->st, cudaStreamDefault) != cudaSuccess) return bad(FI_ERR_CUDA);
    const long long B = max_batch, S2 = h->S2, P = h->o.total;
    bool ok = dalloc(h, &h->params, P) == cudaSuccess && dalloc(h, &h->grads, P) == cudaSuccess &&
              dalloc(h, &h->m, P) == cudaSuccess && dalloc(h, &h->v, P) == cudaSuccess &&
              dalloc(h, &h->Pb, C * XC) == cudaSuccess && dalloc(h, &h->Wm, (size_t)NLAYER * NM * 4096) == cudaSuccess &&
              dalloc(h, &h->WmT, (size_t)NLAYER * NM * 4096) == cudaSuccess &&
              dalloc(h, &h->Wl, NLAYER * C * C) == cudaSuccess && dalloc(h, &h->WlT, NLAYER * C * C) == cudaSuccess &&
              dalloc(h, &h->Q1b, PW * C) == cudaSuccess && dalloc(h, &h->Q1Tb, PW * C) == cudaSuccess &&
              dalloc(h, &h->F1, 32 * S) == cudaSuccess && dalloc(h, &h->F2, 128 * S) == cudaSuccess &&
              dalloc(h, &h->G2, 128 * S) == cudaSuccess && dalloc(h, &h->G1, 32 * S) == cudaSuccess &&
              dalloc(h, &h->F1T, 32 * S) == cudaSuccess && dalloc(h, &h->F2T, 128 * S) == cudaSuccess &&
              dalloc(h, &h->G2T, 128 * S) == cudaSuccess && dalloc(h, &h->G1T, 32 * S) == cudaSuccess &&
              dalloc(h, &h->xe, B * XC * S2) == cudaSuccess &&
              dalloc(h, &h->Tb, (size_t)KX * B * C * 2 * S) == cudaSuccess &&
              dalloc(h, &h->Yb, (size_t)B * C * KX * 64) == cudaSuccess &&
              dalloc(h, &h->Gt, (size_t)B * C * S * 32) == cudaSuccess &&
              dalloc(h, &h->dz, (size_t)B * C * S2) == cudaSuccess &&
              dalloc(h, &h->dYm, (size_t)NM * B * 64) == cudaSuccess &&
              dalloc(h, &h->da_rows, (size_t)B * S2 * PW) == cudaSuccess &&
              dalloc(h, &h->daT, (size_t)B * 2 * PW * S2) == cudaSuccess &&
              dalloc(h, &h->q, (size_t)B * S2) == cudaSuccess &&
              dalloc(h, &h->dq, (size_t)B * S2) == cudaSuccess && dalloc(h, &h->dvf, (size_t)B * C * S2) == cudaSuccess &&
              dalloc(h, &h->part, (size_t)B * h->ns * 2 * PW * VC) == cudaSuccess &&
              dalloc(h, &h->scal, 4) == cudaSuccess && dalloc(h, &h->map_loc, C * (C + 1)) == cudaSuccess &&
              dalloc(h, &h->map_proj, 2 * PW * VC) == cudaSuccess && dalloc(h, &h->map_lift, C * XC) == cudaSuccess &&
              dalloc(h, &h->err, 1) == cudaSuccess;
    for (int l = 0; l <= NLAYER && ok; l++) ok = dalloc(h, &h->vext[l], (size_t)B * VC * S2) == cudaSuccess;
    for (int l = 0; l < NLAYER && ok; l++)
        ok = dalloc(h, &h->zs[l], (size_t)B * C * S2) == cudaSuccess &&
             dalloc(h, &h->Zm[l], (size_t)NM * B * 64) == cudaSuccess;
    if (!ok) return bad(FI_ERR_CUDA);
    // DFT matrices
    std::vector<bf16> mats[8];
    build_dft(S, mats);
    bf16* dst[8] = {h->F1, h->F2, h->G2, h->G1, h->F1T, h->F2T, h->G2T, h->G1T};
    for (int i = 0; i < 8; i++)
        if (cudaMemcpy(dst[i], mats[i].data(), mats[i].size() * sizeof(bf16), cudaMemcpyHostToDevice) != cudaSuccess)
            return bad(FI_ERR_CUDA);
    // split-K gradient maps (targets relative to the base passed to k_reduce_map)
    const Offsets& o = h->o;
    std::vector<int> ml(C * (C + 1)), mp(2 * PW * VC, -1), mf(C * XC, -1);
    for (int co = 0; co < C; co++)
        for (int k = 0; k <= C; k++) ml[co * (C + 1) + k] = (int)(k < C ? SPEC + co * C + k : SPEC + C * C + co);
    for (int j = 0; j < PW; j++) {
        for (int c = 0; c < C; c++) mp[j * VC + c] = (int)(o.Q1 + j * C + c);
        mp[j * VC + C] = (int)(o.b1 + j);
        mp[(PW + j) * VC + C + 1] = (int)(o.Q2 + j);
    }
    for (int c = 0; c < C; c++) {
        for (int k = 0; k < NIN; k++) mf[c * XC + k] = (int)(o.P + c * NIN + k);
        mf[c * XC + NIN] = (int)(o.bP + c);
    }
    if (cudaMemcpy(h->map_loc, ml.data(), ml.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(h->map_proj, mp.data(), mp.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(h->map_lift, mf.data(), mf.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess)
        return bad(FI_ERR_CUDA);
    // ones channel of every NCHW activation buffer (bias gradients)
    for (int l = 0; l <= NLAYER; l++) k_fill_channel<<<(unsigned)((B * S2 + 255) / 256), 256, 0, h->st>>>(
        h->vext[l], (int)B, (int)S2, C, 1.f);
    std::vector<float> p0 = init_params(o, seed);
    if (cudaMemcpy(h->params, p0.data(), P * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
        return bad(FI_ERR_CUDA);
    if (pack(h) != FI_OK || finish(h) != FI_OK) return bad(FI_ERR_CUDA);
    *out = h;
    return FI_OK;
}

int64_t fi_fno_num_params(const fi_fno* h) { return h ? h->o.total : -1; }

int fi_fno_get_params(fi_fno* h, float* out, int64_t n) {
    if (!h || !out || n != h->o.total) return fail(h, FI_ERR_ARG, "parameter count");
    FNO_CK(cudaSetDevice(h->device));
    FNO_CK(cudaStreamSynchronize(h->st));
    FNO_CK(cudaMemcpy(out, h->params, n * sizeof(float), cudaMemcpyDeviceToHost));
    return FI_OK;
}

int fi_fno_set_params(fi_fno* h, const float* in, int64_t n) {
    if (!h || !in || n != h->o.total) return fail(h, FI_ERR_ARG, "parameter count");
    FNO_CK(cudaSetDevice(h->device));
    FNO_CK(cudaStreamSynchronize(h->st));
    FNO_CK(cudaMemcpy(h->params, in, n * sizeof(float), cudaMemcpyHostToDevice));
    FNO_CK(cudaMemset(h->m, 0, n * sizeof(float)));
    FNO_CK(cudaMemset(h->v, 0, n * sizeof(float)));
    h->adam_t = 0;
    h->fwdB = 0;
    int rc = pack(h);
    return rc ? rc : finish(h);
}

int fi_fno_get_grads(fi_fno* h, float* out, int64_t n) {
    if (!h || !out || n != h->o.total) return fail(h, FI_ERR_ARG, "parameter count");
    FNO_CK(cudaSetDevice(h->device));
    FNO_CK(cudaStreamSynchronize(h->st));
    FNO_CK(cudaMemcpy(out, h->grads, n * sizeof(float), cudaMemcpyDeviceToHost));
    return FI_OK;
}

int fi_fno_forward(fi_fno* h, int32_t B, const float* x, float* y) {
    if (!h || !x || !y) return fail(h, FI_ERR_ARG, "null pointer");
    int rc = check_batch(h, B);
    if (rc) return rc;
    FNO_CK(cudaSetDevice(h->device));
    rc = forward(h, B, x, y);
    return rc ? rc : finish(h);
}

int fi_fno_backward(fi_fno* h, int32_t B, const float* dy) {
    if (!h || !dy) return fail(h, FI_ERR_ARG, "null pointer");
    if (B != h->fwdB) return fail(h, FI_ERR_STATE, "backward needs a forward pass of the same batch");
    FNO_CK(cudaSetDevice(h->device));
    int rc = set_loss(h, B, nullptr, nullptr, dy);
    if (!rc) rc = backward(h, B);
    return rc ? rc : finish(h);
}

int fi_fno_train_step(fi_fno* h, int32_t B, const float* x, const float* target, float lr, float* loss) {
    return fi_fno_train_step_weighted(h, B, x, target, nullptr, lr, loss);
}

int fi_fno_train_step_weighted(fi_fno* h, int32_t B, const float* x, const float* target, const float* w, float lr,
                               float* loss) {
    if (!h || !x || !target) return fail(h, FI_ERR_ARG, "null pointer");
    int rc = check_batch(h, B);
    if (rc) return rc;
    FNO_CK(cudaSetDevice(h->device));
    rc = forward(h, B, x, h->q);
    if (!rc) rc = set_loss(h, B, target, w, nullptr);
    if (!rc) rc = backward(h, B);
    if (!rc) rc = adam(h, lr);
    if (!rc) rc = finish(h);
    if (!rc && loss) FNO_CK(cudaMemcpy(loss, h->scal, sizeof(float), cudaMemcpyDeviceToHost));
    return rc;
}

int fi_fno_loss_backward(fi_fno* h, int32_t B, const float* x, const float* target, const float* w, float* loss) {
    if (!h || !x || !target) return fail(h, FI_ERR_ARG, "null pointer");
    int rc = check_batch(h, B);
    if (rc) return rc;
    FNO_CK(cudaSetDevice(h->device));
    rc = forward(h, B, x, h->q);
    if (!rc) rc = set_loss(h, B, target, w, nullptr);
    if (!rc) rc = backward(h, B);
    if (!rc) rc = finish(h);
    if (!rc && loss) FNO_CK(cudaMemcpy(loss, h->scal, sizeof(float), cudaMemcpyDeviceToHost));
    return rc;
}

void* fi_fno_grads_device(fi_fno* h) { return h ? (void*)h->grads : nullptr; }

int fi_fno_adam(fi_fno* h, float lr) {
    if (!h) return FI_ERR_ARG;
    FNO_CK(cudaSetDevice(h->device));
    int rc = adam(h, lr);
    return rc ? rc : finish(h);
}

int fi_fno_set_adam(fi_fno* h, float beta1, float beta2, float eps) {
    if (!h || !(beta1 >= 0.f && beta1 < 1.f) || !(beta2 >= 0.f && beta2 < 1.f) || !(eps > 0.f))
        return fail(h, FI_ERR_ARG, "Adam hyper-parameters");
    h->beta1 = beta1;
    h->beta2 = beta2;
    h->eps = eps;
    return FI_OK;
}

const char* fi_fno_last_error(const fi_fno* h) { return h ? h->msg.c_str() : "null handle"; }

void fi_fno_destroy(fi_fno* h) {
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->st) cudaStreamSynchronize(h->st);
    for (void* p : h->allocs) cudaFree(p);
    if (h->st) cudaStreamDestroy(h->st);
    delete h;
}

}  // extern "C"
