// fi_noalloc.cu -- static device scratch for fi_rhs_noalloc.
//
// The FP32 right-hand side leaves its result in two scratch buffers: the field before
// the dudt corner BC (nx * ny floats, written by every row tile of k_rows_inv) and its
// four corner values (written by row tile 0).  fi_rhs takes them from buffers the
// handle owns and finishes on the host; fi_rhs_noalloc takes them from the file-scope
// array below and finishes on the device, so a call allocates nothing.  Every byte a
// call reads from the scratch is written earlier in the same call: nothing in it has
// to start at zero.  One array serves every handle on a device, so calls that overlap
// in time on the same device race on it.
#include <mutex>

#include "fi_noalloc.cuh"

namespace fi {

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

namespace {
constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
void* g_ptr[MAX_DEVICES] = {};
}  // namespace

cudaError_t noalloc_scratch(void** ptr) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= MAX_DEVICES) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_ptr[dev] = p;
    }
    *ptr = g_ptr[dev];
    return cudaSuccess;
}

__global__ void k_noalloc_finish(const float* __restrict__ v, const double* __restrict__ corners, double border,
                                 size_t n, double* __restrict__ dudt) {
    const double off = 0.25 * (corners[0] + corners[1] + corners[2] + corners[3]) - border;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
        dudt[k] = (double)v[k] - off;
}

cudaError_t noalloc_finish(const void* scratch, double border, size_t n, double* dudt, cudaStream_t stream) {
    const unsigned char* s = (const unsigned char*)scratch;
    const int threads = 256;
    const size_t want = (n + threads - 1) / threads;
    const int blocks = (int)(want < 1184 ? (want ? want : 1) : 1184);  // 148 SMs x 8
    k_noalloc_finish<<<blocks, threads, 0, stream>>>((const float*)s, (const double*)(s + NOALLOC_CORNER_OFFSET),
                                                     border, n, dudt);
    return cudaGetLastError();
}

}  // namespace fi
