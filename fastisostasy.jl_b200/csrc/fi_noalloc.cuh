// fi_noalloc.cuh -- the static device scratch of fi_rhs_noalloc (fi_noalloc.cu).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>

namespace fi {

// Largest grid (nx * ny cells) the static scratch holds: 1024 x 1024.
constexpr size_t NOALLOC_MAX_CELLS = (size_t)1024 * 1024;
// Layout: [0, 4 * NOALLOC_MAX_CELLS) the FP32 field of the right-hand side before its
// corner BC; then 4 doubles, the field's corner values.
constexpr size_t NOALLOC_CORNER_OFFSET = 4 * NOALLOC_MAX_CELLS;
constexpr size_t NOALLOC_SCRATCH_BYTES = NOALLOC_CORNER_OFFSET + 256;

// Address of the scratch on the current device.  The first call on a device looks
// it up with cudaGetSymbolAddress and caches it; later calls only read the cache.
cudaError_t noalloc_scratch(void** ptr);

// dudt[k] = v[k] - (mean of the four corners - border), on `stream`.
cudaError_t noalloc_finish(const void* scratch, double border, size_t n, double* dudt, cudaStream_t stream);

}  // namespace fi
