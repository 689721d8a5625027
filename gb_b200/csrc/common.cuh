// common.cuh -- shared device helpers and the argument blocks of the kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "field.cuh"

namespace gbgpu {

constexpr int kWarp = 32;

// error bits raised by device-side input checks
enum : uint32_t {
    kErrEmptyRow = 1u << 0,
    kErrLeadRange = 1u << 1,     // lead outside the left block
    kErrColRange = 1u << 2,      // column outside [lead, nc)
    kErrCoefRange = 1u << 3,     // coefficient outside [1, p)
    kErrNotMonic = 1u << 4,      // lead coefficient != 1
    kErrMissingPivot = 1u << 5,  // left column without a known pivot
    kErrDupLead = 1u << 6,       // interreduction input with repeated leads
};

// Minimum over a block of a per-thread int; every thread gets the result.
// `scratch` holds one int per warp.  Contains two __syncthreads().
__device__ __forceinline__ int block_min(int v, int* scratch) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    int r = scratch[0];
    const int nw = (blockDim.x + 31) >> 5;
    for (int i = 1; i < nw; ++i) r = min(r, scratch[i]);
    __syncthreads();
    return r;
}

}  // namespace gbgpu
