// Deterministic block / grid reductions (header-only device helpers).
//
// A grid reduction writes one partial per block, and the LAST block to
// finish (atomic ticket after a fence) sums the partials in a fixed order
// and resets the ticket.  For a fixed grid size every run adds the same
// numbers in the same order, so results are bitwise reproducible.
#pragma once
#include <cuda_runtime.h>

namespace transfer {

// Sum over the block; the result is valid in thread 0.  `sh` holds >= 32
// doubles.  Fixed order: butterfly within warps, then over warp sums.
__device__ __forceinline__ double block_sum(double v, double *sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x < 32) {
        t = (l < static_cast<int>(blockDim.x >> 5)) ? sh[l] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    }
    return t;
}

// Completes an NV-value grid reduction.  Every block calls it with its
// thread values; returns true in the last block, where tot[] (valid in
// thread 0) holds the grid totals.  partials: [NV][gridDim.x].
template <int NV>
__device__ __forceinline__ bool grid_reduce(const double (&v)[NV], double *partials, unsigned int *counter,
                                            double (&tot)[NV]) {
    __shared__ double sh[32];
    __shared__ bool am_last;
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        double s = block_sum(v[q], sh);
        if (threadIdx.x == 0) partials[q * gridDim.x + blockIdx.x] = s;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int ticket = atomicAdd(counter, 1u);
        am_last = (ticket == gridDim.x - 1);
    }
    __syncthreads();
    if (!am_last) return false;
    __threadfence();
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        double acc = 0.0;
        for (unsigned int i = threadIdx.x; i < gridDim.x; i += blockDim.x)
            acc += __ldcg(partials + q * gridDim.x + i);
        tot[q] = block_sum(acc, sh);
    }
    if (threadIdx.x == 0) *counter = 0u;
    return true;
}

}  // namespace transfer
