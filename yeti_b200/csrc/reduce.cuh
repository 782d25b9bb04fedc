// Block-level reductions with a fixed summation tree (results do not
// depend on block timing), shared by the Krylov and preconditioner kernels.
#pragma once
#include <cuda_runtime.h>

namespace yeti {

// Last-block-done: every block publishes its partials, then takes a ticket;
// the block that takes the last one sees all partials (fixed summation
// order, so the result does not depend on block timing) and resets the
// ticket for the next reduction.
__device__ __forceinline__ bool last_block(unsigned int *ticket) {
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (last) __threadfence();
    return last;
}

__device__ __forceinline__ double block_sum(double v, double *sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    v = 0.0;
    if (wid == 0) {
        v = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    }
    __syncthreads();
    return v;
}

__device__ __forceinline__ double block_max(double v, double *sh) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    v = 0.0;
    if (wid == 0) {
        v = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    }
    __syncthreads();
    return v;
}

}  // namespace yeti
