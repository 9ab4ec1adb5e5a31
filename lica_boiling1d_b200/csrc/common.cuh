// Shared device/host helpers for the lica B200 kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>

#include "lica_gpu.h"

#define LICA_CUDA_TRY(expr)                                                              \
    do {                                                                                 \
        cudaError_t _e = (expr);                                                         \
        if (_e != cudaSuccess) {                                                         \
            lica_set_last_error(#expr, cudaGetErrorString(_e), __FILE__, __LINE__);       \
            return LICA_ERR_CUDA;                                                        \
        }                                                                                \
    } while (0)

void lica_set_last_error(const char* what, const char* msg, const char* file, int line);

namespace lica {

constexpr int kWarp = 32;

// Deterministic block-wide FP64 sum: fixed-order warp shuffle tree, then warp 0 sums the
// per-warp partials in order.  Every thread must call it; the result is valid in thread 0.
__device__ __forceinline__ double block_sum(double v, double* scratch /* >= 32 doubles */) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = (blockDim.x + 31) >> 5;
    __syncthreads();
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    double r = 0.0;
    if (warp == 0) {
        r = (lane < nwarps) ? scratch[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
    }
    return r;
}

// "Last block" grid reduction: each block stores its partial, the last block to arrive
// sums all partials in index order (deterministic for a fixed grid) and returns true in
// thread 0 with *total set.  counter must be zero before the launch; it is reset here.
__device__ __forceinline__ bool grid_sum_last(double block_partial, double* partials, unsigned* counter,
                                              double* total, double* scratch) {
    __shared__ bool is_last;
    if (threadIdx.x == 0) {
        const unsigned nb = gridDim.x * gridDim.y;
        partials[blockIdx.x + gridDim.x * blockIdx.y] = block_partial;
        __threadfence();
        unsigned prev = atomicAdd(counter, 1u);
        is_last = (prev == nb - 1);
    }
    __syncthreads();
    if (!is_last) return false;
    __threadfence();
    const unsigned nb = gridDim.x * gridDim.y;
    double v = 0.0;
    // fixed assignment: thread t sums partials t, t+blockDim, ... in order
    for (unsigned k = threadIdx.x; k < nb; k += blockDim.x) v += ((volatile double*)partials)[k];
    double s = block_sum(v, scratch);
    if (threadIdx.x == 0) {
        *total = s;
        *counter = 0u;
    }
    return threadIdx.x == 0;
}

}  // namespace lica
