// Shared device/host helpers for the wrapd_b200 CUDA library.
#pragma once
#include <cuda_runtime.h>
#include <cfloat>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>

#include "../../include/wrapd_gpu.h"

namespace wrapd {

struct CudaError : std::runtime_error {
    int code;
    CudaError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define WRAPD_CUDA(call)                                                                         \
    do {                                                                                         \
        cudaError_t err__ = (call);                                                              \
        if (err__ != cudaSuccess)                                                                \
            throw ::wrapd::CudaError(WRAPD_E_CUDA, std::string(#call " failed: ") +              \
                                                       cudaGetErrorString(err__));               \
    } while (0)

#define WRAPD_LAUNCH_CHECK() WRAPD_CUDA(cudaGetLastError())

template <typename T> struct Lim;
template <> struct Lim<double> {
    __host__ __device__ static constexpr double eps() { return DBL_EPSILON; }
    __host__ __device__ static constexpr double min() { return DBL_MIN; }
};
template <> struct Lim<float> {
    __host__ __device__ static constexpr float eps() { return FLT_EPSILON; }
    __host__ __device__ static constexpr float min() { return FLT_MIN; }
};

// 148 SMs on B200; grids for streaming kernels are sized in multiples of it.
constexpr int kNumSMs = 148;

inline int ceil_div(int64_t a, int64_t b) { return static_cast<int>((a + b - 1) / b); }

// Deterministic block sum of one value per thread (blockDim.x a multiple of 32,
// at most 1024).  Returns the total in thread 0.
template <typename T>
__device__ __forceinline__ T block_sum(T v, T* smem) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) smem[warp] = v;
    __syncthreads();
    T r = 0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r += smem[w];
    return r;
}

template <typename T>
__device__ __forceinline__ T block_max(T v, T* smem) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) smem[warp] = v;
    __syncthreads();
    T r = 0;
    if (threadIdx.x == 0) {
        r = smem[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) r = fmax(r, smem[w]);
    }
    return r;
}

}  // namespace wrapd
