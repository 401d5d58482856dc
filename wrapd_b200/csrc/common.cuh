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

// ---- deterministic grid reduction: per-block partials, summed in block order
// by whichever block finishes last. -------------------------------------------
// out[k] = total_k, or for k = 0 with an affine epilogue: (base ? *base : 0) + scale * total_0.
template <int NV, bool MAX = false>
__device__ __forceinline__ void grid_reduce(const double (&v)[NV], double* partials, unsigned* counter, double* out,
                                            const double* base = nullptr, double scale = 1.0) {
    __shared__ double sm[32];
    __shared__ bool last;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        const double r = MAX ? block_max(v[k], sm) : block_sum(v[k], sm);
        if (threadIdx.x == 0) partials[(size_t)blockIdx.x * NV + k] = r;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double acc = MAX ? -1.0e308 : 0.0;
        for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
            const double p = __ldcg(partials + (size_t)b * NV + k);
            acc = MAX ? fmax(acc, p) : acc + p;
        }
        const double r = MAX ? block_max(acc, sm) : block_sum(acc, sm);
        if (threadIdx.x == 0) out[k] = (k == 0 && (base || scale != 1.0)) ? (base ? *base : 0.0) + scale * r : r;
    }
    if (threadIdx.x == 0) *counter = 0u;
}

}  // namespace wrapd
