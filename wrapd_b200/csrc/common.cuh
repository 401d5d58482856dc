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

// ---- bounded waits between CTAs ----------------------------------------------
// A wait on a counter that other CTAs raise (release: their writes, a fence,
// then the atomic) polls it with an acquire load for at most one second of the
// global timer and kWaitPolls polls.  One that gives up sets *status to
// WRAPD_E_TIMEOUT (if it was 0) and returns false; a wait that finds *status
// already set returns false at once, so every waiter of a failed launch ends.
constexpr unsigned long long kWaitNs = 1000000000ull;
constexpr int kWaitPolls = 1 << 24;

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ bool wait_count_geq(const unsigned* count, unsigned target, int* status) {
    const unsigned long long t0 = global_ns();
    for (int i = 0; i < kWaitPolls; ++i) {
        if (ld_acquire(count) >= target) return true;
        if (*reinterpret_cast<volatile int*>(status) != 0) return false;
        if (global_ns() - t0 > kWaitNs) break;
        __nanosleep(64);
    }
    atomicCAS(status, 0, WRAPD_E_TIMEOUT);
    return false;
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

// ---- launches over a batch of meshes ----------------------------------------
// A launch's blocks are tiles: tile b covers items [first, end) of one mesh
// (elements, free vertices or vector entries; each mesh's items are a
// contiguous range).  With a table (t != null) tile b is t[b] = {mesh, first,
// end}; without one (a single mesh) tile b covers [b * per, (b + 1) * per) of
// [0, n).  Every mesh's tiles start at its own first item, so a mesh's blocks
// in a batch do exactly the work of the same mesh's blocks when it is solved
// alone, and the per-mesh sums below add the same partials in the same order:
// a mesh's results in a batch equal its results alone, bit for bit.
struct Tiles {
    const int4* t;       // per tile {mesh, first, end, 0}, or null (one mesh)
    const int* tile0;    // per mesh its first tile, nm + 1 entries (with t)
    int n, per;          // one mesh: item count and items per tile
    int count;           // tiles of the launch
};
struct Tile {
    int mesh, first, end;
};
__device__ __forceinline__ Tile tile_at(const Tiles& T, int b) {
    if (T.t) {
        const int4 v = T.t[b];
        return {v.x, v.y, v.z};
    }
    return {0, b * T.per, min((b + 1) * T.per, T.n)};
}
// `on` (per mesh, null = all) masks whole meshes out of a launch: their tiles
// return before any work or synchronisation.
__device__ __forceinline__ bool mesh_on(const int* on, int mesh) { return !on || on[mesh] != 0; }

// Per-mesh grid reduction: per-tile partials; the last tile of each mesh to
// finish adds that mesh's partials in tile order (thread i takes tiles i,
// i + blockDim.x, ... of the mesh, then a fixed block sum).  Returns true in
// the last tile of the mesh, with the totals in tot[] of thread 0.  With one
// mesh and no table this is grid_reduce's arithmetic.  counters: one per
// mesh, zero between launches (the last tile resets its mesh's).
template <int NV, bool MAX = false>
__device__ __forceinline__ bool seg_reduce(const double (&v)[NV], const Tiles& T, int mesh, double* partials,
                                           unsigned* counters, double (&tot)[NV]) {
    __shared__ double sm[32];
    __shared__ bool last;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        const double r = MAX ? block_max(v[k], sm) : block_sum(v[k], sm);
        if (threadIdx.x == 0) partials[(size_t)blockIdx.x * NV + k] = r;
    }
    const int t0 = T.t ? T.tile0[mesh] : 0, t1 = T.t ? T.tile0[mesh + 1] : (int)gridDim.x;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(counters + mesh, 1u) == (unsigned)(t1 - t0 - 1);
    __syncthreads();
    if (!last) return false;
    __threadfence();
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double acc = MAX ? -1.0e308 : 0.0;
        for (int b = t0 + (int)threadIdx.x; b < t1; b += blockDim.x) {
            const double p = __ldcg(partials + (size_t)b * NV + k);
            acc = MAX ? fmax(acc, p) : acc + p;
        }
        tot[k] = MAX ? block_max(acc, sm) : block_sum(acc, sm);
    }
    if (threadIdx.x == 0) counters[mesh] = 0u;
    return true;
}

// seg_reduce writing the totals to out[mesh * stride + k].
template <int NV, bool MAX = false>
__device__ __forceinline__ void seg_reduce_out(const double (&v)[NV], const Tiles& T, int mesh, double* partials,
                                               unsigned* counters, double* out, int stride) {
    double tot[NV];
    if (seg_reduce<NV, MAX>(v, T, mesh, partials, counters, tot) && threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) out[(size_t)mesh * stride + k] = tot[k];
}

}  // namespace wrapd
