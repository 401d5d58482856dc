// FP64 tensor-core (DMMA, mma.sync m8n8k4 f64) throughput probe: the roofline
// denominator of the numeric factorization, whose dense front updates run on
// this instruction.  Every warp issues independent accumulation chains from
// register operands, so the figure is the instruction's issue limit.
#include "common.cuh"

namespace wrapd {
namespace {

constexpr int kChains = 8;

__global__ void __launch_bounds__(128) k_dmma_peak(int iters, const double* __restrict__ in, double* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    double a = in[lane], b = in[32 + lane];
    double d0[kChains], d1[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) { d0[c] = 0.0; d1[c] = 0.0; }
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < kChains; ++c)
            asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                         : "+d"(d0[c]), "+d"(d1[c])
                         : "d"(a), "d"(b));
    }
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += d0[c] + d1[c];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace
}  // namespace wrapd

using namespace wrapd;

extern "C" WRAPD_API int wrapd_dmma_peak(int iters, double* tflops) {
    if (iters <= 0 || !tflops) return WRAPD_E_INPUT;
    const int blocks = 8 * kNumSMs, threads = 128;
    double *in = nullptr, *out = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = WRAPD_OK;
    if (cudaMalloc(&in, 64 * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&out, (size_t)blocks * threads * sizeof(double)) != cudaSuccess) {
        rc = WRAPD_E_OOM;
    } else {
        double h[64];
        for (int i = 0; i < 64; ++i) h[i] = 1.0 / (1.0 + i);
        float ms = 0.f;
        if (cudaMemcpy(in, h, sizeof h, cudaMemcpyHostToDevice) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
            cudaEventCreate(&e1) != cudaSuccess) {
            rc = WRAPD_E_CUDA;
        } else {
            k_dmma_peak<<<blocks, threads>>>(iters / 10 + 1, in, out);   // warm-up
            cudaEventRecord(e0);
            k_dmma_peak<<<blocks, threads>>>(iters, in, out);
            cudaEventRecord(e1);
            if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
                rc = WRAPD_E_CUDA;
            } else {
                const double flops = 2.0 * 8 * 8 * 4 * kChains * (double)iters * (blocks * threads / 32);
                *tflops = flops / (ms * 1e-3) / 1e12;
            }
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (in) cudaFree(in);
    if (out) cudaFree(out);
    cudaGetLastError();
    return rc;
}
