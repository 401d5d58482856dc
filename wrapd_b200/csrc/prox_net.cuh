// Prox-stretch network: a 5 -> 64 -> 64 -> 3 MLP with GELU (tanh form) that
// maps (sorted singular values of S_in, log(w^2 / (vol mu)), log(mu / lambda))
// to a warm start for the per-element prox (NHProx, src/TetElements.hpp:50-162).
// Operands are BF16, accumulation FP32, on the tensor cores through
// mma.sync.m16n8k16 (one warp = 32 samples = two 16-row tiles).  The prox
// depends only on (sigma_in, w^2/(vol mu), lambda/mu) because psi_NH / mu
// depends only on lambda / mu, so those are the inputs.
//
// Parameters live in an FP32 blob (see the B_* offsets).  Kernels work from a
// shared-memory image of it: BF16 weights in padded rows so that every
// fragment load is bank-conflict free, FP32 biases and the feature
// normalisation.  The output is normalised: sigma_pred = sigma_in + oscale * y.
#pragma once
#include <cuda_bf16.h>

#include <cstdint>

#include "common.cuh"

namespace wrapd {
namespace net {

constexpr int IN = 5, HID = 64, OUT = 3;

// FP32 blob layout (floats).
constexpr int B_MEAN = 0, B_ISTD = 5, B_OSCALE = 10;          // feature mean, 1/std; output scale
constexpr int B_W1 = 16;                                      // W1[64][5]
constexpr int B_B1 = B_W1 + HID * IN;                         // b1[64]
constexpr int B_W2 = B_B1 + HID;                              // W2[64][64]
constexpr int B_B2 = B_W2 + HID * HID;                        // b2[64]
constexpr int B_W3 = B_B2 + HID;                              // W3[3][64]
constexpr int B_B3 = B_W3 + OUT * HID;                        // b3[3]
constexpr int N_BLOB = B_B3 + OUT;                            // 4755
constexpr int N_TRAIN = N_BLOB - B_W1;                        // 4739 trained values
static_assert(N_BLOB == WRAPD_NET_BLOB, "blob size");

// Shared-memory image (bytes).  Row pitches in BF16 elements.
constexpr int LD1 = 24;   // W1s rows (16 used), input staging rows, W3T rows
constexpr int LD2 = 72;   // W2s / W3s / W2T rows (64 used)
constexpr int I_W1 = 0;                        // [64][LD1]
constexpr int I_W2 = I_W1 + HID * LD1 * 2;     // [64][LD2]
constexpr int I_W3 = I_W2 + HID * LD2 * 2;     // [8][LD2], rows 3..7 zero
constexpr int I_B1 = I_W3 + 8 * LD2 * 2;       // float[64]
constexpr int I_B2 = I_B1 + HID * 4;           // float[64]
constexpr int I_B3 = I_B2 + HID * 4;           // float[8], 3..7 zero
constexpr int I_NORM = I_B3 + 8 * 4;           // float[16]: mean[5], istd[5], oscale[3]
constexpr int IMAGE_BYTES = I_NORM + 16 * 4;   // 14048
static_assert(IMAGE_BYTES % 16 == 0, "image copied in 16-byte words");
// Per-warp scratch of the forward pass: inputs [32][LD1] BF16, outputs [32][8] FP32.
constexpr int WARP_SCRATCH = 32 * LD1 * 2 + 32 * 8 * 4;   // 2560

constexpr float kGeluC = 0.7978845608028654f;   // sqrt(2 / pi)
constexpr float kGeluA = 0.044715f;

// tanh x = 1 - 2 / (e^{2x} + 1), with e^{2x} = 2^{2x log2 e} and the reciprocal
// on the special-function unit (ex2.approx, rcp.approx): absolute error ~1e-7,
// far below the BF16 rounding the activations go through next.
__device__ __forceinline__ float tanh_sfu(float x) {
    float e, r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(e) : "f"(x * 2.8853900817779268f));
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(e + 1.0f));
    return 1.0f - 2.0f * r;
}
__device__ __forceinline__ float gelu(float x) {
    return 0.5f * x * (1.0f + tanh_sfu(kGeluC * (x + kGeluA * x * x * x)));
}
__device__ __forceinline__ float gelu_grad(float x) {
    const float x2 = x * x;
    const float t = tanh_sfu(kGeluC * (x + kGeluA * x2 * x));
    return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * kGeluC * (1.0f + 3.0f * kGeluA * x2);
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}
__device__ __forceinline__ uint32_t ld32(const __nv_bfloat16* p) { return *reinterpret_cast<const uint32_t*>(p); }

// D += A B, m16n8k16, A row-major BF16 (4 regs), B col-major BF16 (2 regs), D FP32.
__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Writes the shared-memory image of `blob` with threads [tid, nthreads).
__device__ __forceinline__ void build_image(const float* __restrict__ blob, unsigned char* img, int tid, int nthreads) {
    __nv_bfloat16* W1s = reinterpret_cast<__nv_bfloat16*>(img + I_W1);
    __nv_bfloat16* W2s = reinterpret_cast<__nv_bfloat16*>(img + I_W2);
    __nv_bfloat16* W3s = reinterpret_cast<__nv_bfloat16*>(img + I_W3);
    float* b1 = reinterpret_cast<float*>(img + I_B1);
    float* b2 = reinterpret_cast<float*>(img + I_B2);
    float* b3 = reinterpret_cast<float*>(img + I_B3);
    float* nrm = reinterpret_cast<float*>(img + I_NORM);
    for (int i = tid; i < HID * LD1; i += nthreads) {
        const int o = i / LD1, c = i % LD1;
        W1s[i] = __float2bfloat16_rn(c < IN ? blob[B_W1 + o * IN + c] : 0.0f);
    }
    for (int i = tid; i < HID * LD2; i += nthreads) {
        const int o = i / LD2, c = i % LD2;
        W2s[i] = __float2bfloat16_rn(c < HID ? blob[B_W2 + o * HID + c] : 0.0f);
    }
    for (int i = tid; i < 8 * LD2; i += nthreads) {
        const int o = i / LD2, c = i % LD2;
        W3s[i] = __float2bfloat16_rn(o < OUT && c < HID ? blob[B_W3 + o * HID + c] : 0.0f);
    }
    for (int i = tid; i < HID; i += nthreads) { b1[i] = blob[B_B1 + i]; b2[i] = blob[B_B2 + i]; }
    for (int i = tid; i < 8; i += nthreads) b3[i] = i < OUT ? blob[B_B3 + i] : 0.0f;
    for (int i = tid; i < 16; i += nthreads) nrm[i] = i < 13 ? blob[B_MEAN + i] : 0.0f;
}

// Copies a prebuilt image from global memory (IMAGE_BYTES) with the whole block.
__device__ __forceinline__ void load_image(const unsigned char* __restrict__ g, unsigned char* img) {
    const uint4* src = reinterpret_cast<const uint4*>(g);
    uint4* dst = reinterpret_cast<uint4*>(img);
    for (int i = threadIdx.x; i < IMAGE_BYTES / 16; i += blockDim.x) dst[i] = src[i];
}

// Raw features of one sample: sorted singular values, log of the scale-free
// weight w^2/(vol mu) and log(mu / lambda).
__device__ __forceinline__ void features(const float s[3], float wov, float mu, float lambda, float f[IN]) {
    f[0] = s[0]; f[1] = s[1]; f[2] = s[2];
    f[3] = logf(wov / mu);
    f[4] = logf(mu / lambda);
}

// Forward pass for the 32 samples of a warp; every lane of the warp calls it
// (lanes without a sample pass valid = false and get zeros in).  f: raw
// features of this lane's sample; y: the normalised outputs.
__device__ __forceinline__ void warp_forward(const unsigned char* img, unsigned char* scratch, const float f[IN],
                                             bool valid, float y[OUT]) {
    const float* nrm = reinterpret_cast<const float*>(img + I_NORM);
    const __nv_bfloat16* W1s = reinterpret_cast<const __nv_bfloat16*>(img + I_W1);
    const __nv_bfloat16* W2s = reinterpret_cast<const __nv_bfloat16*>(img + I_W2);
    const __nv_bfloat16* W3s = reinterpret_cast<const __nv_bfloat16*>(img + I_W3);
    const float* b1 = reinterpret_cast<const float*>(img + I_B1);
    const float* b2 = reinterpret_cast<const float*>(img + I_B2);
    const float* b3 = reinterpret_cast<const float*>(img + I_B3);
    __nv_bfloat16* xs = reinterpret_cast<__nv_bfloat16*>(scratch);
    float* os = reinterpret_cast<float*>(scratch + 32 * LD1 * 2);
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;

    uint32_t* xrow = reinterpret_cast<uint32_t*>(xs + lane * LD1);
#pragma unroll
    for (int c = 0; c < 16; c += 2) {
        const float v0 = (valid && c < IN) ? (f[c] - nrm[B_MEAN + c]) * nrm[B_ISTD + c] : 0.0f;
        const float v1 = (valid && c + 1 < IN) ? (f[c + 1] - nrm[B_MEAN + c + 1]) * nrm[B_ISTD + c + 1] : 0.0f;
        xrow[c >> 1] = pack_bf16(v0, v1);
    }
    __syncwarp();
    uint32_t a1[2][4];
#pragma unroll
    for (int m = 0; m < 2; ++m) {
        const int r = m * 16 + g;
        a1[m][0] = ld32(xs + r * LD1 + 2 * t);
        a1[m][1] = ld32(xs + (r + 8) * LD1 + 2 * t);
        a1[m][2] = ld32(xs + r * LD1 + 2 * t + 8);
        a1[m][3] = ld32(xs + (r + 8) * LD1 + 2 * t + 8);
    }
    // layer 1: its output tiles are the A fragments of layer 2
    uint32_t a2[2][4][4];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int n = 8 * j + g;
        const uint32_t w0 = ld32(W1s + n * LD1 + 2 * t), w1 = ld32(W1s + n * LD1 + 2 * t + 8);
        const float c0 = b1[8 * j + 2 * t], c1 = b1[8 * j + 2 * t + 1];
#pragma unroll
        for (int m = 0; m < 2; ++m) {
            float d[4] = {c0, c1, c0, c1};
            mma_bf16(d, a1[m], w0, w1);
            const uint32_t lo = pack_bf16(gelu(d[0]), gelu(d[1])), hi = pack_bf16(gelu(d[2]), gelu(d[3]));
            a2[m][j >> 1][(j & 1) * 2] = lo;
            a2[m][j >> 1][(j & 1) * 2 + 1] = hi;
        }
    }
    // layer 2 in 16-column slices, each slice feeding one K step of layer 3
    float acc[2][4];
#pragma unroll
    for (int m = 0; m < 2; ++m) {
        acc[m][0] = acc[m][2] = b3[2 * t];
        acc[m][1] = acc[m][3] = b3[2 * t + 1];
    }
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        uint32_t a3[2][4];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int j = 2 * s + h, n = 8 * j + g;
            uint32_t w0[4], w1[4];
#pragma unroll
            for (int kt = 0; kt < 4; ++kt) {
                w0[kt] = ld32(W2s + n * LD2 + 16 * kt + 2 * t);
                w1[kt] = ld32(W2s + n * LD2 + 16 * kt + 2 * t + 8);
            }
            const float c0 = b2[8 * j + 2 * t], c1 = b2[8 * j + 2 * t + 1];
#pragma unroll
            for (int m = 0; m < 2; ++m) {
                float d[4] = {c0, c1, c0, c1};
#pragma unroll
                for (int kt = 0; kt < 4; ++kt) mma_bf16(d, a2[m][kt], w0[kt], w1[kt]);
                a3[m][2 * h] = pack_bf16(gelu(d[0]), gelu(d[1]));
                a3[m][2 * h + 1] = pack_bf16(gelu(d[2]), gelu(d[3]));
            }
        }
        const uint32_t v0 = ld32(W3s + g * LD2 + 16 * s + 2 * t), v1 = ld32(W3s + g * LD2 + 16 * s + 2 * t + 8);
#pragma unroll
        for (int m = 0; m < 2; ++m) mma_bf16(acc[m], a3[m], v0, v1);
    }
#pragma unroll
    for (int m = 0; m < 2; ++m) {
        const int r = m * 16 + g;
        os[r * 8 + 2 * t] = acc[m][0];
        os[r * 8 + 2 * t + 1] = acc[m][1];
        os[(r + 8) * 8 + 2 * t] = acc[m][2];
        os[(r + 8) * 8 + 2 * t + 1] = acc[m][3];
    }
    __syncwarp();
#pragma unroll
    for (int i = 0; i < OUT; ++i) y[i] = os[lane * 8 + i];
    __syncwarp();
}

// Warm start of the prox from the network: sigma_in + oscale * y.
__device__ __forceinline__ void predict_start(const unsigned char* img, const float s[3], const float y[OUT],
                                              float out[3]) {
    const float* nrm = reinterpret_cast<const float*>(img + I_NORM);
#pragma unroll
    for (int i = 0; i < 3; ++i) out[i] = s[i] + nrm[B_OSCALE + i] * y[i];
}

// Builds the device image of an FP32 blob (host pointer) into `img`
// (IMAGE_BYTES), staging the blob in `d_blob_scratch` (N_BLOB floats).
void upload_image(const float* h_blob, unsigned char* img, float* d_blob_scratch, cudaStream_t st);

}  // namespace net
}  // namespace wrapd
