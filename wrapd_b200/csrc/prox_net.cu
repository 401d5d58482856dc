// Training and batched inference of the prox-stretch network (prox_net.cuh).
//
// Training step over a batch: k_train_tile runs forward and backward for 128
// samples per CTA (4 warps x 32) on the tensor cores and writes that CTA's
// gradient to a partial buffer; k_reduce_adam adds the partials in CTA order
// (deterministic) and applies Adam to the FP32 blob.  Loss: mean squared error
// of the normalised outputs, t = (sigma* - sigma_in) / oscale.
//
// Backward, per warp (rows = its samples; BF16 operands, FP32 accumulation):
//   dY = 2 (Y - T) / (3 B);  dH2 = dY W3;  dZ2 = dH2 * gelu'(Z2)
//   dH1 = dZ2 W2;  dZ1 = dH1 * gelu'(Z1)
// then per CTA, K = its 128 samples: dW3 = dY^T H2, dW2 = dZ2^T H1,
// dW1 = dZ1^T X, biases = column sums of the FP32 dY / dZ.  Operands of
// these are kept transposed in shared memory ([feature][sample]) so that every
// fragment is two 32-bit loads.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "prox_net.cuh"
#include "prox_net_tc.cuh"

namespace wrapd {
namespace net {
namespace {

constexpr int TILE = 128;          // samples per CTA
constexpr int LDT = TILE + 8;      // transposed rows: [feature][sample]
constexpr int LDZ = HID + 4;       // FP32 activations [sample][LDZ]

// training shared-memory layout (bytes)
constexpr int T_IMG = 0;
constexpr int T_W2T = T_IMG + IMAGE_BYTES;          // [64][LD2] BF16, W2T[in][out]
constexpr int T_W3T = T_W2T + HID * LD2 * 2;        // [64][LD1] BF16, W3T[in][out], out 3..23 zero
constexpr int T_XS = T_W3T + HID * LD1 * 2;         // [128][LD1] BF16 normalised inputs
constexpr int T_XT = T_XS + TILE * LD1 * 2;         // [16][LDT] BF16
constexpr int T_TN = T_XT + 16 * LDT * 2;           // [128][4] FP32 normalised targets
constexpr int T_Z1 = T_TN + TILE * 4 * 4;           // [128][LDZ] FP32: Z1, then dZ1
constexpr int T_Z2 = T_Z1 + TILE * LDZ * 4;         // [128][LDZ] FP32: Z2, then dZ2
constexpr int T_H1T = T_Z2 + TILE * LDZ * 4;        // [64][LDT] BF16
constexpr int T_H2T = T_H1T + HID * LDT * 2;        // [64][LDT] BF16
constexpr int T_DYT = T_H2T + HID * LDT * 2;        // [16][LDT] BF16, rows 3..15 zero
constexpr int T_DYF = T_DYT + 16 * LDT * 2;         // [128][4] FP32 dY
constexpr int T_DZ1T = T_DYF + TILE * 4 * 4;        // [64][LDT] BF16
constexpr int T_DZ2T = T_DZ1T + HID * LDT * 2;      // [64][LDT] BF16
constexpr int T_RED = T_DZ2T + HID * LDT * 2;       // double[4]
constexpr int TRAIN_SMEM = T_RED + 4 * 8;
static_assert(TRAIN_SMEM <= 227 * 1024, "training tile exceeds shared memory");

__device__ __forceinline__ void st_bf16(__nv_bfloat16* p, float v) { *p = __float2bfloat16_rn(v); }

// One CTA: samples [first + 128 * blockIdx.x, ...) of the batch (through perm
// when given), B = batch size for the loss scale.  part: N_TRAIN floats per CTA.
__global__ void __launch_bounds__(128) k_train_tile(const float* __restrict__ blob, const float* __restrict__ X,
                                                    const float* __restrict__ T, const int64_t* __restrict__ perm,
                                                    int64_t first, int64_t last, float inv_b, float* __restrict__ part,
                                                    double* __restrict__ loss_part) {
    extern __shared__ __align__(16) unsigned char sm[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
    build_image(blob, sm + T_IMG, tid, blockDim.x);
    __nv_bfloat16* W2T = reinterpret_cast<__nv_bfloat16*>(sm + T_W2T);
    __nv_bfloat16* W3T = reinterpret_cast<__nv_bfloat16*>(sm + T_W3T);
    for (int i = tid; i < HID * LD2; i += blockDim.x) {
        const int in = i / LD2, o = i % LD2;
        W2T[i] = __float2bfloat16_rn(o < HID ? blob[B_W2 + o * HID + in] : 0.0f);
    }
    for (int i = tid; i < HID * LD1; i += blockDim.x) {
        const int in = i / LD1, o = i % LD1;
        W3T[i] = __float2bfloat16_rn(o < OUT ? blob[B_W3 + o * HID + in] : 0.0f);
    }
    __nv_bfloat16* DYT = reinterpret_cast<__nv_bfloat16*>(sm + T_DYT);
    for (int i = tid; i < 16 * LDT; i += blockDim.x) DYT[i] = __float2bfloat16_rn(0.0f);
    __syncthreads();

    const unsigned char* img = sm + T_IMG;
    const float* nrm = reinterpret_cast<const float*>(img + I_NORM);
    const __nv_bfloat16* W1s = reinterpret_cast<const __nv_bfloat16*>(img + I_W1);
    const __nv_bfloat16* W2s = reinterpret_cast<const __nv_bfloat16*>(img + I_W2);
    const __nv_bfloat16* W3s = reinterpret_cast<const __nv_bfloat16*>(img + I_W3);
    const float* b1 = reinterpret_cast<const float*>(img + I_B1);
    const float* b2 = reinterpret_cast<const float*>(img + I_B2);
    const float* b3 = reinterpret_cast<const float*>(img + I_B3);
    __nv_bfloat16* XS = reinterpret_cast<__nv_bfloat16*>(sm + T_XS);
    __nv_bfloat16* XT = reinterpret_cast<__nv_bfloat16*>(sm + T_XT);
    float* TN = reinterpret_cast<float*>(sm + T_TN);
    float* Z1 = reinterpret_cast<float*>(sm + T_Z1);
    float* Z2 = reinterpret_cast<float*>(sm + T_Z2);
    __nv_bfloat16* H1T = reinterpret_cast<__nv_bfloat16*>(sm + T_H1T);
    __nv_bfloat16* H2T = reinterpret_cast<__nv_bfloat16*>(sm + T_H2T);
    float* DYF = reinterpret_cast<float*>(sm + T_DYF);
    __nv_bfloat16* DZ1T = reinterpret_cast<__nv_bfloat16*>(sm + T_DZ1T);
    __nv_bfloat16* DZ2T = reinterpret_cast<__nv_bfloat16*>(sm + T_DZ2T);
    double* RED = reinterpret_cast<double*>(sm + T_RED);

    // ---- stage this lane's sample ----
    const int row = warp * 32 + lane;
    const int64_t pos = first + (int64_t)blockIdx.x * TILE + row;
    const bool valid = pos < last;
    {
        float f[IN] = {0.f, 0.f, 0.f, 0.f, 0.f}, tg[3] = {0.f, 0.f, 0.f};
        if (valid) {
            const int64_t s = perm ? perm[pos] : pos;
#pragma unroll
            for (int c = 0; c < IN; ++c) f[c] = X[IN * s + c];
#pragma unroll
            for (int c = 0; c < 3; ++c) tg[c] = (T[3 * s + c] - f[c]) / nrm[B_OSCALE + c];
        }
#pragma unroll
        for (int c = 0; c < 16; ++c) {
            const float v = (valid && c < IN) ? (f[c] - nrm[B_MEAN + c]) * nrm[B_ISTD + c] : 0.0f;
            st_bf16(XS + row * LD1 + c, v);
            st_bf16(XT + c * LDT + row, v);
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) TN[row * 4 + c] = tg[c];
        TN[row * 4 + 3] = 0.0f;
    }
    __syncwarp();

    // ---- forward ----
    uint32_t a2[2][4][4];
    {
        uint32_t a1[2][4];
#pragma unroll
        for (int m = 0; m < 2; ++m) {
            const int r = warp * 32 + m * 16 + g;
            a1[m][0] = ld32(XS + r * LD1 + 2 * t);
            a1[m][1] = ld32(XS + (r + 8) * LD1 + 2 * t);
            a1[m][2] = ld32(XS + r * LD1 + 2 * t + 8);
            a1[m][3] = ld32(XS + (r + 8) * LD1 + 2 * t + 8);
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int n = 8 * j + g, col = 8 * j + 2 * t;
            const uint32_t w0 = ld32(W1s + n * LD1 + 2 * t), w1 = ld32(W1s + n * LD1 + 2 * t + 8);
#pragma unroll
            for (int m = 0; m < 2; ++m) {
                const int r = warp * 32 + m * 16 + g;
                float d[4] = {b1[col], b1[col + 1], b1[col], b1[col + 1]};
                mma_bf16(d, a1[m], w0, w1);
                Z1[r * LDZ + col] = d[0]; Z1[r * LDZ + col + 1] = d[1];
                Z1[(r + 8) * LDZ + col] = d[2]; Z1[(r + 8) * LDZ + col + 1] = d[3];
                const float h0 = gelu(d[0]), h1 = gelu(d[1]), h2 = gelu(d[2]), h3 = gelu(d[3]);
                a2[m][j >> 1][(j & 1) * 2] = pack_bf16(h0, h1);
                a2[m][j >> 1][(j & 1) * 2 + 1] = pack_bf16(h2, h3);
                st_bf16(H1T + col * LDT + r, h0); st_bf16(H1T + (col + 1) * LDT + r, h1);
                st_bf16(H1T + col * LDT + r + 8, h2); st_bf16(H1T + (col + 1) * LDT + r + 8, h3);
            }
        }
    }
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
            const int j = 2 * s + h, n = 8 * j + g, col = 8 * j + 2 * t;
            uint32_t w0[4], w1[4];
#pragma unroll
            for (int kt = 0; kt < 4; ++kt) {
                w0[kt] = ld32(W2s + n * LD2 + 16 * kt + 2 * t);
                w1[kt] = ld32(W2s + n * LD2 + 16 * kt + 2 * t + 8);
            }
#pragma unroll
            for (int m = 0; m < 2; ++m) {
                const int r = warp * 32 + m * 16 + g;
                float d[4] = {b2[col], b2[col + 1], b2[col], b2[col + 1]};
#pragma unroll
                for (int kt = 0; kt < 4; ++kt) mma_bf16(d, a2[m][kt], w0[kt], w1[kt]);
                Z2[r * LDZ + col] = d[0]; Z2[r * LDZ + col + 1] = d[1];
                Z2[(r + 8) * LDZ + col] = d[2]; Z2[(r + 8) * LDZ + col + 1] = d[3];
                const float h0 = gelu(d[0]), h1 = gelu(d[1]), h2 = gelu(d[2]), h3 = gelu(d[3]);
                a3[m][2 * h] = pack_bf16(h0, h1);
                a3[m][2 * h + 1] = pack_bf16(h2, h3);
                st_bf16(H2T + col * LDT + r, h0); st_bf16(H2T + (col + 1) * LDT + r, h1);
                st_bf16(H2T + col * LDT + r + 8, h2); st_bf16(H2T + (col + 1) * LDT + r + 8, h3);
            }
        }
        const uint32_t v0 = ld32(W3s + g * LD2 + 16 * s + 2 * t), v1 = ld32(W3s + g * LD2 + 16 * s + 2 * t + 8);
#pragma unroll
        for (int m = 0; m < 2; ++m) mma_bf16(acc[m], a3[m], v0, v1);
    }

    // ---- loss and dY ----
    double lsum = 0.0;
    uint32_t ady[2][4];
#pragma unroll
    for (int m = 0; m < 2; ++m) {
        float dy[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int r = warp * 32 + m * 16 + g + (q >> 1) * 8, col = 2 * t + (q & 1);
            const int64_t p = first + (int64_t)blockIdx.x * TILE + r;
            float v = 0.0f;
            if (col < OUT && p < last) {
                const float e = acc[m][q] - TN[r * 4 + col];
                lsum += (double)e * e;
                v = 2.0f * e * inv_b;
            }
            dy[q] = v;
            if (col < 4) DYF[r * 4 + col] = v;
            if (col < OUT) st_bf16(DYT + col * LDT + r, v);
        }
        ady[m][0] = pack_bf16(dy[0], dy[1]);
        ady[m][1] = pack_bf16(dy[2], dy[3]);
        ady[m][2] = 0u;
        ady[m][3] = 0u;
    }
    // ---- dH2 = dY W3 -> dZ2 ----
    uint32_t adz[2][4][4];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int n = 8 * j + g, col = 8 * j + 2 * t;
        const uint32_t w0 = ld32(W3T + n * LD1 + 2 * t), w1 = ld32(W3T + n * LD1 + 2 * t + 8);
#pragma unroll
        for (int m = 0; m < 2; ++m) {
            const int r = warp * 32 + m * 16 + g;
            float d[4] = {0.f, 0.f, 0.f, 0.f};
            mma_bf16(d, ady[m], w0, w1);
            d[0] *= gelu_grad(Z2[r * LDZ + col]);
            d[1] *= gelu_grad(Z2[r * LDZ + col + 1]);
            d[2] *= gelu_grad(Z2[(r + 8) * LDZ + col]);
            d[3] *= gelu_grad(Z2[(r + 8) * LDZ + col + 1]);
            Z2[r * LDZ + col] = d[0]; Z2[r * LDZ + col + 1] = d[1];
            Z2[(r + 8) * LDZ + col] = d[2]; Z2[(r + 8) * LDZ + col + 1] = d[3];
            adz[m][j >> 1][(j & 1) * 2] = pack_bf16(d[0], d[1]);
            adz[m][j >> 1][(j & 1) * 2 + 1] = pack_bf16(d[2], d[3]);
            st_bf16(DZ2T + col * LDT + r, d[0]); st_bf16(DZ2T + (col + 1) * LDT + r, d[1]);
            st_bf16(DZ2T + col * LDT + r + 8, d[2]); st_bf16(DZ2T + (col + 1) * LDT + r + 8, d[3]);
        }
    }
    // ---- dH1 = dZ2 W2 -> dZ1 ----
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int n = 8 * j + g, col = 8 * j + 2 * t;
        uint32_t w0[4], w1[4];
#pragma unroll
        for (int kt = 0; kt < 4; ++kt) {
            w0[kt] = ld32(W2T + n * LD2 + 16 * kt + 2 * t);
            w1[kt] = ld32(W2T + n * LD2 + 16 * kt + 2 * t + 8);
        }
#pragma unroll
        for (int m = 0; m < 2; ++m) {
            const int r = warp * 32 + m * 16 + g;
            float d[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int kt = 0; kt < 4; ++kt) mma_bf16(d, adz[m][kt], w0[kt], w1[kt]);
            d[0] *= gelu_grad(Z1[r * LDZ + col]);
            d[1] *= gelu_grad(Z1[r * LDZ + col + 1]);
            d[2] *= gelu_grad(Z1[(r + 8) * LDZ + col]);
            d[3] *= gelu_grad(Z1[(r + 8) * LDZ + col + 1]);
            Z1[r * LDZ + col] = d[0]; Z1[r * LDZ + col + 1] = d[1];
            Z1[(r + 8) * LDZ + col] = d[2]; Z1[(r + 8) * LDZ + col + 1] = d[3];
            st_bf16(DZ1T + col * LDT + r, d[0]); st_bf16(DZ1T + (col + 1) * LDT + r, d[1]);
            st_bf16(DZ1T + col * LDT + r + 8, d[2]); st_bf16(DZ1T + (col + 1) * LDT + r + 8, d[3]);
        }
    }
    for (int o = 16; o > 0; o >>= 1) lsum += __shfl_down_sync(0xffffffffu, lsum, o);
    if (lane == 0) RED[warp] = lsum;
    __syncthreads();

    // ---- weight gradients over the CTA's samples (K = 128) ----
    // tiles 0..3: dW1 (m = out/16, n = in 0..7); 4..35: dW2 (4 x 8); 36..43: dW3 (n = in/8)
    float* P = part + (size_t)blockIdx.x * N_TRAIN;
    for (int tile = warp; tile < 44; tile += 4) {
        const __nv_bfloat16 *A, *B;
        int m0, n0, kind;
        if (tile < 4) { kind = 0; A = DZ1T; B = XT; m0 = 16 * tile; n0 = 0; }
        else if (tile < 36) { kind = 1; A = DZ2T; B = H1T; m0 = 16 * ((tile - 4) >> 3); n0 = 8 * ((tile - 4) & 7); }
        else { kind = 2; A = DYT; B = H2T; m0 = 0; n0 = 8 * (tile - 36); }
        float d[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int kk = 0; kk < TILE / 16; ++kk) {
            const int k0 = 16 * kk;
            const uint32_t a[4] = {ld32(A + (m0 + g) * LDT + k0 + 2 * t), ld32(A + (m0 + g + 8) * LDT + k0 + 2 * t),
                                   ld32(A + (m0 + g) * LDT + k0 + 2 * t + 8),
                                   ld32(A + (m0 + g + 8) * LDT + k0 + 2 * t + 8)};
            mma_bf16(d, a, ld32(B + (n0 + g) * LDT + k0 + 2 * t), ld32(B + (n0 + g) * LDT + k0 + 2 * t + 8));
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int o = m0 + g + (q >> 1) * 8, in = n0 + 2 * t + (q & 1);
            if (kind == 0) { if (in < IN) P[B_W1 - B_W1 + o * IN + in] = d[q]; }
            else if (kind == 1) P[B_W2 - B_W1 + o * HID + in] = d[q];
            else if (o < OUT) P[B_W3 - B_W1 + o * HID + in] = d[q];
        }
    }
    {
        const int j = tid & 63;
        const float* Z = tid < 64 ? Z1 : Z2;
        float s = 0.0f;
        for (int r = 0; r < TILE; ++r) s += Z[r * LDZ + j];
        P[(tid < 64 ? B_B1 : B_B2) - B_W1 + j] = s;
        if (tid < OUT) {
            float s3 = 0.0f;
            for (int r = 0; r < TILE; ++r) s3 += DYF[r * 4 + tid];
            P[B_B3 - B_W1 + tid] = s3;
        }
        if (tid == 0) loss_part[blockIdx.x] = ((RED[0] + RED[1]) + RED[2]) + RED[3];
    }
}

// Adds the CTA partials in order; mode 0: write the gradient, mode 1: Adam.
__global__ void k_reduce_adam(int nparts, const float* __restrict__ part, const double* __restrict__ loss_part,
                              float* __restrict__ blob, float* __restrict__ m1, float* __restrict__ m2,
                              float* __restrict__ grad_out, double* __restrict__ loss_out, int mode, float lr_t,
                              float beta1, float beta2, float eps) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < N_TRAIN) {
        float gsum = 0.0f;
        for (int c = 0; c < nparts; ++c) gsum += part[(size_t)c * N_TRAIN + p];
        if (mode == 0) {
            grad_out[p] = gsum;
        } else {
            const float a = beta1 * m1[p] + (1.0f - beta1) * gsum;
            const float b = beta2 * m2[p] + (1.0f - beta2) * gsum * gsum;
            m1[p] = a;
            m2[p] = b;
            blob[B_W1 + p] -= lr_t * a / (sqrtf(b) + eps);
        }
    }
    if (p == 0 && loss_out) {
        double s = 0.0;
        for (int c = 0; c < nparts; ++c) s += loss_part[c];
        *loss_out = s;
    }
}

__global__ void k_image(const float* __restrict__ blob, unsigned char* __restrict__ img) {
    build_image(blob, img, threadIdx.x, blockDim.x);
}

// Batched inference: one warp per 32 samples, the same warp_forward the local
// step inlines.  out = predicted prox stretches.
__global__ void __launch_bounds__(128) k_predict(const unsigned char* __restrict__ gimg, int n,
                                                 const double* __restrict__ sig, const double* __restrict__ wov,
                                                 float mu, float lambda, double* __restrict__ out) {
    extern __shared__ __align__(16) unsigned char sm[];
    load_image(gimg, sm);
    __syncthreads();
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = e < n;
    float s[3] = {1.f, 1.f, 1.f}, f[IN], y[OUT], p[3];
    if (valid) {
#pragma unroll
        for (int i = 0; i < 3; ++i) s[i] = float(sig[3 * (size_t)e + i]);
    }
    features(s, valid ? float(wov[e]) : mu, mu, lambda, f);
    warp_forward(sm, sm + IMAGE_BYTES + (threadIdx.x >> 5) * WARP_SCRATCH, f, valid, y);
    predict_start(sm, s, y, p);
    if (valid) {
#pragma unroll
        for (int i = 0; i < 3; ++i) out[3 * (size_t)e + i] = p[i];
    }
}

__global__ void k_tc_image(const float* __restrict__ blob, unsigned char* __restrict__ img) {
    tc::build_tc_image(blob, img, threadIdx.x, blockDim.x);
}

// Batched inference on the tcgen05 tensor cores: each CTA runs tiles of 128
// samples (tile = blockIdx.x, + gridDim.x, ...) through tc::Cta::forward.
// A bounded wait that gives up sets *err and ends the CTA's work.
__global__ void __launch_bounds__(128) k_predict_tc(const unsigned char* __restrict__ gimg, int n,
                                                    const double* __restrict__ sig, const double* __restrict__ wov,
                                                    float mu, float lambda, double* __restrict__ out,
                                                    int* __restrict__ err) {
    extern __shared__ __align__(128) unsigned char sm[];
    tc::Cta cta;
    cta.img = sm;
    cta.act = sm + tc::T_BYTES;
    cta.bar = reinterpret_cast<uint64_t*>(sm + tc::T_BYTES + tc::A_BYTES);
    cta.tmem_slot = reinterpret_cast<uint32_t*>(sm + tc::T_BYTES + tc::A_BYTES + 8);
    {
        const uint4* src = reinterpret_cast<const uint4*>(gimg);
        uint4* dst = reinterpret_cast<uint4*>(sm);
        for (int i = threadIdx.x; i < tc::T_BYTES / 16; i += blockDim.x) dst[i] = src[i];
    }
    cta.setup();
    const float* nrm = reinterpret_cast<const float*>(sm + tc::T_NORM);
    const int ntiles = (n + tc::M - 1) / tc::M;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int e = tile * tc::M + threadIdx.x;
        const bool valid = e < n;
        float s[3] = {1.f, 1.f, 1.f}, f[IN], y[OUT] = {0.f, 0.f, 0.f};
        if (valid) {
#pragma unroll
            for (int i = 0; i < 3; ++i) s[i] = float(sig[3 * (size_t)e + i]);
        }
        features(s, valid ? float(wov[e]) : mu, mu, lambda, f);
        if (!cta.forward(f, valid, y)) {   // the same verdict in every thread
            if (threadIdx.x == 0) atomicExch(err, 1);
            break;
        }
        if (valid) {
#pragma unroll
            for (int i = 0; i < 3; ++i) out[3 * (size_t)e + i] = s[i] + nrm[B_OSCALE + i] * y[i];
        }
    }
    cta.teardown();
}

}  // namespace

// Device image of a blob, built on `st` into `img` (IMAGE_BYTES).
void upload_image(const float* h_blob, unsigned char* img, float* d_blob_scratch, cudaStream_t st) {
    WRAPD_CUDA(cudaMemcpyAsync(d_blob_scratch, h_blob, N_BLOB * sizeof(float), cudaMemcpyHostToDevice, st));
    k_image<<<1, 256, 0, st>>>(d_blob_scratch, img);
    WRAPD_LAUNCH_CHECK();
}

}  // namespace net
}  // namespace wrapd

using namespace wrapd;
using namespace wrapd::net;

struct wrapd_prox_net {
    float* d_blob = nullptr;
    float* d_m1 = nullptr;
    float* d_m2 = nullptr;
    float* d_part = nullptr;
    double* d_loss = nullptr;      // per-CTA loss partials
    double* d_losses = nullptr;    // per-step loss
    float* d_grad = nullptr;
    float* d_X = nullptr;
    float* d_T = nullptr;
    int64_t* d_perm = nullptr;
    int64_t n = 0;
    int max_parts = 0;
    int64_t step = 0;
    cudaStream_t st = nullptr;
    std::vector<void*> allocs;
    std::string err;

    void* alloc(size_t bytes) {
        void* p = nullptr;
        if (cudaMalloc(&p, bytes ? bytes : 16) != cudaSuccess) {
            cudaGetLastError();
            throw CudaError(WRAPD_E_OOM, "cudaMalloc failed (prox net)");
        }
        allocs.push_back(p);
        return p;
    }
    void release(void* p) {
        if (!p) return;
        cudaFree(p);
        allocs.erase(std::remove(allocs.begin(), allocs.end(), p), allocs.end());
    }
    ~wrapd_prox_net() {
        for (void* p : allocs) cudaFree(p);
        if (st) cudaStreamDestroy(st);
    }
};

namespace {

thread_local std::string g_net_error;

template <typename F>
int net_guarded(wrapd_prox_net* h, F&& f) {
    std::string& err = h ? h->err : g_net_error;
    try {
        f();
        err.clear();
        return WRAPD_OK;
    } catch (const CudaError& e) {
        err = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        err = "host allocation failed";
        return WRAPD_E_OOM;
    } catch (const std::exception& e) {
        err = e.what();
        return WRAPD_E_INPUT;
    }
}

void ensure_parts(wrapd_prox_net* h, int parts) {
    if (parts <= h->max_parts) return;
    h->release(h->d_part);
    h->release(h->d_loss);
    h->d_part = static_cast<float*>(h->alloc((size_t)parts * N_TRAIN * sizeof(float)));
    h->d_loss = static_cast<double*>(h->alloc((size_t)parts * sizeof(double)));
    h->max_parts = parts;
}

void launch_step(wrapd_prox_net* h, int64_t first, int64_t last, const int64_t* perm, int mode, float lr_t,
                 double* loss_out) {
    const int parts = static_cast<int>((last - first + TILE - 1) / TILE);
    ensure_parts(h, parts);
    k_train_tile<<<parts, 128, TRAIN_SMEM, h->st>>>(h->d_blob, h->d_X, h->d_T, perm, first, last,
                                                     1.0f / (3.0f * float(last - first)), h->d_part, h->d_loss);
    WRAPD_LAUNCH_CHECK();
    k_reduce_adam<<<(N_TRAIN + 255) / 256, 256, 0, h->st>>>(parts, h->d_part, h->d_loss, h->d_blob, h->d_m1,
                                                            h->d_m2, h->d_grad, loss_out, mode, lr_t, 0.9f, 0.999f,
                                                            1e-8f);
    WRAPD_LAUNCH_CHECK();
}

uint64_t splitmix(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

}  // namespace

extern "C" {

WRAPD_API const char* wrapd_net_last_error(wrapd_prox_net* h) { return h ? h->err.c_str() : g_net_error.c_str(); }

WRAPD_API int wrapd_net_create(const float* blob, int n_blob, wrapd_prox_net** out) {
    if (!blob || !out || n_blob != N_BLOB) return WRAPD_E_INPUT;
    *out = nullptr;
    wrapd_prox_net* h = nullptr;
    const int rc = net_guarded(nullptr, [&] {
        h = new wrapd_prox_net();
        try {
            WRAPD_CUDA(cudaFuncSetAttribute(k_train_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, TRAIN_SMEM));
            WRAPD_CUDA(cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking));
            h->d_blob = static_cast<float*>(h->alloc(N_BLOB * sizeof(float)));
            h->d_m1 = static_cast<float*>(h->alloc(N_TRAIN * sizeof(float)));
            h->d_m2 = static_cast<float*>(h->alloc(N_TRAIN * sizeof(float)));
            h->d_grad = static_cast<float*>(h->alloc(N_TRAIN * sizeof(float)));
            h->d_losses = static_cast<double*>(h->alloc(sizeof(double)));
            WRAPD_CUDA(cudaMemcpyAsync(h->d_blob, blob, N_BLOB * sizeof(float), cudaMemcpyHostToDevice, h->st));
            WRAPD_CUDA(cudaMemsetAsync(h->d_m1, 0, N_TRAIN * sizeof(float), h->st));
            WRAPD_CUDA(cudaMemsetAsync(h->d_m2, 0, N_TRAIN * sizeof(float), h->st));
            WRAPD_CUDA(cudaStreamSynchronize(h->st));
        } catch (...) {
            delete h;
            h = nullptr;
            throw;
        }
    });
    *out = h;
    return rc;
}

WRAPD_API int wrapd_net_set_data(wrapd_prox_net* h, const float* features, const float* targets, int64_t n) {
    if (!h || n <= 0 || !features || !targets) return WRAPD_E_INPUT;
    return net_guarded(h, [&] {
        h->release(h->d_X);
        h->release(h->d_T);
        h->release(h->d_perm);
        h->d_X = h->d_T = nullptr;
        h->d_perm = nullptr;
        h->d_X = static_cast<float*>(h->alloc((size_t)n * IN * sizeof(float)));
        h->d_T = static_cast<float*>(h->alloc((size_t)n * 3 * sizeof(float)));
        h->d_perm = static_cast<int64_t*>(h->alloc((size_t)n * sizeof(int64_t)));
        WRAPD_CUDA(cudaMemcpyAsync(h->d_X, features, (size_t)n * IN * sizeof(float), cudaMemcpyHostToDevice, h->st));
        WRAPD_CUDA(cudaMemcpyAsync(h->d_T, targets, (size_t)n * 3 * sizeof(float), cudaMemcpyHostToDevice, h->st));
        WRAPD_CUDA(cudaStreamSynchronize(h->st));
        h->n = n;
    });
}

WRAPD_API int wrapd_net_train(wrapd_prox_net* h, int epochs, int batch, float lr, float lr_end, uint64_t seed,
                              double* epoch_loss) {
    if (!h || epochs <= 0 || batch <= 0 || !(lr > 0.0f)) return WRAPD_E_INPUT;
    if (!h->d_X) return WRAPD_E_STATE;
    return net_guarded(h, [&] {
        const int64_t n = h->n;
        const int64_t steps_per_epoch = (n + batch - 1) / batch;
        const int64_t total = steps_per_epoch * epochs;
        std::vector<int64_t> perm(n);
        std::vector<double> losses(steps_per_epoch);
        double* d_losses = static_cast<double*>(h->alloc(steps_per_epoch * sizeof(double)));
        uint64_t rs = seed;
        for (int ep = 0; ep < epochs; ++ep) {
            for (int64_t i = 0; i < n; ++i) perm[i] = i;
            for (int64_t i = n - 1; i > 0; --i) std::swap(perm[i], perm[splitmix(rs) % (uint64_t)(i + 1)]);
            WRAPD_CUDA(cudaMemcpyAsync(h->d_perm, perm.data(), n * sizeof(int64_t), cudaMemcpyHostToDevice, h->st));
            for (int64_t s = 0; s < steps_per_epoch; ++s) {
                const int64_t k = (int64_t)ep * steps_per_epoch + s;
                // cosine schedule from lr to lr_end; Adam bias correction folded into the rate
                const double frac = total > 1 ? double(k) / double(total - 1) : 1.0;
                const double rate = lr_end + 0.5 * (lr - lr_end) * (1.0 + std::cos(3.141592653589793 * frac));
                const int64_t tstep = ++h->step;
                const double corr = std::sqrt(1.0 - std::pow(0.999, double(tstep))) / (1.0 - std::pow(0.9, double(tstep)));
                launch_step(h, s * batch, std::min<int64_t>(n, (s + 1) * batch), h->d_perm, 1, float(rate * corr),
                            d_losses + s);
            }
            WRAPD_CUDA(cudaMemcpyAsync(losses.data(), d_losses, steps_per_epoch * sizeof(double),
                                       cudaMemcpyDeviceToHost, h->st));
            WRAPD_CUDA(cudaStreamSynchronize(h->st));
            if (epoch_loss) {
                double s = 0.0;
                for (double v : losses) s += v;
                epoch_loss[ep] = s / (3.0 * double(n));
            }
        }
        h->release(d_losses);
    });
}

WRAPD_API int wrapd_net_grad(wrapd_prox_net* h, int64_t first, int n, double* loss, float* grad) {
    if (!h || n <= 0 || first < 0 || !grad) return WRAPD_E_INPUT;
    if (!h->d_X || first + n > h->n) return WRAPD_E_INPUT;
    return net_guarded(h, [&] {
        launch_step(h, first, first + n, nullptr, 0, 0.0f, h->d_losses);
        double l = 0.0;
        WRAPD_CUDA(cudaMemcpyAsync(grad, h->d_grad, N_TRAIN * sizeof(float), cudaMemcpyDeviceToHost, h->st));
        WRAPD_CUDA(cudaMemcpyAsync(&l, h->d_losses, sizeof(double), cudaMemcpyDeviceToHost, h->st));
        WRAPD_CUDA(cudaStreamSynchronize(h->st));
        if (loss) *loss = l / (3.0 * double(n));
    });
}

WRAPD_API int wrapd_net_get(wrapd_prox_net* h, float* blob) {
    if (!h || !blob) return WRAPD_E_INPUT;
    return net_guarded(h, [&] {
        WRAPD_CUDA(cudaMemcpyAsync(blob, h->d_blob, N_BLOB * sizeof(float), cudaMemcpyDeviceToHost, h->st));
        WRAPD_CUDA(cudaStreamSynchronize(h->st));
    });
}

WRAPD_API void wrapd_net_destroy(wrapd_prox_net* h) { delete h; }

WRAPD_API int wrapd_net_predict(const float* blob, int n_blob, int n, const double* sigma_in, const double* wov,
                                double mu, double lambda, double* out) {
    if (!blob || n_blob != N_BLOB || n < 0 || (n > 0 && (!sigma_in || !wov || !out))) return WRAPD_E_INPUT;
    if (!(mu > 0.0) || !(lambda > 0.0)) return WRAPD_E_INPUT;
    if (n == 0) return WRAPD_OK;
    return net_guarded(nullptr, [&] {
        struct Bufs {
            std::vector<void*> p;
            ~Bufs() { for (void* q : p) cudaFree(q); }
            void* get(size_t b) {
                void* q = nullptr;
                if (cudaMalloc(&q, b) != cudaSuccess) { cudaGetLastError(); throw CudaError(WRAPD_E_OOM, "cudaMalloc failed"); }
                p.push_back(q);
                return q;
            }
        } bufs;
        float* d_blob = static_cast<float*>(bufs.get(N_BLOB * sizeof(float)));
        unsigned char* d_img = static_cast<unsigned char*>(bufs.get(tc::T_BYTES));
        double* d_s = static_cast<double*>(bufs.get(3 * (size_t)n * sizeof(double)));
        double* d_w = static_cast<double*>(bufs.get((size_t)n * sizeof(double)));
        double* d_o = static_cast<double*>(bufs.get(3 * (size_t)n * sizeof(double)));
        int* d_err = static_cast<int*>(bufs.get(sizeof(int)));
        WRAPD_CUDA(cudaMemcpy(d_blob, blob, N_BLOB * sizeof(float), cudaMemcpyHostToDevice));
        WRAPD_CUDA(cudaMemset(d_err, 0, sizeof(int)));
        k_tc_image<<<1, 256>>>(d_blob, d_img);
        WRAPD_LAUNCH_CHECK();
        WRAPD_CUDA(cudaMemcpy(d_s, sigma_in, 3 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice));
        WRAPD_CUDA(cudaMemcpy(d_w, wov, (size_t)n * sizeof(double), cudaMemcpyHostToDevice));
        const int tiles = (n + tc::M - 1) / tc::M;
        k_predict_tc<<<std::min(tiles, 4 * kNumSMs), 128, tc::SMEM_BYTES>>>(d_img, n, d_s, d_w, float(mu),
                                                                            float(lambda), d_o, d_err);
        WRAPD_LAUNCH_CHECK();
        WRAPD_CUDA(cudaMemcpy(out, d_o, 3 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost));
        int err = 0;
        WRAPD_CUDA(cudaMemcpy(&err, d_err, sizeof(int), cudaMemcpyDeviceToHost));
        if (err) throw CudaError(WRAPD_E_TIMEOUT, "a tensor-core wait of the prox network gave up");
    });
}

}  // extern "C"
