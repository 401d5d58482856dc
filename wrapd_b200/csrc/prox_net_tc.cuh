// The prox network's forward pass on the fifth-generation tensor cores:
// tcgen05.mma (kind::f16, BF16 operands read from shared memory through
// matrix descriptors, FP32 accumulators in tensor memory), 128 samples per
// 128-thread CTA.  Thread t owns sample t of the tile: it writes its
// features (then its hidden activations) as row t of the A operand, one
// elected thread issues each layer's MMAs and commits them to an mbarrier,
// and thread t reads row t of the accumulator back with tcgen05.ld (TMEM lane
// t) for the bias, GELU and BF16 rounding before the next layer.  The
// numerics are those of the mma.sync path in prox_net.cuh: BF16 inputs,
// weights and hidden activations, FP32 accumulation, the same GELU.
//
// Shared-memory operands use the tensor core's no-swizzle K-major layout:
// core matrices of 8 rows x 16 bytes (8 BF16), the one holding rows 8g..8g+7
// and K elements 8c..8c+7 of an R-row operand at byte c * 16 R + 128 g; the
// descriptor's leading-dimension offset (between the two K halves of one
// K = 16 step) is then 16 R bytes and its stride offset (between 8-row groups)
// 128 bytes.  Every wait on the mbarrier is bounded; a wait that gives up sets
// the caller's error flag and the tile's outputs are not written.
#pragma once
#include <cuda_bf16.h>

#include <cstdint>

#include "prox_net.cuh"

namespace wrapd {
namespace net {
namespace tc {

constexpr int M = 128;        // samples per tile: the rows of every layer's A and D
constexpr int K1 = 16;        // layer 1's K: the 5 features padded to one K step
constexpr int N3 = 16;        // layer 3's N: the 3 outputs padded to the smallest N with M = 128
constexpr int TMEM_COLS = 128;   // layer 1 -> columns [0, 64), layer 2 -> [64, 128), layer 3 -> [0, 16)

__host__ __device__ constexpr int cm_off(int R, int row, int k) {
    return (k / 8) * (16 * R) + (row / 8) * 128 + (row % 8) * 16 + (k % 8) * 2;
}

// Weight image (bytes): the B operands W1 (64 x 16), W2 (64 x 64), W3 (16 x 64)
// in the layout above, then b1, b2, b3 (padded to 16) and the normalisation
// (mean[5], 1/std[5], output scale[3]) as FP32.
constexpr int T_W1 = 0;
constexpr int T_W2 = T_W1 + HID * K1 * 2;
constexpr int T_W3 = T_W2 + HID * HID * 2;
constexpr int T_B1 = T_W3 + N3 * HID * 2;
constexpr int T_B2 = T_B1 + HID * 4;
constexpr int T_B3 = T_B2 + HID * 4;
constexpr int T_NORM = T_B3 + N3 * 4;
constexpr int T_BYTES = T_NORM + 16 * 4;
static_assert(T_BYTES % 16 == 0, "image copied in 16-byte words");
// Per-CTA activations: the features (128 x 16), then one hidden layer
// (128 x 64) at a time.
constexpr int A_X = 0;
constexpr int A_H = A_X + M * K1 * 2;
constexpr int A_BYTES = A_H + M * HID * 2;
// Dynamic shared memory of a CTA: image, activations, mbarrier, TMEM address.
constexpr int SMEM_BYTES = T_BYTES + A_BYTES + 16;

// Instruction descriptor of kind::f16: D FP32, A and B BF16, both K-major,
// no negation, M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(n >> 3) << 17) | (uint32_t(m >> 4) << 24);
}

// Shared-memory matrix descriptor: start address, leading- and stride-dimension
// byte offsets (all in 16-byte units), descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t sdesc(const void* p, int lbo_bytes, int sbo_bytes) {
    const uint32_t a = static_cast<uint32_t>(__cvta_generic_to_shared(p));
    return uint64_t((a >> 4) & 0x3FFFu) | (uint64_t((lbo_bytes >> 4) & 0x3FFF) << 16) |
           (uint64_t((sbo_bytes >> 4) & 0x3FFF) << 32) | (uint64_t(1) << 46);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t id, int accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(d_tmem), "l"(a), "l"(b), "r"(id), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}
__device__ __forceinline__ void commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes -> visible to the tensor core's reads
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Waits for the mbarrier phase of parity `phase`, at most `limit` polls.
__device__ __forceinline__ bool wait_bar(uint32_t bar, uint32_t phase, int limit) {
    for (int i = 0; i < limit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}

// 16 FP32 columns of this thread's TMEM lane starting at `taddr`.
__device__ __forceinline__ void ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// The image from an FP32 blob, written by the threads [tid, nthreads).
__device__ __forceinline__ void build_tc_image(const float* __restrict__ blob, unsigned char* img, int tid,
                                               int nthreads) {
    for (int i = tid; i < HID * K1; i += nthreads) {
        const int o = i / K1, c = i % K1;
        *reinterpret_cast<__nv_bfloat16*>(img + T_W1 + cm_off(HID, o, c)) =
            __float2bfloat16_rn(c < IN ? blob[B_W1 + o * IN + c] : 0.0f);
    }
    for (int i = tid; i < HID * HID; i += nthreads) {
        const int o = i / HID, c = i % HID;
        *reinterpret_cast<__nv_bfloat16*>(img + T_W2 + cm_off(HID, o, c)) = __float2bfloat16_rn(blob[B_W2 + o * HID + c]);
    }
    for (int i = tid; i < N3 * HID; i += nthreads) {
        const int o = i / HID, c = i % HID;
        *reinterpret_cast<__nv_bfloat16*>(img + T_W3 + cm_off(N3, o, c)) =
            __float2bfloat16_rn(o < OUT ? blob[B_W3 + o * HID + c] : 0.0f);
    }
    float* b1 = reinterpret_cast<float*>(img + T_B1);
    float* b2 = reinterpret_cast<float*>(img + T_B2);
    float* b3 = reinterpret_cast<float*>(img + T_B3);
    float* nrm = reinterpret_cast<float*>(img + T_NORM);
    for (int i = tid; i < HID; i += nthreads) { b1[i] = blob[B_B1 + i]; b2[i] = blob[B_B2 + i]; }
    for (int i = tid; i < N3; i += nthreads) b3[i] = i < OUT ? blob[B_B3 + i] : 0.0f;
    for (int i = tid; i < 16; i += nthreads) nrm[i] = i < 13 ? blob[B_MEAN + i] : 0.0f;
}

// Per-CTA state of the forward pass: TMEM columns, the mbarrier and its
// phase.  setup() is called by all 128 threads once; teardown() too.
struct Cta {
    unsigned char* img;   // T_BYTES
    unsigned char* act;   // A_BYTES
    uint64_t* bar;
    uint32_t* tmem_slot;
    uint32_t tmem = 0;
    uint32_t phase = 0;

    __device__ __forceinline__ void setup() {
        if (threadIdx.x < 32) {   // warp 0 allocates (a whole warp, sync.aligned)
            asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                         "r"(TMEM_COLS));
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
        }
        if (threadIdx.x == 0) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)));
        fence_before_sync();
        __syncthreads();
        fence_after_sync();
        tmem = *tmem_slot;
        phase = 0;
    }
    __device__ __forceinline__ void teardown() {
        fence_before_sync();
        __syncthreads();
        fence_after_sync();
        if (threadIdx.x < 32)
            asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
    }
    // issues `nk` K steps of one layer (thread 0), commits, and waits (all threads)
    __device__ __forceinline__ bool run_layer(const unsigned char* a, int a_rows_lbo, const unsigned char* b, int b_lbo,
                                              int nk, uint32_t d_col, uint32_t id) {
        fence_async_smem();
        fence_before_sync();
        __syncthreads();
        if (threadIdx.x == 0) {
            fence_after_sync();
#pragma unroll 1
            for (int s = 0; s < nk; ++s)
                mma(tmem + d_col, sdesc(a + 2 * s * a_rows_lbo, a_rows_lbo, 128), sdesc(b + 2 * s * b_lbo, b_lbo, 128),
                    id, s > 0);
            commit(smem_u32(bar));
        }
        // one verdict for the whole CTA, so that every thread takes the same
        // path through the barriers that follow
        const bool ok = __syncthreads_and(wait_bar(smem_u32(bar), phase, 1 << 22)) != 0;
        phase ^= 1u;
        fence_after_sync();
        return ok;
    }
    // row threadIdx.x of the accumulator at column d_col: 64 columns + bias ->
    // GELU -> BF16 row of the hidden activations
    __device__ __forceinline__ void hidden(uint32_t d_col, const float* bias) {
        const uint32_t lane_base = (threadIdx.x & ~31u) << 16;
        const int t = threadIdx.x;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            float v[16];
            ld16(tmem + lane_base + d_col + 16 * q, v);
            wait_ld();
            uint32_t w[8];
#pragma unroll
            for (int i = 0; i < 8; ++i)
                w[i] = pack_bf16(gelu(v[2 * i] + bias[16 * q + 2 * i]), gelu(v[2 * i + 1] + bias[16 * q + 2 * i + 1]));
            // K elements 16q .. 16q + 15 of row t: two core-matrix rows of 16 bytes
            *reinterpret_cast<uint4*>(act + A_H + cm_off(M, t, 16 * q)) = make_uint4(w[0], w[1], w[2], w[3]);
            *reinterpret_cast<uint4*>(act + A_H + cm_off(M, t, 16 * q + 8)) = make_uint4(w[4], w[5], w[6], w[7]);
        }
    }

    // The forward pass of the tile: f = raw features of this thread's sample
    // (any values when !valid); y = normalised outputs.  Returns false if a
    // wait gave up.
    __device__ __forceinline__ bool forward(const float f[IN], bool valid, float y[OUT]) {
        const float* nrm = reinterpret_cast<const float*>(img + T_NORM);
        const int t = threadIdx.x;
        uint32_t x[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const int k0 = 2 * c, k1 = 2 * c + 1;
            const float v0 = (valid && k0 < IN) ? (f[k0] - nrm[B_MEAN + k0]) * nrm[B_ISTD + k0] : 0.0f;
            const float v1 = (valid && k1 < IN) ? (f[k1] - nrm[B_MEAN + k1]) * nrm[B_ISTD + k1] : 0.0f;
            x[c] = pack_bf16(v0, v1);
        }
        *reinterpret_cast<uint4*>(act + A_X + cm_off(M, t, 0)) = make_uint4(x[0], x[1], x[2], x[3]);
        *reinterpret_cast<uint4*>(act + A_X + cm_off(M, t, 8)) = make_uint4(x[4], x[5], x[6], x[7]);
        bool ok = run_layer(act + A_X, 16 * M, img + T_W1, 16 * HID, 1, 0, idesc_bf16(M, HID));
        if (ok) hidden(0, reinterpret_cast<const float*>(img + T_B1));
        ok = ok && run_layer(act + A_H, 16 * M, img + T_W2, 16 * HID, HID / 16, 64, idesc_bf16(M, HID));
        if (ok) hidden(64, reinterpret_cast<const float*>(img + T_B2));
        ok = ok && run_layer(act + A_H, 16 * M, img + T_W3, 16 * N3, HID / 16, 0, idesc_bf16(M, N3));
        if (ok) {
            float v[16];
            ld16(tmem + ((threadIdx.x & ~31u) << 16), v);
            wait_ld();
            const float* b3 = reinterpret_cast<const float*>(img + T_B3);
#pragma unroll
            for (int i = 0; i < OUT; ++i) y[i] = v[i] + b3[i];
        }
        // every lane's reads of this tile are done before the next tile's MMAs
        fence_before_sync();
        __syncthreads();
        return ok;
    }
};

}  // namespace tc
}  // namespace net
}  // namespace wrapd
