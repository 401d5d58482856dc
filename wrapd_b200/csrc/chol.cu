// GPU multifrontal Cholesky and 3-RHS solve; see chol.cuh.
//
// Factorization, per level of the assembly tree (leaves first):
//   extend-add   children's update matrices into the fronts (one launch per
//                child slot, so two children never write one entry at once);
//   then per panel of NB = 32 columns (right-looking partial Cholesky):
//   panel        every CTA factors the NB x NB diagonal block in registers
//                (one warp) and forms its inverse Li (also stored as a diagonal
//                block of Y), then applies it to one tile: the panel rows
//                below the block, P <- P Li^T, or the inverse row block
//                Y[p, 0:p0] <- Li Y[p, 0:p0] (FP64 DMMA tiles);
//   update       blocked right-looking: inside the current OB-column block,
//                F[j0:, j0:be] -= P P^T and Y[j0:be, 0:j0] -= P Y[p, 0:j0];
//                after a block's last panel, the deferred trailing update
//                F[be:, be:] -= B B^T and Y[be:, 0:be] -= B Y[block, 0:be] with
//                K = OB (FP64 DMMA tiles, K-looped), so the large trailing
//                matrix is read and written once per OB columns, not per panel;
//   then         W = L_rs Y for the level's fronts (FP64 DMMA, K-looped).
// A is assembled once per factorization straight into the zeroed F pool.
//
// Every tile product is mma.sync.m8n8k4 f64 (the FP64 tensor-core path of
// sm_100a; tcgen05 has no f64 kind).
#include "chol.cuh"

#include <algorithm>
#include <numeric>

namespace wrapd {

namespace {

constexpr int NB = 32;        // panel width
constexpr int OB = 256;       // outer block: trailing updates beyond it are deferred to one K = OB update
                              // (128: 1.5 % slower on the 3.9M bar; 512: slower on both bars)
constexpr int TL = 64;        // output tile of the DMMA kernels
constexpr int SLD = NB + 4;   // smem row pitch (doubles) for [row][k] operand tiles
constexpr int GEMM_THREADS = 128;
constexpr int kFusedPanelCtas = 4 * 148;   // panel steps up to one wave (4 CTAs per SM) run fused
constexpr int COLS_PER_CTA = 8;    // solve / extend-add column groups (one warp each)

__device__ __forceinline__ int find_item(const int* prefix, int n, int b) {
    int lo = 0, hi = n;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (prefix[mid] <= b) lo = mid; else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// S[i][t] = base[i*rs + t*cs] for i < rows, t < K; zero elsewhere (TL x K4).
__device__ __forceinline__ void load_tile(double* S, const double* __restrict__ base, int64_t rs, int64_t cs,
                                          int rows, int K, int K4) {
    const int total = TL * K4;
    if (rs == 1) {
        for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
            const int i = idx % TL, t = idx / TL;
            S[i * SLD + t] = (i < rows && t < K) ? base[i + t * cs] : 0.0;
        }
    } else {
        for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
            const int t = idx % K4, i = idx / K4;
            S[i * SLD + t] = (i < rows && t < K) ? base[i * rs + t * cs] : 0.0;
        }
    }
}

// acc += As * Bs^T over K4 (multiple of 4); 4 warps in a 2x2 grid of 32x32.
__device__ __forceinline__ void tile_mma(const double* As, const double* Bs, int K4, double (&acc)[4][4][2]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wm = warp & 1, wn = warp >> 1;
    const int r = lane >> 2, c = lane & 3;
    for (int kk = 0; kk < K4; kk += 4) {
        double a[4], b[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = As[(wm * 32 + i * 8 + r) * SLD + kk + c];
#pragma unroll
        for (int j = 0; j < 4; ++j) b[j] = Bs[(wn * 32 + j * 8 + r) * SLD + kk + c];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
    }
}

// C[row*crs + col*ccs] = acc for row < M, col < N.
__device__ __forceinline__ void tile_store(double* C, int64_t crs, int64_t ccs, int M, int N,
                                           const double (&acc)[4][4][2]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wm = warp & 1, wn = warp >> 1;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int row = wm * 32 + i * 8 + (lane >> 2);
                const int col = wn * 32 + j * 8 + 2 * (lane & 3) + h;
                if (row < M && col < N) C[row * crs + col * ccs] = acc[i][j][h];
            }
}

// ---- pipelined GEMM core ------------------------------------------------------
// Operand tiles are staged by cp.async in one of two layouts, chosen by which
// index is contiguous in global memory so that both the staging writes and the
// DMMA fragment reads hit every shared-memory bank evenly:
//   t-major S[t * TP + i] for sources with i contiguous (columns of F),
//   i-major S[i * SLD + t] for sources with t contiguous (row blocks of Y).
// Two stages: chunk c + 1 is in flight while chunk c is multiplied.
constexpr int TP = TL + 8;            // t-major pitch: 8 mod 16 doubles
#ifndef WRAPD_GEMM_KC
#define WRAPD_GEMM_KC 16
#endif
constexpr int KC = WRAPD_GEMM_KC;     // K columns per staged chunk of the trailing-update GEMMs
constexpr int GSLD = KC + 4;          // i-major pitch (KC + 4 = 4 mod 8 doubles: conflict-free fragment reads)
constexpr int TILE_D = (KC * TP > TL * GSLD) ? KC * TP : TL * GSLD;   // doubles per staged operand tile
static_assert(KC % 4 == 0 && KC <= NB, "chunks of whole DMMA k-steps");
#ifndef WRAPD_GEMM_STAGES
#define WRAPD_GEMM_STAGES 2
#endif
constexpr int GEMM_STAGES = WRAPD_GEMM_STAGES;   // cp.async pipeline depth of the trailing-update GEMMs
constexpr int GEMM_SMEM = GEMM_STAGES * 2 * TILE_D * (int)sizeof(double);   // stages x (A, B)

__device__ __forceinline__ void cp_async8(double* s, const double* g, bool valid) {
    const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(s));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(g), "r"(valid ? 8 : 0));
}
// 16-byte copy of which the first src_bytes (16, 8 or 0) come from global
// memory and the rest is zero-filled; both addresses 16-byte aligned.
__device__ __forceinline__ void cp_async16(double* s, const double* g, int src_bytes) {
    const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(s));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(g), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// Element (i, t), i < rows, t < K, of a source with (TMAJOR) i contiguous:
// base[i + t * ld], or t contiguous: base[i * ld + t]; zeros up to K4.
// Where the source is 16-byte aligned and ld even (every front's F and Y
// blocks have an even leading dimension; a job's row offset may still be odd),
// element pairs move as one 16-byte copy: along i in the t-major layout, along
// t in the i-major one.
template <bool TMAJOR>
__device__ __forceinline__ void stage_tile(double* S, const double* base, int64_t ld, int rows, int K, int K4) {
    if ((reinterpret_cast<uintptr_t>(base) & 15) == 0 && (ld & 1) == 0) {
        if constexpr (TMAJOR) {
            const int total = (TL / 2) * K4;
            for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
                const int i = 2 * (idx % (TL / 2)), t = idx / (TL / 2);
                const int nbytes = (t < K && i < rows) ? (i + 1 < rows ? 16 : 8) : 0;
                cp_async16(S + t * TP + i, nbytes ? base + i + (int64_t)t * ld : base, nbytes);
            }
        } else {
            const int total = TL * (K4 / 2);
            for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
                const int t = 2 * (idx % (K4 / 2)), i = idx / (K4 / 2);
                const int nbytes = (i < rows && t < K) ? (t + 1 < K ? 16 : 8) : 0;
                cp_async16(S + i * GSLD + t, nbytes ? base + (int64_t)i * ld + t : base, nbytes);
            }
        }
        return;
    }
    const int total = TL * K4;
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
        if constexpr (TMAJOR) {
            const int i = idx % TL, t = idx / TL;
            const bool v = i < rows && t < K;
            cp_async8(S + t * TP + i, v ? base + i + (int64_t)t * ld : base, v);
        } else {
            const int t = idx % K4, i = idx / K4;
            const bool v = i < rows && t < K;
            cp_async8(S + i * GSLD + t, v ? base + (int64_t)i * ld + t : base, v);
        }
    }
}

template <bool AT, bool BT>
__device__ __forceinline__ void tile_mma2(const double* As, const double* Bs, int K4, double (&acc)[4][4][2]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wm = warp & 1, wn = warp >> 1;
    const int r = lane >> 2, c = lane & 3;
    for (int kk = 0; kk < K4; kk += 4) {
        double a[4], b[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int row = wm * 32 + i * 8 + r;
            a[i] = AT ? As[(kk + c) * TP + row] : As[row * GSLD + kk + c];
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int col = wn * 32 + j * 8 + r;
            b[j] = BT ? Bs[(kk + c) * TP + col] : Bs[col * GSLD + kk + c];
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
    }
}

// acc += A B'^T over t in [0, K): A(i, t) = A0[i + t * lda] (i < M), B'(j, t) =
// B0[j + t * ldb] when BT, else B0[j * ldb + t] (j < N).
template <bool BT>
__device__ __forceinline__ void gemm_pipelined(const double* A0, int64_t lda, int M, const double* B0, int64_t ldb,
                                               int N, int K, double* smem, double (&acc)[4][4][2]) {
    const int nch = (K + KC - 1) / KC;
    auto issue = [&](int c) {
        if (c < nch) {
            const int k0 = c * KC, Kc = min(KC, K - k0), K4 = (Kc + 3) & ~3;
            double* st = smem + (c % GEMM_STAGES) * 2 * TILE_D;
            stage_tile<true>(st, A0 + (int64_t)k0 * lda, lda, M, Kc, K4);
            stage_tile<BT>(st + TILE_D, BT ? B0 + (int64_t)k0 * ldb : B0 + k0, ldb, N, Kc, K4);
        }
        cp_async_commit();   // an empty group past the last chunk keeps the wait count uniform
    };
#pragma unroll
    for (int c = 0; c < GEMM_STAGES - 1; ++c) issue(c);
    for (int c = 0; c < nch; ++c) {
        issue(c + GEMM_STAGES - 1);
        cp_async_wait<GEMM_STAGES - 1>();
        __syncthreads();
        const int Kc = min(KC, K - c * KC), K4 = (Kc + 3) & ~3;
        const double* st = smem + (c % GEMM_STAGES) * 2 * TILE_D;
        tile_mma2<true, BT>(st, st + TILE_D, K4, acc);
        __syncthreads();
    }
}

// ---- assembly ----------------------------------------------------------------
__global__ void k_assemble_A(double* __restrict__ F, const int64_t* __restrict__ pos, const int* __restrict__ ptr,
                             const int* __restrict__ con, int nA, const double* __restrict__ w2,
                             const double* __restrict__ Di, int ne) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nA) return;
    double v = 0.0;
    for (int q = ptr[t]; q < ptr[t + 1]; ++q) {
        const int c = con[q];
        const int e = c >> 4, a = (c >> 2) & 3, b = c & 3;
        double d = 0.0;
#pragma unroll
        for (int r = 0; r < 3; ++r) d += Di[(int64_t)(r + 3 * a) * ne + e] * Di[(int64_t)(r + 3 * b) * ne + e];
        v += w2[e] * d;
    }
    F[pos[t]] = v;
}

__global__ void k_y_identity(double* __restrict__ Y, const FrontDesc* __restrict__ desc, int nfronts) {
    const int f = blockIdx.x;
    if (f >= nfronts) return;
    const FrontDesc d = desc[f];
    for (int i = threadIdx.x; i < d.k; i += blockDim.x) Y[d.y_off + i + (int64_t)i * d.ldy] = 1.0;
}

// children slot `slot` of each front in the list: F_s[rel[i], rel[j]] += U_c[i, j], i >= j
__global__ void k_extend_add(double* __restrict__ F, const FrontDesc* __restrict__ desc, const int* __restrict__ rel,
                             WorkList wl, int slot) {
    const int item = find_item(wl.d_prefix, wl.n, blockIdx.x);
    const int s = wl.d_fronts[item];
    const FrontDesc ds = desc[s];
    const int c = slot == 0 ? ds.child0 : ds.child1;
    const FrontDesc dc = desc[c];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int j = (blockIdx.x - wl.d_prefix[item]) * COLS_PER_CTA + warp;
    if (j >= dc.r) return;
    const int* rc = rel + dc.rel_off;
    const double* Uc = F + dc.f_off + dc.k + (int64_t)(dc.k + j) * dc.ld;
    double* Fs = F + ds.f_off + (int64_t)rc[j] * ds.ld;
    // Uc and Fs live in one pool, so the loads are batched by hand ahead of the
    // stores (rel maps a column's rows to distinct parent rows)
    constexpr int U = 4;
    for (int i0 = j + lane; i0 < dc.r; i0 += 32 * U) {
        double u[U], f[U];
        int ri[U];
#pragma unroll
        for (int q = 0; q < U; ++q) {
            const int i = i0 + 32 * q;
            ri[q] = i < dc.r ? rc[i] : 0;
            u[q] = i < dc.r ? Uc[i] : 0.0;
        }
#pragma unroll
        for (int q = 0; q < U; ++q) f[q] = (i0 + 32 * q < dc.r) ? Fs[ri[q]] : 0.0;
#pragma unroll
        for (int q = 0; q < U; ++q)
            if (i0 + 32 * q < dc.r) Fs[ri[q]] = f[q] + u[q];
    }
}

// ---- panel factorization -------------------------------------------------------
// Cholesky of the nb x nb (nb <= NB = 32) diagonal block at Fd (column-major,
// lower part read) and its inverse, by a CTA of 128 threads in shared memory.
// Right-looking: at pivot j every thread updates a fixed slice of 8 entries
// of row i = tid % 32 (columns tid / 32 + 4m), with all its operands loaded
// before the first store, so one barrier per pivot is the only serial step.
// L(i, j) = A'(i, j) rsqrt(d) goes to Lsm (pitch lp), rsqrt(d) to D.  The
// inverse is right-looking by rows with no barrier: lane c of warp 0 owns
// column c of inv(L), its partial sums P(r, c) in registers; row s of the
// column is (delta(s, c) - P(s, c)) / L(s, s), and the rows below add L(r, s)
// times it (the same fma sequence per entry as a row-by-row sweep).  Row s of
// inv(L) is written to X (pitch xp), columns < nb.  A non-positive (or NaN)
// pivot sets *bad and continues with a unit pivot.
constexpr int LSP = NB + 1;
static_assert(GEMM_THREADS == 128 && NB == 32, "cta_chol_inv maps 128 threads onto 32 rows x 4 column slices");
__device__ __forceinline__ void cta_chol_inv(const double* __restrict__ Fd, int64_t ld, int nb, double* S,
                                             double* Lsm, int lp, double* D, double* X, int xp, bool* bad) {
    const int tid = threadIdx.x;
    for (int idx = tid; idx < NB * NB; idx += GEMM_THREADS) {
        const int i = idx & 31, c = idx >> 5;
        S[i * LSP + c] = (i < nb && c <= i) ? Fd[i + (int64_t)c * ld] : 0.0;
    }
    __syncthreads();
    const int i = tid & 31, q = tid >> 5;
    bool b = false;
    for (int j = 0; j < nb; ++j) {
        double piv = S[j * LSP + j];
        const double sij = S[i * LSP + j];
        double cj[8], ic[8];
#pragma unroll
        for (int m = 0; m < 8; ++m) {
            cj[m] = S[(q + 4 * m) * LSP + j];
            ic[m] = S[i * LSP + q + 4 * m];
        }
        if (!(piv > 0.0)) { b = true; piv = 1.0; }
        const double rs = rsqrt(piv);
        if (q == 0 && i >= j && i < nb) Lsm[i * lp + j] = i == j ? piv * rs : sij * rs;
        if (tid == 0) D[j] = rs;
        const double t = sij * (rs * rs);
#pragma unroll
        for (int m = 0; m < 8; ++m) {
            const int c = q + 4 * m;
            if (c > j && c <= i && i < nb) S[i * LSP + c] = fma(-t, cj[m], ic[m]);
        }
        __syncthreads();
    }
    if (tid < 32) {
        const int c = tid;
        double P[NB];
#pragma unroll
        for (int r = 0; r < NB; ++r) P[r] = 0.0;
#pragma unroll
        for (int s = 0; s < NB; ++s) {
            if (s < nb) {
                const double f = (c <= s) ? ((c == s ? 1.0 : 0.0) - P[s]) * D[s] : 0.0;
                if (c < nb) X[s * xp + c] = f;
#pragma unroll
                for (int r = s + 1; r < NB; ++r)
                    if (r < nb) P[r] = fma(Lsm[r * lp + s], f, P[r]);
            }
        }
    }
    __syncthreads();
    *bad = b;
}

// Diagonal step alone, for panel steps with many CTAs (where redoing the
// block in every CTA would cost more than a launch): one CTA per front
// factors the block and writes Li as the diagonal block of Y.
__global__ void __launch_bounds__(GEMM_THREADS) k_diag(const double* __restrict__ F, double* __restrict__ Y,
                                                       const FrontDesc* __restrict__ desc, WorkList wl, int p,
                                                       int* __restrict__ status) {
    __shared__ double S[NB * LSP];
    __shared__ double Lsm[NB * LSP];
    __shared__ double X[NB * LSP];
    __shared__ double D[NB];
    const FrontDesc d = desc[wl.d_fronts[blockIdx.x]];
    const int p0 = p * NB, nb = min(NB, d.k - p0);
    if (nb <= 0) return;
    bool bad = false;
    cta_chol_inv(F + d.f_off + p0 + (int64_t)p0 * d.ld, d.ld, nb, S, Lsm, LSP, D, X, LSP, &bad);
    if (bad && threadIdx.x == 0) atomicExch(status, WRAPD_E_NOT_SPD);
    double* Yp = Y + d.y_off + p0;   // row block p of Y (column-major, ld = ldy)
    for (int idx = threadIdx.x; idx < NB * NB; idx += GEMM_THREADS) {
        const int i = idx & 31, c = idx >> 5;
        if (i < nb && c < nb) Yp[i + (int64_t)(p0 + c) * d.ldy] = c <= i ? X[i * LSP + c] : 0.0;
    }
}

// The tiles of a panel step after k_diag: nP panel-row tiles (P <- P Li^T),
// then the inverse row-block tiles Y[p, c0:c0+64] <- Li Y[p, c0:c0+64], with
// Li read back from Y's diagonal block.
__global__ void __launch_bounds__(GEMM_THREADS) k_trsm(double* __restrict__ F, double* __restrict__ Y,
                                                       const FrontDesc* __restrict__ desc, WorkList wl,
                                                       const int* __restrict__ nP_of_item, int p) {
    __shared__ double As[TL * SLD];
    __shared__ double Bs[TL * SLD];
    const int item = find_item(wl.d_prefix, wl.n, blockIdx.x);
    const FrontDesc d = desc[wl.d_fronts[item]];
    const int tile = blockIdx.x - wl.d_prefix[item];
    const int nP = nP_of_item[item];
    const int p0 = p * NB, nb = min(NB, d.k - p0), j0 = p0 + nb;
    if (nb <= 0) return;
    const int K4 = (nb + 3) & ~3;
    const double* Li = Y + d.y_off + p0 + (int64_t)p0 * d.ldy;   // Li(i, t) at Li[i + t ldy]
    double acc[4][4][2] = {};
    if (tile < nP) {
        const int m = min(d.ld - j0 - tile * TL, TL);
        double* A = F + d.f_off + j0 + tile * TL + (int64_t)p0 * d.ld;
        load_tile(As, A, 1, d.ld, m, nb, K4);
        load_tile(Bs, Li, 1, d.ldy, nb, nb, K4);
        __syncthreads();
        tile_mma(As, Bs, K4, acc);
        tile_store(A, 1, d.ld, m, nb, acc);
    } else {
        const int c0 = (tile - nP) * TL;
        if (c0 >= p0) return;
        double* Yr = Y + d.y_off + p0 + (int64_t)c0 * d.ldy;   // Y[p0 + t, c0 + j] at Yr[t + j ldy]
        load_tile(As, Li, 1, d.ldy, nb, nb, K4);
        load_tile(Bs, Yr, d.ldy, 1, min(p0 - c0, TL), nb, K4);
        __syncthreads();
        tile_mma(As, Bs, K4, acc);
        tile_store(Yr, 1, d.ldy, nb, min(p0 - c0, TL), acc);
    }
}

// Panel steps with few CTAs (the upper levels: a few large fronts, where the
// step is latency-bound) run as one launch: every CTA first factors the
// front's NB x NB diagonal block itself (warp 0, registers) and keeps its
// inverse Li in shared memory, so no separate diagonal launch precedes it.  Items per front: nP
// panel-row tiles (P <- P Li^T below the diagonal block), then the inverse
// row-block tiles Y[p, c0:c0+64] <- Li Y[p, c0:c0+64], c0 < p0; a front with
// neither has one item that only factors.  The front's first item writes Li
// as the diagonal block of Y.  F's diagonal block is read, never written: the
// solve and the later steps use only Y, W and the panels below it.
__global__ void __launch_bounds__(GEMM_THREADS) k_panel(double* __restrict__ F, double* __restrict__ Y,
                                                        const FrontDesc* __restrict__ desc, WorkList wl,
                                                        const int* __restrict__ nP_of_item, int p,
                                                        int* __restrict__ status) {
    __shared__ __align__(16) double As[TL * SLD];
    __shared__ __align__(16) double Bs[TL * SLD];
    __shared__ double S[NB * LSP];
    __shared__ double D[NB];
    const int item = find_item(wl.d_prefix, wl.n, blockIdx.x);
    const FrontDesc d = desc[wl.d_fronts[item]];
    const int tile = blockIdx.x - wl.d_prefix[item];
    const int nP = nP_of_item[item];
    const int p0 = p * NB, nb = min(NB, d.k - p0), j0 = p0 + nb;
    if (nb <= 0) return;
    const int K4 = (nb + 3) & ~3;
    const bool ptile = tile < nP;
    const int c0 = (tile - nP) * TL;
    const bool ytile = !ptile && c0 < p0;
    // The other operand is staged asynchronously while the diagonal block is
    // factored: the panel rows (A(i, t) = P(i, t)) or the Y row block (B'(j, t)
    // = Y(p0 + t, c0 + j)).
    const int tid = threadIdx.x;
    if (ptile) {
        const int m = min(d.ld - j0 - tile * TL, TL);
        const double* A = F + d.f_off + j0 + tile * TL + (int64_t)p0 * d.ld;
        for (int idx = tid; idx < TL * K4; idx += GEMM_THREADS) {
            const int i = idx % TL, t = idx / TL;
            const bool v = i < m && t < nb;
            cp_async8(As + i * SLD + t, v ? A + i + (int64_t)t * d.ld : A, v);
        }
    } else if (ytile) {
        const int n = min(p0 - c0, TL);
        const double* Yr = Y + d.y_off + p0 + (int64_t)c0 * d.ldy;
        for (int idx = tid; idx < TL * K4; idx += GEMM_THREADS) {
            const int t = idx % K4, j = idx / K4;
            const bool v = j < n && t < nb;
            cp_async8(Bs + j * SLD + t, v ? Yr + t + (int64_t)j * d.ldy : Yr, v);
        }
    }
    cp_async_commit();
    // Li lands in the operand slot of the product: B for panel tiles (B'(j, t) =
    // Li(j, t)), A for inverse row-block tiles (A(i, t) = Li(i, t)); rows 32..63
    // of that slot hold L meanwhile and are cleared afterwards.
    double* Ls = ptile ? Bs : As;
    for (int idx = tid; idx < NB * SLD; idx += GEMM_THREADS) Ls[idx] = 0.0;
    bool bad = false;
    cta_chol_inv(F + d.f_off + p0 + (int64_t)p0 * d.ld, d.ld, nb, S, Ls + NB * SLD, SLD, D, Ls, SLD, &bad);
    if (tile == 0) {
        if (bad && tid == 0) atomicExch(status, WRAPD_E_NOT_SPD);
        double* Yp = Y + d.y_off + p0;   // row block p of Y (column-major, ld = ldy)
        for (int idx = tid; idx < NB * NB; idx += GEMM_THREADS) {
            const int i = idx & 31, c = idx >> 5;
            if (i < nb && c < nb) Yp[i + (int64_t)(p0 + c) * d.ldy] = Ls[i * SLD + c];
        }
    }
    __syncthreads();
    for (int idx = tid; idx < NB * SLD; idx += GEMM_THREADS) Ls[NB * SLD + idx] = 0.0;
    cp_async_wait<0>();
    __syncthreads();
    if (!ptile && !ytile) return;
    double acc[4][4][2] = {};
    tile_mma(As, Bs, K4, acc);
    if (ptile) {
        const int m = min(d.ld - j0 - tile * TL, TL);
        tile_store(F + d.f_off + j0 + tile * TL + (int64_t)p0 * d.ld, 1, d.ld, m, nb, acc);
    } else {
        tile_store(Y + d.y_off + p0 + (int64_t)c0 * d.ldy, 1, d.ldy, nb, min(p0 - c0, TL), acc);
    }
}

#ifndef WRAPD_EPI_BATCH
#define WRAPD_EPI_BATCH 8
#endif
constexpr int EPI_BATCH = WRAPD_EPI_BATCH;   // columns per thread whose reads the staged epilogue issues together
constexpr int EPI_P = TL + 2;   // pitch of the staged output tile: lanes' (row, 2-column) fragments hit distinct banks
static_assert(TL * EPI_P <= 2 * GEMM_STAGES * TILE_D, "the staged output tile reuses the operand stages");
static_assert(TL == 2 * 32 && GEMM_THREADS == 2 * TL, "the staged epilogue maps two threads per row");

// C[row + col*ld] -= acc for row < M, col < N and row + diag >= col, through
// shared memory: the fragments go to a column-major tile, then each warp
// updates 32 consecutive rows of a column (coalesced) with EPI_BATCH columns'
// reads in flight before their writes.  Direct read-modify-writes from the
// fragments would be serialised, since a store through C may alias the next
// read as far as the compiler can tell.  `smem` (the operand stages) must have
// no reads pending from other threads; the call's first barrier ensures that.
__device__ __forceinline__ void tile_sub_staged(double* __restrict__ C, int64_t ld, int M, int N, int diag,
                                                const double (&acc)[4][4][2], double* smem) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wm = warp & 1, wn = warp >> 1;
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int row = wm * 32 + i * 8 + (lane >> 2);
                const int col = wn * 32 + j * 8 + 2 * (lane & 3) + h;
                smem[col * EPI_P + row] = acc[i][j][h];
            }
    __syncthreads();
    const int row = threadIdx.x & (TL - 1), cg = threadIdx.x >> 6;
    if (row >= M) return;
    // columns cg, cg + 2, ... below N and with row + diag >= col
    const int cend = min(N, row + diag + 1);
#pragma unroll 1
    for (int c0 = cg; c0 < cend; c0 += 2 * EPI_BATCH) {
        double v[EPI_BATCH];
#pragma unroll
        for (int q = 0; q < EPI_BATCH; ++q) {
            const int col = c0 + 2 * q;
            v[q] = col < cend ? C[row + (int64_t)col * ld] : 0.0;
        }
#pragma unroll
        for (int q = 0; q < EPI_BATCH; ++q) {
            const int col = c0 + 2 * q;
            if (col < cend) C[row + (int64_t)col * ld] = v[q] - smem[col * EPI_P + row];
        }
    }
}

// Tile t of a job: kind 0 enumerates lower tiles (ti >= tj) column by column,
// kind 1 the full rectangle.
__device__ __forceinline__ void job_tile(const GemmJob& jb, int t, int& ti, int& tj) {
    const int Tr = (jb.r1 - jb.r0 + TL - 1) / TL, Tc = (jb.c1 - jb.c0 + TL - 1) / TL;
    if (jb.kind == 1) { ti = t / Tc; tj = t % Tc; return; }
    for (tj = 0; tj < Tc; ++tj) {
        const int cnt = Tr - tj;
        if (t < cnt) { ti = tj + t; return; }
        t -= cnt;
    }
    ti = Tr;   // not reached for valid t
}

#ifndef WRAPD_GEMM_MINB
#define WRAPD_GEMM_MINB 4
#endif
__global__ void __launch_bounds__(GEMM_THREADS, WRAPD_GEMM_MINB) k_update(double* __restrict__ F, double* __restrict__ Y,
                                                         const FrontDesc* __restrict__ desc, JobList jl) {
    extern __shared__ __align__(16) double gemm_smem[];
    const int item = find_item(jl.d_prefix, jl.n, blockIdx.x);
    const GemmJob jb = jl.d_jobs[item];
    const FrontDesc d = desc[jb.front];
    int ti, tj;
    job_tile(jb, blockIdx.x - jl.d_prefix[item], ti, tj);
    const int r0 = jb.r0 + ti * TL, c0 = jb.c0 + tj * TL;
    const int M = min(TL, jb.r1 - r0), N = min(TL, jb.c1 - c0);
    double acc[4][4][2] = {};
    const double* A0 = F + d.f_off + r0 + (int64_t)jb.k0 * d.ld;
    if (jb.kind == 0)
        gemm_pipelined<true>(A0, d.ld, M, F + d.f_off + c0 + (int64_t)jb.k0 * d.ld, d.ld, N, jb.k1 - jb.k0,
                             gemm_smem, acc);
    else   // B'(j, t) = Y(k0 + t, c0 + j)
        gemm_pipelined<false>(A0, d.ld, M, Y + d.y_off + jb.k0 + (int64_t)c0 * d.ldy, d.ldy, N, jb.k1 - jb.k0,
                              gemm_smem, acc);
    // on tiles of kind 0 crossing the diagonal keep only row >= column (global indices)
    if (jb.kind == 0)
        tile_sub_staged(F + d.f_off + r0 + (int64_t)c0 * d.ld, d.ld, M, N, r0 - c0, acc, gemm_smem);
    else
        tile_sub_staged(Y + d.y_off + r0 + (int64_t)c0 * d.ldy, d.ldy, M, N, TL, acc, gemm_smem);
}

// W = L_rs Y (r x k) with Y lower triangular: tile (ti, tj) of 64 x 64 sums
// t over [64 tj, k) in chunks of NB.
__global__ void __launch_bounds__(GEMM_THREADS) k_wgemm(const double* __restrict__ F, const double* __restrict__ Y,
                                                        double* __restrict__ W, const FrontDesc* __restrict__ desc,
                                                        WorkList wl) {
    extern __shared__ __align__(16) double gemm_smem[];
    const int item = find_item(wl.d_prefix, wl.n, blockIdx.x);
    const FrontDesc d = desc[wl.d_fronts[item]];
    const int t = blockIdx.x - wl.d_prefix[item];
    // column tiles slowest: the tiles with the longest K (c0 = 0) come first in
    // the launch, the short ones fill in behind them
    const int nr = (d.r + TL - 1) / TL;
    const int r0 = (t % nr) * TL, c0 = (t / nr) * TL;
    const int M = min(TL, d.r - r0), N = min(TL, d.k - c0);
    const double* A = F + d.f_off + d.k + r0;   // L_rs(i, t) at A[i + t ld]
    double acc[4][4][2] = {};
    // t over [c0, k): Y(k0 + t, c0 + j) vanishes above the diagonal
    gemm_pipelined<false>(A + (int64_t)c0 * d.ld, d.ld, M, Y + d.y_off + c0 + (int64_t)c0 * d.ldy, d.ldy, N, d.k - c0,
                          gemm_smem, acc);
    tile_store(W + d.y_off + d.k + r0 + (int64_t)c0 * d.ldy, 1, d.ldy, M, N, acc);
}

// ---- solve -----------------------------------------------------------------------
// Per level, one launch per direction.  Forward: a CTA owns a band of 64 rows of
// the front's M = [Y; W] ((k + r) x k, leading dimension ldy) and a chunk of its
// columns (Y rows only up to the diagonal): rows < k give z_s = Y t_s, rows >= k
// give u_s = v_s - W t_s.  Backward: a CTA owns a band of 64 columns and a chunk
// of the rows below the diagonal and of the W rows: y_s = Y^T z_s - W^T y_rows.  The right-hand side is
// read from B (a copy of the input), z from Zb, and y written to x, so no CTA
// reads what another CTA of the same launch writes.

// t_s(i) for i < k, or v_s(i) for i >= k: own b entry plus the children's update
// entries landing on front row i, in child order (inv: offsets in U, or -1).
__device__ __forceinline__ void front_rhs(const double* __restrict__ B, const double* __restrict__ U,
                                          const int64_t* __restrict__ inv, const FrontDesc& d, int i,
                                          double& v0, double& v1, double& v2) {
    if (i < d.k) {
        const double* b = B + 3 * ((int64_t)d.first + i);
        v0 = b[0]; v1 = b[1]; v2 = b[2];
    } else {
        v0 = v1 = v2 = 0.0;
    }
    const int64_t* iv = inv + d.inv_off + 2 * (int64_t)i;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int64_t o = iv[q];
        if (o >= 0) { v0 += __ldcg(U + o); v1 += __ldcg(U + o + 1); v2 += __ldcg(U + o + 2); }
    }
}

// Each CTA takes one item: a 64-wide band (rows forward, columns backward) times
// a chunk of the other dimension (at most SCH).  The CTAs of one band write
// partial sums; the last one to arrive adds them in chunk order (deterministic)
// and writes the band's result, then resets the band counter.
constexpr int SCH = 256;
constexpr int FWD_WARPS = 4;          // warps of a forward solve CTA (eight CTAs per SM)
constexpr int SCH_MIN = 64;
constexpr int kSolveCtas = 2 * 148;   // two 256-thread CTAs per SM of a B200

__device__ __forceinline__ bool band_arrive(unsigned* counter, int nchunk) {
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned old = atomicAdd(counter, 1u);
        last = old == (unsigned)nchunk - 1;
        if (last) *counter = 0u;
    }
    __syncthreads();
    if (last) __threadfence();
    return last;
}

// Forward: lane l of warp w holds rows b0 + 2l and b0 + 2l + 1 of the band (one
// 16-byte load per column: the block's leading dimension and the band start are
// even) and takes columns lo + w, lo + w + FWD_WARPS, ...; the warps' sums
// are added in warp order.  Four-warp CTAs, eight per SM: more items in
// flight for the latency-bound lower levels (eight-warp CTAs, four per SM,
// measured 2 % slower per solve; two-warp CTAs 13 % slower).
// One forward item (q: its index in the item list, which places its partial
// sums in P).  Returns true, in every thread, in the CTA that wrote the band's
// result, after all its writes are visible device-wide.
// The first eight columns of each warp of a forward item (warp w takes columns
// w, w + FWD_WARPS, ...): [Y; W] does not change during a solve, so they are
// loaded before the item's dependency wait and its right-hand-side gather.
constexpr int FWD_PRE = 8;
__device__ __forceinline__ void fwd_pre(const double* __restrict__ YW, const FrontDesc& d, const SolveItem& it,
                                        double2 (&pre)[FWD_PRE]) {
    const int R = d.k + d.r;
    const int nc = it.hi - it.lo;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i0 = it.b0 + 2 * lane;
    const double* M = YW + d.y_off + i0 + (int64_t)it.lo * d.ldy;
#pragma unroll
    for (int u = 0; u < FWD_PRE; ++u) {
        const int j = warp + FWD_WARPS * u;
        pre[u] = (i0 < R && j < nc) ? __ldg(reinterpret_cast<const double2*>(M + (int64_t)j * d.ldy))
                                    : make_double2(0.0, 0.0);
    }
}

__device__ __forceinline__ bool fwd_item(const double* __restrict__ B, double* __restrict__ Zb,
                                         double* __restrict__ U, const int64_t* __restrict__ inv,
                                         const double* __restrict__ YW, const FrontDesc& d, const SolveItem& it, int q,
                                         double* __restrict__ P, unsigned* __restrict__ counters,
                                         const double2 (&pre)[FWD_PRE]) {
    __shared__ double tv[SCH * 3];
    __shared__ double part[FWD_WARPS][TL][3];
    const int R = d.k + d.r;
    const int nc = it.hi - it.lo;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i0 = it.b0 + 2 * lane;
    const double* M = YW + d.y_off + i0 + (int64_t)it.lo * d.ldy;
    constexpr int PRE = FWD_PRE;
    for (int j = threadIdx.x; j < nc; j += blockDim.x) {
        double v0, v1, v2;
        front_rhs(B, U, inv, d, it.lo + j, v0, v1, v2);
        tv[3 * j] = v0; tv[3 * j + 1] = v1; tv[3 * j + 2] = v2;
    }
    __syncthreads();
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, b0 = 0.0, b1 = 0.0, b2 = 0.0;
#pragma unroll
    for (int u = 0; u < PRE; ++u) {
        const int j = warp + FWD_WARPS * u;
        if (j < nc) {
            const double t0 = tv[3 * j], t1 = tv[3 * j + 1], t2 = tv[3 * j + 2];
            a0 = fma(pre[u].x, t0, a0); a1 = fma(pre[u].x, t1, a1); a2 = fma(pre[u].x, t2, a2);
            b0 = fma(pre[u].y, t0, b0); b1 = fma(pre[u].y, t1, b1); b2 = fma(pre[u].y, t2, b2);
        }
    }
    if (i0 < R) {
#pragma unroll 8
        for (int j = warp + FWD_WARPS * PRE; j < nc; j += FWD_WARPS) {
            const double2 m = __ldg(reinterpret_cast<const double2*>(M + (int64_t)j * d.ldy));
            const double t0 = tv[3 * j], t1 = tv[3 * j + 1], t2 = tv[3 * j + 2];
            a0 = fma(m.x, t0, a0); a1 = fma(m.x, t1, a1); a2 = fma(m.x, t2, a2);
            b0 = fma(m.y, t0, b0); b1 = fma(m.y, t1, b1); b2 = fma(m.y, t2, b2);
        }
    }
    part[warp][2 * lane][0] = a0; part[warp][2 * lane][1] = a1; part[warp][2 * lane][2] = a2;
    part[warp][2 * lane + 1][0] = b0; part[warp][2 * lane + 1][1] = b1; part[warp][2 * lane + 1][2] = b2;
    __syncthreads();
    const int row = threadIdx.x;
    const int i = it.b0 + row;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    if (row < TL) {
#pragma unroll
        for (int w = 0; w < FWD_WARPS; ++w) { s0 += part[w][row][0]; s1 += part[w][row][1]; s2 += part[w][row][2]; }
    }
    if (it.nchunk > 1) {
        if (row < TL) {
            double* p = P + 3 * ((int64_t)q * TL + row);
            p[0] = s0; p[1] = s1; p[2] = s2;
        }
        if (!band_arrive(counters + it.band, it.nchunk)) return false;
        if (row < TL) {
            s0 = s1 = s2 = 0.0;
            for (int c = 0; c < it.nchunk; ++c) {
                const double* p = P + 3 * ((int64_t)(it.first + c) * TL + row);
                s0 += __ldcg(p); s1 += __ldcg(p + 1); s2 += __ldcg(p + 2);
            }
        }
    }
    if (row < TL && i < R) {
        if (i < d.k) {
            double* o = Zb + 3 * ((int64_t)d.first + i);
            o[0] = s0; o[1] = s1; o[2] = s2;
        } else {
            double v0, v1, v2;
            front_rhs(B, U, inv, d, i, v0, v1, v2);
            double* u = U + d.u_off + 3 * (int64_t)(i - d.k);
            u[0] = v0 - s0; u[1] = v1 - s1; u[2] = v2 - s2;
        }
    }
    __threadfence();
    __syncthreads();
    return true;
}

__global__ void __launch_bounds__(32 * FWD_WARPS) k_fwd_level(const double* __restrict__ B, double* __restrict__ Zb,
                                                   double* __restrict__ U, const int64_t* __restrict__ inv,
                                                   const double* __restrict__ YW, const FrontDesc* __restrict__ desc,
                                                   const SolveItem* __restrict__ items, double* __restrict__ P,
                                                   unsigned* __restrict__ counters, const int* __restrict__ mesh_on) {
    const SolveItem it = items[blockIdx.x];
    const FrontDesc d = desc[it.front];
    if (mesh_on && !mesh_on[d.mesh]) return;   // the whole band's CTAs: its counter stays 0
    double2 pre[FWD_PRE];
    fwd_pre(YW, d, it, pre);
    fwd_item(B, Zb, U, inv, YW, d, it, blockIdx.x, P, counters, pre);
}

// Backward: a CTA owns a band of 64 columns and a chunk [lo, hi) of the rows
// (lo even; a chunk may cross row k): the input of row i is z_i for i < k and
// minus the solution at the front's row i - k for i >= k.  Warp w takes the
// eight columns b0 + w + 8m; lane l loads rows lo + 2l + 64t and the next one
// of each as one 16-byte load.  The 8 x 3 lane sums are then added across the
// warp by a butterfly that halves the values each lane keeps (12, 6, 3) before
// two plain exchange steps, so the eight columns share 27 shuffles.
// The first row pair of each of the warp's eight columns of a backward item,
// loaded before the item's dependency wait and its input gather.
__device__ __forceinline__ void bwd_pre(const double* __restrict__ YW, const FrontDesc& d, const SolveItem& it,
                                        double2 (&pre)[8]) {
    const int nr = it.hi - it.lo;
    const int nc = min(TL, d.k - it.b0);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const double* M0 = YW + d.y_off + it.lo + (int64_t)(it.b0 + warp) * d.ldy;
#pragma unroll
    for (int m = 0; m < 8; ++m)
        pre[m] = (2 * lane < nr && warp + 8 * m < nc)
                     ? __ldg(reinterpret_cast<const double2*>(M0 + (int64_t)(8 * m) * d.ldy + 2 * lane))
                     : make_double2(0.0, 0.0);
}

__device__ __forceinline__ bool bwd_item(double* __restrict__ x, const double* __restrict__ Zb,
                                         const double* __restrict__ YW, const int* __restrict__ rows,
                                         const FrontDesc& d, const SolveItem& it, int q, double* __restrict__ P,
                                         unsigned* __restrict__ counters, const double2 (&pre)[8]) {
    __shared__ double in[(SCH + 1) * 3];
    __shared__ double res[TL][3];
    const int nr = it.hi - it.lo;
    const int nc = min(TL, d.k - it.b0);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const double* M0 = YW + d.y_off + it.lo + (int64_t)(it.b0 + warp) * d.ldy;
    for (int t = threadIdx.x; t < nr + 1; t += blockDim.x) {
        const int i = it.lo + t;
        double v0 = 0.0, v1 = 0.0, v2 = 0.0;
        if (t < nr) {
            if (i < d.k) {
                const double* z = Zb + 3 * ((int64_t)d.first + i);
                v0 = z[0]; v1 = z[1]; v2 = z[2];
            } else {
                const double* y = x + 3 * (int64_t)rows[d.rows_off + i - d.k];
                v0 = -__ldcg(y); v1 = -__ldcg(y + 1); v2 = -__ldcg(y + 2);
            }
        }
        in[3 * t] = v0; in[3 * t + 1] = v1; in[3 * t + 2] = v2;
    }
    __syncthreads();
    double v[24];
#pragma unroll
    for (int q = 0; q < 24; ++q) v[q] = 0.0;
    if (2 * lane < nr) {
        const int t = 2 * lane;
        const double x0 = in[3 * t], x1 = in[3 * t + 1], x2 = in[3 * t + 2];
        const double y0 = in[3 * t + 3], y1 = in[3 * t + 4], y2 = in[3 * t + 5];
#pragma unroll
        for (int m = 0; m < 8; ++m) {
            v[3 * m] = fma(pre[m].y, y0, fma(pre[m].x, x0, v[3 * m]));
            v[3 * m + 1] = fma(pre[m].y, y1, fma(pre[m].x, x1, v[3 * m + 1]));
            v[3 * m + 2] = fma(pre[m].y, y2, fma(pre[m].x, x2, v[3 * m + 2]));
        }
    }
    for (int t = 2 * lane + 64; t < nr; t += 64) {
        const double x0 = in[3 * t], x1 = in[3 * t + 1], x2 = in[3 * t + 2];
        const double y0 = in[3 * t + 3], y1 = in[3 * t + 4], y2 = in[3 * t + 5];
#pragma unroll
        for (int m = 0; m < 8; ++m) {
            if (warp + 8 * m < nc) {
                const double2 a = __ldg(reinterpret_cast<const double2*>(M0 + (int64_t)(8 * m) * d.ldy + t));
                v[3 * m] = fma(a.y, y0, fma(a.x, x0, v[3 * m]));
                v[3 * m + 1] = fma(a.y, y1, fma(a.x, x1, v[3 * m + 1]));
                v[3 * m + 2] = fma(a.y, y2, fma(a.x, x2, v[3 * m + 2]));
            }
        }
    }
    // reduce-scatter: after the offsets 16, 8, 4 lane l keeps the 3 sums of
    // column slot m = 4 (l>>4 & 1) + 2 (l>>3 & 1) + (l>>2 & 1) over 8 lanes
#pragma unroll
    for (int q = 0; q < 12; ++q) {
        const bool hi = lane & 16;
        const double send = hi ? v[q] : v[q + 12];
        const double keep = hi ? v[q + 12] : v[q];
        v[q] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
    }
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        const bool hi = lane & 8;
        const double send = hi ? v[q] : v[q + 6];
        const double keep = hi ? v[q + 6] : v[q];
        v[q] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
    }
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        const bool hi = lane & 4;
        const double send = hi ? v[q] : v[q + 3];
        const double keep = hi ? v[q + 3] : v[q];
        v[q] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
    }
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        v[q] += __shfl_xor_sync(0xffffffffu, v[q], 2);
        v[q] += __shfl_xor_sync(0xffffffffu, v[q], 1);
    }
    if ((lane & 3) == 0) {
        const int m = ((lane >> 4) & 1) * 4 + ((lane >> 3) & 1) * 2 + ((lane >> 2) & 1);
        const int jj = warp + 8 * m;
        res[jj][0] = v[0]; res[jj][1] = v[1]; res[jj][2] = v[2];
    }
    __syncthreads();
    const int j = threadIdx.x;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    if (j < TL) { s0 = res[j][0]; s1 = res[j][1]; s2 = res[j][2]; }
    if (it.nchunk > 1) {
        if (j < TL) {
            double* p = P + 3 * ((int64_t)q * TL + j);
            p[0] = s0; p[1] = s1; p[2] = s2;
        }
        if (!band_arrive(counters + it.band, it.nchunk)) return false;
        if (j < TL) {
            s0 = s1 = s2 = 0.0;
            for (int c = 0; c < it.nchunk; ++c) {
                const double* p = P + 3 * ((int64_t)(it.first + c) * TL + j);
                s0 += __ldcg(p); s1 += __ldcg(p + 1); s2 += __ldcg(p + 2);
            }
        }
    }
    if (j < nc) {
        double* o = x + 3 * ((int64_t)d.first + it.b0 + j);
        o[0] = s0; o[1] = s1; o[2] = s2;
    }
    __threadfence();
    __syncthreads();
    return true;
}

__global__ void __launch_bounds__(256) k_bwd_level(double* __restrict__ x, const double* __restrict__ Zb,
                                                   const double* __restrict__ YW, const int* __restrict__ rows,
                                                   const FrontDesc* __restrict__ desc,
                                                   const SolveItem* __restrict__ items, double* __restrict__ P,
                                                   unsigned* __restrict__ counters, const int* __restrict__ mesh_on) {
    const SolveItem it = items[blockIdx.x];
    const FrontDesc d = desc[it.front];
    if (mesh_on && !mesh_on[d.mesh]) return;
    double2 pre[8];
    bwd_pre(YW, d, it, pre);
    bwd_item(x, Zb, YW, rows, d, it, blockIdx.x, P, counters, pre);
}

// ---- whole-direction solve over a work queue -------------------------------------
// One launch per direction walks every level: the items of all levels in one
// list (forward: leaves first; backward: root first), taken in list order by
// persistent CTAs through an atomic head (each CTA takes its next item while
// it works on the current one).  An item waits, in thread 0, until the fronts
// it reads are complete -- forward: both children (their update vectors);
// backward: the parent (and through it every ancestor, which own the front's
// rows) -- counted by per-front band counters that each band's writer bumps
// after its writes are visible.  Every item an item waits on comes earlier in
// the list and was taken by a running CTA, so the earliest unfinished item
// never waits and the queue always drains.  A wait (wait_count_geq) is bounded
// by one second of the global timer and a poll count; one that gives up sets
// *status to WRAPD_E_TIMEOUT and skips its item, and every later wait returns at
// once, so the launch ends with the error for the host to read.  The results
// are those of the per-level launches bit for bit: the same items, chunks and
// chunk order per band.
__device__ __forceinline__ bool wait_bands(const unsigned* done, unsigned target, int* status) {
    return wait_count_geq(done, target, status);
}

// Takes the CTA's next item (in every thread).  Thread 0 keeps the index it
// fetched for the item after it in a register (`ahead`), so the atomic's
// round trip runs while the current item is worked on; only its use, one item
// later, waits for it.
__device__ __forceinline__ int next_item(const SolveQueue& Q, int* s_cur, int& ahead) {
    __syncthreads();   // the previous item's shared-memory use is over
    if (threadIdx.x == 0) {
        const int cur = ahead;
        *s_cur = cur;
        if (cur < Q.n) ahead = static_cast<int>(atomicAdd(Q.head, 1u));
    }
    __syncthreads();
    return *s_cur;
}

__global__ void __launch_bounds__(32 * FWD_WARPS, 8) k_fwd_queue(const double* __restrict__ B, double* __restrict__ Zb,
                                                   double* __restrict__ U, const int64_t* __restrict__ inv,
                                                   const double* __restrict__ YW, const FrontDesc* __restrict__ desc,
                                                   SolveQueue Q, double* __restrict__ P, unsigned* __restrict__ counters,
                                                   const int* __restrict__ mesh_on) {
    __shared__ int s_cur, s_ok;
    int ahead = threadIdx.x == 0 ? static_cast<int>(atomicAdd(Q.head, 1u)) : 0;
    for (;;) {
        const int q = next_item(Q, &s_cur, ahead);
        if (q >= Q.n) break;
        const SolveItem it = Q.items[q];
        const FrontDesc d = desc[it.front];
        if (mesh_on && !mesh_on[d.mesh]) continue;
        double2 pre[FWD_PRE];
        fwd_pre(YW, d, it, pre);   // in flight during the wait
        if (threadIdx.x == 0) {
            bool ok = d.child0 < 0 || wait_bands(Q.done + d.child0, Q.nbands[d.child0], Q.status);
            ok = ok && (d.child1 < 0 || wait_bands(Q.done + d.child1, Q.nbands[d.child1], Q.status));
            s_ok = ok;
        }
        __syncthreads();
        if (!s_ok) continue;
        if (fwd_item(B, Zb, U, inv, YW, d, it, q, P, counters, pre) && threadIdx.x == 0 && it.front != Q.hold)
            atomicAdd(Q.done + it.front, 1u);
    }
}

__global__ void __launch_bounds__(256) k_bwd_queue(double* __restrict__ x, const double* __restrict__ Zb,
                                                   const double* __restrict__ YW, const int* __restrict__ rows,
                                                   const FrontDesc* __restrict__ desc, SolveQueue Q,
                                                   double* __restrict__ P, unsigned* __restrict__ counters,
                                                   const int* __restrict__ mesh_on) {
    __shared__ int s_cur, s_ok;
    int ahead = threadIdx.x == 0 ? static_cast<int>(atomicAdd(Q.head, 1u)) : 0;
    for (;;) {
        const int q = next_item(Q, &s_cur, ahead);
        if (q >= Q.n) break;
        const SolveItem it = Q.items[q];
        const FrontDesc d = desc[it.front];
        if (mesh_on && !mesh_on[d.mesh]) continue;
        double2 pre[8];
        bwd_pre(YW, d, it, pre);   // in flight during the wait
        if (threadIdx.x == 0)
            s_ok = d.parent < 0 || wait_bands(Q.done + d.parent, Q.nbands[d.parent], Q.status);
        __syncthreads();
        if (!s_ok) continue;
        if (bwd_item(x, Zb, YW, rows, d, it, q, P, counters, pre) && threadIdx.x == 0 && it.front != Q.hold)
            atomicAdd(Q.done + it.front, 1u);
    }
}

}  // namespace

CholGPU::~CholGPU() {
    if (factor_graph_) cudaGraphExecDestroy(factor_graph_);
    if (solve_graph_) cudaGraphExecDestroy(solve_graph_);
    for (void* p : allocs_) cudaFree(p);
}

template <typename X>
X* CholGPU::upload(const std::vector<X>& v, cudaStream_t st) {
    X* p = nullptr;
    const size_t bytes = std::max<size_t>(1, v.size()) * sizeof(X);
    if (cudaMalloc(&p, bytes) != cudaSuccess) { cudaGetLastError(); throw CudaError(WRAPD_E_OOM, "cudaMalloc failed (factor structures)"); }
    allocs_.push_back(p);
    device_bytes += bytes;
    if (!v.empty()) WRAPD_CUDA(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(X), cudaMemcpyHostToDevice, st));
    return p;
}

JobList CholGPU::make_jobs(const std::vector<GemmJob>& jobs, cudaStream_t st) {
    JobList l;
    std::vector<GemmJob> keep;
    std::vector<int> pre(1, 0);
    for (const GemmJob& jb : jobs) {
        const int Tr = ceil_div(jb.r1 - jb.r0, TL), Tc = ceil_div(jb.c1 - jb.c0, TL);
        if (Tr <= 0 || Tc <= 0 || jb.k1 <= jb.k0) continue;
        int tiles = 0;
        if (jb.kind == 1) tiles = Tr * Tc;
        else for (int tj = 0; tj < Tc; ++tj) tiles += std::max(0, Tr - tj);
        if (tiles <= 0) continue;
        keep.push_back(jb);
        pre.push_back(pre.back() + tiles);
    }
    l.n = static_cast<int>(keep.size());
    l.total = pre.back();
    if (l.n == 0) return l;
    l.d_jobs = upload(keep, st);
    l.d_prefix = upload(pre, st);
    return l;
}

WorkList CholGPU::make_list(const std::vector<int>& fronts, const std::vector<int>& ctas, cudaStream_t st) {
    WorkList w;
    std::vector<int> f, pre(1, 0);
    for (size_t i = 0; i < fronts.size(); ++i)
        if (ctas[i] > 0) { f.push_back(fronts[i]); pre.push_back(pre.back() + ctas[i]); }
    w.n = static_cast<int>(f.size());
    w.total = pre.back();
    if (w.n == 0) return w;
    w.d_fronts = upload(f, st);
    w.d_prefix = upload(pre, st);
    return w;
}

void CholGPU::build(const Symbolic& S, const std::vector<int64_t>& A_pos, const std::vector<int>& A_ptr,
                    const std::vector<int>& A_contrib, cudaStream_t st) {
    WRAPD_CUDA(cudaFuncSetAttribute(k_update, cudaFuncAttributeMaxDynamicSharedMemorySize, GEMM_SMEM));
    WRAPD_CUDA(cudaFuncSetAttribute(k_wgemm, cudaFuncAttributeMaxDynamicSharedMemorySize, GEMM_SMEM));
    n = S.n;
    nfronts = static_cast<int>(S.fronts.size());
    nlevels = static_cast<int>(S.levels.size());
    nnz_L = S.nnz_L;
    flops = S.flops;
    if (S.max_children > 2) throw CudaError(WRAPD_E_INPUT, "assembly tree with more than 2 children");
    h_desc_.resize(nfronts);
    std::vector<int> rows;
    int64_t roff = 0, ioff = 0;
    for (int f = 0; f < nfronts; ++f) {
        const Front& F = S.fronts[f];
        FrontDesc& d = h_desc_[f];
        d.first = F.first; d.k = F.ncols; d.r = F.nrows(); d.ld = F.ld();
        d.f_off = F.f_off; d.y_off = F.y_off; d.u_off = F.u_off; d.rel_off = F.rel_off;
        d.rows_off = roff;
        rows.insert(rows.end(), F.rows.begin(), F.rows.end());
        roff += F.nrows();
        d.inv_off = ioff; ioff += 2 * ((int64_t)d.k + d.r);
        d.nchild = static_cast<int>(F.children.size());
        d.child0 = d.nchild > 0 ? F.children[0] : -1;
        d.child1 = d.nchild > 1 ? F.children[1] : -1;
        d.ldy = static_cast<int>(yw_ld(d.k, d.r));
        d.mesh = front_mesh.empty() ? 0 : front_mesh[f];
        d.parent = F.parent;
    }
    std::vector<int64_t> inv(ioff, -1);
    for (int f = 0; f < nfronts; ++f) {
        const Front& F = S.fronts[f];
        for (size_t q = 0; q < F.children.size(); ++q) {
            const Front& C = S.fronts[F.children[q]];
            for (int i = 0; i < C.nrows(); ++i)
                inv[h_desc_[f].inv_off + 2 * (int64_t)S.relmap[C.rel_off + i] + (int64_t)q] = C.u_off + 3 * (int64_t)i;
        }
    }
    d_inv_ = upload(inv, st);
    d_desc_ = upload(h_desc_, st);
    d_rows_ = upload(rows, st);
    d_rel_ = upload(S.relmap, st);
    nA_ = static_cast<int>(A_pos.size());
    d_Apos_ = upload(A_pos, st);
    d_Aptr_ = upload(A_ptr, st);
    d_Acon_ = upload(A_contrib, st);
    f_pool_ = S.f_pool; y_pool_ = S.y_pool; u_pool_ = S.u_pool;
    auto dalloc = [&](size_t count) {
        double* p = nullptr;
        if (cudaMalloc(&p, std::max<size_t>(1, count) * sizeof(double)) != cudaSuccess) {
            cudaGetLastError();
            throw CudaError(WRAPD_E_OOM, "cudaMalloc failed (factor pools)");
        }
        allocs_.push_back(p);
        device_bytes += std::max<size_t>(1, count) * sizeof(double);
        return p;
    };
    d_F_ = dalloc(f_pool_);
    d_Y_ = dalloc(y_pool_);
    d_U_ = dalloc(u_pool_);
    d_T_ = dalloc(3 * (size_t)n);
    d_Z_ = dalloc(3 * (size_t)n);
    int* st_ptr = nullptr;
    WRAPD_CUDA(cudaMalloc(&st_ptr, sizeof(int)));
    allocs_.push_back(st_ptr);
    d_status = st_ptr;
    WRAPD_CUDA(cudaMemsetAsync(d_status, 0, sizeof(int), st));

    levels_.assign(nlevels, Level());
    fused_ctas_ = kFusedPanelCtas;
    for (int l = 0; l < nlevels; ++l) {
        Level& L = levels_[l];
        L.fronts_sorted = S.levels[l];
        std::stable_sort(L.fronts_sorted.begin(), L.fronts_sorted.end(),
                         [&](int a, int b) { return h_desc_[a].k > h_desc_[b].k; });
        const auto& fs = L.fronts_sorted;
        L.kmax = fs.empty() ? 0 : h_desc_[fs[0]].k;
        std::vector<int> cnt(fs.size());
        for (int slot = 0; slot < 2; ++slot) {
            for (size_t i = 0; i < fs.size(); ++i) {
                const FrontDesc& d = h_desc_[fs[i]];
                const int c = slot == 0 ? d.child0 : d.child1;
                cnt[i] = c < 0 ? 0 : ceil_div(h_desc_[c].r, COLS_PER_CTA);
            }
            L.extend.push_back(make_list(fs, cnt, st));
        }
        const int steps = ceil_div(L.kmax, NB);
        for (int p = 0; p < steps; ++p) {
            std::vector<int> act, ct, nP;
            std::vector<GemmJob> jobs;
            for (int f : fs) {
                const FrontDesc& d = h_desc_[f];
                const int p0 = p * NB;
                if (d.k <= p0) continue;
                const int nb = std::min(NB, d.k - p0), j0 = p0 + nb;
                const int m = d.ld - j0;
                const int bs = (p0 / OB) * OB, be = std::min(d.k, bs + OB);
                act.push_back(f);
                nP.push_back(ceil_div(m, TL));
                ct.push_back(ceil_div(m, TL) + ceil_div(p0, TL));
                if (j0 < be) {
                    // inside the outer block: only the block's remaining columns, K = this panel
                    jobs.push_back(GemmJob{f, 0, j0, d.ld, j0, be, p0, j0});
                    jobs.push_back(GemmJob{f, 1, j0, be, 0, j0, p0, j0});
                } else {
                    // the block's last panel: the deferred trailing update, K = the whole block
                    jobs.push_back(GemmJob{f, 0, be, d.ld, be, d.ld, bs, be});
                    jobs.push_back(GemmJob{f, 1, be, d.k, 0, be, bs, be});
                }
            }
            // every active front gets at least one item (its diagonal block is factored there)
            for (int& c : ct) c = std::max(c, 1);
            // both forms of the step are kept; factor_launches picks one by the step's size
            L.diag.push_back(make_list(act, std::vector<int>(act.size(), 1), st));
            L.trsm.push_back(make_list(act, ct, st));
            L.trsm_split.push_back(nP);
            L.update.push_back(make_jobs(jobs, st));
        }
        std::vector<int> wg(fs.size());
        for (size_t q = 0; q < fs.size(); ++q) {
            const FrontDesc& d = h_desc_[fs[q]];
            wg[q] = ceil_div(d.r, TL) * ceil_div(d.k, TL);
        }
        // Solve items with chunks of sch_of(front) (<= SCH) along the streamed dimension.
        auto fwd_items = [&](auto sch_of, std::vector<SolveItem>& fwd, int& fbands) {
            fwd.clear();
            fbands = 0;
            for (int f : fs) {
                const int sch = sch_of(f);
                const FrontDesc& d = h_desc_[f];
                const int R = d.k + d.r;
                // forward: row bands; Y bands use columns up to their last row
                for (int b0 = 0; b0 < R; b0 += TL) {
                    const int cend = b0 < d.k ? std::min(d.k, b0 + TL) : d.k;
                    const int nch = ceil_div(cend, sch), first = static_cast<int>(fwd.size());
                    for (int c = 0; c < nch; ++c)
                        fwd.push_back({f, b0, c * sch, std::min(cend, (c + 1) * sch), nch, first, fbands});
                    fbands++;
                }
            }
        };
        auto bwd_items = [&](auto sch_of, std::vector<SolveItem>& bwd, int& bbands) {
            bwd.clear();
            bbands = 0;
            for (int f : fs) {
                const int sch = sch_of(f);
                const FrontDesc& d = h_desc_[f];
                const int R = d.k + d.r;
                // backward: column bands over rows [b0, R) (Y rows below the band, then the W rows)
                for (int b0 = 0; b0 < d.k; b0 += TL) {
                    const int nch = ceil_div(R - b0, sch), first = static_cast<int>(bwd.size());
                    for (int lo = b0; lo < R; lo += sch) bwd.push_back({f, b0, lo, std::min(R, lo + sch), nch, first, bbands});
                    bbands++;
                }
            }
        };
        // Candidate chunk lengths SCH, SCH/2, ..., SCH_MIN, all uploaded.  The fixed
        // rule takes chunks as long as possible (fewer partial sums) while the
        // launch still has kSolveCtas CTAs: the upper levels of a large system
        // hold a few large fronts, and long chunks there leave most SMs idle with
        // each CTA latency-bound.  When not even the shortest chunks fill the GPU
        // (a small system) the longest are kept.  autotune() may pick another
        // candidate by timing.
        std::vector<SolveItem> fwd, bwd;
        int fbands = 0, bbands = 0;
        L.cfwd = -1;
        L.cbwd = -1;
        // per mesh of a batch: its item counts for each candidate (the rule
        // below applied to the mesh alone)
        const int nmesh = front_mesh.empty() ? 1 : 1 + *std::max_element(front_mesh.begin(), front_mesh.end());
        std::vector<std::vector<int>> mfwd(nmesh), mbwd(nmesh);
        for (int sch = SCH, c = 0; sch >= SCH_MIN; sch /= 2, ++c) {
            fwd_items([&](int) { return sch; }, fwd, fbands);
            bwd_items([&](int) { return sch; }, bwd, bbands);
            L.cand.push_back({sch, upload(fwd, st), static_cast<int>(fwd.size()), upload(bwd, st),
                              static_cast<int>(bwd.size()), fwd, bwd});
            if (L.cfwd < 0 && (int)fwd.size() >= kSolveCtas) L.cfwd = c;
            if (L.cbwd < 0 && (int)bwd.size() >= kSolveCtas) L.cbwd = c;
            solve_parts_ = std::max<int64_t>(solve_parts_, std::max<int64_t>(fwd.size(), bwd.size()));
            solve_bands_ = std::max(solve_bands_, std::max(fbands, bbands));
            if (nmesh > 1) {
                for (int m = 0; m < nmesh; ++m) { mfwd[m].push_back(0); mbwd[m].push_back(0); }
                for (const SolveItem& it : fwd) mfwd[front_mesh[it.front]][c]++;
                for (const SolveItem& it : bwd) mbwd[front_mesh[it.front]][c]++;
            }
        }
        if (L.cfwd < 0) L.cfwd = 0;
        if (L.cbwd < 0) L.cbwd = 0;
        if (nmesh > 1) {
            // a batch: every front takes its own mesh's choice
            std::vector<int> sf(nmesh, SCH), sb(nmesh, SCH);
            for (int m = 0; m < nmesh; ++m) {
                int cf = -1, cb = -1;
                for (int c = 0; c < (int)mfwd[m].size(); ++c) {
                    if (cf < 0 && mfwd[m][c] >= kSolveCtas) cf = c;
                    if (cb < 0 && mbwd[m][c] >= kSolveCtas) cb = c;
                }
                sf[m] = SCH >> std::max(cf, 0);
                sb[m] = SCH >> std::max(cb, 0);
            }
            fwd_items([&](int f) { return sf[front_mesh[f]]; }, fwd, fbands);
            bwd_items([&](int f) { return sb[front_mesh[f]]; }, bwd, bbands);
            L.cand.push_back({0, upload(fwd, st), static_cast<int>(fwd.size()), upload(bwd, st),
                              static_cast<int>(bwd.size()), fwd, bwd});
            L.cfwd = L.cbwd = static_cast<int>(L.cand.size()) - 1;
            solve_parts_ = std::max<int64_t>(solve_parts_, std::max<int64_t>(fwd.size(), bwd.size()));
            solve_bands_ = std::max(solve_bands_, std::max(fbands, bbands));
        }
        L.wgemm = make_list(fs, wg, st);
    }
    trsm_nP_.clear();
    for (auto& L : levels_) {
        std::vector<int*> w;
        for (auto& nP : L.trsm_split) w.push_back(nP.empty() ? nullptr : upload(nP, st));
        trsm_nP_.push_back(w);
    }
    count_launches();
    // work queues: room for every level's longest candidate list; the band
    // counts do not depend on the chunk length
    int64_t qcap_f = 0, qcap_b = 0;
    qbands_f_ = qbands_b_ = 0;
    for (const Level& L : levels_) {
        int64_t mf = 0, mb = 0;
        for (const Level::SolveCand& c : L.cand) { mf = std::max<int64_t>(mf, c.nfwd); mb = std::max<int64_t>(mb, c.nbwd); }
        qcap_f += mf;
        qcap_b += mb;
        if (!L.cand.empty()) {
            const Level::SolveCand& c = L.cand[0];
            qbands_f_ += c.hfwd.empty() ? 0 : c.hfwd.back().band + 1;
            qbands_b_ += c.hbwd.empty() ? 0 : c.hbwd.back().band + 1;
        }
    }
    solve_parts_ = std::max<int64_t>(solve_parts_, std::max(qcap_f, qcap_b));
    d_P_ = dalloc(3 * TL * (size_t)solve_parts_);
    {
        unsigned* c = nullptr;
        WRAPD_CUDA(cudaMalloc(&c, std::max(1, solve_bands_) * sizeof(unsigned)));
        allocs_.push_back(c);
        device_bytes += std::max(1, solve_bands_) * sizeof(unsigned);
        d_cnt_ = c;
        WRAPD_CUDA(cudaMemsetAsync(d_cnt_, 0, std::max(1, solve_bands_) * sizeof(unsigned), st));
    }
    d_qf_ = upload(std::vector<SolveItem>(std::max<int64_t>(1, qcap_f)), st);
    d_qb_ = upload(std::vector<SolveItem>(std::max<int64_t>(1, qcap_b)), st);
    d_qnb_ = upload(std::vector<unsigned>(2 * (size_t)std::max(1, nfronts)), st);
    qcap_f_ = qcap_f;
    qcap_b_ = qcap_b;
    qctl_words_ = 2 + 2 * (size_t)nfronts + qbands_f_ + qbands_b_;
    d_qctl_ = upload(std::vector<unsigned>(qctl_words_), st);
    {
        int dev = 0, sms = 0, bf = 0, bb = 0;
        WRAPD_CUDA(cudaGetDevice(&dev));
        WRAPD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        WRAPD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bf, k_fwd_queue, 32 * FWD_WARPS, 0));
        WRAPD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bb, k_bwd_queue, 256, 0));
        qgrid_f_ = std::max(1, bf) * sms;
        qgrid_b_ = std::max(1, bb) * sms;
    }
    build_queues(st);
    WRAPD_CUDA(cudaStreamSynchronize(st));
}

// The chosen candidate of every level, concatenated: forward leaves first,
// backward root first, with item and band indexes made global (each
// direction's bands numbered from 0 in its own counter range).  Every index
// the kernels will use is checked against its buffer here.
void CholGPU::build_queues(cudaStream_t st) {
    std::vector<SolveItem> qf, qb;
    std::vector<unsigned> nb(2 * (size_t)std::max(1, nfronts), 0u);
    auto append = [&](const std::vector<SolveItem>& src, std::vector<SolveItem>& q, int& bands, unsigned* nbands) {
        const int i0 = static_cast<int>(q.size()), b0 = bands;
        for (size_t i = 0; i < src.size(); ++i) {
            SolveItem g = src[i];
            if ((int)i == g.first) nbands[g.front]++;   // the first chunk of a band
            g.first += i0;
            g.band += b0;
            bands = std::max(bands, g.band + 1);
            q.push_back(g);
        }
    };
    int bf = 0, bb = 0;
    for (int l = 0; l < nlevels; ++l) {
        const Level& L = levels_[l];
        if (!L.cand.empty()) append(L.cand[L.cfwd].hfwd, qf, bf, nb.data());
    }
    for (int l = nlevels - 1; l >= 0; --l) {
        const Level& L = levels_[l];
        if (!L.cand.empty()) append(L.cand[L.cbwd].hbwd, qb, bb, nb.data() + nfronts);
    }
    auto check = [&](const std::vector<SolveItem>& q, int64_t cap, int nbands, const char* what) {
        if ((int64_t)q.size() > cap || (int64_t)q.size() > solve_parts_)
            throw CudaError(WRAPD_E_INPUT, std::string("solve queue longer than its buffers: ") + what);
        for (size_t i = 0; i < q.size(); ++i) {
            const SolveItem& g = q[i];
            const bool ok = g.front >= 0 && g.front < nfronts && g.band >= 0 && g.band < nbands && g.nchunk >= 1 &&
                            g.first >= 0 && g.first <= (int)i && (int64_t)g.first + g.nchunk <= (int64_t)q.size() &&
                            (int)i < g.first + g.nchunk;
            if (!ok) throw CudaError(WRAPD_E_INPUT, std::string("solve queue item out of range: ") + what);
        }
    };
    if (bf != qbands_f_ || bb != qbands_b_) throw CudaError(WRAPD_E_INPUT, "solve queue band count mismatch");
    check(qf, qcap_f_, qbands_f_, "forward");
    check(qb, qcap_b_, qbands_b_, "backward");
    nqf_ = static_cast<int>(qf.size());
    nqb_ = static_cast<int>(qb.size());
    if (!qf.empty()) WRAPD_CUDA(cudaMemcpyAsync(d_qf_, qf.data(), qf.size() * sizeof(SolveItem), cudaMemcpyHostToDevice, st));
    if (!qb.empty()) WRAPD_CUDA(cudaMemcpyAsync(d_qb_, qb.data(), qb.size() * sizeof(SolveItem), cudaMemcpyHostToDevice, st));
    WRAPD_CUDA(cudaMemcpyAsync(d_qnb_, nb.data(), nb.size() * sizeof(unsigned), cudaMemcpyHostToDevice, st));
    WRAPD_CUDA(cudaStreamSynchronize(st));   // the host vectors go out of scope
    if (solve_graph_) { cudaGraphExecDestroy(solve_graph_); solve_graph_ = nullptr; }
}

void CholGPU::count_launches() {
    launches_factor = 4;   // memsets + assembly + identity
    launches_solve = 2;    // the two queue launches (plus a copy and a memset)
    for (const Level& L : levels_) {
        for (const WorkList& e : L.extend) launches_factor += e.total ? 1 : 0;
        for (size_t p = 0; p < L.trsm.size(); ++p) {
            if (L.trsm[p].total > fused_ctas_) launches_factor += L.diag[p].n ? 1 : 0;
            launches_factor += (L.trsm[p].total ? 1 : 0) + (L.update[p].total ? 1 : 0);
        }
        launches_factor += L.wgemm.total ? 1 : 0;
    }
}

std::vector<int> CholGPU::tuning() const {
    std::vector<int> t{fused_ctas_, nlevels};
    for (const Level& L : levels_) t.push_back(L.cand.empty() ? 0 : L.cand[L.cfwd].sch);
    for (const Level& L : levels_) t.push_back(L.cand.empty() ? 0 : L.cand[L.cbwd].sch);
    return t;
}

// Each candidate is timed by CUDA events on the handle's stream: one level's
// solve launch (the mean of three after one untimed), or one whole
// factorization launched directly (after one untimed at the fixed rule).  The
// solve launches run on scratch vectors; the factorizations on the current
// weights, so the factor is valid afterwards whatever the choice.
void CholGPU::autotune(const double* d_w2, const double* d_Di, int ne, cudaStream_t st) {
    cudaEvent_t e0, e1;
    WRAPD_CUDA(cudaEventCreate(&e0));
    WRAPD_CUDA(cudaEventCreate(&e1));
    auto timed = [&](int reps, auto&& launch) {
        launch();
        WRAPD_CUDA(cudaEventRecord(e0, st));
        for (int r = 0; r < reps; ++r) launch();
        WRAPD_CUDA(cudaEventRecord(e1, st));
        WRAPD_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        WRAPD_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        return ms / reps;
    };
    // (a batch keeps its per-mesh chunk lengths: a mesh's solve stays its own)
    for (Level& L : levels_) {
        if (!front_mesh.empty()) break;
        float best_f = 1e30f, best_b = 1e30f;
        for (int c = 0; c < (int)L.cand.size(); ++c) {
            const Level::SolveCand& C = L.cand[c];
            const float tf = timed(3, [&] {
                k_fwd_level<<<C.nfwd, 32 * FWD_WARPS, 0, st>>>(d_T_, d_Z_, d_U_, d_inv_, d_Y_, d_desc_, C.fwd, d_P_, d_cnt_,
                                                    nullptr);
            });
            const float tb = timed(3, [&] {
                k_bwd_level<<<C.nbwd, 256, 0, st>>>(d_T_, d_Z_, d_Y_, d_rows_, d_desc_, C.bwd, d_P_, d_cnt_,
                                                    nullptr);
            });
            WRAPD_LAUNCH_CHECK();
            if (tf < best_f) { best_f = tf; L.cfwd = c; }
            if (tb < best_b) { best_b = tb; L.cbwd = c; }
        }
    }
    if (front_mesh.empty()) build_queues(st);
    const int candidates[] = {0, kNumSMs, kFusedPanelCtas, 4 * kFusedPanelCtas, 1 << 30};
    float best = 1e30f;
    int pick = kFusedPanelCtas;
    fused_ctas_ = kFusedPanelCtas;
    factor_launches(d_w2, d_Di, ne, st);   // untimed first run
    for (int c : candidates) {
        fused_ctas_ = c;
        const float t = timed(1, [&] { factor_launches(d_w2, d_Di, ne, st); });
        if (t < best) { best = t; pick = c; }
    }
    fused_ctas_ = pick;
    count_launches();
    WRAPD_CUDA(cudaMemsetAsync(d_status, 0, sizeof(int), st));
    WRAPD_CUDA(cudaStreamSynchronize(st));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
}

void CholGPU::factor_launches(const double* d_w2, const double* d_Di, int ne, cudaStream_t st) {
    WRAPD_CUDA(cudaMemsetAsync(d_F_, 0, f_pool_ * sizeof(double), st));
    WRAPD_CUDA(cudaMemsetAsync(d_Y_, 0, y_pool_ * sizeof(double), st));
    if (nA_ > 0) {
        k_assemble_A<<<ceil_div(nA_, 256), 256, 0, st>>>(d_F_, d_Apos_, d_Aptr_, d_Acon_, nA_, d_w2, d_Di, ne);
        WRAPD_LAUNCH_CHECK();
    }
    k_y_identity<<<nfronts, 128, 0, st>>>(d_Y_, d_desc_, nfronts);
    WRAPD_LAUNCH_CHECK();
    for (int l = 0; l < nlevels; ++l) {
        Level& L = levels_[l];
        for (int slot = 0; slot < 2; ++slot)
            if (L.extend[slot].total) {
                k_extend_add<<<L.extend[slot].total, 32 * COLS_PER_CTA, 0, st>>>(d_F_, d_desc_, d_rel_, L.extend[slot], slot);
                WRAPD_LAUNCH_CHECK();
            }
        for (size_t p = 0; p < L.trsm.size(); ++p) {
            if (L.trsm[p].total <= fused_ctas_) {
                if (L.trsm[p].total) {
                    k_panel<<<L.trsm[p].total, GEMM_THREADS, 0, st>>>(d_F_, d_Y_, d_desc_, L.trsm[p],
                                                                      trsm_nP_[l][p], (int)p, d_status);
                    WRAPD_LAUNCH_CHECK();
                }
            } else {
                if (L.diag[p].n) {
                    k_diag<<<L.diag[p].n, GEMM_THREADS, 0, st>>>(d_F_, d_Y_, d_desc_, L.diag[p], (int)p, d_status);
                    WRAPD_LAUNCH_CHECK();
                }
                if (L.trsm[p].total) {
                    k_trsm<<<L.trsm[p].total, GEMM_THREADS, 0, st>>>(d_F_, d_Y_, d_desc_, L.trsm[p],
                                                                     trsm_nP_[l][p], (int)p);
                    WRAPD_LAUNCH_CHECK();
                }
            }
            if (L.update[p].total) {
                k_update<<<L.update[p].total, GEMM_THREADS, GEMM_SMEM, st>>>(d_F_, d_Y_, d_desc_, L.update[p]);
                WRAPD_LAUNCH_CHECK();
            }
        }
        if (L.wgemm.total) {
            k_wgemm<<<L.wgemm.total, GEMM_THREADS, GEMM_SMEM, st>>>(d_F_, d_Y_, d_Y_, d_desc_, L.wgemm);
            WRAPD_LAUNCH_CHECK();
        }
    }
}

void CholGPU::factor(const double* d_w2, const double* d_Di, int ne, cudaStream_t st) {
    if (!use_graphs) { factor_launches(d_w2, d_Di, ne, st); return; }
    if (!factor_graph_) {
        cudaGraph_t g;
        WRAPD_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        try {
            factor_launches(d_w2, d_Di, ne, st);
        } catch (...) {
            cudaStreamEndCapture(st, &g);
            throw;
        }
        WRAPD_CUDA(cudaStreamEndCapture(st, &g));
        WRAPD_CUDA(cudaGraphInstantiate(&factor_graph_, g, 0));
        cudaGraphDestroy(g);
    }
    WRAPD_CUDA(cudaGraphLaunch(factor_graph_, st));
}

void CholGPU::solve_launches(double* d_x, cudaStream_t st, const int* mesh_on, int hold) {
    WRAPD_CUDA(cudaMemcpyAsync(d_T_, d_x, 3 * (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    WRAPD_CUDA(cudaMemsetAsync(d_qctl_, 0, qctl_words_ * sizeof(unsigned), st));
    unsigned* bands = d_qctl_ + 2 + 2 * (size_t)nfronts;
    if (nqf_ > 0) {
        const SolveQueue Q{d_qf_, nqf_, d_qctl_, d_qctl_ + 2, d_qnb_, d_status, hold};
        k_fwd_queue<<<std::min(qgrid_f_, nqf_), 32 * FWD_WARPS, 0, st>>>(d_T_, d_Z_, d_U_, d_inv_, d_Y_, d_desc_, Q, d_P_, bands,
                                                           mesh_on);
        WRAPD_LAUNCH_CHECK();
    }
    if (nqb_ > 0) {
        const SolveQueue Q{d_qb_, nqb_, d_qctl_ + 1, d_qctl_ + 2 + nfronts, d_qnb_ + nfronts, d_status, hold};
        k_bwd_queue<<<std::min(qgrid_b_, nqb_), 256, 0, st>>>(d_x, d_Z_, d_Y_, d_rows_, d_desc_, Q, d_P_,
                                                           bands + qbands_f_, mesh_on);
        WRAPD_LAUNCH_CHECK();
    }
}

void CholGPU::solve_holding(double* d_x, int hold, cudaStream_t st) {
    if (hold < 0 || hold >= nfronts) throw CudaError(WRAPD_E_INPUT, "front index out of range");
    solve_launches(d_x, st, nullptr, hold);
}

void CholGPU::solve(double* d_x, cudaStream_t st, const int* mesh_on) {
    if (!use_graphs) { solve_launches(d_x, st, mesh_on); return; }
    if (!solve_graph_ || solve_graph_x_ != d_x || solve_graph_mask_ != mesh_on) {
        if (solve_graph_) { cudaGraphExecDestroy(solve_graph_); solve_graph_ = nullptr; }
        cudaGraph_t g;
        WRAPD_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        try {
            solve_launches(d_x, st, mesh_on);
        } catch (...) {
            cudaStreamEndCapture(st, &g);
            throw;
        }
        WRAPD_CUDA(cudaStreamEndCapture(st, &g));
        WRAPD_CUDA(cudaGraphInstantiate(&solve_graph_, g, 0));
        cudaGraphDestroy(g);
        solve_graph_x_ = d_x;
        solve_graph_mask_ = mesh_on;
    }
    WRAPD_CUDA(cudaGraphLaunch(solve_graph_, st));
}

}  // namespace wrapd
