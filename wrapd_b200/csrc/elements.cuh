// Per-element kernels of the ADMM loop (one thread per tet) and the free-vertex
// vector kernels.  Element arrays are SoA: component k of element e is at
// [k * ne + e], so every load and store of a warp is coalesced.  All state is
// stored in FP64; the local step's SVD and prox can run in FP32 (mixed mode),
// everything else (gradient assembly, reductions, the global step) is FP64.
#pragma once
#include "elem_math.cuh"
#include "elem_types.cuh"
#include "prox_net.cuh"

namespace wrapd {

// Candidate-weight modes of update_all_candidate_weights (src/TetElements.cpp:391-432).
enum { CAND_NONE = 0, CAND_REST = 1, CAND_HESSIAN = 2 };

template <typename T>
__device__ __forceinline__ void load9(const double* a, int ne, int e, T* m) {
#pragma unroll
    for (int k = 0; k < 9; ++k) m[k] = T(a[(size_t)k * ne + e]);
}
template <typename T>
__device__ __forceinline__ void store9(double* a, int ne, int e, const T* m) {
#pragma unroll
    for (int k = 0; k < 9; ++k) a[(size_t)k * ne + e] = double(m[k]);
}

// F = (D_free x_free + D_fix x_fix)^T, src/TetElements.cpp:568-586, computed
// in FP64.  `split` sums free then pinned slots as the reference does for
// partially pinned tets; otherwise the four slots in order (Di * x_local).
__device__ __forceinline__ void deformation(const ElemView& E, int e, const double* __restrict__ x,
                                            const double* __restrict__ xfix, bool split, double* F) {
    const int4 id = E.idx[e];
    const int ids[4] = {id.x, id.y, id.z, id.w};
    double xa[4][3];
    bool fixed[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        fixed[a] = ids[a] < 0;
        const double* p = fixed[a] ? xfix + 3 * (size_t)(-ids[a] - 1) : x + 3 * (size_t)ids[a];
        xa[a][0] = p[0]; xa[a][1] = p[1]; xa[a][2] = p[2];
    }
    const bool any_fixed = fixed[0] || fixed[1] || fixed[2] || fixed[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        double d[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) d[a] = E.Di[(size_t)(c + 3 * a) * E.ne + e];
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            if (split && any_fixed) {
                double vf = 0.0, vx = 0.0;
#pragma unroll
                for (int a = 0; a < 4; ++a) {
                    if (fixed[a]) vx += d[a] * xa[a][r];
                    else vf += d[a] * xa[a][r];
                }
                F[r + 3 * c] = vf + vx;
            } else {
                double v = 0.0;
#pragma unroll
                for (int a = 0; a < 4; ++a) v += d[a] * xa[a][r];
                F[r + 3 * c] = v;
            }
        }
    }
}

// potential_energy_x per element (src/TetElements.cpp:598-635) from the
// sign-fixed singular values: NH psi(sigma); ARAP |F - R|^2 / 2 with
// R = U V^T, i.e. sum (sigma_i - 1)^2 / 2 (k = 1).
__device__ __forceinline__ double elastic_energy(const Material& m, const double* s) {
    if (m.model == MODEL_ARAP)
        return 0.5 * ((s[0] - 1.0) * (s[0] - 1.0) + (s[1] - 1.0) * (s[1] - 1.0) + (s[2] - 1.0) * (s[2] - 1.0));
    return NH<double>{m.mu, m.lambda}.psi_plain(s[0], s[1], s[2]);
}

// ---- the defo cache + gradient of the global AL objective -------------------
// update_defo_cache (src/TetElements.cpp:564-596) fused with
// global_obj_grad (src/TetElements.cpp:691-738): F, SVD, symF, Q = V^T P V,
// K + K^T, M = F - U diag(s) (K+K^T) V^T and g_e = w^2 Di^T M^T, plus the AL
// value 0.5 w^2 |symF - P|^2, the potential energy and the inversion count at
// x (src/TetElements.cpp:444-468, 598-635).  Outputs out[0..2] = value, pe, flips.
// SEG: a batch (per-mesh sums); a single mesh takes grid_reduce, the same
// arithmetic.  Register budgets: the single-mesh form compiles to 128 with no
// occupancy hint; the segmented one and the UV forms below are held to 128
// (16 warps per SM) by the hint, without which they took 164-168.  Launched
// on 256-element tiles (two CTAs per SM).
// UV (single mesh only): 0 = SVD as usual; 1 = also keep U and V of the SVD
// in uv (U then V, 9 SoA components each); 2 = x is the point of the last
// UV = 1 launch, so F's SVD is that launch's: sig, U, V and symF are read
// back instead of recomputed (the same values, so the same results).
template <bool SEG, int UV = 0>
static __global__ void __launch_bounds__(256, (SEG || UV != 0) ? 2 : 0) k_grad(ElemView E, Tiles T, const int* on, const double* __restrict__ x,
                                              const double* __restrict__ xfix, Material mat0, int write_gel,
                                              double* partials, unsigned* counters, double* out, int stride,
                                              double* __restrict__ uv = nullptr) {
    const Tile tl = tile_at(T, blockIdx.x);
    if (!mesh_on(on, tl.mesh)) return;
    const int e = tl.first + threadIdx.x;
    const Material mat = elem_material(E, mat0, e < tl.end ? e : E.ne);
    double red[3] = {0.0, 0.0, 0.0};
    if (e < tl.end) {
        double Fd[9];
        deformation(E, e, x, xfix, true, Fd);
        double F[9], s[3], Us[9], Vs[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) F[i] = double(Fd[i]);
        double S[9];
        if constexpr (UV == 2) {
            load9(uv, E.ne, e, Us);
            load9(uv + (size_t)9 * E.ne, E.ne, e, Vs);
#pragma unroll
            for (int i = 0; i < 3; ++i) s[i] = E.sig[(size_t)i * E.ne + e];
            load9(E.symF, E.ne, e, S);
        } else {
            svd3(F, s, Us, Vs);
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    M3(S, r, c) = M3(Vs, r, 0) * s[0] * M3(Vs, c, 0) + M3(Vs, r, 1) * s[1] * M3(Vs, c, 1) +
                                  M3(Vs, r, 2) * s[2] * M3(Vs, c, 2);
            store9(E.symF, E.ne, e, S);
#pragma unroll
            for (int i = 0; i < 3; ++i) E.sig[(size_t)i * E.ne + e] = s[i];
            if constexpr (UV == 1) {
                store9(uv, E.ne, e, Us);
                store9(uv + (size_t)9 * E.ne, E.ne, e, Vs);
            }
        }
        double Zm[9], Um[9], P[9];
        load9(E.Z, E.ne, e, Zm);
        load9(E.U, E.ne, e, Um);
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c) M3(P, r, c) = M3(Zm, c, r) - M3(Um, c, r);
        const double w2 = E.w2[e];
        {
            double v = 0.0;
#pragma unroll
            for (int i = 0; i < 9; ++i) { const double d = double(S[i]) - double(P[i]); v += d * d; }
            red[0] = (0.5 * w2) * v;
        }
        red[1] = E.vol[e] * elastic_energy(mat, s);
        red[2] = (s[0] < double(0) || s[1] < double(0) || s[2] < double(0)) ? 1.0 : 0.0;
        if (write_gel) {
            double Tm[9], Q[9], K[9], Mm[9];
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    M3(Tm, r, c) = M3(Vs, 0, r) * M3(P, 0, c) + M3(Vs, 1, r) * M3(P, 1, c) + M3(Vs, 2, r) * M3(P, 2, c);
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    M3(Q, r, c) = M3(Tm, r, 0) * M3(Vs, 0, c) + M3(Tm, r, 1) * M3(Vs, 1, c) + M3(Tm, r, 2) * M3(Vs, 2, c);
            M3(K, 0, 0) = M3(Q, 0, 0) / s[0];
            M3(K, 1, 1) = M3(Q, 1, 1) / s[1];
            M3(K, 2, 2) = M3(Q, 2, 2) / s[2];
            M3(K, 0, 1) = M3(K, 1, 0) = (M3(Q, 0, 1) + M3(Q, 1, 0)) / (s[0] + s[1]);
            M3(K, 0, 2) = M3(K, 2, 0) = (M3(Q, 0, 2) + M3(Q, 2, 0)) / (s[0] + s[2]);
            M3(K, 1, 2) = M3(K, 2, 1) = (M3(Q, 1, 2) + M3(Q, 2, 1)) / (s[1] + s[2]);
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    double v = double(0);
#pragma unroll
                    for (int a = 0; a < 3; ++a) {
                        const double t = M3(K, a, 0) * M3(Vs, c, 0) + M3(K, a, 1) * M3(Vs, c, 1) + M3(K, a, 2) * M3(Vs, c, 2);
                        v += M3(Us, r, a) * s[a] * t;
                    }
                    M3(Mm, r, c) = F[r + 3 * c] - v;
                }
            const double w2t = double(w2);
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int r = 0; r < 3; ++r) {
                    double v = double(0);
#pragma unroll
                    for (int c = 0; c < 3; ++c) v += double(E.Di[(size_t)(c + 3 * a) * E.ne + e]) * (w2t * M3(Mm, r, c));
                    E.gel[(size_t)(r + 3 * a) * E.ne + e] = v;
                }
        }
    }
    if constexpr (SEG)
        seg_reduce_out<3>(red, T, tl.mesh, partials, counters, out, stride);
    else
        grid_reduce<3>(red, partials, counters, out);
}

// ---- per-mesh vectors of the global step (MeshCtl, VecPools: elem_types.cuh) --
__device__ __forceinline__ int hist_slot(const MeshCtl& c, int i, int M) { return (c.head + i) % (M + 1); }
__device__ __forceinline__ double* g_cur(const VecPools& P, const MeshCtl& c) { return P.G[c.grot % 3]; }
__device__ __forceinline__ double* g_new(const VecPools& P, const MeshCtl& c) { return P.G[(c.grot + 1) % 3]; }
__device__ __forceinline__ double* g_old(const VecPools& P, const MeshCtl& c) { return P.G[(c.grot + 2) % 3]; }

// Gather modes: at the start of an ADMM iteration the gradient goes to the
// mesh's cur buffer and is compared with old (|grad - grad_old|^2, the early
// return of SplitLBFGS.hpp:138-142); inside the L-BFGS loop it goes to new,
// y = new - cur is staged with <s, y>; GATHER_PLAIN writes `plain` only.
enum { GATHER_START = 0, GATHER_LBFGS = 1, GATHER_PLAIN = 2 };

// Free-vertex gather of the element gradients (atomic-free; each vertex's
// incidences, in element order, are added by eight lanes in a fixed order, so
// the sum is deterministic):
//   grad[i] = sum over (e, a) incident to i of gel(a, :)[e].
// Tiles of 32 free vertices (eight lanes each).  Per mesh: out[0] = |d|^2 with
// d = grad - gold, out[1] = <s_stage, d> (GATHER_LBFGS), out[2] = |x - xs|^2
// (the x error of AlgorithmData, at the point the gradient was taken; x may be
// null).
static __global__ void __launch_bounds__(256) k_gather(Tiles T, const int* on, int mode, const MeshCtl* __restrict__ ctl,
                                                VecPools P, double* __restrict__ plain, const int* __restrict__ inc_ptr,
                                                const int* __restrict__ inc, const double* __restrict__ gel, int ne,
                                                const double* __restrict__ x, const double* __restrict__ xs,
                                                double* partials, unsigned* counters, double* out, int stride) {
    const Tile tl = tile_at(T, blockIdx.x);
    if (!mesh_on(on, tl.mesh)) return;
    double *grad = plain, *ystage = nullptr;
    const double *gold = nullptr, *sstage = nullptr;
    if (mode != GATHER_PLAIN) {
        const MeshCtl c = ctl[tl.mesh];
        if (mode == GATHER_START) {
            grad = g_cur(P, c);
            gold = g_old(P, c);
        } else {
            grad = g_new(P, c);
            gold = g_cur(P, c);
            ystage = P.Y[c.stage];
            sstage = P.S[c.stage];
        }
    }
    // eight lanes per vertex: lane s of the group adds incidences s, s + 8, ...
    // of the vertex, then the group adds its lanes in a fixed xor tree
    const int i = tl.first + (threadIdx.x >> 3), sub = threadIdx.x & 7;
    double red[3] = {0.0, 0.0, 0.0};
    double g0 = 0.0, g1 = 0.0, g2 = 0.0;
    if (i < tl.end) {
        for (int t = inc_ptr[i] + sub; t < inc_ptr[i + 1]; t += 8) {
            const int c = inc[t];
            const int e = c >> 2, a = c & 3;
            g0 += gel[(size_t)(0 + 3 * a) * ne + e];
            g1 += gel[(size_t)(1 + 3 * a) * ne + e];
            g2 += gel[(size_t)(2 + 3 * a) * ne + e];
        }
    }
#pragma unroll
    for (int o = 4; o > 0; o >>= 1) {
        g0 += __shfl_xor_sync(0xffffffffu, g0, o);
        g1 += __shfl_xor_sync(0xffffffffu, g1, o);
        g2 += __shfl_xor_sync(0xffffffffu, g2, o);
    }
    if (i < tl.end && sub == 0) {
        grad[3 * (size_t)i] = g0; grad[3 * (size_t)i + 1] = g1; grad[3 * (size_t)i + 2] = g2;
        if (gold) {
            const double d0 = g0 - gold[3 * (size_t)i], d1 = g1 - gold[3 * (size_t)i + 1], d2 = g2 - gold[3 * (size_t)i + 2];
            if (ystage) { ystage[3 * (size_t)i] = d0; ystage[3 * (size_t)i + 1] = d1; ystage[3 * (size_t)i + 2] = d2; }
            red[0] = d0 * d0 + d1 * d1 + d2 * d2;
            if (sstage) red[1] = sstage[3 * (size_t)i] * d0 + sstage[3 * (size_t)i + 1] * d1 + sstage[3 * (size_t)i + 2] * d2;
        }
        if (x) {
            const double e0 = x[3 * (size_t)i] - xs[3 * (size_t)i], e1 = x[3 * (size_t)i + 1] - xs[3 * (size_t)i + 1],
                         e2 = x[3 * (size_t)i + 2] - xs[3 * (size_t)i + 2];
            red[2] = e0 * e0 + e1 * e1 + e2 * e2;
        }
    }
    seg_reduce_out<3>(red, T, tl.mesh, partials, counters, out, stride);
}

// ---- local step ---------------------------------------------------------------
// TetElements::polar_update, NH branch (src/TetElements.cpp:284-346), fused
// per element: S_in = (symF + U)^T, SVD, prox from the last stretches, Z and
// U update, and the candidate weight (src/TetElements.cpp:391-432).  C is the
// arithmetic of the SVD and the prox (double, or float in mixed mode); loads,
// stores, the dual update and every sum are FP64.
// out[0..4] = bef_penalty, aft_penalty, curr_pe, negative-stretch count, prox
// iterations.
// prox_mode 0: the reference's L-BFGS prox; 1: Newton (prox_newton); 2 (NET):
// Newton from the better (lower prox objective) of the last stretches and the
// prox network's prediction.  The FP32 instantiation always uses Newton.
// NET needs dynamic shared memory: the network image plus one scratch per warp.
template <typename C, bool NET>
__global__ void __launch_bounds__(512, 1) k_local(ElemView E, Tiles T, const int* on, Material mat0, int prox_iters,
                                               int cand_mode, int prox_mode, const unsigned char* __restrict__ net_img,
                                               double* partials, unsigned* counters, double* out, int stride) {
    const Tile tl = tile_at(T, blockIdx.x);
    if (!mesh_on(on, tl.mesh)) return;
    double red[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    extern __shared__ __align__(16) unsigned char local_smem[];
    if constexpr (NET) {
        net::load_image(net_img, local_smem);
        __syncthreads();
    }
    const int e = tl.first + threadIdx.x;
    const bool valid = e < tl.end;
    const Material mat = elem_material(E, mat0, valid ? e : E.ne);
    double S[9], Um[9];
    double w2 = 0.0, vol = 1.0;
    C sg[3] = {C(1), C(1), C(1)}, Ue[9], Ve[9];
    if (valid) {
        double Zm[9];
        load9(E.symF, E.ne, e, S);
        load9(E.U, E.ne, e, Um);
        load9(E.Z, E.ne, e, Zm);
        w2 = E.w2[e];
        vol = E.vol[e];
        C Sin[9];
        double bef = 0.0;
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                M3(Sin, r, c) = C(M3(S, c, r) + M3(Um, c, r));
                const double d = M3(S, r, c) - (M3(Zm, r, c) - M3(Um, r, c));
                bef += d * d;
            }
        red[0] += 0.5 * w2 * bef;
        svd3(Sin, sg, Ue, Ve);
    }
    Prox<C> P;
    P.nh.mu = C(mat.mu);
    P.nh.lambda = C(mat.lambda);
    P.x0[0] = sg[0]; P.x0[1] = sg[1]; P.x0[2] = sg[2];
    P.wov = C(w2 / vol);
    C xs[3] = {C(1), C(1), C(1)};
    if (valid) {
#pragma unroll
        for (int i = 0; i < 3; ++i) xs[i] = C(E.slast[(size_t)i * E.ne + e]);
    }
    if constexpr (NET) {
        // warp-collective: every lane runs the network, lanes past the end on dummies
        const float sf[3] = {float(sg[0]), float(sg[1]), float(sg[2])};
        float f[net::IN], y[net::OUT], pr[3];
        net::features(sf, valid ? float(w2 / vol) : float(mat.mu), float(mat.mu), float(mat.lambda), f);
        net::warp_forward(local_smem, local_smem + net::IMAGE_BYTES + (threadIdx.x >> 5) * net::WARP_SCRATCH, f,
                          valid, y);
        net::predict_start(local_smem, sf, y, pr);
        if (valid) {
            const C cand[3] = {C(pr[0]), C(pr[1]), C(pr[2])};
            if (isfinite(cand[0]) && isfinite(cand[1]) && isfinite(cand[2]) && P.value(cand) < P.value(xs)) {
                xs[0] = cand[0]; xs[1] = cand[1]; xs[2] = cand[2];
            }
        }
    }
    if (valid) {
        int iters;
        if constexpr (sizeof(C) == sizeof(double)) {
            if (NET || prox_mode == 1) {
                iters = prox_newton(P, xs, prox_iters, C(1e-12));
            } else {
                extern __shared__ double prox_hist[];   // 48 x blockDim doubles
                iters = prox_lbfgs(P, xs, prox_iters, ProxHistory<double>{prox_hist + threadIdx.x, (int)blockDim.x});
                if (iters < 0) iters = prox_iters;
            }
        } else {
            iters = prox_newton(P, xs, prox_iters, C(8) * Lim<C>::eps());
        }
        if (sizeof(C) < sizeof(double) &&
            !(isfinite(xs[0]) && isfinite(xs[1]) && isfinite(xs[2]) && xs[0] >= C(0) && xs[1] >= C(0) && xs[2] >= C(0))) {
            // FP32 range guard: near a vanishing stretch 1/x overflows in single
            // precision; redo this element's prox in FP64 from the same inputs.
            Prox<double> Pd;
            Pd.nh.mu = mat.mu;
            Pd.nh.lambda = mat.lambda;
            Pd.x0[0] = double(sg[0]); Pd.x0[1] = double(sg[1]); Pd.x0[2] = double(sg[2]);
            Pd.wov = w2 / vol;
            double xd[3];
#pragma unroll
            for (int i = 0; i < 3; ++i) xd[i] = E.slast[(size_t)i * E.ne + e];
            iters += prox_newton(Pd, xd, prox_iters, 1e-12);
#pragma unroll
            for (int i = 0; i < 3; ++i) xs[i] = C(xd[i]);
        }
        red[4] += double(iters);
        double xo[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) { xo[i] = double(xs[i]); E.slast[(size_t)i * E.ne + e] = xo[i]; }
        red[3] += (xo[0] < 0.0 || xo[1] < 0.0 || xo[2] < 0.0) ? 1.0 : 0.0;
        C Soc[9];
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c)
                M3(Soc, r, c) = M3(Ve, r, 0) * xs[0] * M3(Ue, c, 0) + M3(Ve, r, 1) * xs[1] * M3(Ue, c, 1) +
                                M3(Ve, r, 2) * xs[2] * M3(Ue, c, 2);
        red[2] += vol * NH<double>{mat.mu, mat.lambda}.psi_plain(xo[0], xo[1], xo[2]);
        double aft = 0.0, Zm[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            const double So = double(Soc[i]);
            const double d = S[i] - (So - Um[i]);
            aft += d * d;
            Zm[i] = So;
            Um[i] = Um[i] + (S[i] - So);
        }
        red[1] += 0.5 * w2 * aft;
        store9(E.Z, E.ne, e, Zm);
        store9(E.U, E.ne, e, Um);
        if (cand_mode == CAND_REST) {
            E.w2c[e] = vol * mat.wr;
        } else if (cand_mode == CAND_HESSIAN) {
            const double lm = NH<double>{mat.mu, mat.lambda}.hess_lmax(xo);
            double c = lm;
            if (lm < mat.wmin) c = mat.wmin;
            if (lm > mat.wmax) c = mat.wmax;
            E.w2c[e] = vol * c;
        }
    }
    seg_reduce_out<5>(red, T, tl.mesh, partials, counters, out, stride);
}

// initialize_dual_vars (src/TetElements.cpp:145-166): Z = (V diag(s) V^T)^T of
// F(X) with all four slots read from X, U = 0; then polar_potential_energy
// (src/TetElements.cpp:638-675) of the new Z.  out[0] = that energy.
static __global__ void __launch_bounds__(128) k_init_dual(ElemView E, Tiles T, const int* on, const double* __restrict__ x,
                                                   const double* __restrict__ xfix, Material mat0,
                                                   double* partials, unsigned* counters, double* out, int stride) {
    const Tile tl = tile_at(T, blockIdx.x);
    if (!mesh_on(on, tl.mesh)) return;
    const int e = tl.first + threadIdx.x;
    const Material mat = elem_material(E, mat0, e < tl.end ? e : E.ne);
    double red[1] = {0.0};
    if (e < tl.end) {
        double Fd[9];
        deformation(E, e, x, xfix, false, Fd);
        double F[9], s[3], Us[9], Vs[9], Zm[9], Zt[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) F[i] = double(Fd[i]);
        svd3(F, s, Us, Vs);
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c)
                M3(Zm, r, c) = M3(Vs, c, 0) * s[0] * M3(Vs, r, 0) + M3(Vs, c, 1) * s[1] * M3(Vs, r, 1) +
                               M3(Vs, c, 2) * s[2] * M3(Vs, r, 2);
        store9(E.Z, E.ne, e, Zm);
        double zero[9] = {};
        store9(E.U, E.ne, e, zero);
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c) M3(Zt, r, c) = M3(Zm, c, r);
        if (mat.model == MODEL_ARAP) {
            // ARAP polar_potential_energy (src/TetElements.cpp:640-646): |Z - I|^2 / 2
            double n2 = 0.0;
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int c = 0; c < 3; ++c) { const double d = M3(Zm, r, c) - (r == c ? 1.0 : 0.0); n2 += d * d; }
            red[0] = 0.5 * E.vol[e] * n2;
        } else {
            svd3(Zt, s, Us, Vs);
            red[0] = E.vol[e] * NH<double>{mat.mu, mat.lambda}.psi_plain(double(s[0]), double(s[1]), double(s[2]));
        }
    }
    seg_reduce_out<1>(red, T, tl.mesh, partials, counters, out, stride);
}

// Candidate weights of midupdate_weights (src/TetElements.cpp:360-388): from
// F(X) (from_x = 1) or from the cached singular values.
static __global__ void __launch_bounds__(128) k_mid_candidates(ElemView E, Tiles T, const int* on,
                                                        const double* __restrict__ x, const double* __restrict__ xfix,
                                                        Material mat0, int from_x, int cand_mode) {
    const Tile tl = tile_at(T, blockIdx.x);
    if (!mesh_on(on, tl.mesh)) return;
    const int e = tl.first + threadIdx.x;
    if (e >= tl.end) return;
    const Material mat = elem_material(E, mat0, e);
    double s[3];
    if (from_x) {
        double Fd[9];
        deformation(E, e, x, xfix, false, Fd);
        double F[9], st[3], Us[9], Vs[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) F[i] = double(Fd[i]);
        svd3(F, st, Us, Vs);
        s[0] = st[0]; s[1] = st[1]; s[2] = st[2];
    } else {
#pragma unroll
        for (int i = 0; i < 3; ++i) s[i] = double(E.sig[(size_t)i * E.ne + e]);
    }
    const double vol = E.vol[e];
    if (cand_mode == CAND_HESSIAN) {
        const double lm = NH<double>{mat.mu, mat.lambda}.hess_lmax(s);
        double c = lm;
        if (lm < mat.wmin) c = mat.wmin;
        if (lm > mat.wmax) c = mat.wmax;
        E.w2c[e] = vol * c;
    } else {
        E.w2c[e] = vol * mat.wr;
    }
}

// max_wsq_ratio (src/Elements.hpp:56-69): out[0] = max_e max(w2/w2c, w2c/w2).
// Per mesh (System::possibly_update_weights takes the max over its own elements).
static __global__ void __launch_bounds__(256) k_ratio(ElemView E, Tiles T, const int* on, double* partials,
                                               unsigned* counters, double* out, int stride) {
    const Tile tl = tile_at(T, blockIdx.x);
    if (!mesh_on(on, tl.mesh)) return;
    const int e = tl.first + threadIdx.x;
    double red[1] = {0.0};
    if (e < tl.end) {
        const double a = E.w2[e] / E.w2c[e], b = 1.0 / a;
        red[0] = fmax(a, b);
    }
    seg_reduce_out<1, true>(red, T, tl.mesh, partials, counters, out, stride);
}

// update_actual_weights (src/TetElements.cpp:435-442), on the meshes that reweight.
static __global__ void __launch_bounds__(256) k_apply_weights(ElemView E, Tiles T, const int* on) {
    const Tile tl = tile_at(T, blockIdx.x);
    if (!mesh_on(on, tl.mesh)) return;
    const int e = tl.first + threadIdx.x;
    if (e >= tl.end) return;
    const double r = E.w2[e] / E.w2c[e];
#pragma unroll
    for (int k = 0; k < 9; ++k) E.U[(size_t)k * E.ne + e] = r * E.U[(size_t)k * E.ne + e];
    E.w2[e] = E.w2c[e];
}

// ---- global-step vector kernels (n x 3 FP64, dissection order) ----------------
// Tiles of kVecTile doubles of one mesh's range (thread t takes entries t,
// t + 256, ...).  The two-loop recursion of SplitLBFGS::minimize
// (SplitLBFGS.hpp:152-177) runs as a chain of steps, each an axpy and an inner
// product per mesh; every mesh walks its own history length `it`:
//   first loop, step j = it-1 .. 0: q = g (j = it-1) or q -= alpha_{j+1} y_{j+1};
//     alpha_j = rho_j <s_j, q>;  step -1: q -= alpha_0 y_0 (q = g when it = 0);
//   second loop, step j = 0 .. it-1: q += c_{j-1} s_{j-1} (j > 0);
//     c_j = alpha_j - rho_j <y_j, q>;  step it: q += c_{it-1} s_{it-1};
//     dir = <g, q>.
// A launch serves one step index j for every mesh; meshes whose walk has no
// step j return.  alpha_j, c_j and dir are per mesh in the scalar block
// (scal + mesh * stride + S_ALPHA / S_C / S_DIR).
constexpr int kVecTile = 2048;


static __global__ void __launch_bounds__(256) k_lbfgs_first(Tiles T, const int* on, const MeshCtl* __restrict__ ctl,
                                                     VecPools P, const double* __restrict__ rho,
                                                     double* __restrict__ q, int j, TwoLoopSlots sl, double* partials,
                                                     unsigned* counters, double* scal, int stride) {
    const Tile tl = tile_at(T, blockIdx.x);
    if (!mesh_on(on, tl.mesh)) return;
    const MeshCtl c = ctl[tl.mesh];
    if (j >= c.it || (j == -1 && false)) return;
    double* sc = scal + (size_t)tl.mesh * stride;
    const bool first = j == c.it - 1;                  // q = g (also j = -1 with it = 0)
    const double* g = g_cur(P, c);
    const double* yv = first ? nullptr : P.Y[hist_slot(c, j + 1, P.M)];
    const double cf = first ? 0.0 : -__ldcg(sc + sl.alpha + j + 1);
    const double* sv = j >= 0 ? P.S[hist_slot(c, j, P.M)] : nullptr;
    double red[1] = {0.0};
    for (int i = tl.first + (int)threadIdx.x; i < tl.end; i += blockDim.x) {
        double qi = first ? g[i] : q[i];
        if (yv) qi = qi + cf * yv[i];
        q[i] = qi;
        if (sv) red[0] += sv[i] * qi;
    }
    if (j < 0) return;
    double tot[1];
    if (seg_reduce<1>(red, T, tl.mesh, partials, counters, tot) && threadIdx.x == 0)
        sc[sl.alpha + j] = rho[(size_t)tl.mesh * kHistSlots + hist_slot(c, j, P.M)] * tot[0];
}

static __global__ void __launch_bounds__(256) k_lbfgs_second(Tiles T, const int* on, const MeshCtl* __restrict__ ctl,
                                                      VecPools P, const double* __restrict__ rho,
                                                      double* __restrict__ q, int j, TwoLoopSlots sl, double* partials,
                                                      unsigned* counters, double* scal, int stride) {
    const Tile tl = tile_at(T, blockIdx.x);
    if (!mesh_on(on, tl.mesh)) return;
    const MeshCtl c = ctl[tl.mesh];
    if (j > c.it) return;
    double* sc = scal + (size_t)tl.mesh * stride;
    const double* sv = j > 0 ? P.S[hist_slot(c, j - 1, P.M)] : nullptr;
    const double cf = j > 0 ? __ldcg(sc + sl.c + j - 1) : 0.0;
    const double* w = j < c.it ? P.Y[hist_slot(c, j, P.M)] : g_cur(P, c);
    double red[1] = {0.0};
    for (int i = tl.first + (int)threadIdx.x; i < tl.end; i += blockDim.x) {
        double qi = q[i];
        if (sv) {
            qi = qi + cf * sv[i];
            q[i] = qi;
        }
        red[0] += w[i] * qi;
    }
    double tot[1];
    if (seg_reduce<1>(red, T, tl.mesh, partials, counters, tot) && threadIdx.x == 0) {
        if (j < c.it)
            sc[sl.c + j] = __ldcg(sc + sl.alpha + j) + (-rho[(size_t)tl.mesh * kHistSlots + hist_slot(c, j, P.M)]) * tot[0];
        else
            sc[sl.dir] = tot[0];
    }
}

// ---- the two-loop recursion in one cooperative launch per loop (one mesh) ---------
// For a single mesh above the one-CTA size the M + 1 steps of each loop are
// the k_lbfgs_first / k_lbfgs_second steps above, run by one cooperative launch
// (all CTAs resident): CTA b takes vector tiles b, b + G, ... and keeps them
// for the whole loop, each step's inner product is the same per-tile block sum
// in partials (two buffers, alternating by step), and after a grid barrier
// every CTA adds the tile partials in the seg_reduce order -- the same alpha_i,
// c_i and decrement as the per-step launches, bit for bit, in every CTA.  The
// barrier is a counter the CTAs raise, waited on with wait_count_geq (bounded;
// a wait that gives up leaves WRAPD_E_TIMEOUT in *status and the CTA returns).
// REG (when the grid has a CTA per tile at the register form's occupancy):
// a CTA's kTwoLoopPT entries per thread stay in registers for the whole loop,
// q is stored once at the end, and the two history vectors of the next step
// (which do not change during the loop) are loaded before the grid barrier, so
// no step waits on a memory round trip after its barrier.  The per-entry
// operations and the order of every sum are those of the tile loop.
constexpr int kTwoLoopGridThreads = 256;
constexpr int kTwoLoopPT = kVecTile / kTwoLoopGridThreads;
static_assert(kVecTile % kTwoLoopGridThreads == 0, "whole entries per thread");
__device__ __forceinline__ bool grid_barrier(unsigned* bar, unsigned target, int* status) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(bar, 1u);
        ok = wait_count_geq(bar, target, status) ? 1 : 0;
    }
    __syncthreads();
    return ok != 0;
}

// The total over the mesh's tiles of partials[] in seg_reduce's order (every thread gets it).
__device__ __forceinline__ double grid_total(const double* partials, int ntiles) {
    __shared__ double sm[32];
    __shared__ double total;
    double acc = 0.0;
    for (int b = threadIdx.x; b < ntiles; b += blockDim.x) acc += __ldcg(partials + b);
    const double r = block_sum(acc, sm);
    if (threadIdx.x == 0) total = r;
    __syncthreads();
    return total;
}

template <bool SECOND, bool REG>
static __global__ void __launch_bounds__(kTwoLoopGridThreads) k_two_loop_grid(Tiles T, const MeshCtl* __restrict__ ctl, VecPools P,
                                                       const double* __restrict__ rho, double* __restrict__ q,
                                                       TwoLoopSlots sl, double* partials, unsigned* bar,
                                                       int* status, double* scal) {
    __shared__ double sm[32];
    const MeshCtl c = ctl[0];
    const int ntiles = T.count, G = gridDim.x;
    unsigned nbar = 0;
    if constexpr (REG) {
        // one tile per CTA (the host launches REG only with ntiles <= G), kept in registers
        const int t = blockIdx.x;
        const Tile tl = t < ntiles ? tile_at(T, t) : Tile{0, 0, 0};
        const int i0 = tl.first + (int)threadIdx.x;
        double qv[kTwoLoopPT], av[kTwoLoopPT], bv[kTwoLoopPT];
        auto load = [&](double (&v)[kTwoLoopPT], const double* src) {
#pragma unroll
            for (int k = 0; k < kTwoLoopPT; ++k) {
                const int i = i0 + k * kTwoLoopGridThreads;
                v[k] = (src && i < tl.end) ? src[i] : 0.0;
            }
        };
        auto store_q = [&]() {
#pragma unroll
            for (int k = 0; k < kTwoLoopPT; ++k) {
                const int i = i0 + k * kTwoLoopGridThreads;
                if (i < tl.end) q[i] = qv[k];
            }
        };
        if constexpr (!SECOND) {
            // av: y_{j+1} (the update), bv: s_j (the inner product) of step j
            double alpha_next = 0.0;
            load(qv, g_cur(P, c));
            load(bv, c.it - 1 >= 0 ? P.S[hist_slot(c, c.it - 1, P.M)] : nullptr);
            for (int j = c.it - 1; j >= -1; --j) {
                const bool first = j == c.it - 1;
                const double cf = first ? 0.0 : -alpha_next;
                double red = 0.0;
#pragma unroll
                for (int k = 0; k < kTwoLoopPT; ++k) {
                    if (i0 + k * kTwoLoopGridThreads < tl.end) {
                        double qi = qv[k];
                        if (!first) qi = qi + cf * av[k];
                        qv[k] = qi;
                        if (j >= 0) red += bv[k] * qi;
                    }
                }
                if (j < 0) break;
                double* part = partials + (size_t)(j & 1) * ntiles;
                const double r = block_sum(red, sm);
                if (threadIdx.x == 0 && t < ntiles) part[t] = r;
                load(av, P.Y[hist_slot(c, j, P.M)]);
                load(bv, j - 1 >= 0 ? P.S[hist_slot(c, j - 1, P.M)] : nullptr);
                nbar += G;
                if (!grid_barrier(bar, nbar, status)) return;
                alpha_next = rho[hist_slot(c, j, P.M)] * grid_total(part, ntiles);
                if (blockIdx.x == 0 && threadIdx.x == 0) scal[sl.alpha + j] = alpha_next;
            }
            store_q();
        } else {
            // av: s_{j-1} (the update), bv: y_j or g (the inner product) of step j
            double c_prev = 0.0;
            load(qv, q);
            load(bv, 0 < c.it ? P.Y[hist_slot(c, 0, P.M)] : g_cur(P, c));
            for (int j = 0; j <= c.it; ++j) {
                const double cf = j > 0 ? c_prev : 0.0;
                double red = 0.0;
#pragma unroll
                for (int k = 0; k < kTwoLoopPT; ++k) {
                    if (i0 + k * kTwoLoopGridThreads < tl.end) {
                        double qi = qv[k];
                        if (j > 0) {
                            qi = qi + cf * av[k];
                            qv[k] = qi;
                        }
                        red += bv[k] * qi;
                    }
                }
                double* part = partials + (size_t)(j & 1) * ntiles;
                const double r = block_sum(red, sm);
                if (threadIdx.x == 0 && t < ntiles) part[t] = r;
                if (j < c.it) {
                    load(av, P.S[hist_slot(c, j, P.M)]);
                    load(bv, j + 1 < c.it ? P.Y[hist_slot(c, j + 1, P.M)] : g_cur(P, c));
                }
                nbar += G;
                if (!grid_barrier(bar, nbar, status)) return;
                const double tot = grid_total(part, ntiles);
                if (j < c.it) {
                    c_prev = __ldcg(scal + sl.alpha + j) + (-rho[hist_slot(c, j, P.M)]) * tot;
                    if (blockIdx.x == 0 && threadIdx.x == 0) scal[sl.c + j] = c_prev;
                } else if (blockIdx.x == 0 && threadIdx.x == 0) {
                    scal[sl.dir] = tot;
                }
            }
            store_q();
        }
        return;
    } else if constexpr (!SECOND) {
        // first loop, j = it - 1 .. -1: q = (first ? g : q) - alpha_{j+1} y_{j+1}; alpha_j = rho_j <s_j, q>
        double alpha_next = 0.0;
        for (int j = c.it - 1; j >= -1; --j) {
            const bool first = j == c.it - 1;
            const double* g = g_cur(P, c);
            const double* yv = first ? nullptr : P.Y[hist_slot(c, j + 1, P.M)];
            const double cf = first ? 0.0 : -alpha_next;
            const double* sv = j >= 0 ? P.S[hist_slot(c, j, P.M)] : nullptr;
            double* part = partials + (size_t)(j & 1) * ntiles;
            for (int t = blockIdx.x; t < ntiles; t += G) {
                const Tile tl = tile_at(T, t);
                double red = 0.0;
                for (int i = tl.first + (int)threadIdx.x; i < tl.end; i += blockDim.x) {
                    double qi = first ? g[i] : q[i];
                    if (yv) qi = qi + cf * yv[i];
                    q[i] = qi;
                    if (sv) red += sv[i] * qi;
                }
                if (j >= 0) {
                    const double r = block_sum(red, sm);
                    if (threadIdx.x == 0) part[t] = r;
                }
            }
            if (j < 0) break;
            nbar += G;
            if (!grid_barrier(bar, nbar, status)) return;
            alpha_next = rho[hist_slot(c, j, P.M)] * grid_total(part, ntiles);
            if (blockIdx.x == 0 && threadIdx.x == 0) scal[sl.alpha + j] = alpha_next;
        }
    } else {
        // second loop, j = 0 .. it: q += c_{j-1} s_{j-1}; c_j = alpha_j - rho_j <y_j, q>, dir = <g, q>
        double c_prev = 0.0;
        for (int j = 0; j <= c.it; ++j) {
            const double* sv = j > 0 ? P.S[hist_slot(c, j - 1, P.M)] : nullptr;
            const double cf = j > 0 ? c_prev : 0.0;
            const double* w = j < c.it ? P.Y[hist_slot(c, j, P.M)] : g_cur(P, c);
            double* part = partials + (size_t)(j & 1) * ntiles;
            for (int t = blockIdx.x; t < ntiles; t += G) {
                const Tile tl = tile_at(T, t);
                double red = 0.0;
                for (int i = tl.first + (int)threadIdx.x; i < tl.end; i += blockDim.x) {
                    double qi = q[i];
                    if (sv) {
                        qi = qi + cf * sv[i];
                        q[i] = qi;
                    }
                    red += w[i] * qi;
                }
                const double r = block_sum(red, sm);
                if (threadIdx.x == 0) part[t] = r;
            }
            nbar += G;
            if (!grid_barrier(bar, nbar, status)) return;
            const double tot = grid_total(part, ntiles);
            if (j < c.it) {
                c_prev = __ldcg(scal + sl.alpha + j) + (-rho[hist_slot(c, j, P.M)]) * tot;
                if (blockIdx.x == 0 && threadIdx.x == 0) scal[sl.c + j] = c_prev;
            } else if (blockIdx.x == 0 && threadIdx.x == 0) {
                scal[sl.dir] = tot;
            }
        }
    }
}

// ---- the two-loop recursion in one CTA per mesh, for small meshes -----------------
// With 3 x free vertices <= kTwoLoopMaxN the chain of short reductions above is
// latency-bound: one 1024-thread CTA per mesh runs each half of the
// recursion, q in registers (kTwoLoopPerThread entries per thread), each inner
// product a block sum in a fixed order.  Same formulas and the same alpha_i,
// c_i and decrement slots.  Block b serves mesh b (meshes that are off or not
// small return).
constexpr int kTwoLoopThreads = 1024;
constexpr int kTwoLoopPerThread = 16;
constexpr int kTwoLoopMaxN = kTwoLoopThreads * kTwoLoopPerThread;

__device__ __forceinline__ double cta_sum_all(double v, double* sm) {
    __shared__ double total;
    const double r = block_sum(v, sm);
    if (threadIdx.x == 0) total = r;
    __syncthreads();
    return total;
}

// First loop (SplitLBFGS.hpp:152-158): q = g; for i = it-1 .. 0:
// alpha_i = rho_i <s_i, q>, q -= alpha_i y_i.
static __global__ void __launch_bounds__(kTwoLoopThreads) k_two_loop_first(const int* on, const MeshCtl* __restrict__ ctl,
                                                                           VecPools P, const double* __restrict__ rho,
                                                                           double* __restrict__ q, TwoLoopSlots sl,
                                                                           double* scal, int stride) {
    const int m = blockIdx.x;
    const MeshCtl c = ctl[m];
    if (!mesh_on(on, m) || !c.small) return;
    __shared__ double sm[32];
    const int n = c.v1 - c.v0;
    const double* g = g_cur(P, c) + c.v0;
    double* qm = q + c.v0;
    double* alpha = scal + (size_t)m * stride + sl.alpha;
    double qr[kTwoLoopPerThread];
#pragma unroll
    for (int k = 0; k < kTwoLoopPerThread; ++k) {
        const int i = threadIdx.x + k * kTwoLoopThreads;
        qr[k] = i < n ? g[i] : 0.0;
    }
    for (int h = c.it - 1; h >= 0; --h) {
        const int hs = hist_slot(c, h, P.M);
        const double* sp = P.S[hs] + c.v0;
        const double* yp = P.Y[hs] + c.v0;
        double d = 0.0;
#pragma unroll
        for (int k = 0; k < kTwoLoopPerThread; ++k) {
            const int i = threadIdx.x + k * kTwoLoopThreads;
            if (i < n) d += sp[i] * qr[k];
        }
        const double a = rho[(size_t)m * kHistSlots + hs] * cta_sum_all(d, sm);
        if (threadIdx.x == 0) alpha[h] = a;
#pragma unroll
        for (int k = 0; k < kTwoLoopPerThread; ++k) {
            const int i = threadIdx.x + k * kTwoLoopThreads;
            if (i < n) qr[k] = qr[k] + (-a) * yp[i];
        }
    }
#pragma unroll
    for (int k = 0; k < kTwoLoopPerThread; ++k) {
        const int i = threadIdx.x + k * kTwoLoopThreads;
        if (i < n) qm[i] = qr[k];
    }
}

// Second loop (SplitLBFGS.hpp:170-173) after q = A^-1 q: for i = 0 .. it-1:
// c_i = alpha_i - rho_i <y_i, q>, q += c_i s_i; then dir = <g, q>.
static __global__ void __launch_bounds__(kTwoLoopThreads) k_two_loop_second(const int* on, const MeshCtl* __restrict__ ctl,
                                                                            VecPools P, const double* __restrict__ rho,
                                                                            double* __restrict__ q, TwoLoopSlots sl,
                                                                            double* scal, int stride) {
    const int m = blockIdx.x;
    const MeshCtl c = ctl[m];
    if (!mesh_on(on, m) || !c.small) return;
    __shared__ double sm[32];
    const int n = c.v1 - c.v0;
    const double* g = g_cur(P, c) + c.v0;
    double* qm = q + c.v0;
    double* sc = scal + (size_t)m * stride;
    double qr[kTwoLoopPerThread];
#pragma unroll
    for (int k = 0; k < kTwoLoopPerThread; ++k) {
        const int i = threadIdx.x + k * kTwoLoopThreads;
        qr[k] = i < n ? qm[i] : 0.0;
    }
    for (int h = 0; h < c.it; ++h) {
        const int hs = hist_slot(c, h, P.M);
        const double* sp = P.S[hs] + c.v0;
        const double* yp = P.Y[hs] + c.v0;
        double d = 0.0;
#pragma unroll
        for (int k = 0; k < kTwoLoopPerThread; ++k) {
            const int i = threadIdx.x + k * kTwoLoopThreads;
            if (i < n) d += yp[i] * qr[k];
        }
        const double cc = sc[sl.alpha + h] + (-rho[(size_t)m * kHistSlots + hs]) * cta_sum_all(d, sm);
        if (threadIdx.x == 0) sc[sl.c + h] = cc;
#pragma unroll
        for (int k = 0; k < kTwoLoopPerThread; ++k) {
            const int i = threadIdx.x + k * kTwoLoopThreads;
            if (i < n) qr[k] = qr[k] + cc * sp[i];
        }
    }
    double d = 0.0;
#pragma unroll
    for (int k = 0; k < kTwoLoopPerThread; ++k) {
        const int i = threadIdx.x + k * kTwoLoopThreads;
        if (i < n) {
            qm[i] = qr[k];
            d += g[i] * qr[k];
        }
    }
    const double dd = cta_sum_all(d, sm);
    if (threadIdx.x == 0) sc[sl.dir] = dd;
}

// x <- x - rate * step with step = q, or grad when the mesh's decrement
// dir <= 0 (the steepest-descent restart of SplitLBFGS.hpp:189-194);
// s = x_new - x_old into the mesh's stage slot.  rate is 1 unless the global
// line search chose another (SplitLBFGS.hpp:196-206).
static __global__ void __launch_bounds__(256) k_xupdate(Tiles T, const int* on, const MeshCtl* __restrict__ ctl,
                                                 VecPools P, double* __restrict__ x, const double* __restrict__ q,
                                                 const double* scal, int dir_slot, int stride, double rate) {
    const Tile tl = tile_at(T, blockIdx.x);
    if (!mesh_on(on, tl.mesh)) return;
    const MeshCtl c = ctl[tl.mesh];
    const bool restart = !(__ldcg(scal + (size_t)tl.mesh * stride + dir_slot) > 0.0);
    const double* grad = g_cur(P, c);
    double* s = P.S[c.stage];
    for (int i = tl.first + (int)threadIdx.x; i < tl.end; i += blockDim.x) {
        const double xo = x[i];
        const double xn = xo - rate * (restart ? grad[i] : q[i]);
        s[i] = xn - xo;
        x[i] = xn;
    }
}

// grad_old = 0 (SplitLBFGS keeps grad_old across ADMM iterations and zeroes
// it with the history, SplitLBFGS.hpp:118-121) on the meshes that are on.
static __global__ void __launch_bounds__(256) k_zero_old(Tiles T, const int* on, const MeshCtl* __restrict__ ctl,
                                                  VecPools P) {
    const Tile tl = tile_at(T, blockIdx.x);
    if (!mesh_on(on, tl.mesh)) return;
    double* g = g_old(P, ctl[tl.mesh]);
    for (int i = tl.first + (int)threadIdx.x; i < tl.end; i += blockDim.x) g[i] = 0.0;
}

// Per mesh |x - xs|^2 (the x error of AlgorithmData::update_per_iter_data).
static __global__ void __launch_bounds__(256) k_xerr(Tiles T, const int* on, const double* __restrict__ x,
                                              const double* __restrict__ xs, double* partials, unsigned* counters,
                                              double* out, int stride) {
    const Tile tl = tile_at(T, blockIdx.x);
    if (!mesh_on(on, tl.mesh)) return;
    double red[1] = {0.0};
    for (int i = tl.first + (int)threadIdx.x; i < tl.end; i += blockDim.x) {
        const double d = x[i] - xs[i];
        red[0] += d * d;
    }
    seg_reduce_out<1>(red, T, tl.mesh, partials, counters, out, stride);
}

// Inputs of the global line search (Backtracking::search,
// deps/mcloptlib/include/MCL/Backtracking.hpp:71-98): out[0] = <q, q>,
// out[1] = <grad, grad> (sums); then, in k_ls_gmax, out[0] = max |grad|.
static __global__ void __launch_bounds__(256) k_ls_norms(int n, const double* __restrict__ q,
                                                  const double* __restrict__ grad, double* partials,
                                                  unsigned* counter, double* out) {
    double red[2] = {0.0, 0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        red[0] += q[i] * q[i];
        red[1] += grad[i] * grad[i];
    }
    grid_reduce<2>(red, partials, counter, out);
}

static __global__ void __launch_bounds__(256) k_ls_gmax(int n, const double* __restrict__ grad, double* partials,
                                                 unsigned* counter, double* out) {
    double red[1] = {0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        red[0] = fmax(red[0], fabs(grad[i]));
    grid_reduce<1, true>(red, partials, counter, out);
}

// Trial point of the line search: xt = x + alpha * p with p = -step.
static __global__ void __launch_bounds__(256) k_ls_trial(int n, double* __restrict__ xt, const double* __restrict__ x,
                                                  const double* __restrict__ step, double alpha) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        xt[i] = x[i] + alpha * -step[i];
}

// ---- ARAP local step (rotation-aware) ------------------------------------------
// polar_update, ARAP branch (src/TetElements.cpp:265-282): S = symF + U (both
// symmetric), Z = (S + I) / 2, U += symF - Z; curr_pe = sum vol |symF - I|^2 / 2.
// out[0..4] as k_local (no prox: [3] = [4] = 0).
static __global__ void __launch_bounds__(128) k_local_arap(ElemView E, Tiles T, const int* on, double* partials,
                                                         unsigned* counters, double* out, int stride) {
    const Tile tl = tile_at(T, blockIdx.x);
    if (!mesh_on(on, tl.mesh)) return;
    const int e = tl.first + threadIdx.x;
    double red[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (e < tl.end) {
        double S[9], Um[9], Zm[9];
        load9(E.symF, E.ne, e, S);
        load9(E.U, E.ne, e, Um);
        load9(E.Z, E.ne, e, Zm);
        const double w2 = E.w2[e], vol = E.vol[e];
        double bef = 0.0, aft = 0.0, n2 = 0.0;
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            const double d = S[i] - (Zm[i] - Um[i]);
            bef += d * d;
        }
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            const double id = (i % 4 == 0) ? 1.0 : 0.0;
            const double So = 0.5 * ((S[i] + Um[i]) + id);
            n2 += (S[i] - id) * (S[i] - id);
            const double d = S[i] - (So - Um[i]);
            aft += d * d;
            Zm[i] = So;
            Um[i] = Um[i] + (S[i] - So);
        }
        red[0] = 0.5 * w2 * bef;
        red[1] = 0.5 * w2 * aft;
        red[2] = 0.5 * vol * n2;
        store9(E.Z, E.ne, e, Zm);
        store9(E.U, E.ne, e, Um);
    }
    seg_reduce_out<5>(red, T, tl.mesh, partials, counters, out, stride);
}

// ---- rotation-unaware ADMM (-ra 0) -----------------------------------------------
// initialize_dual_vars, rotation-unaware branch (src/TetElements.cpp:167-181):
// Z = Di x = F^T with all four slots read from X, U = 0.
static __global__ void __launch_bounds__(128) k_init_dual_unaware(ElemView E, const double* __restrict__ x,
                                                                const double* __restrict__ xfix) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E.ne) return;
    double F[9], Zm[9], zero[9] = {};
    deformation(E, e, x, xfix, false, F);
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) M3(Zm, r, c) = F[c + 3 * r];
    store9(E.Z, E.ne, e, Zm);
    store9(E.U, E.ne, e, zero);
}

// TetElements::update (src/TetElements.cpp:193-254) from F at the current x
// (the defo cache): Dx = F^T, F' = (Dx + U)^T; NH: SVD of F', the prox from the
// last stretches, Z = V diag(sigma*) U^T; ARAP: Z = (F' + rot(F'))^T / 2; then
// U += Dx - Z.  C: arithmetic of the SVD and prox as in k_local (float in mixed
// mode, with the same FP64 rescue).  out[0..4] = 0, 0, 0, negative stretches,
// prox iterations.
template <typename C>
__global__ void __launch_bounds__(128, 4) k_local_unaware(ElemView E, const double* __restrict__ x,
                                                       const double* __restrict__ xfix, Material mat0, int prox_iters,
                                                       int cand_mode, int prox_mode, double* partials,
                                                       unsigned* counter, double* out) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    double red[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (e < E.ne) {
        const Material mat = elem_material(E, mat0, e);
        double F[9], Um[9], Zn[9];
        deformation(E, e, x, xfix, true, F);
        load9(E.U, E.ne, e, Um);
        C Fp[9];
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c) M3(Fp, r, c) = C(F[r + 3 * c] + M3(Um, c, r));   // (F^T + U)^T
        C sg[3], Ue[9], Ve[9];
        svd3(Fp, sg, Ue, Ve);
        if (mat.model == MODEL_ARAP) {
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    // rot(F') = Ue Ve^T; Z(r, c) = (F'(c, r) + R(c, r)) / 2
                    const double Rcr = double(M3(Ue, c, 0) * M3(Ve, r, 0) + M3(Ue, c, 1) * M3(Ve, r, 1) +
                                              M3(Ue, c, 2) * M3(Ve, r, 2));
                    M3(Zn, r, c) = 0.5 * (double(M3(Fp, c, r)) + Rcr);
                }
        } else {
            const double w2 = E.w2[e], vol = E.vol[e];
            Prox<C> P;
            P.nh.mu = C(mat.mu);
            P.nh.lambda = C(mat.lambda);
            P.x0[0] = sg[0]; P.x0[1] = sg[1]; P.x0[2] = sg[2];
            P.wov = C(w2 / vol);
            C xs[3];
#pragma unroll
            for (int i = 0; i < 3; ++i) xs[i] = C(E.slast[(size_t)i * E.ne + e]);
            int iters;
            if constexpr (sizeof(C) == sizeof(double)) {
                if (prox_mode != 0) {
                    iters = prox_newton(P, xs, prox_iters, C(1e-12));
                } else {
                    extern __shared__ double prox_hist[];
                    iters = prox_lbfgs(P, xs, prox_iters, ProxHistory<double>{prox_hist + threadIdx.x, (int)blockDim.x});
                    if (iters < 0) iters = prox_iters;
                }
            } else {
                iters = prox_newton(P, xs, prox_iters, C(8) * Lim<C>::eps());
                if (!(isfinite(xs[0]) && isfinite(xs[1]) && isfinite(xs[2]) && xs[0] >= C(0) && xs[1] >= C(0) &&
                      xs[2] >= C(0))) {
                    Prox<double> Pd;
                    Pd.nh.mu = mat.mu;
                    Pd.nh.lambda = mat.lambda;
                    Pd.x0[0] = double(sg[0]); Pd.x0[1] = double(sg[1]); Pd.x0[2] = double(sg[2]);
                    Pd.wov = w2 / vol;
                    double xd[3];
#pragma unroll
                    for (int i = 0; i < 3; ++i) xd[i] = E.slast[(size_t)i * E.ne + e];
                    iters += prox_newton(Pd, xd, prox_iters, 1e-12);
#pragma unroll
                    for (int i = 0; i < 3; ++i) xs[i] = C(xd[i]);
                }
            }
            red[4] = double(iters);
            double xo[3];
#pragma unroll
            for (int i = 0; i < 3; ++i) { xo[i] = double(xs[i]); E.slast[(size_t)i * E.ne + e] = xo[i]; }
            red[3] = (xo[0] < 0.0 || xo[1] < 0.0 || xo[2] < 0.0) ? 1.0 : 0.0;
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    M3(Zn, r, c) = double(M3(Ve, r, 0) * xs[0] * M3(Ue, c, 0) + M3(Ve, r, 1) * xs[1] * M3(Ue, c, 1) +
                                          M3(Ve, r, 2) * xs[2] * M3(Ue, c, 2));
            if (cand_mode == CAND_REST) {
                E.w2c[e] = vol * mat.wr;
            } else if (cand_mode == CAND_HESSIAN) {
                const double lm = NH<double>{mat.mu, mat.lambda}.hess_lmax(xo);
                double cnd = lm;
                if (lm < mat.wmin) cnd = mat.wmin;
                if (lm > mat.wmax) cnd = mat.wmax;
                E.w2c[e] = vol * cnd;
            }
        }
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c) M3(Um, r, c) = M3(Um, r, c) + (F[c + 3 * r] - M3(Zn, r, c));
        store9(E.Z, E.ne, e, Zn);
        store9(E.U, E.ne, e, Um);
    }
    grid_reduce<5>(red, partials, counter, out);
}

// UnawareGS right-hand side per element (TetElements::add_to_b,
// src/TetElements.cpp:470-481): b_e(a, r) = w^2 sum_c Di(c, a) (Z - U - Dfix xfix)(c, r),
// into the gradient rows gel (the gather adds the free slots).
static __global__ void __launch_bounds__(128) k_rhs_unaware(ElemView E, const double* __restrict__ xfix) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E.ne) return;
    double Zm[9], Um[9], Ffix[9] = {};
    load9(E.Z, E.ne, e, Zm);
    load9(E.U, E.ne, e, Um);
    const int4 id = E.idx[e];
    const int s[4] = {id.x, id.y, id.z, id.w};
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        if (s[a] >= 0) continue;
        const double* p = xfix + 3 * (size_t)(-s[a] - 1);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double d = E.Di[(size_t)(c + 3 * a) * E.ne + e];
#pragma unroll
            for (int r = 0; r < 3; ++r) Ffix[c + 3 * r] += d * p[r];   // (Dfix xfix)(c, r)
        }
    }
    const double w2 = E.w2[e];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            double v = 0.0;
#pragma unroll
            for (int c = 0; c < 3; ++c)
                v += E.Di[(size_t)(c + 3 * a) * E.ne + e] * (M3(Zm, c, r) - M3(Um, c, r) - Ffix[c + 3 * r]);
            E.gel[(size_t)(r + 3 * a) * E.ne + e] = w2 * v;
        }
}

}  // namespace wrapd
