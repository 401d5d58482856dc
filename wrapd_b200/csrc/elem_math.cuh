// Per-element device math, in registers, templated on the arithmetic type
// (double for the FP64 path, float for the FP32 local step of mixed mode).
// 3x3 matrices are 9 scalars column-major: a[r + 3*c].
#pragma once
#include "common.cuh"

namespace wrapd {

#define M3(a, r, c) (a)[(r) + 3 * (c)]

template <typename T>
__device__ __forceinline__ T det3(const T* m) {
    return M3(m, 0, 0) * (M3(m, 1, 1) * M3(m, 2, 2) - M3(m, 1, 2) * M3(m, 2, 1)) -
           M3(m, 0, 1) * (M3(m, 1, 0) * M3(m, 2, 2) - M3(m, 1, 2) * M3(m, 2, 0)) +
           M3(m, 0, 2) * (M3(m, 1, 0) * M3(m, 2, 1) - M3(m, 1, 1) * M3(m, 2, 0));
}

// Two-sided Jacobi SVD of a 3x3 matrix with the rotation sign fix.  Restates
// Eigen 3.3.7 JacobiSVD::compute for square inputs (scale by the max |entry|,
// sweep the (1,0),(2,0),(2,1) pairs with real_2x2_jacobi_svd until every
// off-diagonal entry is below max(min_normal, 2 eps max|diag|), make the
// diagonal non-negative, sort descending), then wrapd's math::svd sign fix
// (src/Math.hpp:147-160): a reflection in U or V negates column 2 and sigma_2.
// The sweep loop is capped at 64 (Jacobi needs < 10 sweeps on finite 3x3
// input; the cap only bounds non-finite input).
template <typename T>
__device__ __forceinline__ void svd3(const T* A, T* sig, T* U, T* V) {
    T W[9];
    T scale = T(0);
#pragma unroll
    for (int i = 0; i < 9; ++i) scale = fmax(scale, fabs(A[i]));
    if (scale == T(0)) scale = T(1);
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        W[i] = A[i] / scale;
        U[i] = V[i] = (i % 4 == 0) ? T(1) : T(0);
    }
    const T prec = T(2) * Lim<T>::eps(), tiny = Lim<T>::min();
    T maxd = fmax(fabs(W[0]), fmax(fabs(W[4]), fabs(W[8])));
    bool finished = false;
    for (int sweep = 0; sweep < 64 && !finished; ++sweep) {
        finished = true;
#pragma unroll
        for (int p = 1; p < 3; ++p) {
#pragma unroll
            for (int q = 0; q < p; ++q) {
                const T thr = fmax(tiny, prec * maxd);
                if (fabs(M3(W, p, q)) > thr || fabs(M3(W, q, p)) > thr) {
                    finished = false;
                    const T m00 = M3(W, p, p), m01 = M3(W, p, q), m10 = M3(W, q, p), m11 = M3(W, q, q);
                    const T t = m00 + m11, d = m10 - m01;
                    T c1, s1;
                    if (fabs(d) < tiny) { s1 = T(0); c1 = T(1); }
                    else { const T u = t / d, tmp = sqrt(T(1) + u * u); s1 = T(1) / tmp; c1 = u / tmp; }
                    const T a00 = c1 * m00 + s1 * m10, a01 = c1 * m01 + s1 * m11;
                    const T a11 = -s1 * m01 + c1 * m11;
                    T cr, sr;
                    const T deno = T(2) * fabs(a01);
                    if (deno < tiny) { cr = T(1); sr = T(0); }
                    else {
                        const T tau = (a00 - a11) / deno, w = sqrt(tau * tau + T(1));
                        const T tt = tau > T(0) ? T(1) / (tau + w) : T(1) / (tau - w);
                        const T sgn = tt > T(0) ? T(1) : T(-1);
                        const T n = T(1) / sqrt(tt * tt + T(1));
                        sr = -sgn * (a01 / fabs(a01)) * fabs(tt) * n;
                        cr = n;
                    }
                    const T cl = c1 * cr + s1 * sr;
                    const T sl = -c1 * sr + s1 * cr;
#pragma unroll
                    for (int i = 0; i < 3; ++i) {
                        const T x = M3(W, p, i), y = M3(W, q, i);
                        M3(W, p, i) = cl * x + sl * y;
                        M3(W, q, i) = -sl * x + cl * y;
                    }
#pragma unroll
                    for (int i = 0; i < 3; ++i) {
                        const T x = M3(U, i, p), y = M3(U, i, q);
                        M3(U, i, p) = cl * x + sl * y;
                        M3(U, i, q) = -sl * x + cl * y;
                    }
#pragma unroll
                    for (int i = 0; i < 3; ++i) {
                        const T x = M3(W, i, p), y = M3(W, i, q);
                        M3(W, i, p) = cr * x - sr * y;
                        M3(W, i, q) = sr * x + cr * y;
                    }
#pragma unroll
                    for (int i = 0; i < 3; ++i) {
                        const T x = M3(V, i, p), y = M3(V, i, q);
                        M3(V, i, p) = cr * x - sr * y;
                        M3(V, i, q) = sr * x + cr * y;
                    }
                    maxd = fmax(maxd, fmax(fabs(M3(W, p, p)), fabs(M3(W, q, q))));
                }
            }
        }
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const T a = M3(W, i, i);
        sig[i] = fabs(a);
        if (a < T(0)) {
#pragma unroll
            for (int r = 0; r < 3; ++r) M3(U, r, i) = -M3(U, r, i);
        }
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) sig[i] *= scale;
    // selection sort, descending, first maximum wins (Eigen's maxCoeff)
    auto swapcol = [&](int i, int j) {
        T t = sig[i]; sig[i] = sig[j]; sig[j] = t;
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            t = M3(U, r, i); M3(U, r, i) = M3(U, r, j); M3(U, r, j) = t;
            t = M3(V, r, i); M3(V, r, i) = M3(V, r, j); M3(V, r, j) = t;
        }
    };
    {
        int pos = 0;
        T mx = sig[0];
        if (sig[1] > mx) { mx = sig[1]; pos = 1; }
        if (sig[2] > mx) { mx = sig[2]; pos = 2; }
        if (mx != T(0)) {
            if (pos == 1) swapcol(0, 1);
            else if (pos == 2) swapcol(0, 2);
            if (sig[2] > sig[1] && sig[2] != T(0)) swapcol(1, 2);
        }
    }
    if (det3(U) < T(0)) {
#pragma unroll
        for (int r = 0; r < 3; ++r) M3(U, r, 2) = -M3(U, r, 2);
        sig[2] = -sig[2];
    }
    if (det3(V) < T(0)) {
#pragma unroll
        for (int r = 0; r < 3; ++r) M3(V, r, 2) = -M3(V, r, 2);
        sig[2] = -sig[2];
    }
}

// ---- compressible Neo-Hookean with the extended log (J0 = 0.1) -------------
// src/TetElements.hpp:61-144; energies of src/TetElements.cpp:619-628.
template <typename T>
struct NH {
    T mu, lambda;
    static constexpr double J0 = 0.1;

    __device__ __forceinline__ T fJ_ext(T J) const {
        const T r = J / T(J0) - T(1);
        return log(T(J0)) + ((J - T(J0)) / T(J0)) - T(0.5) * r * r;
    }
    // energy density without the negative-stretch guard (energies)
    __device__ __forceinline__ T psi_plain(T x0, T x1, T x2) const {
        const T I1 = x0 * x0 + x1 * x1 + x2 * x2;
        const T J = x0 * x1 * x2;
        T e = T(0.5) * mu * (I1 - T(3));
        if (J > T(J0)) {
            const T lj = log(J);
            e += -mu * lj + T(0.5) * lambda * lj * lj;
        } else {
            const T fJ = fJ_ext(J);
            e += -mu * fJ + T(0.5) * lambda * fJ * fJ;
        }
        return e;
    }
    // NHProx::energy_density: 1e15 for a negative stretch
    __device__ __forceinline__ T psi(T x0, T x1, T x2) const {
        if (x0 < T(0) || x1 < T(0) || x2 < T(0)) return T(1.e15);
        return psi_plain(x0, x1, x2);
    }
    // gradient of the density (without the prox penalty)
    __device__ __forceinline__ void dpsi(const T* x, T* g) const {
        const T J = x[0] * x[1] * x[2];
        T f;
        if (J > T(J0)) {
            f = lambda * log(J) - mu;
        } else {
            const T fJ = fJ_ext(J);
            const T dfJdJ = T(1) / T(J0) - (J - T(J0)) / (T(J0) * T(J0));
            f = (lambda * fJ - mu) * dfJdJ * J;
        }
#pragma unroll
        for (int i = 0; i < 3; ++i) g[i] = mu * x[i] + f * (T(1) / x[i]);
    }
    // lambda_max of makePD(hessian_density(x)) = max(lambda_max(H), 0); the
    // PSD projection of src/Math.hpp:243-261 only zeroes negative eigenvalues.
    __device__ __forceinline__ T hess_lmax(const T* x) const;
    // hessian_density before the PSD projection (src/TetElements.hpp:109-142):
    // h = {h00, h11, h22, h01, h02, h12}
    __device__ __forceinline__ void hess(const T* x, T* h) const;
};

// Largest eigenvalue of a symmetric 3x3 (cyclic Jacobi, at most 12 sweeps).
template <typename T>
__device__ __forceinline__ T sym3_lmax(T a00, T a11, T a22, T a01, T a02, T a12) {
    T a[9] = {a00, a01, a02, a01, a11, a12, a02, a12, a22};
    for (int sweep = 0; sweep < 12; ++sweep) {
        const T off = M3(a, 0, 1) * M3(a, 0, 1) + M3(a, 0, 2) * M3(a, 0, 2) + M3(a, 1, 2) * M3(a, 1, 2);
        const T dn = M3(a, 0, 0) * M3(a, 0, 0) + M3(a, 1, 1) * M3(a, 1, 1) + M3(a, 2, 2) * M3(a, 2, 2);
        if (off <= T(1e-40) * dn || off == T(0)) break;
#pragma unroll
        for (int p = 0; p < 2; ++p)
#pragma unroll
            for (int q = p + 1; q < 3; ++q) {
                const T apq = M3(a, p, q);
                if (apq != T(0)) {
                    const T theta = (M3(a, q, q) - M3(a, p, p)) / (T(2) * apq);
                    const T t = (theta >= T(0) ? T(1) : T(-1)) / (fabs(theta) + sqrt(theta * theta + T(1)));
                    const T c = T(1) / sqrt(t * t + T(1)), s = t * c;
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        const T akp = M3(a, k, p), akq = M3(a, k, q);
                        M3(a, k, p) = c * akp - s * akq;
                        M3(a, k, q) = s * akp + c * akq;
                    }
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        const T apk = M3(a, p, k), aqk = M3(a, q, k);
                        M3(a, p, k) = c * apk - s * aqk;
                        M3(a, q, k) = s * apk + c * aqk;
                    }
                }
            }
    }
    return fmax(M3(a, 0, 0), fmax(M3(a, 1, 1), M3(a, 2, 2)));
}

template <typename T>
__device__ __forceinline__ void NH<T>::hess(const T* x, T* h) const {
    const T J = x[0] * x[1] * x[2];
    if (J > T(J0)) {
        const T lj = log(J);
        const T ct = mu - lambda * (lj - T(1));
        h[0] = mu + ct / (x[0] * x[0]);
        h[1] = mu + ct / (x[1] * x[1]);
        h[2] = mu + ct / (x[2] * x[2]);
        h[3] = lambda / (x[0] * x[1]);
        h[4] = lambda / (x[0] * x[2]);
        h[5] = lambda / (x[1] * x[2]);
    } else {
        const T fJ = fJ_ext(J);
        const T dfJdJ = T(1) / T(J0) - (J - T(J0)) / (T(J0) * T(J0));
        const T lfm = lambda * fJ - mu;
        const T a = x[1] * x[2], b = x[0] * x[2], c = x[0] * x[1];
        h[0] = mu - lfm * (a / T(J0)) * (a / T(J0)) + lambda * (dfJdJ * a) * (dfJdJ * a);
        h[1] = mu - lfm * (b / T(J0)) * (b / T(J0)) + lambda * (dfJdJ * b) * (dfJdJ * b);
        h[2] = mu - lfm * (c / T(J0)) * (c / T(J0)) + lambda * (dfJdJ * c) * (dfJdJ * c);
        const T ct = lfm * (dfJdJ - J / (T(J0) * T(J0))) + lambda * J * dfJdJ * dfJdJ;
        h[3] = x[2] * ct;
        h[4] = x[1] * ct;
        h[5] = x[0] * ct;
    }
}

template <typename T>
__device__ __forceinline__ T NH<T>::hess_lmax(const T* x) const {
    T h[6];
    hess(x, h);
    const T m = sym3_lmax(h[0], h[1], h[2], h[3], h[4], h[5]);
    return m > T(0) ? m : T(0);
}

// ---- the proximal stretch solve --------------------------------------------
// min_x psi(x) + (wov/2)|x - x0|^2 by LBFGS<3, M=8> with cubic-interpolating
// Armijo backtracking, restating deps/mcloptlib/include/MCL/LBFGS.hpp:52-152,
// Backtracking.hpp:268-332 and Prox::converged (src/TetElements.hpp:40-42).
// The history is kept in registers (fully unrolled, predicated loops); the
// line search is capped at 4096 trials instead of 100000 (the step shrinks by
// at least 2x per trial, so it underflows to zero long before).
template <typename T>
struct Prox {
    NH<T> nh;
    T x0[3];
    T wov;

    __device__ __forceinline__ T value(const T* x) const {
        const T d0 = x[0] - x0[0], d1 = x[1] - x0[1], d2 = x[2] - x0[2];
        return nh.psi(x[0], x[1], x[2]) + (wov * T(0.5)) * (d0 * d0 + d1 * d1 + d2 * d2);
    }
    // The value with its byproducts J = x0 x1 x2 and lf = log(J) (or the
    // extension fJ below J0): the same operations as value().
    __device__ __forceinline__ T value_lf(const T* x, T& J, T& lf) const {
        const T mu = nh.mu, lambda = nh.lambda;
        J = x[0] * x[1] * x[2];
        lf = J > T(NH<T>::J0) ? log(J) : nh.fJ_ext(J);
        T e;
        if (x[0] < T(0) || x[1] < T(0) || x[2] < T(0)) {
            e = T(1.e15);
        } else {
            const T I1 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
            e = T(0.5) * mu * (I1 - T(3));
            e += -mu * lf + T(0.5) * lambda * lf * lf;
        }
        const T d0 = x[0] - x0[0], d1 = x[1] - x0[1], d2 = x[2] - x0[2];
        return e + (wov * T(0.5)) * (d0 * d0 + d1 * d1 + d2 * d2);
    }
    // The gradient (dpsi plus the penalty's) from the J and lf of value_lf at
    // the same x.
    __device__ __forceinline__ void grad_lf(const T* x, T J, T lf, T* g) const {
        const T mu = nh.mu, lambda = nh.lambda;
        T f;
        if (J > T(NH<T>::J0)) {
            f = lambda * lf - mu;
        } else {
            const T dfJdJ = T(1) / T(NH<T>::J0) - (J - T(NH<T>::J0)) / (T(NH<T>::J0) * T(NH<T>::J0));
            f = (lambda * lf - mu) * dfJdJ * J;
        }
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            g[i] = mu * x[i] + f * (T(1) / x[i]);
            g[i] = g[i] + wov * (x[i] - x0[i]);
        }
    }
    // The gradient and the value together, log(J) taken once for both.
    __device__ __forceinline__ T value_grad(const T* x, T* g) const {
        T J, lf;
        const T e = value_lf(x, J, lf);
        grad_lf(x, J, lf, g);
        return e;
    }
};

template <typename T>
__device__ __forceinline__ T dot3(const T* a, const T* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

template <typename T>
__device__ __forceinline__ T cubic_step(T fx0, T gtp, T fxa, T alpha, T fxp, T alphap) {
    const T mult = T(1) / (alpha * alpha * alphap * alphap * (alpha - alphap));
    const T a00 = mult * (alphap * alphap), a01 = mult * (-alpha * alpha);
    const T a10 = mult * (-alphap * alphap * alphap), a11 = mult * (alpha * alpha * alpha);
    const T b0 = fxa - fx0 - alpha * gtp, b1 = fxp - fx0 - alphap * gtp;
    const T r0 = a00 * b0 + a01 * b1, r1 = a10 * b0 + a11 * b1;
    if (fabs(r0) <= T(0)) return -gtp / (T(2) * r1);
    const T d = sqrt(r1 * r1 - T(3) * r0 * gtp);
    return (-r1 + d) / (T(3) * r0);
}

// The value and the log term at the accepted point of a line search (valid
// only when the search evaluated a trial and accepted it).
template <typename T>
struct LsPoint {
    T f, J, lf;
    bool ok;
};

// fx0 and g: the objective and its gradient at x, which the callers already
// hold (the reference's search evaluates them again at the same x; the values
// are the same).  When acc is given, the value and the log term at the
// accepted trial point are stored there, so the caller's next gradient needs
// no second log.
template <typename T>
__device__ __forceinline__ T linesearch_cubic(const Prox<T>& P, const T* x, const T* p, T alpha0, T fx0, const T* g,
                                              int max_trials = 4096, LsPoint<T>* acc = nullptr) {
    if (sqrt(dot3(p, p)) <= Lim<T>::eps()) return T(1e-4);
    T alpha = alpha0;
    const T gtp = dot3(g, p);
    T fxp = fx0, alphap = alpha;
    for (int it = 0; it < max_trials; ++it) {
        const T xa[3] = {x[0] + alpha * p[0], x[1] + alpha * p[1], x[2] + alpha * p[2]};
        T J, lf;
        const T fxa = P.value_lf(xa, J, lf);
        if (fxa <= fx0 + alpha * T(1e-4) * gtp) {
            if (acc) {
                acc->f = fxa; acc->J = J; acc->lf = lf; acc->ok = true;
            }
            return alpha;
        }
        const T at = it == 0 ? (gtp / (T(2) * (fx0 + gtp - fxa))) : cubic_step(fx0, gtp, fxa, alpha, fxp, alphap);
        fxp = fxa;
        alphap = alpha;
        const T lo = T(0.1) * alpha, hi = T(0.5) * alpha;
        alpha = at < lo ? lo : (at > hi ? hi : at);
    }
    return T(-1);
}

// History of the 3-D L-BFGS: M pairs (s_i, y_i) kept outside registers, in a
// thread-private strided slice of shared memory (entry (i, c) of s at
// base[(6 i + c) * stride], of y at base[(6 i + 3 + c) * stride]); with the
// thread index as offset and the block size as stride, a warp's accesses fall
// in distinct banks.
template <typename T>
struct ProxHistory {
    T* base;
    int stride;
    __device__ __forceinline__ T& s(int i, int c) const { return base[(6 * i + c) * stride]; }
    __device__ __forceinline__ T& y(int i, int c) const { return base[(6 * i + 3 + c) * stride]; }
};

// Returns the iteration count (or -1 when the line search fails; x keeps the
// last iterate, as in the reference).
template <typename T>
__device__ __forceinline__ int prox_lbfgs(const Prox<T>& P, T* x, int max_iters, const ProxHistory<T>& H) {
    constexpr int M = 8;
    T alpha[M], rho[M];
    T grad[3], q[3], gold[3], xold[3];
    T fx = P.value_grad(x, grad);
    T gamma_k = T(1), alpha_init = T(1);
    int global_iter = 0;
    int head = 0;   // ring position of the oldest pair once the history is full
    for (int k = 0; k < max_iters; ++k) {
#pragma unroll
        for (int c = 0; c < 3; ++c) { xold[c] = x[c]; gold[c] = grad[c]; q[c] = grad[c]; }
        global_iter++;
        const int iter = k < M ? k : M;
        for (int i = iter - 1; i >= 0; --i) {
            const int slot = k < M ? i : (head + i) % M;
            const T s0 = H.s(slot, 0), s1 = H.s(slot, 1), s2 = H.s(slot, 2);
            const T y0 = H.y(slot, 0), y1 = H.y(slot, 1), y2 = H.y(slot, 2);
            const T r = T(1) / (s0 * y0 + s1 * y1 + s2 * y2);
            const T a = r * (s0 * q[0] + s1 * q[1] + s2 * q[2]);
            rho[i] = r;
            alpha[i] = a;
            q[0] = q[0] - a * y0; q[1] = q[1] - a * y1; q[2] = q[2] - a * y2;
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) q[c] = gamma_k * q[c];
        for (int i = 0; i < iter; ++i) {
            const int slot = k < M ? i : (head + i) % M;
            const T beta = rho[i] * (q[0] * H.y(slot, 0) + q[1] * H.y(slot, 1) + q[2] * H.y(slot, 2));
            const T cf = alpha[i] - beta;
            q[0] = q[0] + cf * H.s(slot, 0); q[1] = q[1] + cf * H.s(slot, 1); q[2] = q[2] + cf * H.s(slot, 2);
        }
        const T dir = dot3(q, grad);
        if (dir <= T(0)) {
#pragma unroll
            for (int c = 0; c < 3; ++c) q[c] = grad[c];
            max_iters -= k;
            k = 0;
            head = 0;
            const T ninf = fmax(fabs(grad[0]), fmax(fabs(grad[1]), fabs(grad[2])));
            alpha_init = fmin(T(1), T(1) / ninf);
        }
        const T mq[3] = {-q[0], -q[1], -q[2]};
        LsPoint<T> acc;
        acc.ok = false;
        const T rate = linesearch_cubic(P, x, mq, alpha_init, fx, grad, 4096, &acc);
        if (rate <= T(0)) return -1;
        T xl[3];
        // x - rate q is the accepted trial point x + rate (-q), bit for bit
        // (one rounding each, a fused multiply-add)
#pragma unroll
        for (int c = 0; c < 3; ++c) { xl[c] = x[c]; x[c] -= rate * q[c]; }
        {
            const T dx[3] = {xl[0] - x[0], xl[1] - x[1], xl[2] - x[2]};
            if (sqrt(dot3(grad, grad)) < T(1e-8) || sqrt(dot3(dx, dx)) < T(1e-8)) break;
        }
        if (acc.ok) {   // the search's value and log term at this x
            fx = acc.f;
            P.grad_lf(x, acc.J, acc.lf, grad);
        } else {
            fx = P.value_grad(x, grad);
        }
        T st[3], yt[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) { st[c] = x[c] - xold[c]; yt[c] = grad[c] - gold[c]; }
        // history push: column k while k < M, else drop the oldest (ring head)
        const int slot = k < M ? k : head;
#pragma unroll
        for (int c = 0; c < 3; ++c) { H.s(slot, c) = st[c]; H.y(slot, c) = yt[c]; }
        if (k >= M) head = (head + 1) % M;
        const T denom = dot3(yt, yt);
        if (fabs(denom) <= T(0)) break;
        gamma_k = dot3(st, yt) / denom;
        alpha_init = T(1);
    }
    return global_iter;
}

// Newton's method on the same prox objective -- the reference's commented-out
// alternative prox solver (src/TetElements.cpp:215, 304;
// deps/mcloptlib/include/MCL/Newton.hpp:30-74) -- with the same cubic
// backtracking.  The step solves (hess_density + wov I) d = -g by a 3x3
// Cholesky; where that matrix is not positive definite the step falls back to
// -g / (wov + |H|_max).  Stops when |g| or the step is below tol * max(1, |x|).
// Quadratic convergence reaches the arithmetic's resolution in a few steps,
// which is what lets the prox run in FP32 (where the L-BFGS prox's absolute
// 1e-8 stop is below the type's resolution).
template <typename T>
__device__ __forceinline__ int prox_newton(const Prox<T>& P, T* x, int max_iters, T tol) {
    int it = 0;
    for (; it < max_iters; ++it) {
        T g[3], h[6];
        const T fx = P.value_grad(x, g);
        const T xs = fmax(T(1), fmax(fabs(x[0]), fmax(fabs(x[1]), fabs(x[2]))));
        if (sqrt(dot3(g, g)) <= tol * P.wov * xs) break;
        P.nh.hess(x, h);
        h[0] += P.wov; h[1] += P.wov; h[2] += P.wov;
        T d[3];
        // 3x3 Cholesky of [h0 h3 h4; h3 h1 h5; h4 h5 h2]
        const T l00 = h[0];
        bool pd = l00 > T(0);
        T L00 = 0, L10 = 0, L20 = 0, L11 = 0, L21 = 0, L22 = 0;
        if (pd) {
            L00 = sqrt(l00); L10 = h[3] / L00; L20 = h[4] / L00;
            const T a11 = h[1] - L10 * L10;
            pd = a11 > T(0);
            if (pd) {
                L11 = sqrt(a11); L21 = (h[5] - L20 * L10) / L11;
                const T a22 = h[2] - L20 * L20 - L21 * L21;
                pd = a22 > T(0);
                if (pd) L22 = sqrt(a22);
            }
        }
        if (pd) {
            const T y0 = -g[0] / L00;
            const T y1 = (-g[1] - L10 * y0) / L11;
            const T y2 = (-g[2] - L20 * y0 - L21 * y1) / L22;
            d[2] = y2 / L22;
            d[1] = (y1 - L21 * d[2]) / L11;
            d[0] = (y0 - L10 * d[1] - L20 * d[2]) / L00;
        } else {
            const T sc = P.wov + fmax(fabs(h[0]), fmax(fabs(h[1]), fabs(h[2])));
            d[0] = -g[0] / sc; d[1] = -g[1] / sc; d[2] = -g[2] / sc;
        }
        if (dot3(d, g) >= T(0)) { d[0] = -g[0] / P.wov; d[1] = -g[1] / P.wov; d[2] = -g[2] / P.wov; }
        if (sqrt(dot3(d, d)) <= tol * xs) {   // converged: take the last (tiny) step without a search
            x[0] += d[0]; x[1] += d[1]; x[2] += d[2];
            ++it;
            break;
        }
        const T rate = linesearch_cubic(P, x, d, T(1), fx, g, 40);
        if (rate <= T(0)) break;
        const T st[3] = {rate * d[0], rate * d[1], rate * d[2]};
        x[0] += st[0]; x[1] += st[1]; x[2] += st[2];
        if (sqrt(dot3(st, st)) <= tol * xs) { ++it; break; }
    }
    return it;
}

}  // namespace wrapd
