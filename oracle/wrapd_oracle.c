/* Test infrastructure: the CPU restatement of the reference's ADMM solve loop.
 * See wrapd_oracle.h.  Reference paths are relative to the wrapd project root.
 * Runs single-threaded and in element order, which is the summation order of
 * the reference run with OMP_NUM_THREADS=1. */
#include "wrapd_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define A3(a, r, c) ((a)[(r) + 3 * (c)])
enum { E_OK = 0, E_INPUT = -1, E_INVERTED = -2, E_NOT_SPD = -3, E_NAN = -4, E_PROX_NEG = -5 };

/* ------------------------------------------------------------------------ */
/* 3x3 helpers                                                               */
/* ------------------------------------------------------------------------ */

/* Eigen's 3x3 determinant (cofactor expansion along the first row). */
static double det3(const double* m) {
    return A3(m, 0, 0) * (A3(m, 1, 1) * A3(m, 2, 2) - A3(m, 1, 2) * A3(m, 2, 1)) -
           A3(m, 0, 1) * (A3(m, 1, 0) * A3(m, 2, 2) - A3(m, 1, 2) * A3(m, 2, 0)) +
           A3(m, 0, 2) * (A3(m, 1, 0) * A3(m, 2, 1) - A3(m, 1, 1) * A3(m, 2, 0));
}

static void inv3(const double* m, double* out) {
    double c00 = A3(m, 1, 1) * A3(m, 2, 2) - A3(m, 1, 2) * A3(m, 2, 1);
    double c01 = A3(m, 1, 2) * A3(m, 2, 0) - A3(m, 1, 0) * A3(m, 2, 2);
    double c02 = A3(m, 1, 0) * A3(m, 2, 1) - A3(m, 1, 1) * A3(m, 2, 0);
    double det = A3(m, 0, 0) * c00 + A3(m, 0, 1) * c01 + A3(m, 0, 2) * c02;
    double id = 1.0 / det;
    A3(out, 0, 0) = c00 * id;
    A3(out, 1, 0) = c01 * id;
    A3(out, 2, 0) = c02 * id;
    A3(out, 0, 1) = (A3(m, 0, 2) * A3(m, 2, 1) - A3(m, 0, 1) * A3(m, 2, 2)) * id;
    A3(out, 1, 1) = (A3(m, 0, 0) * A3(m, 2, 2) - A3(m, 0, 2) * A3(m, 2, 0)) * id;
    A3(out, 2, 1) = (A3(m, 0, 1) * A3(m, 2, 0) - A3(m, 0, 0) * A3(m, 2, 1)) * id;
    A3(out, 0, 2) = (A3(m, 0, 1) * A3(m, 1, 2) - A3(m, 0, 2) * A3(m, 1, 1)) * id;
    A3(out, 1, 2) = (A3(m, 0, 2) * A3(m, 1, 0) - A3(m, 0, 0) * A3(m, 1, 2)) * id;
    A3(out, 2, 2) = (A3(m, 0, 0) * A3(m, 1, 1) - A3(m, 0, 1) * A3(m, 1, 0)) * id;
}

static double fro2_diff(const double* a, const double* b) {
    double s = 0.0;
    for (int i = 0; i < 9; ++i) { double d = a[i] - b[i]; s += d * d; }
    return s;
}

/* ------------------------------------------------------------------------ */
/* SVD: two-sided Jacobi, restating Eigen 3.3.7 JacobiSVD::compute for a     */
/* square 3x3 (deps/Eigen3/Eigen/src/SVD/JacobiSVD.h:681-776, with          */
/* real_2x2_jacobi_svd from misc/RealSvd2x2.h and makeJacobi from            */
/* Jacobi/Jacobi.h:83-113), then wrapd's rotation sign fix                   */
/* (src/Math.hpp:147-160).                                                   */
/* ------------------------------------------------------------------------ */
void orc_svd3(const double* A, double* sig, double* U, double* V) {
    double W[9];
    double scale = 0.0;
    for (int i = 0; i < 9; ++i) scale = fmax(scale, fabs(A[i]));
    if (scale == 0.0) scale = 1.0;
    for (int i = 0; i < 9; ++i) W[i] = A[i] / scale;
    for (int i = 0; i < 9; ++i) U[i] = V[i] = (i % 4 == 0) ? 1.0 : 0.0;
    const double prec = 2.0 * DBL_EPSILON, tiny = DBL_MIN;
    double maxd = fmax(fabs(W[0]), fmax(fabs(W[4]), fabs(W[8])));
    int finished = 0;
    while (!finished) {
        finished = 1;
        for (int p = 1; p < 3; ++p) {
            for (int q = 0; q < p; ++q) {
                double thr = fmax(tiny, prec * maxd);
                if (!(fabs(A3(W, p, q)) > thr || fabs(A3(W, q, p)) > thr)) continue;
                finished = 0;
                double m00 = A3(W, p, p), m01 = A3(W, p, q), m10 = A3(W, q, p), m11 = A3(W, q, q);
                double t = m00 + m11, d = m10 - m01, c1, s1;
                if (fabs(d) < DBL_MIN) { s1 = 0.0; c1 = 1.0; }
                else { double u = t / d, tmp = sqrt(1.0 + u * u); s1 = 1.0 / tmp; c1 = u / tmp; }
                double a00 = c1 * m00 + s1 * m10, a01 = c1 * m01 + s1 * m11;
                double a11 = -s1 * m01 + c1 * m11;
                double cr, sr;
                double deno = 2.0 * fabs(a01);
                if (deno < DBL_MIN) { cr = 1.0; sr = 0.0; }
                else {
                    double tau = (a00 - a11) / deno, w = sqrt(tau * tau + 1.0);
                    double tt = tau > 0.0 ? 1.0 / (tau + w) : 1.0 / (tau - w);
                    double sgn = tt > 0.0 ? 1.0 : -1.0;
                    double n = 1.0 / sqrt(tt * tt + 1.0);
                    sr = -sgn * (a01 / fabs(a01)) * fabs(tt) * n;
                    cr = n;
                }
                double cl = c1 * cr + s1 * sr;   /* rot1 * j_right^T */
                double sl = -c1 * sr + s1 * cr;
                for (int i = 0; i < 3; ++i) { /* W rows p,q by j_left */
                    double x = A3(W, p, i), y = A3(W, q, i);
                    A3(W, p, i) = cl * x + sl * y;
                    A3(W, q, i) = -sl * x + cl * y;
                }
                for (int i = 0; i < 3; ++i) { /* U cols p,q by j_left^T on the right */
                    double x = A3(U, i, p), y = A3(U, i, q);
                    A3(U, i, p) = cl * x + sl * y;
                    A3(U, i, q) = -sl * x + cl * y;
                }
                for (int i = 0; i < 3; ++i) { /* W cols p,q by j_right */
                    double x = A3(W, i, p), y = A3(W, i, q);
                    A3(W, i, p) = cr * x - sr * y;
                    A3(W, i, q) = sr * x + cr * y;
                }
                for (int i = 0; i < 3; ++i) {
                    double x = A3(V, i, p), y = A3(V, i, q);
                    A3(V, i, p) = cr * x - sr * y;
                    A3(V, i, q) = sr * x + cr * y;
                }
                maxd = fmax(maxd, fmax(fabs(A3(W, p, p)), fabs(A3(W, q, q))));
            }
        }
    }
    for (int i = 0; i < 3; ++i) {
        double a = A3(W, i, i);
        sig[i] = fabs(a);
        if (a < 0.0) for (int r = 0; r < 3; ++r) A3(U, r, i) = -A3(U, r, i);
    }
    for (int i = 0; i < 3; ++i) sig[i] *= scale;
    for (int i = 0; i < 3; ++i) {
        int pos = i;
        double mx = sig[i];
        for (int j = i + 1; j < 3; ++j) if (sig[j] > mx) { mx = sig[j]; pos = j; }
        if (mx == 0.0) break;
        if (pos != i) {
            double t = sig[i]; sig[i] = sig[pos]; sig[pos] = t;
            for (int r = 0; r < 3; ++r) {
                t = A3(U, r, i); A3(U, r, i) = A3(U, r, pos); A3(U, r, pos) = t;
                t = A3(V, r, i); A3(V, r, i) = A3(V, r, pos); A3(V, r, pos) = t;
            }
        }
    }
    if (det3(U) < 0.0) { for (int r = 0; r < 3; ++r) A3(U, r, 2) = -A3(U, r, 2); sig[2] = -sig[2]; }
    if (det3(V) < 0.0) { for (int r = 0; r < 3; ++r) A3(V, r, 2) = -A3(V, r, 2); sig[2] = -sig[2]; }
}

/* ------------------------------------------------------------------------ */
/* Neo-Hookean (extended log, J0 = 0.1), src/TetElements.hpp:50-144          */
/* ------------------------------------------------------------------------ */
#define NH_J0 0.1

double orc_nh_psi_plain(double mu, double lambda, const double* x) {
    /* src/TetElements.cpp:619-628 (no negative-stretch guard) */
    double I1 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
    double J = x[0] * x[1] * x[2];
    double e = 0.5 * mu * (I1 - 3.0);
    if (J > NH_J0) {
        double lj = log(J);
        e += -mu * lj + 0.5 * lambda * lj * lj;
    } else {
        double r = J / NH_J0 - 1.0;
        double fJ = log(NH_J0) + ((J - NH_J0) / NH_J0) - 0.5 * r * r;
        e += -mu * fJ + 0.5 * lambda * fJ * fJ;
    }
    return e;
}

double orc_nh_psi(double mu, double lambda, const double* x) {
    /* energy_density, src/TetElements.hpp:61-77 */
    if (x[0] < 0.0 || x[1] < 0.0 || x[2] < 0.0) return 1.e15;
    return orc_nh_psi_plain(mu, lambda, x);
}

static double prox_value(double mu, double lambda, const double* x0, double wov, const double* x) {
    double d0 = x[0] - x0[0], d1 = x[1] - x0[1], d2 = x[2] - x0[2];
    return orc_nh_psi(mu, lambda, x) + (wov * 0.5) * (d0 * d0 + d1 * d1 + d2 * d2);
}

double orc_prox_value_grad(double mu, double lambda, const double* x0, double wov,
                           const double* x, double* g) {
    /* NHProx::gradient, src/TetElements.hpp:93-107 */
    double J = x[0] * x[1] * x[2];
    double f;
    if (J > NH_J0) {
        f = lambda * log(J) - mu;
    } else {
        double r = J / NH_J0 - 1.0;
        double fJ = log(NH_J0) + ((J - NH_J0) / NH_J0) - 0.5 * r * r;
        double dfJdJ = 1.0 / NH_J0 - (J - NH_J0) / (NH_J0 * NH_J0);
        f = (lambda * fJ - mu) * dfJdJ * J;
    }
    for (int i = 0; i < 3; ++i) g[i] = mu * x[i] + f * (1.0 / x[i]) + wov * (x[i] - x0[i]);
    return prox_value(mu, lambda, x0, wov, x);
}

static double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* BacktrackingCubic::search, deps/mcloptlib/include/MCL/Backtracking.hpp:268-332 */
static double cubic_step(double fx0, double gtp, double fxa, double alpha, double fxp, double alphap) {
    double mult = 1.0 / (alpha * alpha * alphap * alphap * (alpha - alphap));
    double a00 = mult * (alphap * alphap), a01 = mult * (-alpha * alpha);
    double a10 = mult * (-alphap * alphap * alphap), a11 = mult * (alpha * alpha * alpha);
    double b0 = fxa - fx0 - alpha * gtp, b1 = fxp - fx0 - alphap * gtp;
    double r0 = a00 * b0 + a01 * b1, r1 = a10 * b0 + a11 * b1;
    if (fabs(r0) <= 0.0) return -gtp / (2.0 * r1);
    double d = sqrt(r1 * r1 - 3.0 * r0 * gtp);
    return (-r1 + d) / (3.0 * r0);
}

static double linesearch_cubic(double mu, double lambda, const double* x0, double wov,
                               const double* x, const double* p, double alpha0) {
    if (sqrt(dot3(p, p)) <= DBL_EPSILON) return 1e-4;
    double alpha = alpha0, g[3];
    double fx0 = orc_prox_value_grad(mu, lambda, x0, wov, x, g);
    double gtp = dot3(g, p);
    double fxp = fx0, alphap = alpha;
    for (int it = 0; it < 100000; ++it) {
        double xa[3] = {x[0] + alpha * p[0], x[1] + alpha * p[1], x[2] + alpha * p[2]};
        double fxa = prox_value(mu, lambda, x0, wov, xa);
        if (fxa <= fx0 + alpha * 1e-4 * gtp) return alpha;
        double at = it == 0 ? (gtp / (2.0 * (fx0 + gtp - fxa))) : cubic_step(fx0, gtp, fxa, alpha, fxp, alphap);
        fxp = fxa;
        alphap = alpha;
        double lo = 0.1 * alpha, hi = 0.5 * alpha;
        alpha = at < lo ? lo : (at > hi ? hi : at);
    }
    return -1.0;
}

/* LBFGS<double,3,8>::minimize, deps/mcloptlib/include/MCL/LBFGS.hpp:52-152, with
 * Prox::converged (src/TetElements.hpp:40-42). Returns iterations, -1 on failure. */
int orc_prox_lbfgs(double mu, double lambda, const double* x0, double wov, double* x, int max_iters_in) {
    enum { M = 8 };
    double s[M][3], y[M][3], alpha[M], rho[M];
    double grad[3], q[3], grad_old[3], x_old[3], x_last[3];
    orc_prox_value_grad(mu, lambda, x0, wov, x, grad);
    double gamma_k = 1.0, alpha_init = 1.0;
    int global_iter = 0, max_iters = max_iters_in;
    for (int k = 0; k < max_iters; ++k) {
        memcpy(x_old, x, sizeof x_old);
        memcpy(grad_old, grad, sizeof grad_old);
        memcpy(q, grad, sizeof q);
        global_iter++;
        int iter = k < M ? k : M;
        for (int i = iter - 1; i >= 0; --i) {
            rho[i] = 1.0 / dot3(s[i], y[i]);
            alpha[i] = rho[i] * dot3(s[i], q);
            for (int c = 0; c < 3; ++c) q[c] = q[c] - alpha[i] * y[i][c];
        }
        for (int c = 0; c < 3; ++c) q[c] = gamma_k * q[c];
        for (int i = 0; i < iter; ++i) {
            double beta = rho[i] * dot3(q, y[i]);
            for (int c = 0; c < 3; ++c) q[c] = q[c] + (alpha[i] - beta) * s[i][c];
        }
        double dir = dot3(q, grad);
        if (dir <= 0.0) {
            memcpy(q, grad, sizeof q);
            max_iters -= k;
            k = 0;
            double ninf = fmax(fabs(grad[0]), fmax(fabs(grad[1]), fabs(grad[2])));
            alpha_init = fmin(1.0, 1.0 / ninf);
        }
        double mq[3] = {-q[0], -q[1], -q[2]};
        double rate = linesearch_cubic(mu, lambda, x0, wov, x, mq, alpha_init);
        if (rate <= 0.0) return -1;
        memcpy(x_last, x, sizeof x_last);
        for (int c = 0; c < 3; ++c) x[c] -= rate * q[c];
        {
            double dx[3] = {x_last[0] - x[0], x_last[1] - x[1], x_last[2] - x[2]};
            if (sqrt(dot3(grad, grad)) < 1e-8 || sqrt(dot3(dx, dx)) < 1e-8) break;
        }
        orc_prox_value_grad(mu, lambda, x0, wov, x, grad);
        double st[3], yt[3];
        for (int c = 0; c < 3; ++c) { st[c] = x[c] - x_old[c]; yt[c] = grad[c] - grad_old[c]; }
        if (k < M) {
            memcpy(s[k], st, sizeof st);
            memcpy(y[k], yt, sizeof yt);
        } else {
            memmove(s[0], s[1], sizeof(double) * 3 * (M - 1));
            memmove(y[0], y[1], sizeof(double) * 3 * (M - 1));
            memcpy(s[M - 1], st, sizeof st);
            memcpy(y[M - 1], yt, sizeof yt);
        }
        double denom = dot3(yt, yt);
        if (fabs(denom) <= 0.0) break;
        gamma_k = dot3(st, yt) / denom;
        alpha_init = 1.0;
    }
    return global_iter;
}

/* Symmetric 3x3 eigenvalues by cyclic Jacobi (own). */
static void sym_eig3(const double* H, double* ev) {
    double a[9];
    memcpy(a, H, sizeof a);
    for (int sweep = 0; sweep < 50; ++sweep) {
        double off = A3(a, 0, 1) * A3(a, 0, 1) + A3(a, 0, 2) * A3(a, 0, 2) + A3(a, 1, 2) * A3(a, 1, 2);
        double dn = A3(a, 0, 0) * A3(a, 0, 0) + A3(a, 1, 1) * A3(a, 1, 1) + A3(a, 2, 2) * A3(a, 2, 2);
        if (off <= 1e-40 * dn || off == 0.0) break;
        for (int p = 0; p < 2; ++p)
            for (int q = p + 1; q < 3; ++q) {
                double apq = A3(a, p, q);
                if (apq == 0.0) continue;
                double theta = (A3(a, q, q) - A3(a, p, p)) / (2.0 * apq);
                double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < 3; ++k) { /* columns */
                    double akp = A3(a, k, p), akq = A3(a, k, q);
                    A3(a, k, p) = c * akp - s * akq;
                    A3(a, k, q) = s * akp + c * akq;
                }
                for (int k = 0; k < 3; ++k) { /* rows */
                    double apk = A3(a, p, k), aqk = A3(a, q, k);
                    A3(a, p, k) = c * apk - s * aqk;
                    A3(a, q, k) = s * apk + c * aqk;
                }
            }
    }
    ev[0] = A3(a, 0, 0); ev[1] = A3(a, 1, 1); ev[2] = A3(a, 2, 2);
}

/* Max eigenvalue of makePD(hessian_density(sigma)) (src/TetElements.hpp:109-144,
 * src/Math.hpp:243-261, src/TetElements.cpp:414-416).  makePD zeroes the
 * negative eigenvalues, so the max eigenvalue of the projected matrix is
 * max(lambda_max(H), 0). */
double orc_hess_lmax(double mu, double lambda, const double* x) {
    double H[9];
    double J = x[0] * x[1] * x[2];
    if (J > NH_J0) {
        double lj = log(J);
        double ct = mu - lambda * (lj - 1.0);
        A3(H, 0, 0) = mu + ct / (x[0] * x[0]);
        A3(H, 1, 1) = mu + ct / (x[1] * x[1]);
        A3(H, 2, 2) = mu + ct / (x[2] * x[2]);
        A3(H, 0, 1) = A3(H, 1, 0) = lambda / (x[0] * x[1]);
        A3(H, 0, 2) = A3(H, 2, 0) = lambda / (x[0] * x[2]);
        A3(H, 1, 2) = A3(H, 2, 1) = lambda / (x[1] * x[2]);
    } else {
        double r = J / NH_J0 - 1.0;
        double fJ = log(NH_J0) + ((J - NH_J0) / NH_J0) - 0.5 * r * r;
        double dfJdJ = 1.0 / NH_J0 - (J - NH_J0) / (NH_J0 * NH_J0);
        double lfm = lambda * fJ - mu;
        double a = x[1] * x[2], b = x[0] * x[2], c = x[0] * x[1];
        A3(H, 0, 0) = mu - lfm * (a / NH_J0) * (a / NH_J0) + lambda * (dfJdJ * a) * (dfJdJ * a);
        A3(H, 1, 1) = mu - lfm * (b / NH_J0) * (b / NH_J0) + lambda * (dfJdJ * b) * (dfJdJ * b);
        A3(H, 2, 2) = mu - lfm * (c / NH_J0) * (c / NH_J0) + lambda * (dfJdJ * c) * (dfJdJ * c);
        double ct = lfm * (dfJdJ - J / (NH_J0 * NH_J0)) + lambda * J * dfJdJ * dfJdJ;
        A3(H, 0, 1) = A3(H, 1, 0) = x[2] * ct;
        A3(H, 0, 2) = A3(H, 2, 0) = x[1] * ct;
        A3(H, 1, 2) = A3(H, 2, 1) = x[0] * ct;
    }
    double ev[3];
    sym_eig3(H, ev);
    double m = fmax(ev[0], fmax(ev[1], ev[2]));
    return m > 0.0 ? m : 0.0;
}

/* ------------------------------------------------------------------------ */
/* Sparse LDL^T of the free-vertex weighted Laplacian.  The reference uses    */
/* Eigen's SimplicialLDLT with AMD (deps/mcloptlib/include/MCL/               */
/* LinearSolver.hpp:279-298); any symmetric ordering gives the same solve up  */
/* to rounding, so the oracle uses reverse Cuthill-McKee and an envelope      */
/* (profile) LDL^T.                                                           */
/* ------------------------------------------------------------------------ */
typedef struct {
    int n;
    int *adj_ptr, *adj;   /* symmetric adjacency (no diagonal) */
    int *perm, *iperm;    /* new -> old, old -> new */
    int *first;           /* first column of row i's envelope (new numbering) */
    long *rowptr;         /* offsets of row i's envelope entries */
    double *L;            /* envelope of L (unit lower), row-wise */
    double *D;
    /* A values in (new) envelope layout, assembled per factorization */
    double* Aenv;
    double* Adiag;
    /* linear_solver 1: A in CSR (row i: the diagonal, then adj of i in order) */
    long* cptr;
    int* ccol;
    double* cval;
} env_ldl;

static int cmp_int(const void* a, const void* b) { return (*(const int*)a > *(const int*)b) - (*(const int*)a < *(const int*)b); }

static void env_free(env_ldl* f) {
    free(f->adj_ptr); free(f->adj); free(f->perm); free(f->iperm); free(f->first);
    free(f->rowptr); free(f->L); free(f->D); free(f->Aenv); free(f->Adiag);
    free(f->cptr); free(f->ccol); free(f->cval);
    memset(f, 0, sizeof *f);
}

/* Reverse Cuthill-McKee from a minimum-degree start, per connected component. */
static void rcm(int n, const int* ptr, const int* adj, int* perm) {
    char* seen = calloc((size_t)n, 1);
    int* queue = perm;
    int head = 0, tail = 0;
    int* nb = malloc(sizeof(int) * (size_t)(n + 1));
    while (tail < n) {
        int start = -1, bestdeg = 1 << 30;
        for (int i = 0; i < n; ++i)
            if (!seen[i] && ptr[i + 1] - ptr[i] < bestdeg) { bestdeg = ptr[i + 1] - ptr[i]; start = i; }
        seen[start] = 1;
        queue[tail++] = start;
        while (head < tail) {
            int v = queue[head++], cnt = 0;
            for (int k = ptr[v]; k < ptr[v + 1]; ++k) if (!seen[adj[k]]) { nb[cnt++] = adj[k]; seen[adj[k]] = 1; }
            /* order neighbours by degree, ties by id */
            for (int a = 1; a < cnt; ++a) {
                int x = nb[a], dx = ptr[x + 1] - ptr[x], b = a - 1;
                while (b >= 0 && (ptr[nb[b] + 1] - ptr[nb[b]] > dx ||
                                  (ptr[nb[b] + 1] - ptr[nb[b]] == dx && nb[b] > x))) { nb[b + 1] = nb[b]; --b; }
                nb[b + 1] = x;
            }
            for (int a = 0; a < cnt; ++a) queue[tail++] = nb[a];
        }
    }
    for (int i = 0; i < n / 2; ++i) { int t = perm[i]; perm[i] = perm[n - 1 - i]; perm[n - 1 - i] = t; }
    free(seen);
    free(nb);
}

/* ------------------------------------------------------------------------ */
/* Solver state                                                              */
/* ------------------------------------------------------------------------ */
struct orc_state {
    orc_problem p;
    int ne, nv, nf, np;
    double mu, lambda, k_rest;
    double *mu_e, *lambda_e;   /* per element (the uniform values unless the problem gives arrays) */
    int* fidx;   /* ne x 4: free index or -1 */
    int* xidx;   /* ne x 4: fixed index or -1 */
    int* tet;    /* ne x 4 */
    int* nfree;  /* ne */
    int* free_of_vert; int* fix_of_vert; /* nv */
    double *Di, *vol, *w2, *w2c, *DtD, *Dfx;
    double *Z, *U, *slast;
    double *F, *sig, *Us, *Vs, *symF;
    double *xfree, *xfix;
    double curr_pe;
    int count;   /* the reweight delay counter (src/TetElements.cpp:404) */
    env_ldl A;
    /* SplitLBFGS state (deps/mcloptlib/include/MCL/SplitLBFGS.hpp:48-80) */
    int M, m_k;
    double m_tol;
    double **s, **y;  /* logical order via head index */
    int head;
    double *alpha, *rho, *q, *grad, *grad_old, *x_old;
    /* logs */
    int iter;
    double *objectives, *ls_dal, *gs_dal;
    int *flips, *reweighted, *inner;
    int setup_done;
};

int orc_n_free(const orc_state* s) { return s->nf; }
int orc_iters(const orc_state* s) { return s->iter; }

void orc_problem_defaults(orc_problem* p) {
    memset(p, 0, sizeof *p);
    p->youngs = 1e7; p->poisson = 0.45;
    p->max_iters = 5000; p->tol = 1e-11; p->lbfgs_m = 6; p->global_iters = 100; p->kappa = 1.0;
    p->reweighting = 1; p->rw_delay = 50; p->gamma = 1.5;
    p->beta_static = 1.0; p->beta_min = 0.1; p->beta_max = 10.0; p->rw_every = 0;
    p->rot_aware = 1; p->model = 0; p->global_ls = 0;
}

#define NEWD(n) ((double*)calloc((size_t)(n) ? (size_t)(n) : 1, sizeof(double)))
#define NEWI(n) ((int*)calloc((size_t)(n) ? (size_t)(n) : 1, sizeof(int)))

void orc_destroy(orc_state* s) {
    if (!s) return;
    free(s->mu_e); free(s->lambda_e);
    free(s->fidx); free(s->xidx); free(s->tet); free(s->nfree); free(s->free_of_vert); free(s->fix_of_vert);
    free(s->Di); free(s->vol); free(s->w2); free(s->w2c); free(s->DtD); free(s->Dfx);
    free(s->Z); free(s->U); free(s->slast); free(s->F); free(s->sig); free(s->Us); free(s->Vs); free(s->symF);
    free(s->xfree); free(s->xfix);
    env_free(&s->A);
    if (s->s) for (int i = 0; i < s->M; ++i) { free(s->s[i]); free(s->y[i]); }
    free(s->s); free(s->y); free(s->alpha); free(s->rho); free(s->q); free(s->grad); free(s->grad_old); free(s->x_old);
    free(s->objectives); free(s->ls_dal); free(s->gs_dal); free(s->flips); free(s->reweighted); free(s->inner);
    free(s);
}

/* Lame(E, nu), src/Lame.hpp:50-53 */
static void lame(double E, double nu, double* mu, double* lambda) {
    *mu = E / (2.0 * (1.0 + nu));
    *lambda = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
}

orc_state* orc_create(const orc_problem* p, int* err) {
    if (err) *err = E_OK;
    if (!p || p->n_verts <= 0 || p->n_tets <= 0 || p->n_pins < 0 || p->n_pins >= p->n_verts || p->lbfgs_m < 1) {
        if (err) *err = E_INPUT;
        return NULL;
    }
    orc_state* s = calloc(1, sizeof *s);
    s->p = *p;
    s->ne = p->n_tets; s->nv = p->n_verts; s->np = p->n_pins; s->nf = p->n_verts - p->n_pins;
    lame(p->youngs, p->poisson, &s->mu, &s->lambda);
    s->k_rest = 2.0066 * s->mu + 1.0122 * s->lambda;   /* src/TetElements.cpp:84 */
    s->mu_e = NEWD(s->ne); s->lambda_e = NEWD(s->ne);
    for (int e = 0; e < s->ne; ++e) {
        if (p->youngs_e && p->poisson_e) lame(p->youngs_e[e], p->poisson_e[e], &s->mu_e[e], &s->lambda_e[e]);
        else { s->mu_e[e] = s->mu; s->lambda_e[e] = s->lambda; }
    }
    /* free/fixed maps from the sorted pins, samples/utils/AddMeshes.hpp:268-289 */
    int* sp = NEWI(s->np);
    memcpy(sp, p->pins, sizeof(int) * (size_t)s->np);
    qsort(sp, (size_t)s->np, sizeof(int), cmp_int);
    for (int j = 0; j < s->np; ++j)
        if (sp[j] < 0 || sp[j] >= s->nv || (j > 0 && sp[j] == sp[j - 1])) {
            if (err) *err = E_INPUT;
            free(sp);
            orc_destroy(s);
            return NULL;
        }
    s->free_of_vert = NEWI(s->nv); s->fix_of_vert = NEWI(s->nv);
    for (int i = 0, j = 0, k = 0; i < s->nv; ++i) {
        if (j < s->np && i == sp[j]) { s->free_of_vert[i] = -1; s->fix_of_vert[i] = j++; }
        else { s->free_of_vert[i] = k++; s->fix_of_vert[i] = -1; }
    }
    int ne = s->ne;
    s->tet = NEWI(4 * ne); s->fidx = NEWI(4 * ne); s->xidx = NEWI(4 * ne); s->nfree = NEWI(ne);
    s->Di = NEWD(12 * ne); s->vol = NEWD(ne); s->w2 = NEWD(ne); s->w2c = NEWD(ne); s->DtD = NEWD(16 * ne); s->Dfx = NEWD(9 * ne);
    s->Z = NEWD(9 * ne); s->U = NEWD(9 * ne); s->slast = NEWD(3 * ne);
    s->F = NEWD(9 * ne); s->sig = NEWD(3 * ne); s->Us = NEWD(9 * ne); s->Vs = NEWD(9 * ne); s->symF = NEWD(9 * ne);
    s->xfree = NEWD(3 * s->nf); s->xfix = NEWD(3 * s->np);
    /* TetElements ctor, src/TetElements.cpp:90-142 */
    for (int e = 0; e < ne; ++e) {
        const int* t = p->tets + 4 * e;
        for (int a = 0; a < 4; ++a) {
            if (t[a] < 0 || t[a] >= s->nv) { if (err) *err = E_INPUT; free(sp); orc_destroy(s); return NULL; }
            s->tet[4 * e + a] = t[a];
            s->fidx[4 * e + a] = s->free_of_vert[t[a]];
            s->xidx[4 * e + a] = s->fix_of_vert[t[a]];
            if (s->fidx[4 * e + a] >= 0) s->nfree[e]++;
        }
        double ed[9], ei[9];
        for (int c = 0; c < 3; ++c)
            for (int r = 0; r < 3; ++r) A3(ed, r, c) = p->rest[3 * t[c + 1] + r] - p->rest[3 * t[0] + r];
        inv3(ed, ei);
        s->vol[e] = det3(ed) / 6.0;
        if (s->vol[e] < 0.0) { if (err) *err = E_INVERTED; free(sp); orc_destroy(s); return NULL; }
        double* Di = s->Di + 12 * e;  /* Di = (S * Dm^-1)^T, 3x4 col-major: Di[r + 3a] */
        for (int r = 0; r < 3; ++r) {
            Di[r + 0] = -A3(ei, 0, r) - A3(ei, 1, r) - A3(ei, 2, r);
            for (int a = 1; a < 4; ++a) Di[r + 3 * a] = A3(ei, a - 1, r);
        }
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b) {
                double v = 0.0;
                for (int r = 0; r < 3; ++r) v += Di[r + 3 * a] * Di[r + 3 * b];
                s->DtD[16 * e + a + 4 * b] = v;
            }
        /* k = 1 for ARAP, 2.0066 mu + 1.0122 lambda for NH (src/TetElements.cpp:80-87) */
        const double k = p->model == 1 ? 1.0 : 2.0066 * s->mu_e[e] + 1.0122 * s->lambda_e[e];
        s->w2[e] = p->beta_static * k * s->vol[e];
        s->slast[3 * e] = s->slast[3 * e + 1] = s->slast[3 * e + 2] = 1.0;
    }
    free(sp);
    s->M = p->lbfgs_m;
    s->s = calloc((size_t)s->M, sizeof(double*));
    s->y = calloc((size_t)s->M, sizeof(double*));
    for (int i = 0; i < s->M; ++i) { s->s[i] = NEWD(3 * s->nf); s->y[i] = NEWD(3 * s->nf); }
    s->alpha = NEWD(s->M); s->rho = NEWD(s->M);
    s->q = NEWD(3 * s->nf); s->grad = NEWD(3 * s->nf); s->grad_old = NEWD(3 * s->nf); s->x_old = NEWD(3 * s->nf);
    int cap = p->max_iters + 2;
    s->objectives = NEWD(cap); s->ls_dal = NEWD(cap); s->gs_dal = NEWD(cap);
    s->flips = NEWI(cap); s->reweighted = NEWI(cap); s->inner = NEWI(cap);
    s->m_tol = 1e-15;
    return s;
}

/* x_local of element e from the full positions X (n_verts x 3) */
static void F_from_X(const orc_state* s, int e, const double* X, double* F) {
    const double* Di = s->Di + 12 * e;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            double v = 0.0;
            for (int a = 0; a < 4; ++a) v += Di[c + 3 * a] * X[3 * s->tet[4 * e + a] + r];
            A3(F, r, c) = v;
        }
}

/* update_fix_cache, src/TetElements.cpp:547-562 (Dfx holds Dfix * x_fix = a part of F^T) */
static void update_fix_cache(orc_state* s) {
    for (int e = 0; e < s->ne; ++e) {
        if (s->nfree[e] == 4) continue;
        const double* Di = s->Di + 12 * e;
        double* D = s->Dfx + 9 * e;
        for (int c = 0; c < 3; ++c)
            for (int r = 0; r < 3; ++r) {
                double v = 0.0;
                for (int a = 0; a < 4; ++a) {
                    int j = s->xidx[4 * e + a];
                    if (j >= 0) v += Di[c + 3 * a] * s->xfix[3 * j + r];
                }
                A3(D, c, r) = v;  /* (Dfix * xfix)(c, r) */
            }
    }
}

/* update_defo_cache, src/TetElements.cpp:564-596 */
static void defo_cache_at(orc_state* s, const double* xfree) {
    for (int e = 0; e < s->ne; ++e) {
        const double* Di = s->Di + 12 * e;
        double* F = s->F + 9 * e;
        for (int c = 0; c < 3; ++c)
            for (int r = 0; r < 3; ++r) {
                double v = 0.0;
                for (int a = 0; a < 4; ++a) {
                    int j = s->fidx[4 * e + a];
                    if (j >= 0) v += Di[c + 3 * a] * xfree[3 * j + r];
                }
                if (s->nfree[e] < 4) v += A3(s->Dfx + 9 * e, c, r);
                A3(F, r, c) = v;
            }
        double* sg = s->sig + 3 * e;
        double* Uu = s->Us + 9 * e;
        double* Vv = s->Vs + 9 * e;
        orc_svd3(F, sg, Uu, Vv);
        double* S = s->symF + 9 * e;
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) {
                double v = 0.0;
                for (int k = 0; k < 3; ++k) v += A3(Vv, r, k) * sg[k] * A3(Vv, c, k);
                A3(S, r, c) = v;
            }
    }
}

void orc_update_defo_cache(orc_state* s) { defo_cache_at(s, s->xfree); }

/* rot(F) = U V^T of the sign-fixed SVD, math::polar (src/Math.hpp:218-225) */
static void rot3(const double* F, double* R) {
    double sg[3], Uu[9], Vv[9];
    orc_svd3(F, sg, Uu, Vv);
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            double v = 0.0;
            for (int k = 0; k < 3; ++k) v += A3(Uu, r, k) * A3(Vv, c, k);
            A3(R, r, c) = v;
        }
}

/* potential_energy_x, src/TetElements.cpp:598-635 (ARAP: k = 1) */
double orc_potential_energy(const orc_state* s) {
    double pe = 0.0;
    if (s->p.model == 1) {
        for (int e = 0; e < s->ne; ++e) {
            double R[9];
            rot3(s->F + 9 * e, R);
            pe += 0.5 * 1.0 * s->vol[e] * fro2_diff(s->F + 9 * e, R);
        }
        return pe;
    }
    for (int e = 0; e < s->ne; ++e) pe += s->vol[e] * orc_nh_psi_plain(s->mu_e[e], s->lambda_e[e], s->sig + 3 * e);
    return pe;
}

int orc_inversion_count(const orc_state* s) {
    int c = 0;
    for (int e = 0; e < s->ne; ++e) {
        const double* g = s->sig + 3 * e;
        if (g[0] < 0.0 || g[1] < 0.0 || g[2] < 0.0) c++;
    }
    return c;
}

/* update_all_candidate_weights, src/TetElements.cpp:391-432 */
static void candidate_weights(orc_state* s, const double* sig) {
    if (s->count > s->p.rw_delay) {
        for (int e = 0; e < s->ne; ++e) {
            double wr = 2.0066 * s->mu_e[e] + 1.0122 * s->lambda_e[e];
            double wmin = wr * s->p.beta_min, wmax = wr * s->p.beta_max;
            double lm = orc_hess_lmax(s->mu_e[e], s->lambda_e[e], sig + 3 * e);
            double c = lm;
            if (lm < wmin) c = wmin;
            if (lm > wmax) c = wmax;
            s->w2c[e] = s->vol[e] * c;
        }
    } else {
        for (int e = 0; e < s->ne; ++e) s->w2c[e] = s->vol[e] * (2.0066 * s->mu_e[e] + 1.0122 * s->lambda_e[e]);
    }
    s->count++;
}

/* update_actual_weights, src/TetElements.cpp:435-442 */
static void update_actual_weights(orc_state* s) {
    for (int e = 0; e < s->ne; ++e) {
        double r = s->w2[e] / s->w2c[e];
        for (int i = 0; i < 9; ++i) s->U[9 * e + i] = r * s->U[9 * e + i];
        s->w2[e] = s->w2c[e];
    }
}

/* max_wsq_ratio, src/Elements.hpp:56-69 */
static double max_wsq_ratio(const orc_state* s) {
    double m = 0.0;
    for (int e = 0; e < s->ne; ++e) {
        double a = s->w2[e] / s->w2c[e], b = 1.0 / a;
        if (a > m) m = a;
        if (b > m) m = b;
    }
    return m;
}

/* ---- the weighted Laplacian A = sum_e w_e^2 D_e^T D_e over free vertices --- */
static void build_pattern(orc_state* s) {
    env_ldl* f = &s->A;
    int n = s->nf;
    f->n = n;
    /* adjacency via element pairs */
    int* deg = NEWI(n + 1);
    for (int e = 0; e < s->ne; ++e)
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b) {
                int i = s->fidx[4 * e + a], j = s->fidx[4 * e + b];
                if (i >= 0 && j >= 0 && i != j) deg[i]++;
            }
    f->adj_ptr = NEWI(n + 1);
    for (int i = 0; i < n; ++i) f->adj_ptr[i + 1] = f->adj_ptr[i] + deg[i];
    f->adj = NEWI(f->adj_ptr[n]);
    int* fill = NEWI(n);
    for (int e = 0; e < s->ne; ++e)
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b) {
                int i = s->fidx[4 * e + a], j = s->fidx[4 * e + b];
                if (i >= 0 && j >= 0 && i != j) f->adj[f->adj_ptr[i] + fill[i]++] = j;
            }
    /* dedupe */
    int* np = NEWI(n + 1);
    int w = 0;
    for (int i = 0; i < n; ++i) {
        int b = f->adj_ptr[i], en = f->adj_ptr[i + 1];
        qsort(f->adj + b, (size_t)(en - b), sizeof(int), cmp_int);
        np[i] = w;
        for (int k = b; k < en; ++k) if (k == b || f->adj[k] != f->adj[k - 1]) f->adj[w++] = f->adj[k];
    }
    np[n] = w;
    memcpy(f->adj_ptr, np, sizeof(int) * (size_t)(n + 1));
    free(np); free(deg); free(fill);
    if (s->p.linear_solver == 1) {
        /* CSR with the diagonal first in each row; no ordering, no envelope */
        f->cptr = (long*)calloc((size_t)n + 1, sizeof(long));
        for (int i = 0; i < n; ++i) f->cptr[i + 1] = f->cptr[i] + 1 + (f->adj_ptr[i + 1] - f->adj_ptr[i]);
        f->ccol = NEWI(f->cptr[n]);
        f->cval = NEWD(f->cptr[n]);
        for (int i = 0; i < n; ++i) {
            long o = f->cptr[i];
            f->ccol[o++] = i;
            for (int k = f->adj_ptr[i]; k < f->adj_ptr[i + 1]; ++k) f->ccol[o++] = f->adj[k];
        }
        f->D = NEWD(n);
        return;
    }
    f->perm = NEWI(n); f->iperm = NEWI(n);
    rcm(n, f->adj_ptr, f->adj, f->perm);
    for (int i = 0; i < n; ++i) f->iperm[f->perm[i]] = i;
    f->first = NEWI(n);
    f->rowptr = (long*)calloc((size_t)n + 1, sizeof(long));
    for (int i = 0; i < n; ++i) {
        int old = f->perm[i], fi = i;
        for (int k = f->adj_ptr[old]; k < f->adj_ptr[old + 1]; ++k) {
            int j = f->iperm[f->adj[k]];
            if (j < fi) fi = j;
        }
        f->first[i] = fi;
        f->rowptr[i + 1] = f->rowptr[i] + (i - fi);
    }
    f->L = NEWD(f->rowptr[n]);
    f->Aenv = NEWD(f->rowptr[n]);
    f->D = NEWD(n);
    f->Adiag = NEWD(n);
}

/* get_A_triplets / update_A_coeffs values (src/TetElements.cpp:483-510), stored
 * as the lower envelope in the oracle ordering. */
static void assemble_A(orc_state* s) {
    env_ldl* f = &s->A;
    memset(f->Aenv, 0, sizeof(double) * (size_t)f->rowptr[f->n]);
    memset(f->Adiag, 0, sizeof(double) * (size_t)f->n);
    for (int e = 0; e < s->ne; ++e)
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b) {
                int i = s->fidx[4 * e + a], j = s->fidx[4 * e + b];
                if (i < 0 || j < 0 || i > j) continue;  /* upper triangle incl. diagonal */
                double v = s->w2[e] * s->DtD[16 * e + a + 4 * b];
                int ni = f->iperm[i], nj = f->iperm[j];
                if (ni == nj) f->Adiag[ni] += v;
                else {
                    int r = ni > nj ? ni : nj, c = ni > nj ? nj : ni;
                    f->Aenv[f->rowptr[r] + (c - f->first[r])] += v;
                }
            }
}

/* The same values as a full symmetric CSR matrix (both triangles). */
static int csr_slot(const env_ldl* f, int i, int j) {
    long lo = f->cptr[i] + 1, hi = f->cptr[i + 1] - 1;   /* neighbours are sorted */
    if (i == j) return 0;
    while (lo <= hi) {
        long m = (lo + hi) / 2;
        if (f->ccol[m] == j) return (int)(m - f->cptr[i]);
        if (f->ccol[m] < j) lo = m + 1; else hi = m - 1;
    }
    return -1;
}

static int assemble_A_csr(orc_state* s) {
    env_ldl* f = &s->A;
    memset(f->cval, 0, sizeof(double) * (size_t)f->cptr[f->n]);
    for (int e = 0; e < s->ne; ++e)
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b) {
                int i = s->fidx[4 * e + a], j = s->fidx[4 * e + b];
                if (i < 0 || j < 0 || i > j) continue;
                double v = s->w2[e] * s->DtD[16 * e + a + 4 * b];
                f->cval[f->cptr[i] + csr_slot(f, i, j)] += v;
                if (i != j) f->cval[f->cptr[j] + csr_slot(f, j, i)] += v;
            }
    for (int i = 0; i < f->n; ++i) {
        f->D[i] = f->cval[f->cptr[i]];
        if (!(f->D[i] > 0.0)) return E_NOT_SPD;
    }
    return E_OK;
}

/* Up-looking envelope LDL^T. */
static int factor_A(orc_state* s) {
    env_ldl* f = &s->A;
    if (s->p.linear_solver == 1) return assemble_A_csr(s);
    assemble_A(s);
    for (int i = 0; i < f->n; ++i) {
        double* Li = f->L + f->rowptr[i];
        const double* Ai = f->Aenv + f->rowptr[i];
        int fi = f->first[i];
        for (int j = fi; j < i; ++j) {
            /* w_j = A_ij - sum_k L_ik D_k L_jk ;  L_ij = w_j / D_j */
            double v = Ai[j - fi];
            int fj = f->first[j], lo = fi > fj ? fi : fj;
            const double* Lj = f->L + f->rowptr[j];
            for (int k = lo; k < j; ++k) v -= Li[k - fi] * f->D[k] * Lj[k - fj];
            Li[j - fi] = v / f->D[j];
        }
        double d = f->Adiag[i];
        for (int k = fi; k < i; ++k) d -= Li[k - fi] * Li[k - fi] * f->D[k];
        if (!(d > 0.0)) return E_NOT_SPD;
        f->D[i] = d;
    }
    return E_OK;
}

/* Column c of y = A x (n x 3 row-major blocks), rows split over host threads. */
static void csr_mv(const env_ldl* f, const double* x, double* y) {
    #pragma omp parallel for schedule(static)
    for (int i = 0; i < f->n; ++i) {
        double a0 = 0.0, a1 = 0.0, a2 = 0.0;
        for (long k = f->cptr[i]; k < f->cptr[i + 1]; ++k) {
            const double v = f->cval[k];
            const double* xj = x + 3L * f->ccol[k];
            a0 += v * xj[0]; a1 += v * xj[1]; a2 += v * xj[2];
        }
        y[3L * i] = a0; y[3L * i + 1] = a1; y[3L * i + 2] = a2;
    }
}

/* Per-column dot products of two n x 3 blocks: fixed chunks, partials summed in
 * chunk order (the same result for any thread count). */
static void dot3n(int n, const double* a, const double* b, double out[3]) {
    enum { CH = 4096 };
    const int nch = (n + CH - 1) / CH;
    double* part = NEWD(3L * nch);
    #pragma omp parallel for schedule(static)
    for (int c = 0; c < nch; ++c) {
        double s0 = 0.0, s1 = 0.0, s2 = 0.0;
        const int hi = (c + 1) * CH < n ? (c + 1) * CH : n;
        for (int i = c * CH; i < hi; ++i) {
            s0 += a[3L * i] * b[3L * i]; s1 += a[3L * i + 1] * b[3L * i + 1]; s2 += a[3L * i + 2] * b[3L * i + 2];
        }
        part[3 * c] = s0; part[3 * c + 1] = s1; part[3 * c + 2] = s2;
    }
    out[0] = out[1] = out[2] = 0.0;
    for (int c = 0; c < nch; ++c) { out[0] += part[3 * c]; out[1] += part[3 * c + 1]; out[2] += part[3 * c + 2]; }
    free(part);
}

/* x = A^-1 b by Jacobi-preconditioned conjugate gradients, the three columns
 * side by side, to |b - A x| <= 1e-14 |b| per column (restarted from the true
 * residual when the recurrence has drifted). */
static void cg_solve(orc_state* s, const double* b, double* x) {
    env_ldl* f = &s->A;
    const int n = f->n;
    const size_t m = 3 * (size_t)n;
    double *r = NEWD(m), *z = NEWD(m), *p = NEWD(m), *q = NEWD(m), *xx = NEWD(m);
    double bb[3], tol2[3];
    dot3n(n, b, b, bb);
    for (int c = 0; c < 3; ++c) tol2[c] = 1e-28 * bb[c];
    for (int restart = 0; restart < 4; ++restart) {
        csr_mv(f, xx, q);
        for (size_t i = 0; i < m; ++i) r[i] = b[i] - q[i];
        double rr[3];
        dot3n(n, r, r, rr);
        if (rr[0] <= tol2[0] && rr[1] <= tol2[1] && rr[2] <= tol2[2]) break;
        for (int i = 0; i < n; ++i) for (int c = 0; c < 3; ++c) z[3L * i + c] = r[3L * i + c] / f->D[i];
        memcpy(p, z, sizeof(double) * m);
        double rz[3];
        dot3n(n, r, z, rz);
        int done[3] = {rr[0] <= tol2[0], rr[1] <= tol2[1], rr[2] <= tol2[2]};
        for (int it = 0; it < 50000 && !(done[0] && done[1] && done[2]); ++it) {
            csr_mv(f, p, q);
            double pq[3], al[3];
            dot3n(n, p, q, pq);
            for (int c = 0; c < 3; ++c) al[c] = done[c] ? 0.0 : rz[c] / pq[c];
            #pragma omp parallel for schedule(static)
            for (int i = 0; i < n; ++i)
                for (int c = 0; c < 3; ++c) {
                    xx[3L * i + c] += al[c] * p[3L * i + c];
                    r[3L * i + c] -= al[c] * q[3L * i + c];
                    z[3L * i + c] = r[3L * i + c] / f->D[i];
                }
            double rz2[3], be[3];
            dot3n(n, r, z, rz2);
            dot3n(n, r, r, rr);
            for (int c = 0; c < 3; ++c) {
                if (rr[c] <= tol2[c]) done[c] = 1;
                be[c] = done[c] ? 0.0 : rz2[c] / rz[c];
                rz[c] = rz2[c];
            }
            #pragma omp parallel for schedule(static)
            for (int i = 0; i < n; ++i)
                for (int c = 0; c < 3; ++c) p[3L * i + c] = z[3L * i + c] + be[c] * p[3L * i + c];
        }
    }
    memcpy(x, xx, sizeof(double) * m);
    free(r); free(z); free(p); free(q); free(xx);
}

void orc_solve_A(orc_state* s, const double* b, double* x) {
    env_ldl* f = &s->A;
    int n = f->n;
    if (s->p.linear_solver == 1) { cg_solve(s, b, x); return; }
    double* z = NEWD(3 * n);
    for (int i = 0; i < n; ++i) for (int c = 0; c < 3; ++c) z[3 * i + c] = b[3 * f->perm[i] + c];
    for (int i = 0; i < n; ++i) {
        const double* Li = f->L + f->rowptr[i];
        for (int k = f->first[i]; k < i; ++k)
            for (int c = 0; c < 3; ++c) z[3 * i + c] -= Li[k - f->first[i]] * z[3 * k + c];
    }
    for (int i = 0; i < n; ++i) for (int c = 0; c < 3; ++c) z[3 * i + c] /= f->D[i];
    for (int i = n - 1; i >= 0; --i) {
        const double* Li = f->L + f->rowptr[i];
        for (int k = f->first[i]; k < i; ++k)
            for (int c = 0; c < 3; ++c) z[3 * k + c] -= Li[k - f->first[i]] * z[3 * i + c];
    }
    for (int i = 0; i < n; ++i) for (int c = 0; c < 3; ++c) x[3 * f->perm[i] + c] = z[3 * i + c];
    free(z);
}

/* ---- global objective ---------------------------------------------------- */
/* global_obj_grad() on the cache, src/TetElements.cpp:742-787 (gradient) and
 * the value term of global_obj_value, src/TetElements.cpp:678-688. */
double orc_global_grad_cached(orc_state* s, double* grad) {
    memset(grad, 0, sizeof(double) * 3 * (size_t)s->nf);
    double val = 0.0;
    for (int e = 0; e < s->ne; ++e) {
        const double *sg = s->sig + 3 * e, *Uu = s->Us + 9 * e, *Vv = s->Vs + 9 * e, *F = s->F + 9 * e;
        double P[9], T[9], Q[9], K[9], Mm[9];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) A3(P, r, c) = s->Z[9 * e + c + 3 * r] - s->U[9 * e + c + 3 * r];
        for (int r = 0; r < 3; ++r)  /* T = V^T P */
            for (int c = 0; c < 3; ++c) {
                double v = 0.0;
                for (int k = 0; k < 3; ++k) v += A3(Vv, k, r) * A3(P, k, c);
                A3(T, r, c) = v;
            }
        for (int r = 0; r < 3; ++r)  /* Q = T V */
            for (int c = 0; c < 3; ++c) {
                double v = 0.0;
                for (int k = 0; k < 3; ++k) v += A3(T, r, k) * A3(Vv, k, c);
                A3(Q, r, c) = v;
            }
        A3(K, 0, 0) = A3(Q, 0, 0) / sg[0];
        A3(K, 1, 1) = A3(Q, 1, 1) / sg[1];
        A3(K, 2, 2) = A3(Q, 2, 2) / sg[2];
        A3(K, 0, 1) = A3(K, 1, 0) = (A3(Q, 0, 1) + A3(Q, 1, 0)) / (sg[0] + sg[1]);
        A3(K, 0, 2) = A3(K, 2, 0) = (A3(Q, 0, 2) + A3(Q, 2, 0)) / (sg[0] + sg[2]);
        A3(K, 1, 2) = A3(K, 2, 1) = (A3(Q, 1, 2) + A3(Q, 2, 1)) / (sg[1] + sg[2]);
        /* M = F - U diag(s) K V^T */
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) {
                double v = 0.0;
                for (int a = 0; a < 3; ++a) {
                    double t = 0.0;
                    for (int b = 0; b < 3; ++b) t += A3(K, a, b) * A3(Vv, c, b);
                    v += A3(Uu, r, a) * sg[a] * t;
                }
                A3(Mm, r, c) = A3(F, r, c) - v;
            }
        const double* Di = s->Di + 12 * e;
        double w2 = s->w2[e];
        for (int a = 0; a < 4; ++a) {
            int j = s->fidx[4 * e + a];
            if (j < 0) continue;
            for (int r = 0; r < 3; ++r) {
                double v = 0.0;
                for (int c = 0; c < 3; ++c) v += Di[c + 3 * a] * (w2 * A3(Mm, r, c));
                grad[3 * j + r] += v;
            }
        }
        val += (0.5 * w2) * fro2_diff(s->symF + 9 * e, P);
    }
    return val;
}

double orc_global_grad(orc_state* s, const double* xfree, double* grad) {
    defo_cache_at(s, xfree);
    return orc_global_grad_cached(s, grad);
}

static double global_value(orc_state* s, const double* xfree) {
    defo_cache_at(s, xfree);
    double val = 0.0;
    for (int e = 0; e < s->ne; ++e) {
        double P[9];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) A3(P, r, c) = s->Z[9 * e + c + 3 * r] - s->U[9 * e + c + 3 * r];
        val += (0.5 * s->w2[e]) * fro2_diff(s->symF + 9 * e, P);
    }
    return val;
}

/* ---- local step: polar_update (NH), src/TetElements.cpp:256-356 ------------ */
static int prox_error;

double orc_polar_update(orc_state* s, int update_candidates) {
    double bef_pe = s->curr_pe, pe = 0.0, bef = 0.0, aft = 0.0;
    prox_error = 0;
    if (s->p.model == 1) {   /* ARAP branch, src/TetElements.cpp:265-282 */
        for (int e = 0; e < s->ne; ++e) {
            double *Z = s->Z + 9 * e, *U = s->U + 9 * e;
            const double* S = s->symF + 9 * e;
            double Sio[9], ZmU[9], SmI[9], SmU[9];
            for (int i = 0; i < 9; ++i) { Sio[i] = S[i] + U[i]; ZmU[i] = Z[i] - U[i]; SmI[i] = S[i]; }
            bef += 0.5 * s->w2[e] * fro2_diff(S, ZmU);
            for (int i = 0; i < 9; ++i) Sio[i] = 0.5 * Sio[i];
            for (int d = 0; d < 3; ++d) { Sio[4 * d] += 0.5; SmI[4 * d] -= 1.0; }
            double n2 = 0.0;
            for (int i = 0; i < 9; ++i) n2 += SmI[i] * SmI[i];
            pe += 0.5 * 1.0 * s->vol[e] * n2;
            for (int i = 0; i < 9; ++i) SmU[i] = Sio[i] - U[i];
            aft += 0.5 * s->w2[e] * fro2_diff(S, SmU);
            for (int i = 0; i < 9; ++i) { Z[i] = Sio[i]; U[i] += S[i] - Sio[i]; }
        }
        s->curr_pe = pe;
        return aft - bef + pe - bef_pe;
    }
    double* tmp = NEWD(3 * s->ne);
    for (int e = 0; e < s->ne; ++e) {
        double *Z = s->Z + 9 * e, *U = s->U + 9 * e;
        const double* S = s->symF + 9 * e;
        double Sin[9], ZmU[9], sg[3], Ue[9], Ve[9];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) {
                A3(Sin, r, c) = A3(S, c, r) + A3(U, c, r);
                A3(ZmU, r, c) = A3(Z, r, c) - A3(U, r, c);
            }
        bef += 0.5 * s->w2[e] * fro2_diff(S, ZmU);
        orc_svd3(Sin, sg, Ue, Ve);
        double* x = s->slast + 3 * e;
        double xs[3] = {x[0], x[1], x[2]};
        /* the reference ignores a failed line search and keeps the last iterate */
        (void)orc_prox_lbfgs(s->mu_e[e], s->lambda_e[e], sg, s->w2[e] / s->vol[e], xs, 20);
        memcpy(x, xs, sizeof xs);
        memcpy(tmp + 3 * e, xs, sizeof xs);
        if (xs[0] < 0.0 || xs[1] < 0.0 || xs[2] < 0.0) prox_error = 1;
        double So[9];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) {
                double v = 0.0;
                for (int k = 0; k < 3; ++k) v += A3(Ve, r, k) * xs[k] * A3(Ue, c, k);
                A3(So, r, c) = v;
            }
        pe += s->vol[e] * orc_nh_psi_plain(s->mu_e[e], s->lambda_e[e], xs);
        double SomU[9];
        for (int i = 0; i < 9; ++i) SomU[i] = So[i] - U[i];
        aft += 0.5 * s->w2[e] * fro2_diff(S, SomU);
        for (int i = 0; i < 9; ++i) { Z[i] = So[i]; U[i] += S[i] - So[i]; }
    }
    s->curr_pe = pe;
    if (update_candidates && s->p.reweighting) candidate_weights(s, tmp);
    free(tmp);
    return aft - bef + pe - bef_pe;
}

/* ---- global step: SplitLBFGS::minimize, deps/mcloptlib/include/MCL/SplitLBFGS.hpp:114-256 */
static double dotn(const double* a, const double* b, int n) {
    double v = 0.0;
    for (int i = 0; i < n; ++i) v += a[i] * b[i];
    return v;
}

static double* hist(double** v, int head, int M, int i) { return v[(head + i) % M]; }

/* Backtracking::search (deps/mcloptlib/include/MCL/Backtracking.hpp:71-98),
 * called by SplitMinimizer::linesearch for -global_ls 1 with p = -q: Armijo
 * sufficient decrease 1e-4, step factor 0.7, from alpha0; a direction of norm
 * <= machine epsilon returns the decrease constant.  `work` holds n doubles. */
static double backtracking(orc_state* s, const double* x, const double* q, double alpha0, double* work) {
    const int n = 3 * s->nf;
    const double decrease = 1.e-4, tau = 0.7;
    if (sqrt(dotn(q, q, n)) <= DBL_EPSILON) return decrease;
    double* g = NEWD(n);
    const double fx0 = orc_global_grad(s, x, g);
    const double gtp = -dotn(g, q, n);
    free(g);
    double alpha = alpha0;
    int iter = 0;
    for (; iter < 100000; ++iter) {
        for (int k = 0; k < n; ++k) work[k] = x[k] + alpha * -q[k];
        const double fxa = global_value(s, work);
        if (fxa <= fx0 + alpha * decrease * gtp) break;
        alpha *= tau;
    }
    return iter >= 100000 ? -1.0 : alpha;
}

static int lbfgs_minimize(orc_state* s, int* err) {
    int n = 3 * s->nf, M = s->M;
    double *q = s->q, *grad = s->grad, *gold = s->grad_old, *xo = s->x_old, *x = s->xfree;
    *err = E_OK;
    if (s->m_k == 0) {
        memset(q, 0, sizeof(double) * (size_t)n);
        memset(grad, 0, sizeof(double) * (size_t)n);
        memset(gold, 0, sizeof(double) * (size_t)n);
        memset(xo, 0, sizeof(double) * (size_t)n);
    }
    orc_global_grad_cached(s, grad);
    double dd = 0.0;
    for (int i = 0; i < n; ++i) { double d = grad[i] - gold[i]; dd += d * d; }
    if (dd < 1.e-13) return 0;
    int global_iter = 1, max_iters = s->p.global_iters, breaking = 0;
    double* st = NEWD(n);
    double* yt = NEWD(n);
    for (; global_iter <= max_iters; ++global_iter) {
        memcpy(xo, x, sizeof(double) * (size_t)n);
        memcpy(gold, grad, sizeof(double) * (size_t)n);
        memcpy(q, grad, sizeof(double) * (size_t)n);
        int iter = s->m_k < M ? s->m_k : M;
        for (int i = iter - 1; i >= 0; --i) {
            double *si = hist(s->s, s->head, M, i), *yi = hist(s->y, s->head, M, i);
            s->rho[i] = 1.0 / dotn(si, yi, n);
            s->alpha[i] = s->rho[i] * dotn(si, q, n);
            for (int k = 0; k < n; ++k) q[k] = q[k] - s->alpha[i] * yi[k];
        }
        orc_solve_A(s, q, q);
        for (int i = 0; i < iter; ++i) {
            double *si = hist(s->s, s->head, M, i), *yi = hist(s->y, s->head, M, i);
            double beta = s->rho[i] * dotn(yi, q, n);
            for (int k = 0; k < n; ++k) q[k] = q[k] + si[k] * (s->alpha[i] - beta);
        }
        double dir = dotn(grad, q, n);
        if (isnan(dir)) { *err = E_NAN; free(st); free(yt); return global_iter; }
        double alpha_init = 1.0;
        if (dir <= 0.0) {
            memcpy(q, grad, sizeof(double) * (size_t)n);
            max_iters -= s->m_k;
            s->m_k = 0;
            double gmax = 0.0;
            for (int k = 0; k < n; ++k) gmax = fabs(grad[k]) > gmax ? fabs(grad[k]) : gmax;
            alpha_init = 1.0 / gmax < 1.0 ? 1.0 / gmax : 1.0;
        }
        double rate = 1.0;   /* LSMethod::None -> rate 1 */
        if (s->p.global_ls && s->m_tol > 1.e-12) {
            rate = backtracking(s, x, q, alpha_init, st);
            if (rate <= 0.0) { free(st); free(yt); return -1; }   /* SplitMinimizer::FAILURE */
        }
        for (int k = 0; k < n; ++k) x[k] -= rate * q[k];
        orc_global_grad(s, x, grad);
        for (int k = 0; k < n; ++k) { st[k] = x[k] - xo[k]; yt[k] = grad[k] - gold[k]; }
        if (s->m_k < M) {
            memcpy(hist(s->s, s->head, M, s->m_k), st, sizeof(double) * (size_t)n);
            memcpy(hist(s->y, s->head, M, s->m_k), yt, sizeof(double) * (size_t)n);
        } else {
            /* erase(begin) + push_back: the oldest slot becomes the newest */
            memcpy(hist(s->s, s->head, M, 0), st, sizeof(double) * (size_t)n);
            memcpy(hist(s->y, s->head, M, 0), yt, sizeof(double) * (size_t)n);
            s->head = (s->head + 1) % M;
        }
        if (dir > 0.0 && (dir < s->p.kappa * s->m_tol || dir < s->p.kappa * 1.e-12)) {
            s->m_k += 1;
            memcpy(xo, x, sizeof(double) * (size_t)n);
            breaking = 1;
            break;
        }
        double denom = dotn(yt, yt, n);
        if (fabs(denom) <= 0.0) { breaking = 1; break; }
        s->m_k++;
    }
    free(st);
    free(yt);
    if (s->m_k > M) s->m_k = M;
    return breaking ? global_iter : global_iter - 1;
}

/* ---- rotation-unaware ADMM (-ra 0) ----------------------------------------- */
/* TetElements::update, src/TetElements.cpp:193-254: from F at the current x
 * (update_defo_cache), Ft = F^T + U; NH: SVD of Ft^T, prox from the last
 * stretches, Ft = V sigma* U^T; ARAP: Ft = (F' + rot(F'))^T / 2 with F' = Ft^T;
 * then U += F^T - Ft, Z = Ft. */
static void local_update_unaware(orc_state* s, int update_candidates) {
    double* tmp = NEWD(3 * s->ne);
    prox_error = 0;
    for (int e = 0; e < s->ne; ++e) {
        double *Z = s->Z + 9 * e, *U = s->U + 9 * e;
        const double* F = s->F + 9 * e;
        double Dx[9], Fp[9], Ft[9];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) A3(Dx, r, c) = A3(F, c, r);
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) A3(Fp, r, c) = A3(Dx, c, r) + A3(U, c, r);   /* (Dx + U)^T */
        if (s->p.model == 1) {
            double R[9];
            rot3(Fp, R);
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) A3(Ft, r, c) = 0.5 * (A3(Fp, c, r) + A3(R, c, r));
        } else {
            double sg[3], Ue[9], Ve[9];
            orc_svd3(Fp, sg, Ue, Ve);
            double* x = s->slast + 3 * e;
            double xs[3] = {x[0], x[1], x[2]};
            (void)orc_prox_lbfgs(s->mu_e[e], s->lambda_e[e], sg, s->w2[e] / s->vol[e], xs, 20);
            memcpy(x, xs, sizeof xs);
            memcpy(tmp + 3 * e, xs, sizeof xs);
            if (xs[0] < 0.0 || xs[1] < 0.0 || xs[2] < 0.0) prox_error = 1;
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) {
                    double v = 0.0;
                    for (int k = 0; k < 3; ++k) v += A3(Ve, r, k) * xs[k] * A3(Ue, c, k);
                    A3(Ft, r, c) = v;
                }
        }
        for (int i = 0; i < 9; ++i) { U[i] += Dx[i] - Ft[i]; Z[i] = Ft[i]; }
    }
    if (update_candidates && s->p.reweighting) candidate_weights(s, tmp);
    free(tmp);
}

/* UnawareGS::global_step, src/GlobalStepBehavior.hpp:162-180: b = sum_e w^2
 * Di^T (Z - U - Dfix xfix) (TetElements::add_to_b, src/TetElements.cpp:470-481),
 * x = A^-1 b per column, then the defo cache at the new x. */
static void global_step_unaware(orc_state* s) {
    const int n = 3 * s->nf;
    double* b = NEWD(n);
    for (int e = 0; e < s->ne; ++e) {
        const double* Di = s->Di + 12 * e;
        double T[9];
        for (int i = 0; i < 9; ++i) T[i] = s->Z[9 * e + i] - s->U[9 * e + i];
        if (s->nfree[e] < 4)
            for (int i = 0; i < 9; ++i) T[i] -= s->Dfx[9 * e + i];
        for (int a = 0; a < 4; ++a) {
            const int j = s->fidx[4 * e + a];
            if (j < 0) continue;
            for (int r = 0; r < 3; ++r) {
                double v = 0.0;
                for (int c = 0; c < 3; ++c) v += Di[c + 3 * a] * A3(T, c, r);
                b[3 * j + r] += s->w2[e] * v;
            }
        }
    }
    orc_solve_A(s, b, s->xfree);
    free(b);
    defo_cache_at(s, s->xfree);
}

/* ---- ADMM driver --------------------------------------------------------- */
static void load_positions(orc_state* s) {
    const orc_problem* p = &s->p;
    for (int i = 0; i < s->nv; ++i) {
        if (s->fix_of_vert[i] >= 0) for (int c = 0; c < 3; ++c) s->xfix[3 * s->fix_of_vert[i] + c] = p->init[3 * i + c];
        else for (int c = 0; c < 3; ++c) s->xfree[3 * s->free_of_vert[i] + c] = p->init[3 * i + c];
    }
    update_fix_cache(s);
}

/* initialize_dual_vars, src/TetElements.cpp:145-166, then m_curr_pe =
 * polar_potential_energy (src/TetElements.cpp:638-675). */
static void init_dual(orc_state* s) {
    double pe = 0.0;
    for (int e = 0; e < s->ne; ++e) {
        double F[9], sg[3], Uu[9], Vv[9];
        F_from_X(s, e, s->p.init, F);
        double* Z = s->Z + 9 * e;
        memset(s->U + 9 * e, 0, 9 * sizeof(double));
        if (!s->p.rot_aware) {   /* Z = Di x = F^T (src/TetElements.cpp:167-181) */
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) A3(Z, r, c) = A3(F, c, r);
            continue;
        }
        orc_svd3(F, sg, Uu, Vv);
        for (int r = 0; r < 3; ++r)   /* Z = S^T with S = V diag(s) V^T */
            for (int c = 0; c < 3; ++c) {
                double v = 0.0;
                for (int k = 0; k < 3; ++k) v += A3(Vv, c, k) * sg[k] * A3(Vv, r, k);
                A3(Z, r, c) = v;
            }
    }
    if (!s->p.rot_aware) return;
    for (int e = 0; e < s->ne; ++e) {
        if (s->p.model == 1) {   /* ARAP polar_potential_energy, src/TetElements.cpp:640-646 */
            const double* Z = s->Z + 9 * e;
            double n2 = 0.0;
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) { const double d = A3(Z, r, c) - (r == c ? 1.0 : 0.0); n2 += d * d; }
            pe += 0.5 * 1.0 * s->vol[e] * n2;
            continue;
        }
        double Zt[9], sg[3], Uu[9], Vv[9];
        for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) A3(Zt, r, c) = A3(s->Z + 9 * e, c, r);
        orc_svd3(Zt, sg, Uu, Vv);
        pe += s->vol[e] * orc_nh_psi_plain(s->mu_e[e], s->lambda_e[e], sg);
    }
    s->curr_pe = pe;
}

/* The TetElements-only sequence of a fresh mesh: positions at init, fix and
 * defo caches, dual variables (no weights update, no factorization). */
void orc_init_state(orc_state* s) {
    load_positions(s);
    defo_cache_at(s, s->xfree);
    init_dual(s);
}

int orc_setup(orc_state* s) {
    const orc_problem* p = &s->p;
    int rc;
    /* update_all_candidate_weights throws for any model but NH (src/TetElements.cpp:393-395) */
    if (p->reweighting && p->model != 0) return E_INPUT;
    load_positions(s);
    /* GlobalStepBehavior ctor: midupdate_weights(X_init), src/TetElements.cpp:360-381 */
    if (p->reweighting) {
        double* sg = NEWD(3 * s->ne);
        for (int e = 0; e < s->ne; ++e) {
            double F[9], Uu[9], Vv[9];
            F_from_X(s, e, p->init, F);
            orc_svd3(F, sg + 3 * e, Uu, Vv);
        }
        candidate_weights(s, sg);
        update_actual_weights(s);
        free(sg);
    }
    build_pattern(s);
    if ((rc = factor_A(s)) != E_OK) return rc;
    s->m_k = 0;
    /* ADMM::setup_solve, src/ADMM.cpp:89-107 */
    load_positions(s);
    defo_cache_at(s, s->xfree);
    init_dual(s);
    s->iter = 0;
    s->objectives[0] = orc_potential_energy(s);
    s->flips[0] = orc_inversion_count(s);
    s->reweighted[0] = 1;
    /* initialize_weights, src/GlobalStepBehavior.hpp:223-230 */
    if (p->reweighting) {
        candidate_weights(s, s->sig);
        update_actual_weights(s);
        if ((rc = factor_A(s)) != E_OK) return rc;
        s->m_k = 0;
    }
    s->setup_done = 1;
    return E_OK;
}

/* ADMM::iterate, src/ADMM.cpp:109-156; ADMM::converged, src/ADMM.cpp:158-169 */
int orc_iterate(orc_state* s) {
    const orc_problem* p = &s->p;
    int rc;
    if (!s->setup_done) return E_INPUT;
    if (s->iter >= p->max_iters) return E_INPUT;
    double dal = 0.0, obj_bef = 0.0, obj_aft = 0.0;
    int its = 1;
    if (!p->rot_aware) {
        /* local_update, update_defo_cache, UnawareGS::global_step (ADMM.cpp:117-133) */
        local_update_unaware(s, 1);
        if (prox_error) return E_PROX_NEG;
        global_step_unaware(s);
        obj_aft = 1.e8;   /* UnawareGS::last_step_delta_auglag */
    } else {
        dal = orc_polar_update(s, 1);
        if (prox_error) return E_PROX_NEG;
        defo_cache_at(s, s->xfree);
        obj_bef = global_value(s, s->xfree);
        s->m_tol = fabs(dal);
        its = lbfgs_minimize(s, &rc);
        if (rc != E_OK) return rc;
        obj_aft = global_value(s, s->xfree);
    }
    int rw = 0;
    if (p->reweighting) {
        if (p->rw_every > 0) rw = ((s->iter + 1) % p->rw_every) == 0;
        else rw = max_wsq_ratio(s) > p->gamma;
        if (rw) {
            update_actual_weights(s);
            if ((rc = factor_A(s)) != E_OK) return rc;
            s->m_k = 0;
        }
    }
    int k = s->iter;
    s->reweighted[k + 1] = rw;
    s->ls_dal[k] = fabs(dal);
    s->gs_dal[k] = fabs(obj_aft - obj_bef);
    s->inner[k] = its;
    s->objectives[k + 1] = orc_potential_energy(s);
    s->flips[k + 1] = orc_inversion_count(s);
    s->iter = k + 1;
    double res = fabs(s->objectives[k + 1] - s->objectives[k]) / (fabs(s->objectives[k + 1]) + 1.0);
    int conv = s->flips[k + 1] == 0 && s->flips[k] == 0 && res < p->tol;
    return conv ? 1 : 0;
}

int orc_solve(orc_state* s) {
    int rc = orc_setup(s);
    if (rc != E_OK) return rc;
    while (s->iter < s->p.max_iters) {
        rc = orc_iterate(s);
        if (rc < 0) return rc;
        if (rc == 1) break;
    }
    return s->iter;
}

/* ---- accessors ------------------------------------------------------------ */
long orc_get(const orc_state* s, const char* name, double* buf) {
    struct { const char* n; const double* p; long cnt; } tab[] = {
        {"Z", s->Z, 9L * s->ne}, {"U", s->U, 9L * s->ne}, {"F", s->F, 9L * s->ne},
        {"symF", s->symF, 9L * s->ne}, {"Usvd", s->Us, 9L * s->ne}, {"Vsvd", s->Vs, 9L * s->ne},
        {"sigma", s->sig, 3L * s->ne}, {"slast", s->slast, 3L * s->ne}, {"w2", s->w2, s->ne},
        {"w2c", s->w2c, s->ne}, {"vol", s->vol, s->ne}, {"xfree", s->xfree, 3L * s->nf},
        {"grad", s->grad, 3L * s->nf}, {"objectives", s->objectives, s->iter + 1L},
        {"ls_dal", s->ls_dal, s->iter}, {"gs_dal", s->gs_dal, s->iter},
    };
    for (size_t i = 0; i < sizeof tab / sizeof tab[0]; ++i)
        if (!strcmp(name, tab[i].n)) {
            if (buf) memcpy(buf, tab[i].p, sizeof(double) * (size_t)tab[i].cnt);
            return tab[i].cnt;
        }
    const int* ip = NULL;
    long cnt = 0;
    if (!strcmp(name, "flips")) { ip = s->flips; cnt = s->iter + 1L; }
    else if (!strcmp(name, "reweighted")) { ip = s->reweighted; cnt = s->iter + 1L; }
    else if (!strcmp(name, "inner_iters")) { ip = s->inner; cnt = s->iter; }
    if (ip) {
        if (buf) for (long i = 0; i < cnt; ++i) buf[i] = ip[i];
        return cnt;
    }
    if (!strcmp(name, "X")) {
        if (buf)
            for (int i = 0; i < s->nv; ++i)
                for (int c = 0; c < 3; ++c)
                    buf[3 * i + c] = s->free_of_vert[i] >= 0 ? s->xfree[3 * s->free_of_vert[i] + c]
                                                              : s->xfix[3 * s->fix_of_vert[i] + c];
        return 3L * s->nv;
    }
    return -1;
}

int orc_set(orc_state* s, const char* name, const double* buf) {
    double* dst = NULL;
    long cnt = 0;
    if (!strcmp(name, "Z")) { dst = s->Z; cnt = 9L * s->ne; }
    else if (!strcmp(name, "U")) { dst = s->U; cnt = 9L * s->ne; }
    else if (!strcmp(name, "w2")) { dst = s->w2; cnt = s->ne; }
    else if (!strcmp(name, "slast")) { dst = s->slast; cnt = 3L * s->ne; }
    else if (!strcmp(name, "xfree")) { dst = s->xfree; cnt = 3L * s->nf; }
    if (!dst) return E_INPUT;
    memcpy(dst, buf, sizeof(double) * (size_t)cnt);
    return E_OK;
}
