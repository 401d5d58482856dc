/* Test infrastructure: a CPU restatement, in plain C, of the reference's ADMM
 * solve loop (georgbrown/wrapd, Eigen-fallback path).  It is the checker the
 * CUDA implementation is compared against; nothing in the product links it.
 * Each function cites the reference code it restates.  It is pinned against
 * the reference itself (oracle/_ref, built from the reference sources) by
 * tests/test_oracle.py and by the golden vectors under tests/golden/.
 *
 * Conventions: 3x3 matrices are 9 doubles column-major (a[r + 3*c]), like
 * Eigen's default storage; per-vertex arrays are n x 3 row-major.
 */
#ifndef WRAPD_ORACLE_H
#define WRAPD_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- per-element math ---------------------------------------------------- */
void orc_svd3(const double F[9], double sigma[3], double U[9], double V[9]);
double orc_nh_psi(double mu, double lambda, const double x[3]);          /* energy_density */
double orc_nh_psi_plain(double mu, double lambda, const double x[3]);    /* energies (no x<0 guard) */
double orc_prox_value_grad(double mu, double lambda, const double x0[3], double wov,
                           const double x[3], double g[3]);
int orc_prox_lbfgs(double mu, double lambda, const double x0[3], double wov, double x[3], int max_iters);
double orc_hess_lmax(double mu, double lambda, const double sigma[3]);

/* ---- whole solve ---------------------------------------------------------- */
typedef struct {
    int n_verts, n_tets, n_pins;
    const double* rest;   /* n_verts x 3 */
    const double* init;   /* n_verts x 3 */
    const int* tets;      /* n_tets x 4, 0-based */
    const int* pins;      /* n_pins, any order */
    double youngs, poisson;
    int max_iters;        /* -it      (5000) */
    double tol;           /* -tol     (1e-11) */
    int lbfgs_m;          /* history  (6) */
    int global_iters;     /* -global_it (100) */
    double kappa;         /* -kappa   (1) */
    int reweighting;      /* -rw      (1) */
    int rw_delay;         /* -rw_delay (50) */
    double gamma;         /* -gamma   (1.5) */
    double beta_static, beta_min, beta_max;  /* (1, 0.1, 10) */
    int rw_every;         /* extension: >0 reweights every rw_every iterations instead of the gamma rule */
    const double* youngs_e;   /* extension: per-element Young's modulus (a batch of meshes), or NULL */
    const double* poisson_e;  /* extension: per-element Poisson ratio, or NULL */
    int rot_aware;        /* -ra      (1); 0 = UnawareGS (src/GlobalStepBehavior.hpp:118-193) */
    int model;            /* -model   (0 = nh, 1 = arap) */
    int global_ls;        /* -global_ls (0); 1 = Backtracking Armijo line search in the global step */
    int linear_solver;    /* 0: envelope LDL^T (default); 1: Jacobi-preconditioned conjugate gradients to a
                             relative residual of 1e-14, for systems whose envelope factor does not fit in
                             memory (the 3.9M-tet bar); same solve up to that residual */
} orc_problem;

void orc_problem_defaults(orc_problem* p);

typedef struct orc_state orc_state;

/* Returns NULL and sets *err (if given) on bad input; err codes match the C ABI. */
orc_state* orc_create(const orc_problem* p, int* err);
void orc_destroy(orc_state* s);

/* Everything ADMM::initialize + ADMM::solve do before the first iteration. */
int orc_setup(orc_state* s);
/* One ADMM iteration; returns 1 if converged after it, 0 if not, <0 on error. */
int orc_iterate(orc_state* s);
/* orc_setup + iterate until converged or max_iters; returns iterations or <0. */
int orc_solve(orc_state* s);

int orc_n_free(const orc_state* s);
int orc_iters(const orc_state* s);

/* Read a state array or log by name:
 *  per element:  "Z","U","F","symF","Usvd","Vsvd" (9), "sigma","slast" (3), "w2","w2c","vol" (1)
 *  per free vertex: "xfree","grad" (3)
 *  whole mesh: "X" (n_verts x 3)
 *  logs (iters+1 or iters entries): "objectives","flips","reweighted","inner_iters","ls_dal","gs_dal"
 * Returns the number of doubles written (buf may be NULL to query), or <0. */
long orc_get(const orc_state* s, const char* name, double* buf);
/* Overwrite a state array ("Z","U","w2","slast","xfree"). */
int orc_set(orc_state* s, const char* name, const double* buf);

/* Components, for per-stage parity checks. */
void orc_init_state(orc_state* s);                           /* positions, caches, dual variables */
void orc_update_defo_cache(orc_state* s);                   /* F, SVD, symF at xfree */
double orc_polar_update(orc_state* s, int update_candidates); /* local step, returns delta-AL */
double orc_global_grad_cached(orc_state* s, double* grad);   /* uses the cache */
double orc_global_grad(orc_state* s, const double* xfree, double* grad); /* refreshes cache at xfree */
double orc_potential_energy(const orc_state* s);
int orc_inversion_count(const orc_state* s);
/* Apply A^-1 (the factored weighted Laplacian) to an n_free x 3 block. */
void orc_solve_A(orc_state* s, const double* b, double* x);

#ifdef __cplusplus
}
#endif
#endif
