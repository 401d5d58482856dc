/* wrapd_gpu.h -- C ABI of the B200 implementation of WRAPD's ADMM solve loop.
 *
 * The reference (georgbrown/wrapd) exposes the path as C++ classes, not a C
 * ABI: wrapd::Solver (src/Solver.hpp:37-72), wrapd::System (src/System.hpp:
 * 41-174) and wrapd::TetElements (src/TetElements.hpp:165-247), driven by the
 * `quasi` front end (samples/tests/quasi.cpp:44-144) and
 * binding::add_tetmesh (samples/utils/AddMeshes.hpp:61-132).  Each entry point
 * below names the reference interface it replaces.
 *
 * Conventions
 *   - Every function returns 0 on success or a negative WRAPD_E_* code; no C++
 *     exception crosses this boundary.  wrapd_last_error() gives the message.
 *   - The caller owns every host buffer; the library owns device memory.
 *   - Positions are n x 3 row-major doubles; tets are n_tets x 4 0-based ids.
 *   - One handle per host thread.  Each handle has its own CUDA stream.
 *   - There is no CPU fallback: without a usable CUDA device wrapd_create
 *     fails with WRAPD_E_CUDA.
 */
#ifndef WRAPD_GPU_H
#define WRAPD_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WRAPD_ABI_VERSION 1

#if defined(__GNUC__)
#define WRAPD_API __attribute__((visibility("default")))
#else
#define WRAPD_API
#endif

enum {
    WRAPD_OK = 0,
    WRAPD_E_INPUT = -1,          /* bad argument (std::runtime_error in Settings.cpp:164, MeshIO.hpp:309-311) */
    WRAPD_E_INVERTED_REST = -2,  /* inverted rest tet (src/TetElements.cpp:99-101) */
    WRAPD_E_NOT_SPD = -3,        /* non-positive pivot while factoring D^T W D */
    WRAPD_E_NAN = -4,            /* NaN L-BFGS decrement (deps/mcloptlib/include/MCL/SplitLBFGS.hpp:181-184) */
    WRAPD_E_PROX_NEG = -5,       /* negative prox stretch (src/TetElements.cpp:320-323) */
    WRAPD_E_TIMEOUT = -6,        /* a bounded device wait gave up */
    WRAPD_E_OOM = -7,            /* device allocation failed */
    WRAPD_E_CUDA = -8,           /* any other CUDA error, or no device */
    WRAPD_E_STATE = -9,          /* call out of order (e.g. solve before initialize) */
    WRAPD_E_UNSUPPORTED = -10    /* an option this library does not implement */
};

/* Solver options.  Field meanings and defaults follow wrapd::Settings
 * (src/Settings.hpp:103-162), ModelSettings (src/ModelSettings.hpp:33-41),
 * Settings::GStep (src/Settings.hpp:121-149) and the flags parsed in
 * src/Settings.cpp:31-176; the fields after `prox_iters` are extensions. */
typedef struct wrapd_settings {
    int max_iters;        /* -it         5000  */
    double tol;           /* -tol        1e-11 */
    int rot_aware;        /* -ra         1 (0: rotation-unaware global step, x = A^-1 b) */
    int reweighting;      /* -rw         1     */
    int rw_delay;         /* -rw_delay   50    */
    double gamma;         /* -gamma      1.5   */
    int global_iters;     /* -global_it  100   */
    int global_ls;        /* -global_ls  0 (1: backtracking line search in the global step) */
    double kappa;         /* -kappa      1     */
    int model;            /* -model      0 = nh, 1 = arap */
    double poisson;       /* -poisson    0.45  */
    double beta_static;   /* -beta_static 1    */
    double beta_min;      /* -beta_min   0.1   */
    double beta_max;      /* -beta_max   10    */
    int prox_iters;       /* prox L-BFGS iterations, 20 (src/ModelSettings.hpp:40) */
    /* extensions */
    double youngs;        /* Young's modulus, 1e7 Pa (hard-coded in src/Lame.hpp:38) */
    int lbfgs_m;          /* global L-BFGS history, 6 (SplitLBFGS.hpp:41) */
    int rw_every;         /* 0: gamma rule; N > 0: reweight (and refactor) every N iterations */
    int precision;        /* 0: FP64 throughout; 1: FP32 local step (SVD + Newton prox), FP64 elsewhere */
    int prox_mode;        /* 0: L-BFGS prox as the reference (parity mode); 1: Newton prox;
                             2: Newton prox warm-started by the prox network (wrapd_set_prox_net) on
                             the first local step and the one after each reweight, from the last
                             stretches elsewhere */
    int leaf_size;        /* nested-dissection leaf size for the factorization, 64 */
    int verbose;          /* -p          0 here (1 prints the reference's table) */
    int device;           /* CUDA device ordinal, 0 */
    int autotune;         /* 0; 1: wrapd_initialize times the candidate tile shapes of the triangular
                             solve (chunk length per level and direction) and of the factorization's
                             panel steps (fused or split, by the number of tiles), and the first
                             wrapd_begin_solve the local step's tile (64, 128, 256 or 512 elements per
                             CTA), on this system, and keeps the fastest (see wrapd_get_tuning) */
} wrapd_settings;

typedef struct wrapd_handle wrapd_handle;

/* Log channels of wrapd_get_log (AlgorithmData, src/AlgorithmData.hpp:43-73). */
enum {
    WRAPD_LOG_OBJECTIVES = 0,       /* iters + 1 entries: potential energy per iterate */
    WRAPD_LOG_REWEIGHTED = 1,       /* iters + 1 entries (entry 0 is 1, as the reference logs) */
    WRAPD_LOG_FLIPS = 2,            /* iters + 1 entries: inverted elements */
    WRAPD_LOG_INNER_ITERS = 3,      /* iters entries: global L-BFGS iterations */
    WRAPD_LOG_LS_DELTA_AL = 4,      /* iters entries: |delta AL| of the local step */
    WRAPD_LOG_GS_DELTA_AL = 5,      /* iters entries: |delta AL| of the global step */
    WRAPD_LOG_ACCUMULATED_TIME_S = 6, /* iters + 1 entries: local + global + refactor seconds */
    WRAPD_LOG_X_ERRORS = 7,         /* iters + 1 entries: |x - x_soln| / |x_init - x_soln| */
    WRAPD_LOG_PROX_ITERS = 8        /* iters entries: mean prox iterations per element (extension) */
};

/* Defaults of wrapd::Settings() + ModelSettings() (src/Settings.hpp:154-162,
 * src/ModelSettings.hpp:33-41). */
WRAPD_API int wrapd_settings_default(wrapd_settings* s);

/* wrapd::Solver::Solver(const Settings&) (src/Solver.cpp:32-35). */
WRAPD_API int wrapd_create(const wrapd_settings* s, wrapd_handle** out);

/* binding::add_tetmesh + System::add_nodes + create_tets_from_mesh +
 * Solver::set_pins (samples/utils/AddMeshes.hpp:61-132, src/System.hpp:75-92,
 * src/TetElements.hpp:250-288, src/System.cpp:33-44).  Pins are vertex ids
 * held in place at init_xyz.  soln_xyz may be NULL.  Called again before
 * wrapd_initialize, it appends another mesh (vertex ids of each call are its
 * own, shifted as add_tetmesh's prev_tet_verts does): the meshes form a
 * batch.  Each mesh is solved as the reference solves it alone -- its own
 * L-BFGS history, early exits, reweighting decisions and convergence test,
 * bit for bit the same as a handle holding that mesh only -- while the work
 * of all of them shares the launches: one local-step and one gradient launch
 * over the unconverged meshes' element tiles, one factorization holding one
 * tree per mesh.  A converged mesh drops out of the launches.  Batches take
 * the rotation-aware global step without line search (rot_aware = 1,
 * global_ls = 0; others give WRAPD_E_UNSUPPORTED at wrapd_initialize).  (The
 * reference's add_tetmesh replaces the element set on a second call; the
 * batch is an extension.)  Positions are returned in the order added. */
WRAPD_API int wrapd_add_tetmesh(wrapd_handle* h, const double* rest_xyz, const double* init_xyz,
                      const double* soln_xyz, int n_verts, const int32_t* tets, int n_tets,
                      const int32_t* pins, int n_pins);

/* wrapd_add_tetmesh with the mesh's own material (extension): Young's
 * modulus and Poisson ratio of this mesh in place of the settings' youngs and
 * poisson, for batches of meshes of different materials. */
WRAPD_API int wrapd_add_tetmesh_material(wrapd_handle* h, const double* rest_xyz, const double* init_xyz,
                                         const double* soln_xyz, int n_verts, const int32_t* tets, int n_tets,
                                         const int32_t* pins, int n_pins, double youngs, double poisson);

/* wrapd::Solver::initialize (src/Solver.cpp:48-60) -> ADMM::initialize
 * (src/ADMM.cpp:34-56): element precompute, initial weights, symbolic
 * analysis (one nested dissection per mesh) and the first numeric
 * factorization, all on the device. */
WRAPD_API int wrapd_initialize(wrapd_handle* h);

/* wrapd::Solver::solve (src/Solver.cpp:38-46) -> ADMM::solve
 * (src/ADMM.cpp:59-84): iterate to convergence or max_iters and write the
 * final positions (n_verts x 3) to x_out (may be NULL). */
WRAPD_API int wrapd_solve(wrapd_handle* h, double* x_out);

/* The two halves of ADMM::solve, for stepping: wrapd_begin_solve runs
 * setup_solve + initialize_weights (src/ADMM.cpp:60-72, 89-107);
 * wrapd_iterate runs up to n iterations of ADMM::iterate + converged
 * (src/ADMM.cpp:109-169) and reports *converged; wrapd_get_positions is
 * ADMM::finish_solve (src/ADMM.cpp:171-182). */
WRAPD_API int wrapd_begin_solve(wrapd_handle* h);
WRAPD_API int wrapd_iterate(wrapd_handle* h, int n, int* iters_done, int* converged);
WRAPD_API int wrapd_get_positions(wrapd_handle* h, double* x_out);

/* AlgorithmData per-iteration logs (src/AlgorithmData.hpp:43-73).  Copies up
 * to cap entries into out; *len receives the channel's length. */
WRAPD_API int wrapd_get_log(wrapd_handle* h, int which, double* out, int cap, int* len);

/* The log channel of one mesh of a batch (meshes numbered in the order they
 * were added): each mesh is an independent ADMM solve -- its own L-BFGS
 * history and early exits, reweighting decisions and convergence test, as a
 * reference Solver holding that mesh alone -- and stops logging when it
 * converges.  wrapd_get_log gives, for a batch, the sums over its meshes of
 * the energies, flips, inner iterations and |delta AL|, 1 where any mesh
 * reweighted, and the batch's x error.  (No reference counterpart: the
 * reference solves one mesh per Solver.) */
WRAPD_API int wrapd_get_mesh_log(wrapd_handle* h, int mesh, int which, double* out, int cap, int* len);

/* RuntimeData (src/RuntimeData.hpp:30-44): ms[0..5] = setup, local, global,
 * refactor, finish, inner iterations (as a double).  Device times from CUDA
 * events on the handle's stream. */
WRAPD_API int wrapd_get_runtime(wrapd_handle* h, double ms[6]);

/* Problem sizes: out[0..7] = n_verts, n_tets, n_free, n_pins, fronts, levels,
 * nnz(L), factorization flops. */
WRAPD_API int wrapd_get_info(wrapd_handle* h, double out[8]);

/* Work counters since wrapd_create: out[0..3] = kernel launches issued by the
 * handle, numeric factorizations, triangular solves (3 RHS each), host
 * synchronisations.  (No reference counterpart: instrumentation.) */
WRAPD_API int wrapd_get_counters(wrapd_handle* h, int64_t out[4]);

/* The tile shapes in use (no reference counterpart): out[0] = the largest
 * panel step (in tiles) whose diagonal block is factored inside the tile
 * launch, out[1] = levels L, then L forward and L backward solve chunk
 * lengths (0: each mesh of a batch takes its own), then the local step's
 * tile (elements per CTA).  *len receives 3 + 2 L.  Chosen by timing when
 * autotune = 1 (the local tile at the first wrapd_begin_solve), by fixed
 * rules otherwise. */
WRAPD_API int wrapd_get_tuning(wrapd_handle* h, int* out, int cap, int* len);

/* Per-phase device timeline (no reference counterpart; the reference's
 * MicroTimer splits only local/global/refactor).  wrapd_set_profiling(h, 1)
 * records CUDA events at phase boundaries of every later iteration;
 * wrapd_get_profile returns accumulated ms and interval counts for the slots
 * 0 local step, 1 gradient + gather, 2 two-loop and x-update vector kernels,
 * 3 triangular solves, 4 (unused), 5 device idle around host synchronisations
 * and the reweight/refactor phase. */
WRAPD_API int wrapd_set_profiling(wrapd_handle* h, int on);
WRAPD_API int wrapd_get_profile(wrapd_handle* h, double ms[6], int64_t counts[6]);

WRAPD_API const char* wrapd_last_error(const wrapd_handle* h);
WRAPD_API void wrapd_destroy(wrapd_handle* h);

/* ---- TetElements-level entry points (public methods of wrapd::TetElements,
 * src/TetElements.hpp:165-207), used by the parity tests. ---------------- */

/* Read or overwrite a state array by name.  Per element, in input order:
 * "Z","U","symF" (9, the reference's column-major Mat3x3), "slast" (3),
 * "w2","w2c","vol" (1).  Per free vertex in ascending vertex id order:
 * "xfree","grad" (3).  Returns the element count written via *len.  Under
 * rw_every, wrapd_solve/wrapd_iterate refresh "w2c" only in the local step of
 * a reweighting iteration (the one that reads it). */
WRAPD_API int wrapd_get_state(wrapd_handle* h, const char* name, double* out, int64_t cap, int64_t* len);
WRAPD_API int wrapd_set_state(wrapd_handle* h, const char* name, const double* in, int64_t n);

/* TetElements::update_defo_cache(x_free) (src/TetElements.cpp:564-596). */
WRAPD_API int wrapd_update_defo_cache(wrapd_handle* h);

/* TetElements::polar_update (src/TetElements.cpp:256-356): returns delta-AL. */
WRAPD_API int wrapd_polar_update(wrapd_handle* h, int update_candidates, double* delta_al);

/* TetElements::global_obj_grad(x_free, g) (src/TetElements.cpp:691-738):
 * refreshes the cache at x_free (n_free x 3, NULL = current), writes the
 * gradient (n_free x 3) and the AL value. */
WRAPD_API int wrapd_global_grad(wrapd_handle* h, const double* x_free, double* grad, double* value);

/* TetElements::potential_energy_x + inversion_count on the cache
 * (src/TetElements.cpp:444-468, 598-635). */
WRAPD_API int wrapd_potential_energy(wrapd_handle* h, double* pe, int* flips);

/* LinearSolver::solve applied to the 3 columns (SplitLBFGS.hpp:165-167):
 * x = A^-1 b for an n_free x 3 block (free vertices in ascending id order). */
WRAPD_API int wrapd_solve_A(wrapd_handle* h, const double* b, double* x);

/* The bounded waits of the solve (no reference counterpart): wrapd_solve_A
 * with front `front` of the assembly tree never reporting completion, so the
 * wait of its parent's forward items runs out after about a second.  Returns
 * WRAPD_E_TIMEOUT when it did (x then holds no solution) and leaves the handle
 * usable; WRAPD_E_INPUT for a front outside [0, fronts) (wrapd_get_info). */
WRAPD_API int wrapd_solve_A_holding(wrapd_handle* h, const double* b, double* x, int front);

/* ---- per-element math over a batch, on the current device (handle-free) --
 * The same device functions the ADMM kernels inline.  fp32 = 1 runs them in
 * single precision (the element math of mixed mode). */

/* math::svd with the rotation sign fix (src/Math.hpp:140-193): F is n x 9
 * column-major 3x3 matrices; sigma n x 3; U, V n x 9. */
WRAPD_API int wrapd_svd3_batch(int n, int fp32, const double* F, double* sigma, double* U, double* V);

/* The per-element prox of polar_update (src/TetElements.cpp:312-317): NHProx
 * with x0 = sigma0 and w^2/vol = wov, minimised by LBFGS<3> with cubic
 * backtracking (deps/mcloptlib/include/MCL/LBFGS.hpp:52-152) from `start`;
 * out n x 3, iters n (LBFGS::minimize's return value). */
WRAPD_API int wrapd_prox_batch(int n, int fp32, double mu, double lambda, int max_iters, const double* sigma0,
                               const double* wov, const double* start, double* out, int* iters);

/* Candidate stiffness before the volume factor: max eigenvalue of
 * makePD(hessian_density(sigma)) (src/TetElements.cpp:414-416). */
WRAPD_API int wrapd_hess_lmax_batch(int n, double mu, double lambda, const double* sigma, double* out);

/* TetElements::potential_energy_x + inversion_count (src/TetElements.cpp:
 * 598-635, 444-468) over a batch of stretch triples: *pe = sum vol * psi(sigma),
 * *flips = triples with a negative entry.  sigma n x 3, vol n (host). */
WRAPD_API int wrapd_potential_energy_batch(int n, double mu, double lambda, const double* sigma, const double* vol,
                                           double* pe, int* flips);

/* The batched potential energy and inversion count above, for callers that may
 * not allocate device memory: host code that has handed the GPU's memory to its
 * own allocator, or that runs under a rule of no device allocation after
 * start-up (an application that reserves all GPU memory up front, a loop that
 * cannot take the implicit synchronisation of cudaMalloc).  No counterpart in
 * the reference.
 *   d_sigma (n x 3), d_vol (n) and d_out (2 doubles: sum vol * psi, inverted
 *   count) are device pointers owned by the caller; the work is queued on
 *   `stream` (a cudaStream_t, NULL for the default stream) and d_out is ready
 *   when that stream has reached it.
 *   Nothing is allocated: the reduction's scratch is a fixed array of about
 *   1 MiB inside the library, held by every GPU that loads it until exit.
 *   n may be at most 16,777,216; larger n returns WRAPD_E_INPUT without work.
 *   The first call on each device looks up that array's device address (with
 *   the device current); make that first call before any stream capture.  The
 *   address is kept for the life of the process: do not call this entry point
 *   after resetting the device (cudaDeviceReset) in the same process.
 *   All calls share the one array: calls that overlap on the GPU (other
 *   streams or threads) race and give wrong sums, so serialise them. */
WRAPD_API int wrapd_potential_energy_batch_noalloc(int n, double mu, double lambda, const double* d_sigma,
                                                   const double* d_vol, double* d_out, void* stream);

/* The Newton prox of prox_mode 1 (no reference counterpart: the reference
 * keeps mcloptlib's Newton commented out, src/TetElements.cpp:215, 304):
 * NHProx with x0 = sigma0, w^2/vol = wov, from `start`, until |g| <= tol *
 * wov * max(1, |x|) or the step is below tol * max(1, |x|); out n x 3, iters n
 * (nullable). */
WRAPD_API int wrapd_prox_newton_batch(int n, int fp32, double mu, double lambda, double tol, int max_iters,
                                      const double* sigma0, const double* wov, const double* start, double* out,
                                      int* iters);

/* ---- prox network (no reference counterpart) --------------------------------
 * A 5 -> 64 -> 64 -> 3 GELU MLP that predicts the prox stretches from
 * (sorted singular values of S_in, log(w^2 / (vol mu)), log(mu / lambda)); it
 * warm-starts the Newton prox under prox_mode 2.  Parameters are an FP32 blob
 * of WRAPD_NET_BLOB floats: feature mean[5], 1/std[5], output scale[3], 3 pad,
 * W1[64][5], b1[64], W2[64][64], b2[64], W3[3][64], b3[3]; the prediction is
 * sigma_in + scale * y.  Kernels compute with BF16 operands and FP32
 * accumulation.  Training: features n x 5 (raw, as above), targets n x 3 (the
 * converged prox stretches); loss = mean squared error of the normalised
 * output (sigma* - sigma_in) / scale; Adam (0.9, 0.999, 1e-8) with a cosine
 * rate from lr to lr_end.  Deterministic for a given seed. */
#define WRAPD_NET_BLOB 4755
typedef struct wrapd_prox_net wrapd_prox_net;
WRAPD_API int wrapd_net_create(const float* blob, int n_blob, wrapd_prox_net** out);
WRAPD_API int wrapd_net_set_data(wrapd_prox_net* h, const float* features, const float* targets, int64_t n);
/* epoch_loss: `epochs` entries (nullable), the mean loss seen over each epoch. */
WRAPD_API int wrapd_net_train(wrapd_prox_net* h, int epochs, int batch, float lr, float lr_end, uint64_t seed,
                              double* epoch_loss);
/* Loss and gradient (WRAPD_NET_BLOB - 16 floats, the trained part of the blob)
 * over samples [first, first + n) of the data, without an update. */
WRAPD_API int wrapd_net_grad(wrapd_prox_net* h, int64_t first, int n, double* loss, float* grad);
WRAPD_API int wrapd_net_get(wrapd_prox_net* h, float* blob);
WRAPD_API const char* wrapd_net_last_error(wrapd_prox_net* h);   /* h may be NULL: last create/predict error */
WRAPD_API void wrapd_net_destroy(wrapd_prox_net* h);
/* Predicted prox stretches for n samples: sigma_in n x 3 (sorted singular
 * values), wov n (w^2 / vol); out n x 3. */
WRAPD_API int wrapd_net_predict(const float* blob, int n_blob, int n, const double* sigma_in, const double* wov,
                                double mu, double lambda, double* out);
/* Installs the network used by prox_mode 2 (copied; call before begin_solve). */
WRAPD_API int wrapd_set_prox_net(wrapd_handle* h, const float* blob, int n_blob);

/* Measured FP64 tensor-core throughput of this GPU (TFLOP/s): back-to-back
 * mma.sync m8n8k4 f64 from registers on every SM for `iters` rounds, timed by
 * CUDA events.  The roofline denominator of the factorization (no reference
 * counterpart). */
WRAPD_API int wrapd_dmma_peak(int iters, double* tflops);

/* ---- Host-only planning: no CUDA call, no device memory ------------------
 * The symbolic analysis that wrapd_initialize runs on the host, for one mesh,
 * with no GPU needed: the nested-dissection order of the free vertices, the
 * assembly tree of dense fronts, and the sizes of the factor's device pools,
 * so a job can be sized against the GPU's memory before a handle exists.
 * Stands for the analyzePattern step of the reference's SimplicialLDLT
 * (deps/mcloptlib/include/MCL/LinearSolver.hpp:279-298, AMD ordering there;
 * geometric nested dissection here).  Errors: wrapd_last_error(NULL). */
typedef struct wrapd_plan wrapd_plan;

/* Mesh arguments as wrapd_add_tetmesh (rest positions n_verts x 3, tets
 * n_tets x 4 0-based, distinct pinned vertex ids); leaf_size <= 0 takes the
 * default of the settings (64).  Free vertices are numbered in ascending
 * vertex id order with the pinned ones skipped, as the solver numbers them. */
WRAPD_API int wrapd_plan_create(const double* rest_xyz, int n_verts, const int32_t* tets, int n_tets,
                                const int32_t* pins, int n_pins, int leaf_size, wrapd_plan** out);

/* out[0..7] = free vertices, fronts, levels, stored factor entries (dense
 * fronts: k(k+1)/2 + k r each), F-pool bytes and Y-pool bytes (FP64; the two
 * largest device allocations of a solve), total front rows (the length of
 * the row and relative-index arrays), factorization flops (rounded). */
WRAPD_API int wrapd_plan_info(const wrapd_plan* p, int64_t out[8]);

/* perm (free vertices): the free index of the vertex in each column of the
 * new order.  Per front, in post-order (children before their parent): first
 * column, column count, parent front (-1 for a root), level (one more than
 * its highest child, 0 for a leaf); row_ptr (fronts + 1) delimits its rows
 * (new numbering, sorted, after its own columns) in `rows`, and `relmap`
 * gives where each row lands in the parent's front (t < k_parent: the
 * parent's column t; k_parent + t: the parent's row t).  Any output may be
 * NULL. */
WRAPD_API int wrapd_plan_fronts(const wrapd_plan* p, int32_t* perm, int32_t* first, int32_t* ncols,
                                int32_t* parent, int32_t* level, int64_t* row_ptr, int32_t* rows,
                                int32_t* relmap);
WRAPD_API void wrapd_plan_destroy(wrapd_plan* p);

#ifdef __cplusplus
}
#endif
#endif /* WRAPD_GPU_H */
