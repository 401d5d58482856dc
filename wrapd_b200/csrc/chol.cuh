// GPU multifrontal Cholesky of the free-vertex weighted Laplacian
// A = sum_e w_e^2 D_e^T D_e and its 3-right-hand-side solve.  Replaces the
// reference's Eigen SimplicialLDLT (deps/mcloptlib/include/MCL/
// LinearSolver.hpp:279-298): `factor` is LinearSolver::factorize,
// `solve` is the three LinearSolver::solve calls of SplitLBFGS.hpp:165-167.
//
// Storage (all device, FP64):
//   F pool  one (k+r) x (k+r) column-major frontal matrix per front.  After
//           factoring, columns 0..k-1 hold the front's panel of L
//           (L_ss on top, L_rs below) and the trailing r x r block holds the
//           update matrix that the parent assembles.
//   Y pool  one (k + r) x k block per front, column-major with an even
//           leading dimension ldy >= k + r: rows 0..k-1 hold Y = inv(L_ss)
//           (lower triangular, built during the factorization), rows k..k+r-1
//           hold W = L_rs inv(L_ss).
//   With Y and W the solve needs no serial substitution: per front, forward
//   x_s = Y t_s and u_s = v_s - W t_s, backward y_s = Y^T z_s - W^T y_rows,
//   i.e. one pass of 2D-tiled matrix-vector products over [Y; W] per level.
//   vectors n x 3 row-major in the nested-dissection order (3 RHS at once).
#pragma once
#include <vector>

#include "common.cuh"
#include "symbolic.hpp"

namespace wrapd {

struct FrontDesc {
    int first, k, r, ld;
    int64_t f_off, y_off, u_off, rows_off, rel_off, inv_off;
    int nchild, child0, child1, ldy;   // ldy: leading dimension of the front's [Y; W] block
    int mesh;                          // the mesh of a batch the front belongs to (0: one mesh)
    int parent;                        // -1 at a root
};

// A trailing-update job of the blocked factorization: C -= A B'^T over a K range
// of panel columns.  kind 0: C is F[r0:r1, c0:c1] of the front (lower part
// where rows and columns overlap), A = F[r0:r1, k0:k1], B' = F[c0:c1, k0:k1];
// kind 1: C is Y[r0:r1, c0:c1], A = F[r0:r1, k0:k1], B'(j, t) = Y[k0 + t, c0 + j].
// A solve work item: a 64-wide band starting at b0 (rows forward, columns
// backward) times the chunk [lo, hi) of the other dimension.  The band's items
// are contiguous, starting at `first`, `nchunk` of them; `band` indexes the
// arrival counter.
struct SolveItem {
    int front, b0, lo, hi, nchunk, first, band;
};

// The items of every level of one direction as one work list (see k_fwd_queue):
// head is the next item to take; done[f] counts the bands of front f written,
// complete at nbands[f]; status receives WRAPD_E_TIMEOUT from a wait that gave
// up; hold is a front whose completion is never counted (-1: none), which
// makes the waits on it run out (the test of that path).
struct SolveQueue {
    const SolveItem* items;
    int n;
    unsigned* head;
    unsigned* done;
    const unsigned* nbands;
    int* status;
    int hold;
};

struct GemmJob {
    int front, kind, r0, r1, c0, c1, k0, k1;
};

struct JobList {
    int n = 0;
    int total = 0;       // total CTAs (64 x 64 output tiles)
    GemmJob* d_jobs = nullptr;
    int* d_prefix = nullptr;
};

// One launch's work: `n` fronts (ids), each owning prefix[i+1]-prefix[i] CTAs.
struct WorkList {
    int n = 0;
    int total = 0;       // total CTAs
    int* d_fronts = nullptr;
    int* d_prefix = nullptr;
};

class CholGPU {
public:
    CholGPU() = default;
    ~CholGPU();
    bool use_graphs = true;
    CholGPU(const CholGPU&) = delete;
    CholGPU& operator=(const CholGPU&) = delete;

    // Upload the symbolic structures.  A_pos/A_ptr/A_contrib describe the
    // lower-triangle entries of A: entry t goes to F-pool offset A_pos[t] and
    // sums w2[e] * (D_e^T D_e)(a, b) over contributions c = e*16 + a*4 + b in
    // A_contrib[A_ptr[t] .. A_ptr[t+1]).
    void build(const Symbolic& S, const std::vector<int64_t>& A_pos, const std::vector<int>& A_ptr,
               const std::vector<int>& A_contrib, cudaStream_t st);
    // Numeric factorization from the element weights w2 (ne) and the element
    // matrices Di (12 x ne, SoA, Di[(r + 3a) * ne + e]).  Sets *d_status to
    // WRAPD_E_NOT_SPD on a non-positive pivot (checked by the caller later).
    // The launch sequence is captured once into a CUDA graph and replayed
    // (the pointers must stay the same between calls).
    void factor(const double* d_w2, const double* d_Di, int ne, cudaStream_t st);
    // In place: x <- A^-1 x for an n x 3 block in the dissection order
    // (graph-replayed per vector and mask pointer): one queue-driven launch per
    // direction.  With mesh_on (device, one int per mesh) the fronts of a mesh
    // whose entry is 0 are skipped: that mesh's rows of x keep their input
    // values.  A dependency wait that gives up leaves WRAPD_E_TIMEOUT in
    // *d_status.
    void solve(double* d_x, cudaStream_t st, const int* mesh_on = nullptr);
    // One solve of x in which front `hold` never reports completion, so that the
    // waits on it run out (not graph-captured; the test of the bounded waits).
    void solve_holding(double* d_x, int hold, cudaStream_t st);
    // Times the candidate tile shapes on this system (the solve's chunk length
    // per level and direction; the largest panel step, in tiles, that factors
    // its diagonal block inside the tile launch) and keeps the fastest.  Runs
    // real factorizations of the current weights; call before the first factor.
    void autotune(const double* d_w2, const double* d_Di, int ne, cudaStream_t st);
    // [fused panel-step limit, levels, forward chunk per level..., backward chunk per level...]
    std::vector<int> tuning() const;

    // Per front, the mesh of a batch it belongs to (empty: one mesh).  Set
    // before build(): each mesh's solve then takes the chunk lengths it would
    // take alone, so its partial sums, and results, are those of its own solve.
    std::vector<int> front_mesh;

    int n = 0;
    int* d_status = nullptr;
    int64_t nnz_L = 0;
    double flops = 0.0;
    int nfronts = 0, nlevels = 0;
    size_t device_bytes = 0;
    int launches_factor = 0, launches_solve = 0;

private:
    struct Level {
        std::vector<int> fronts_sorted;   // by k descending
        int kmax = 0;
        std::vector<WorkList> extend;    // per child slot: CTAs over child columns
        std::vector<WorkList> diag;      // per panel step (steps not fused): one CTA per front
        std::vector<WorkList> trsm;      // per panel step: panel row tiles + Y row-block tiles
        std::vector<JobList> update;     // per panel step: blocked trailing-update jobs (F and Y)
        std::vector<std::vector<int>> trsm_split;  // per step: panel-row tiles per item
        WorkList wgemm;                  // W = L_rs Y tiles
        // solve items for each candidate chunk length: forward (64-row band,
        // column chunk) and backward (64-column band, row chunk)
        struct SolveCand {
            int sch;
            SolveItem* fwd;
            int nfwd;
            SolveItem* bwd;
            int nbwd;
            std::vector<SolveItem> hfwd, hbwd;   // host copies, for the work queues
        };
        std::vector<SolveCand> cand;
        int cfwd = 0, cbwd = 0;          // the candidates in use
    };
    std::vector<Level> levels_;
    FrontDesc* d_desc_ = nullptr;
    int* d_rows_ = nullptr;
    int* d_rel_ = nullptr;
    int64_t* d_inv_ = nullptr;   // per front row: the (up to 2) children's update-vector entries that add into it
    int64_t* d_Apos_ = nullptr;
    int* d_Aptr_ = nullptr;
    int* d_Acon_ = nullptr;
    int nA_ = 0;
    double* d_F_ = nullptr;
    double* d_Y_ = nullptr;
    double* d_U_ = nullptr;      // solve update vectors
    double* d_T_ = nullptr;      // solve: copy of the right-hand side (n x 3)
    double* d_Z_ = nullptr;      // solve: forward result (n x 3)
    double* d_P_ = nullptr;      // solve: per-item partial sums (64 x 3 per item)
    unsigned* d_cnt_ = nullptr;  // solve: per-band arrival counters (zero between launches)
    int64_t solve_parts_ = 0;
    int solve_bands_ = 0;
    int64_t f_pool_ = 0, y_pool_ = 0, u_pool_ = 0;
    cudaGraphExec_t factor_graph_ = nullptr;
    cudaGraphExec_t solve_graph_ = nullptr;
    double* solve_graph_x_ = nullptr;
    const int* solve_graph_mask_ = nullptr;
    int fused_ctas_ = 0;                 // panel steps of at most this many tiles run fused (k_panel)
    void count_launches();
    void factor_launches(const double* d_w2, const double* d_Di, int ne, cudaStream_t st);
    void solve_launches(double* d_x, cudaStream_t st, const int* mesh_on, int hold = -1);
    // the work queues of the chosen per-level candidates (after build and autotune)
    void build_queues(cudaStream_t st);
    SolveItem* d_qf_ = nullptr;   // forward items, leaves first (capacity: the longest candidates)
    SolveItem* d_qb_ = nullptr;   // backward items, root first
    int nqf_ = 0, nqb_ = 0;
    unsigned* d_qnb_ = nullptr;   // bands per front: forward [0, nfronts), backward [nfronts, 2 nfronts)
    unsigned* d_qctl_ = nullptr;  // zeroed per solve: 2 heads, done counters (2 nfronts), band counters
    size_t qctl_words_ = 0;
    int qbands_f_ = 0, qbands_b_ = 0;   // band counters: forward, then backward
    int64_t qcap_f_ = 0, qcap_b_ = 0;   // item capacity of d_qf_, d_qb_
    int qgrid_f_ = 0, qgrid_b_ = 0;   // persistent CTAs per queue launch (resident at once)
    std::vector<void*> allocs_;
    std::vector<FrontDesc> h_desc_;
    std::vector<std::vector<int*>> trsm_nP_;   // per level, per panel step: panel-row tile counts
    JobList make_jobs(const std::vector<GemmJob>& jobs, cudaStream_t st);

    template <typename X> X* upload(const std::vector<X>& v, cudaStream_t st);
    WorkList make_list(const std::vector<int>& fronts, const std::vector<int>& ctas, cudaStream_t st);
};

}  // namespace wrapd
