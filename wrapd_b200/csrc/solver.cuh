// Host orchestration of the ADMM solve loop on one GPU (the role of the
// reference's ADMM, RotAwareGS, SplitLBFGS, System and AlgorithmData classes:
// src/ADMM.cpp, src/GlobalStepBehavior.hpp:196-268,
// deps/mcloptlib/include/MCL/SplitLBFGS.hpp, src/System.cpp,
// src/AlgorithmData.cpp).  All numeric work runs in the CUDA kernels of
// elements.cuh and chol.cu; the host keeps only the integer bookkeeping and
// the scalar decisions (L-BFGS history ring, early exits, reweight trigger).
#pragma once
#include <memory>
#include <string>
#include <vector>

#include "chol.cuh"
#include "elem_types.cuh"
#include "symbolic.hpp"

namespace wrapd {

struct Logs {
    std::vector<double> objectives, ls_dal, gs_dal, acc_time_s, x_errors, prox_iters;
    std::vector<int> flips, reweighted, inner;
};

// One tiling of a launch over the batch (see Tiles in common.cuh): device
// table of {mesh, first, end} per tile and each mesh's first tile.  With one
// mesh no table is used (tile b covers [b * per, (b + 1) * per)).
struct TileSet {
    int4* d_t = nullptr;
    int* d_tile0 = nullptr;
    int n = 0, per = 0, count = 0;
    Tiles view() const { return Tiles{d_t, d_tile0, n, per, count}; }
};

class SolverGPU {
public:
    explicit SolverGPU(const wrapd_settings& s);
    ~SolverGPU();

    // Appends one mesh (pins: its own vertex ids).  Several meshes make a
    // batch: one launch per kernel over all their elements and one
    // factorization of the block-diagonal system, while each mesh keeps the
    // decisions of its own reference Solver (L-BFGS early exit and history,
    // reweighting, convergence) and stops when it converges; youngs/poisson > 0
    // give the mesh its own material (else the settings').
    Material material(double youngs, double poisson) const;
    void add_mesh(const double* rest, const double* init, const double* soln, int nv, const int32_t* tets, int ne,
                  const int32_t* pins, int np, double youngs = 0.0, double poisson = 0.0);
    void initialize();
    void begin_solve();
    // runs up to n iterations; returns iterations done; *converged set when the test passes
    int iterate(int n, bool* converged);
    void positions(double* out);
    // installs the prox network (FP32 blob, net::N_BLOB floats) used by prox_mode 2
    void set_prox_net(const float* blob);
    void solve(double* out);

    // components
    void get_state(const std::string& name, std::vector<double>& out);
    void set_state(const std::string& name, const double* in, int64_t n);
    void update_defo_cache();
    double polar_update(bool update_candidates);
    double global_grad(const double* xfree, double* grad);
    void potential_energy(double* pe, int* flips);
    // x = A^-1 b; with hold >= 0, front `hold` never reports completion (the
    // bounded-wait test: throws WRAPD_E_TIMEOUT)
    void solve_A(const double* b, double* x, int hold = -1);
    int n_fronts() const { return chol.nfronts; }

    // The logs of a single mesh; of a batch, the sums over its meshes
    // (energies, flips, inner iterations), any reweight, and the x error of
    // the whole batch.  mesh_logs(m): the logs of mesh m of a batch.
    const Logs& logs() const { return nm == 1 ? runs_[0].logs : logs_; }
    const Logs& mesh_logs(int m) const;
    int meshes() const { return nm; }
    int local_tile() const { return local_per_; }
    bool initialized() const { return initialized_; }
    // Optional per-phase device timeline (CUDA events on the handle's stream):
    // slots of kProfileNames, accumulated ms and counts.
    static constexpr int kProfileSlots = 6;
    bool profiling = false;
    double profile_ms[kProfileSlots] = {};
    int64_t profile_n[kProfileSlots] = {};
    double runtime_ms[6] = {0, 0, 0, 0, 0, 0};
    wrapd_settings cfg;
    int nv = 0, ne = 0, np = 0, nf = 0;
    int iter = 0;
    CholGPU chol;
    int64_t kernel_launches = 0;   // launches issued by this handle (element, vector and factor kernels)
    int64_t n_factor = 0, n_solve = 0, n_sync = 0;

private:
    static constexpr int kScalStride = 96;   // scalars per mesh in the device scalar block
    bool fp32() const { return cfg.precision == 1; }
    ElemView view();
    void* dalloc(size_t bytes);
    template <typename X> X* dupload(const std::vector<X>& v);
    void sync_read();
    void mark(int slot);          // close the running profile slot at this point of the stream
    void profile_flush();         // turn recorded event pairs into milliseconds
    std::vector<std::pair<cudaEvent_t, int>> marks_;
    std::vector<cudaEvent_t> event_pool_;
    size_t event_next_ = 0;
    void check_status();
    void grad_at_x(bool write_gel, int mask);
    void gather(int mode, int mask, bool xerr, double* plain = nullptr);
    void local_step_unaware(int cand_mode, bool fp32_compute);
    void global_step_unaware();
    void local_step(int cand_mode);
    void mid_candidates(bool from_x, int cand_mode);
    void apply_weights(int mask);
    void factor();
    int lbfgs_minimize();
    double line_search();
    int cand_mode_now() const;
    void download_elem(const double* d, int comps, std::vector<double>& out);
    void upload_elem(double* d, int comps, const double* in);
    void x_error_launch(int mask);
    // batch plumbing
    void build_tiles(TileSet& t, int per, const std::vector<std::pair<int, int>>& ranges);
    const int* mask(int which) const { return d_ctl_block_masks_ + (size_t)which * nm; }
    void set_mask(int which, int m, bool on) {
        ctl_writable();
        h_masks_[(size_t)which * nm + m] = on ? 1 : 0;
    }
    void ctl_writable();          // waits for the last control-block upload to be read
    bool any_mask(int which) const;
    void push_ctl();
    VecPools pools() const;
    double& hs(int m, int slot) { return h_scal_[(size_t)m * kScalStride + slot]; }
    double* ds(int slot) const { return d_scal_ + slot; }
    void union_logs(int k);

    // host mesh
    std::vector<double> rest_, init_, soln_;
    std::vector<int> tets_, pins_;         // pins sorted (batch vertex ids)
    struct MeshIn { int v_off, nv, e_off, ne, mat; bool soln; };
    std::vector<MeshIn> meshes_;
    std::vector<Material> mats_;           // distinct materials of the batch
    std::vector<int> free_of_vert_, fix_of_vert_;
    std::vector<int> perm_, iperm_;        // dissection order over free vertices
    bool have_soln_ = false;
    Material mat_{};
    int* d_mid_ = nullptr;                 // per-element material index (several materials only)
    Material* d_mats_ = nullptr;
    // device
    cudaStream_t st_ = nullptr;
    // phase events of two consecutive iterations (local, global, reweight): an
    // iteration's times are read once a later host synchronisation has passed them
    cudaEvent_t evs_[2][4] = {};
    struct PendingTiming { bool on = false; int k = 0; cudaEvent_t* ev = nullptr; };
    PendingTiming pend_;
    void settle_timing(bool wait);
    std::vector<void*> allocs_;
    int4* d_idx_ = nullptr;
    double *d_Di_ = nullptr, *d_vol_ = nullptr, *d_w2_ = nullptr, *d_w2c_ = nullptr;
    double* d_uv_ = nullptr;     // U, V of the last gradient's SVD (one mesh), valid at x while uv_valid_
    bool uv_valid_ = false;
    double *d_Z_ = nullptr, *d_U_ = nullptr, *d_symF_ = nullptr, *d_sig_ = nullptr, *d_slast_ = nullptr, *d_gel_ = nullptr;
    int *d_inc_ptr_ = nullptr, *d_inc_ = nullptr;
    double *d_x_ = nullptr, *d_xfix_ = nullptr, *d_xsoln_ = nullptr, *d_xinit_ = nullptr;
    double* d_q_ = nullptr;
    double* d_G_[3] = {};                  // gradient ring (see VecPools)
    std::vector<double*> d_S_, d_Y_;       // history slots, lbfgs_m + 1 each
    double* d_partials_ = nullptr;
    unsigned char* d_net_img_ = nullptr;   // prox network image + FP32 blob staging
    unsigned* d_counters_ = nullptr;       // one grid-reduction counter per mesh
    double* d_scal_ = nullptr;             // kScalStride scalars per mesh
    double* h_scal_ = nullptr;
    int* h_status_ = nullptr;    // pinned: the device status word, read with the scalars
    unsigned* d_bar_ = nullptr;  // grid-barrier counter of the cooperative two-loop recursion
    int coop_grid_ = 0;          // its CTAs (0: not used -- a batch, or no cooperative launch)
    bool coop_reg_ = false;      // its register form (one vector tile per CTA)
    void two_loop_grid(bool second, const VecPools& P, const TwoLoopSlots& sl);
    // ---- the meshes of the batch: each its own ADMM and L-BFGS state ----
    int nm = 0;
    struct MeshRun {
        int e0 = 0, e1 = 0, f0 = 0, f1 = 0;    // element range, free-vertex range (dissection order)
        MeshCtl ctl{};                          // rings and history length, as the kernels see them
        double rho[kHistSlots] = {};            // 1 / <s, y> per history slot
        double m_tol = 1e-15, curr_pe = 0.0, init_xerr = 1.0, obj_bef = 0.0;
        bool converged = false, fp64_phase = false;
        Logs logs;
        // one SplitLBFGS::minimize call
        int max_iters = 0, its = 0;
        bool in_loop = false;
    };
    std::vector<MeshRun> runs_;
    TileSet te128_, te256_, tv32_, tvec_;
    TileSet te_local_;                     // the local step's element tiles (local_per_ elements each)
    // 512 elements (16 warps, one CTA per SM): the FP64 local step takes 0.577
    // ms on the 786k bar (0.587 at 256, 0.71 at 128, 0.96 at 64, 1.67 at 32)
    // and 2.60 ms on the 3.9M bar (2.79 at 256, 3.65 at 128)
    int local_per_ = 512;
    bool local_tuned_ = false;
    void autotune_local();
    // control block on the device and its pinned mirror: masks (kMasks x nm
    // ints), then MeshCtl (nm), then rho (nm x kHistSlots doubles)
    void* d_ctl_block_ = nullptr;
    void* h_ctl_block_ = nullptr;
    size_t ctl_bytes_ = 0;
    int* d_ctl_block_masks_ = nullptr;
    int* h_masks_ = nullptr;
    MeshCtl* d_ctl_ = nullptr;
    MeshCtl* h_ctl_ = nullptr;
    double* d_rho_ = nullptr;
    double* h_rho_ = nullptr;
    bool ctl_pending_ = false;             // an upload not yet passed by a stream synchronisation
    std::vector<double> acc_time_s_;       // local + global + refactor seconds after each iteration
    // algorithm state
    int count_ = 0;          // reweight-delay counter (src/TetElements.cpp:404)
    bool ls_restart_ = false;   // the last line search followed a non-descent restart
    bool initialized_ = false, solving_ = false, converged_ = false;
    Logs logs_;              // a batch's summary logs
};

}  // namespace wrapd
