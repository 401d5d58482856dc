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

class SolverGPU {
public:
    explicit SolverGPU(const wrapd_settings& s);
    ~SolverGPU();

    // Appends one mesh (pins: its own vertex ids).  Several meshes make a
    // batch solved as one block-diagonal system; youngs/poisson > 0 give the
    // mesh its own material (else the settings').
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
    void solve_A(const double* b, double* x);

    const Logs& logs() const { return logs_; }
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
    void grad_at_x(bool write_gel);
    void gather(double* grad, const double* gold, double* ystage, const double* sstage, bool xerr = false);
    void local_step_unaware(int cand_mode, bool fp32_compute);
    void global_step_unaware();
    void local_step(int cand_mode, bool fp32_compute);
    void mid_candidates(bool from_x, int cand_mode);
    void apply_weights();
    void factor();
    int lbfgs_minimize();
    double line_search();
    int cand_mode_now() const;
    void download_elem(const double* d, int comps, std::vector<double>& out);
    void upload_elem(double* d, int comps, const double* in);
    double x_error();
    void x_error_launch();

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
    double *d_Z_ = nullptr, *d_U_ = nullptr, *d_symF_ = nullptr, *d_sig_ = nullptr, *d_slast_ = nullptr, *d_gel_ = nullptr;
    int *d_inc_ptr_ = nullptr, *d_inc_ = nullptr;
    double *d_x_ = nullptr, *d_xfix_ = nullptr, *d_xsoln_ = nullptr, *d_xinit_ = nullptr;
    double *d_q_ = nullptr, *d_gcur_ = nullptr, *d_gold_ = nullptr, *d_gnew_ = nullptr;
    double *d_sstage_ = nullptr, *d_ystage_ = nullptr;
    std::vector<double*> s_, y_;
    std::vector<double> rho_;
    double* d_partials_ = nullptr;
    unsigned char* d_net_img_ = nullptr;   // prox network image + FP32 blob staging
    unsigned* d_counter_ = nullptr;
    double* d_scal_ = nullptr;
    double* h_scal_ = nullptr;
    // algorithm state
    int count_ = 0;          // reweight-delay counter (src/TetElements.cpp:404)
    int m_k_ = 0;
    double m_tol_ = 1e-15;
    bool ls_restart_ = false;   // the last line search followed a non-descent restart
    double curr_pe_ = 0.0;
    double init_xerr_ = 1.0;
    bool initialized_ = false, solving_ = false, converged_ = false;
    bool fp64_phase_ = false;   // mixed mode: switched to FP64 local steps (refinement)
    Logs logs_;
};

}  // namespace wrapd
