// Host orchestration of the ADMM solve loop; see solver.cuh.
#include "solver.cuh"

#include "elements.cuh"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <numeric>

namespace wrapd {

namespace {

// Slots of the device scalar block (one pinned download per sync point).
enum : int {
    S_GRAD = 0,      // value, pe, flips
    S_GATHER = 4,    // |grad - gold|^2, <s, y>, |x - x_soln|^2
    S_LOCAL = 8,     // bef, aft, pe, negative stretches, prox iterations
    S_INIT = 13,     // polar potential energy after initialize_dual_vars
    S_RATIO = 14,    // max weight ratio
    S_DIR = 16,      // L-BFGS decrement
    S_XERR = 18,     // |x - x_soln|^2
    S_DUMMY = 19,
    S_ALPHA = 20,    // alpha_i, up to 32 entries
    S_C = 52,        // alpha_i - beta_i, up to 32 entries
    S_ONE = 84,      // constant 1 (a device-side coefficient)
    S_LSN = 85,      // line search: <q, q>, <grad, grad>
    S_LSM = 87,      // line search: max |grad|
    S_LSV = 88,      // line search: AL value, pe, flips at the trial point
    S_COUNT = 91
};
// Dynamic shared memory of k_local<double>: the prox L-BFGS history, 48 doubles
// per thread of a 128-thread block.
constexpr int kLocalHistBytes = 48 * 128 * (int)sizeof(double);
// Mixed mode switches its local step to FP64 when the normalized energy
// residual drops below this (the FP32 local step's noise floor is ~1e-7).
constexpr double kMixedSwitch = 1e-7;

int blocks_for(int64_t n, int threads) { return std::max(1, ceil_div(n, threads)); }

// Vector kernels use a fixed grid of 2 CTAs per SM (grid-stride loops).
int vec_blocks(int64_t n) { return std::max(1, std::min(2 * kNumSMs, ceil_div(n, 256))); }

// (S * Dm^-1)^T and the rest volume of one tet, src/TetElements.cpp:93-118.
void element_geometry(const double* p0, const double* p1, const double* p2, const double* p3, double* Di,
                      double* vol) {
    double ed[9];
    for (int r = 0; r < 3; ++r) {
        ed[r + 0] = p1[r] - p0[r];
        ed[r + 3] = p2[r] - p0[r];
        ed[r + 6] = p3[r] - p0[r];
    }
    auto m = [&](int r, int c) { return ed[r + 3 * c]; };
    const double c00 = m(1, 1) * m(2, 2) - m(1, 2) * m(2, 1);
    const double c01 = m(1, 2) * m(2, 0) - m(1, 0) * m(2, 2);
    const double c02 = m(1, 0) * m(2, 1) - m(1, 1) * m(2, 0);
    const double det = m(0, 0) * c00 + m(0, 1) * c01 + m(0, 2) * c02;
    const double id = 1.0 / det;
    double inv[9];
    inv[0 + 3 * 0] = c00 * id;
    inv[1 + 3 * 0] = c01 * id;
    inv[2 + 3 * 0] = c02 * id;
    inv[0 + 3 * 1] = (m(0, 2) * m(2, 1) - m(0, 1) * m(2, 2)) * id;
    inv[1 + 3 * 1] = (m(0, 0) * m(2, 2) - m(0, 2) * m(2, 0)) * id;
    inv[2 + 3 * 1] = (m(0, 1) * m(2, 0) - m(0, 0) * m(2, 1)) * id;
    inv[0 + 3 * 2] = (m(0, 1) * m(1, 2) - m(0, 2) * m(1, 1)) * id;
    inv[1 + 3 * 2] = (m(0, 2) * m(1, 0) - m(0, 0) * m(1, 2)) * id;
    inv[2 + 3 * 2] = (m(0, 0) * m(1, 1) - m(0, 1) * m(1, 0)) * id;
    // Di(r, a): a = 0 -> minus the column sums of Dm^-1 rows; a >= 1 -> row a-1 of Dm^-1
    for (int r = 0; r < 3; ++r) {
        Di[r + 0] = -inv[0 + 3 * r] - inv[1 + 3 * r] - inv[2 + 3 * r];
        for (int a = 1; a < 4; ++a) Di[r + 3 * a] = inv[(a - 1) + 3 * r];
    }
    *vol = det / 6.0;
}

}  // namespace

SolverGPU::SolverGPU(const wrapd_settings& s) : cfg(s) {
    if (cfg.rot_aware != 0 && cfg.rot_aware != 1) throw CudaError(WRAPD_E_INPUT, "rot_aware must be 0 or 1");
    if (cfg.global_ls != 0 && cfg.global_ls != 1) throw CudaError(WRAPD_E_INPUT, "global_ls must be 0 or 1");
    if (cfg.model != MODEL_NH && cfg.model != MODEL_ARAP) throw CudaError(WRAPD_E_INPUT, "model must be 0 (nh) or 1 (arap)");
    if (cfg.prox_mode < 0 || cfg.prox_mode > 2)
        throw CudaError(WRAPD_E_UNSUPPORTED, "prox_mode must be 0 (L-BFGS), 1 (Newton) or 2 (Newton from the prox network)");
    if (cfg.lbfgs_m < 1 || cfg.lbfgs_m > kMaxHistory) throw CudaError(WRAPD_E_INPUT, "lbfgs_m must be in [1, 32]");
    if (cfg.max_iters < 0 || cfg.global_iters < 1 || cfg.prox_iters < 1) throw CudaError(WRAPD_E_INPUT, "bad iteration limits");
    if (!(cfg.poisson > -1.0 && cfg.poisson < 0.5) || !(cfg.youngs > 0.0)) throw CudaError(WRAPD_E_INPUT, "bad material");
    if (cfg.precision != 0 && cfg.precision != 1) throw CudaError(WRAPD_E_INPUT, "precision must be 0 or 1");
    if (cfg.autotune != 0 && cfg.autotune != 1) throw CudaError(WRAPD_E_INPUT, "autotune must be 0 or 1");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) throw CudaError(WRAPD_E_CUDA, "no CUDA device");
    if (cfg.device < 0 || cfg.device >= ndev) throw CudaError(WRAPD_E_INPUT, "bad device ordinal");
    WRAPD_CUDA(cudaSetDevice(cfg.device));
    WRAPD_CUDA(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
    for (auto& set : evs_)
        for (auto& e : set) WRAPD_CUDA(cudaEventCreate(&e));
    WRAPD_CUDA(cudaMallocHost(&h_scal_, S_COUNT * sizeof(double)));
    WRAPD_CUDA(cudaFuncSetAttribute(k_local<double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kLocalHistBytes));
    WRAPD_CUDA(cudaFuncSetAttribute(k_local_unaware<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    kLocalHistBytes));
    mat_ = material(cfg.youngs, cfg.poisson);
}

// Lame(E, nu), src/Lame.hpp:50-53; k = 2.0066 mu + 1.0122 lambda, src/TetElements.cpp:84
Material SolverGPU::material(double youngs, double poisson) const {
    Material m{};
    m.mu = youngs / (2.0 * (1.0 + poisson));
    m.lambda = youngs * poisson / ((1.0 + poisson) * (1.0 - 2.0 * poisson));
    m.model = cfg.model;
    // rest stiffness k: 1 for ARAP (src/TetElements.cpp:80-87)
    m.wr = cfg.model == MODEL_ARAP ? 1.0 : 2.0066 * m.mu + 1.0122 * m.lambda;
    m.wmin = m.wr * cfg.beta_min;
    m.wmax = m.wr * cfg.beta_max;
    return m;
}

SolverGPU::~SolverGPU() {
    if (st_) cudaStreamSynchronize(st_);
    for (cudaEvent_t e : event_pool_) cudaEventDestroy(e);
    for (void* p : allocs_) cudaFree(p);
    if (d_net_img_) cudaFree(d_net_img_);
    for (auto& set : evs_)
        for (auto& e : set) if (e) cudaEventDestroy(e);
    if (h_scal_) cudaFreeHost(h_scal_);
    if (st_) cudaStreamDestroy(st_);
}

void* SolverGPU::dalloc(size_t bytes) {
    void* p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(bytes, 16)) != cudaSuccess) {
        cudaGetLastError();
        throw CudaError(WRAPD_E_OOM, "cudaMalloc of " + std::to_string(bytes) + " bytes failed");
    }
    allocs_.push_back(p);
    return p;
}

template <typename X>
X* SolverGPU::dupload(const std::vector<X>& v) {
    X* p = static_cast<X*>(dalloc(v.size() * sizeof(X)));
    if (!v.empty()) WRAPD_CUDA(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(X), cudaMemcpyHostToDevice, st_));
    return p;
}

ElemView SolverGPU::view() {
    ElemView v;
    v.ne = ne;
    v.idx = d_idx_;
    v.Di = d_Di_;
    v.vol = d_vol_;
    v.w2 = d_w2_;
    v.w2c = d_w2c_;
    v.Z = d_Z_;
    v.U = d_U_;
    v.symF = d_symF_;
    v.sig = d_sig_;
    v.slast = d_slast_;
    v.gel = d_gel_;
    v.mid = d_mid_;
    v.mats = d_mats_;
    return v;
}

void SolverGPU::add_mesh(const double* rest, const double* init, const double* soln, int nv_, const int32_t* tets,
                         int ne_, const int32_t* pins, int np_, double youngs, double poisson) {
    if (initialized_) throw CudaError(WRAPD_E_STATE, "add_tetmesh after initialize");
    if (!rest || !init || !tets || nv_ <= 0 || ne_ <= 0 || np_ < 0 || np_ >= nv_ || (np_ > 0 && !pins))
        throw CudaError(WRAPD_E_INPUT, "bad mesh arguments");
    if (!meshes_.empty() && meshes_[0].soln != (soln != nullptr))
        throw CudaError(WRAPD_E_INPUT, "give a solution mesh for every mesh of a batch or for none");
    if ((youngs > 0.0) != (poisson > 0.0) || (poisson > 0.0 && !(poisson < 0.5)))
        throw CudaError(WRAPD_E_INPUT, "bad mesh material");
    for (int i = 0; i < 4 * ne_; ++i)
        if (tets[i] < 0 || tets[i] >= nv_) throw CudaError(WRAPD_E_INPUT, "tet vertex id out of range");
    std::vector<int> p(pins, pins + np_);
    std::sort(p.begin(), p.end());
    for (int j = 0; j < np_; ++j)
        if (p[j] < 0 || p[j] >= nv_ || (j > 0 && p[j] == p[j - 1]))
            throw CudaError(WRAPD_E_INPUT, "pin ids must be distinct vertex ids");
    // the mesh's material: one entry per distinct (mu, lambda)
    const Material m = youngs > 0.0 ? material(youngs, poisson) : mat_;
    int mi = 0;
    while (mi < (int)mats_.size() && !(mats_[mi].mu == m.mu && mats_[mi].lambda == m.lambda)) ++mi;
    if (mi == (int)mats_.size()) mats_.push_back(m);
    meshes_.push_back({nv, nv_, ne, ne_, mi, soln != nullptr});
    // append, vertex ids shifted by the vertices before (binding::add_tetmesh's
    // prev_tet_verts, samples/utils/AddMeshes.hpp:70-84)
    rest_.insert(rest_.end(), rest, rest + 3 * (size_t)nv_);
    init_.insert(init_.end(), init, init + 3 * (size_t)nv_);
    if (soln) soln_.insert(soln_.end(), soln, soln + 3 * (size_t)nv_);
    else soln_.insert(soln_.end(), rest, rest + 3 * (size_t)nv_);
    have_soln_ = soln != nullptr;
    for (int i = 0; i < 4 * ne_; ++i) tets_.push_back(tets[i] + nv);
    for (int v : p) pins_.push_back(v + nv);
    nv += nv_; ne += ne_; np += np_; nf = nv - np;
    // free/fixed maps over the batch, samples/utils/AddMeshes.hpp:89-110 (meshes
    // follow each other and pins stay sorted, so each mesh's free vertices are
    // contiguous)
    free_of_vert_.assign(nv, -1);
    fix_of_vert_.assign(nv, -1);
    for (int i = 0, j = 0, k = 0; i < nv; ++i) {
        if (j < np && i == pins_[j]) fix_of_vert_[i] = j++;
        else free_of_vert_[i] = k++;
    }
}

void SolverGPU::initialize() {
    if (nv == 0) throw CudaError(WRAPD_E_STATE, "initialize before add_tetmesh");
    if (initialized_) throw CudaError(WRAPD_E_STATE, "already initialized");
    // update_all_candidate_weights (src/TetElements.cpp:393-395)
    if (cfg.model != MODEL_NH && cfg.reweighting)
        throw CudaError(WRAPD_E_INPUT, "Adaptive weights are only supported for the NH model (use reweighting = 0)");
    auto t0 = std::chrono::steady_clock::now();
    // host phase timings, printed to stderr with verbose >= 2
    std::vector<std::pair<const char*, double>> laps;
    auto tl = t0;
    auto lap = [&](const char* name) {
        const auto now = std::chrono::steady_clock::now();
        laps.emplace_back(name, std::chrono::duration<double, std::milli>(now - tl).count());
        tl = now;
    };
    // ---- element geometry (TetElements ctor, src/TetElements.cpp:90-142) ----
    std::vector<double> Di(12 * (size_t)ne), vol(ne), w2(ne);
    for (int e = 0; e < ne; ++e) {
        const int* t = &tets_[4 * (size_t)e];
        double d[12], v;
        element_geometry(&rest_[3 * (size_t)t[0]], &rest_[3 * (size_t)t[1]], &rest_[3 * (size_t)t[2]],
                         &rest_[3 * (size_t)t[3]], d, &v);
        if (v < 0.0) throw CudaError(WRAPD_E_INVERTED_REST, "inverted tet " + std::to_string(e) + " in the rest mesh");
        for (int k = 0; k < 12; ++k) Di[(size_t)k * ne + e] = d[k];
        vol[e] = v;
    }
    std::vector<int> mid(ne);
    for (const MeshIn& M : meshes_)
        for (int e = M.e_off; e < M.e_off + M.ne; ++e) {
            mid[e] = M.mat;
            w2[e] = cfg.beta_static * mats_[M.mat].wr * vol[e];
        }
    lap("element geometry");
    // ---- free-vertex graph, nested dissection, symbolic factorization ----
    // element incidences per free vertex (free numbering), in element order
    // (entry e * 4 + a for vertex slot a of element e), and the adjacency: the
    // other free vertices of the incident elements, sorted and unique
    std::vector<int> vinc_ptr, vinc, ptr, adj;
    free_vertex_graph(nf, ne, tets_.data(), free_of_vert_.data(), vinc_ptr, vinc, ptr, adj);
    std::vector<double> coords(3 * (size_t)nf);
    for (int i = 0; i < nv; ++i)
        if (free_of_vert_[i] >= 0)
            for (int c = 0; c < 3; ++c) coords[3 * (size_t)free_of_vert_[i] + c] = rest_[3 * (size_t)i + c];
    lap("free-vertex graph");
    // one nested dissection per mesh (their graphs are disjoint), then the forest
    std::vector<Symbolic> parts;
    for (const MeshIn& M : meshes_) {
        int f0 = -1, f1 = -1;
        for (int i = M.v_off; i < M.v_off + M.nv; ++i)
            if (free_of_vert_[i] >= 0) { if (f0 < 0) f0 = free_of_vert_[i]; f1 = free_of_vert_[i] + 1; }
        if (f0 < 0) throw CudaError(WRAPD_E_INPUT, "a mesh without free vertices");
        const int n = f1 - f0;
        std::vector<int> p(n + 1), a(adj.begin() + ptr[f0], adj.begin() + ptr[f1]);
        for (int i = 0; i <= n; ++i) p[i] = ptr[f0 + i] - ptr[f0];
        for (int& v : a) v -= f0;
        std::vector<double> c(coords.begin() + 3 * (size_t)f0, coords.begin() + 3 * (size_t)f1);
        parts.push_back(analyse(n, p, a, c, cfg.leaf_size > 0 ? cfg.leaf_size : 64));
    }
    Symbolic S = merge(parts);
    lap("nested dissection + symbolic");
    std::vector<Symbolic>().swap(parts);
    perm_ = S.perm;
    iperm_ = S.iperm;
    // element slots: free -> dissection index, pinned -> -(pin + 1)
    std::vector<int4> idx(ne);
    for (int e = 0; e < ne; ++e) {
        int s[4];
        for (int a = 0; a < 4; ++a) {
            const int v = tets_[4 * (size_t)e + a];
            s[a] = free_of_vert_[v] >= 0 ? iperm_[free_of_vert_[v]] : -(fix_of_vert_[v] + 1);
        }
        idx[e] = make_int4(s[0], s[1], s[2], s[3]);
    }
    // lower-triangle entries of A in front storage, with their element
    // contributions in the order of the reference's triplet list
    std::vector<int64_t> A_pos;
    std::vector<int> A_ptr, A_con;
    assembly_map(S, vinc_ptr, vinc, ptr, adj, A_pos, A_ptr, A_con);
    lap("A pattern (scatter map)");
    // gather incidences, element order per free vertex
    std::vector<int> inc_ptr(nf + 1, 0), inc;
    for (int e = 0; e < ne; ++e) {
        const int s[4] = {idx[e].x, idx[e].y, idx[e].z, idx[e].w};
        for (int a = 0; a < 4; ++a) if (s[a] >= 0) inc_ptr[s[a] + 1]++;
    }
    for (int i = 0; i < nf; ++i) inc_ptr[i + 1] += inc_ptr[i];
    inc.resize(inc_ptr[nf]);
    {
        std::vector<int> fill(inc_ptr.begin(), inc_ptr.end() - 1);
        for (int e = 0; e < ne; ++e) {
            const int s[4] = {idx[e].x, idx[e].y, idx[e].z, idx[e].w};
            for (int a = 0; a < 4; ++a) if (s[a] >= 0) inc[fill[s[a]]++] = e * 4 + a;
        }
    }
    lap("gather incidences");
    // ---- device state ----
    const size_t TS = sizeof(double);
    d_idx_ = dupload(idx);
    d_Di_ = dupload(Di);
    d_vol_ = dupload(vol);
    d_w2_ = dupload(w2);
    if (mats_.size() > 1) {
        d_mid_ = dupload(mid);
        d_mats_ = dupload(mats_);
    }
    d_w2c_ = static_cast<double*>(dalloc(ne * sizeof(double)));
    d_Z_ = static_cast<double*>(dalloc(9 * (size_t)ne * TS));
    d_U_ = static_cast<double*>(dalloc(9 * (size_t)ne * TS));
    d_symF_ = static_cast<double*>(dalloc(9 * (size_t)ne * TS));
    d_sig_ = static_cast<double*>(dalloc(3 * (size_t)ne * TS));
    d_slast_ = static_cast<double*>(dalloc(3 * (size_t)ne * TS));
    d_gel_ = static_cast<double*>(dalloc(12 * (size_t)ne * TS));
    WRAPD_CUDA(cudaMemsetAsync(d_U_, 0, 9 * (size_t)ne * TS, st_));
    WRAPD_CUDA(cudaMemsetAsync(d_Z_, 0, 9 * (size_t)ne * TS, st_));
    {
        // m_last_sigma = (1, 1, 1)
        std::vector<double> ones(3 * (size_t)ne, 1.0);
        WRAPD_CUDA(cudaMemcpyAsync(d_slast_, ones.data(), ones.size() * 8, cudaMemcpyHostToDevice, st_));
        WRAPD_CUDA(cudaStreamSynchronize(st_));
    }
    d_inc_ptr_ = dupload(inc_ptr);
    d_inc_ = dupload(inc);
    std::vector<double> xp(3 * (size_t)nf), xs(3 * (size_t)nf), xfix(3 * (size_t)std::max(np, 1));
    for (int i = 0; i < nv; ++i) {
        if (free_of_vert_[i] >= 0) {
            const int p = iperm_[free_of_vert_[i]];
            for (int c = 0; c < 3; ++c) { xp[3 * (size_t)p + c] = init_[3 * (size_t)i + c]; xs[3 * (size_t)p + c] = soln_[3 * (size_t)i + c]; }
        } else {
            for (int c = 0; c < 3; ++c) xfix[3 * (size_t)fix_of_vert_[i] + c] = init_[3 * (size_t)i + c];
        }
    }
    d_x_ = dupload(xp);
    d_xinit_ = dupload(xp);
    d_xsoln_ = dupload(xs);
    d_xfix_ = dupload(xfix);
    const size_t vb = 3 * (size_t)nf * sizeof(double);
    d_q_ = static_cast<double*>(dalloc(vb));
    d_gcur_ = static_cast<double*>(dalloc(vb));
    d_gold_ = static_cast<double*>(dalloc(vb));
    d_gnew_ = static_cast<double*>(dalloc(vb));
    d_sstage_ = static_cast<double*>(dalloc(vb));
    d_ystage_ = static_cast<double*>(dalloc(vb));
    WRAPD_CUDA(cudaMemsetAsync(d_gold_, 0, vb, st_));
    WRAPD_CUDA(cudaMemsetAsync(d_gcur_, 0, vb, st_));
    s_.assign(cfg.lbfgs_m, nullptr);
    y_.assign(cfg.lbfgs_m, nullptr);
    for (int i = 0; i < cfg.lbfgs_m; ++i) {
        s_[i] = static_cast<double*>(dalloc(vb));
        y_[i] = static_cast<double*>(dalloc(vb));
    }
    rho_.assign(cfg.lbfgs_m, 0.0);
    const size_t nblk = (size_t)std::max(blocks_for(std::max(ne, nf), 128), blocks_for(8 * (int64_t)nf, 256)) +
                        2 * kNumSMs + 8;
    d_partials_ = static_cast<double*>(dalloc(nblk * 5 * sizeof(double)));
    d_counter_ = static_cast<unsigned*>(dalloc(sizeof(unsigned)));
    d_scal_ = static_cast<double*>(dalloc(S_COUNT * sizeof(double)));
    WRAPD_CUDA(cudaMemsetAsync(d_counter_, 0, sizeof(unsigned), st_));
    WRAPD_CUDA(cudaMemsetAsync(d_scal_, 0, S_COUNT * sizeof(double), st_));
    {
        static const double one = 1.0;
        WRAPD_CUDA(cudaMemcpyAsync(d_scal_ + S_ONE, &one, sizeof(double), cudaMemcpyHostToDevice, st_));
    }
    lap("element state upload");
    chol.build(S, A_pos, A_ptr, A_con, st_);
    WRAPD_CUDA(cudaStreamSynchronize(st_));
    lap("factor structures upload");
    // ---- GlobalStepBehavior ctor: midupdate_weights(X_init) and the first factorization ----
    if (cfg.reweighting) {
        mid_candidates(true, cand_mode_now());
        count_++;
        apply_weights();
    }
    if (cfg.autotune) {
        chol.autotune(d_w2_, d_Di_, ne, st_);
        lap("autotune (solve chunks, panel steps)");
    }
    factor();
    m_k_ = 0;
    check_status();
    lap("first factorization (graph capture + run)");
    initialized_ = true;
    runtime_ms[0] += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (cfg.verbose >= 2)
        for (const auto& l : laps) std::fprintf(stderr, "wrapd setup: %-42s %9.1f ms\n", l.first, l.second);
}

int SolverGPU::cand_mode_now() const {
    if (!cfg.reweighting) return CAND_NONE;
    return count_ > cfg.rw_delay ? CAND_HESSIAN : CAND_REST;
}

#define WRAPD_ELEM_LAUNCH(kernel, grid, block, ...)                    \
    do {                                                               \
        kernel<<<grid, block, 0, st_>>>(view(), __VA_ARGS__);          \
        WRAPD_LAUNCH_CHECK();                                          \
        kernel_launches++;                                             \
    } while (0)

void SolverGPU::grad_at_x(bool write_gel) {
    WRAPD_ELEM_LAUNCH(k_grad, blocks_for(ne, 128), 128, d_x_, d_xfix_, mat_, write_gel ? 1 : 0, d_partials_,
                      d_counter_, d_scal_ + S_GRAD);
}

void SolverGPU::gather(double* grad, const double* gold, double* ystage, const double* sstage, bool xerr) {
    k_gather<<<blocks_for(8 * (int64_t)nf, 256), 256, 0, st_>>>(nf, d_inc_ptr_, d_inc_, d_gel_, ne, grad, gold, ystage, sstage,
                                                   xerr ? d_x_ : nullptr, d_xsoln_, d_partials_, d_counter_,
                                                   d_scal_ + S_GATHER);
    WRAPD_LAUNCH_CHECK();
    kernel_launches++;
}

void SolverGPU::local_step(int cand_mode, bool fp32_compute) {
    if (cfg.model == MODEL_ARAP) {
        k_local_arap<<<blocks_for(ne, 128), 128, 0, st_>>>(view(), d_partials_, d_counter_, d_scal_ + S_LOCAL);
        WRAPD_LAUNCH_CHECK();
        kernel_launches++;
        return;
    }
    // prox_mode 2 runs the network where the last stretches are a stale warm
    // start: the first local step and the one after each reweight (the weight
    // w^2 / vol, an input of the prox, has just changed); elsewhere the last
    // stretches start the Newton prox at least as well and cost nothing.
    const bool net = cfg.prox_mode == 2 && (logs_.reweighted.empty() || logs_.reweighted.back() != 0);
    const int nb = blocks_for(ne, 128);
    const int net_smem = net::IMAGE_BYTES + 4 * net::WARP_SCRATCH;
    if (net && !d_net_img_) throw CudaError(WRAPD_E_STATE, "prox_mode 2 needs a network (wrapd_set_prox_net)");
    if (fp32_compute) {
        if (net)
            k_local<float, true><<<nb, 128, net_smem, st_>>>(view(), mat_, cfg.prox_iters, cand_mode, 2, d_net_img_,
                                                             d_partials_, d_counter_, d_scal_ + S_LOCAL);
        else
            k_local<float, false><<<nb, 128, 0, st_>>>(view(), mat_, cfg.prox_iters, cand_mode, 1, nullptr,
                                                       d_partials_, d_counter_, d_scal_ + S_LOCAL);
    } else {
        if (net)
            k_local<double, true><<<nb, 128, net_smem, st_>>>(view(), mat_, cfg.prox_iters, cand_mode, 2, d_net_img_,
                                                              d_partials_, d_counter_, d_scal_ + S_LOCAL);
        else
            k_local<double, false><<<nb, 128, kLocalHistBytes, st_>>>(view(), mat_, cfg.prox_iters, cand_mode,
                                                                      (fp32() || cfg.prox_mode == 2) ? 1 : cfg.prox_mode,
                                                                      nullptr, d_partials_, d_counter_,
                                                                      d_scal_ + S_LOCAL);
    }
    WRAPD_LAUNCH_CHECK();
    kernel_launches++;
}

void SolverGPU::local_step_unaware(int cand_mode, bool fp32_compute) {
    const int nb = blocks_for(ne, 128);
    if (fp32_compute && cfg.model == MODEL_NH)
        k_local_unaware<float><<<nb, 128, 0, st_>>>(view(), d_x_, d_xfix_, mat_, cfg.prox_iters, cand_mode, 1,
                                                    d_partials_, d_counter_, d_scal_ + S_LOCAL);
    else
        k_local_unaware<double><<<nb, 128, kLocalHistBytes, st_>>>(view(), d_x_, d_xfix_, mat_, cfg.prox_iters,
                                                                   cand_mode, (fp32() || cfg.prox_mode != 0) ? 1 : 0,
                                                                   d_partials_, d_counter_, d_scal_ + S_LOCAL);
    WRAPD_LAUNCH_CHECK();
    kernel_launches++;
}

void SolverGPU::global_step_unaware() {
    WRAPD_ELEM_LAUNCH(k_rhs_unaware, blocks_for(ne, 128), 128, d_xfix_);
    gather(d_q_, nullptr, nullptr, nullptr);
    mark(1);
    chol.solve(d_q_, st_);
    kernel_launches += chol.launches_solve;
    n_solve++;
    mark(3);
    WRAPD_CUDA(cudaMemcpyAsync(d_x_, d_q_, 3 * (size_t)nf * sizeof(double), cudaMemcpyDeviceToDevice, st_));
    // update_defo_cache(x, true): singular values for the energy and flips
    grad_at_x(false);
    mark(1);
}

void SolverGPU::set_prox_net(const float* blob) {
    if (!d_net_img_) {
        void* p = nullptr;
        if (cudaMalloc(&p, net::IMAGE_BYTES + net::N_BLOB * sizeof(float)) != cudaSuccess) {
            cudaGetLastError();
            throw CudaError(WRAPD_E_OOM, "cudaMalloc failed (prox network)");
        }
        d_net_img_ = static_cast<unsigned char*>(p);
    }
    net::upload_image(blob, d_net_img_, reinterpret_cast<float*>(d_net_img_ + net::IMAGE_BYTES), st_);
    WRAPD_CUDA(cudaStreamSynchronize(st_));
}

void SolverGPU::mid_candidates(bool from_x, int cand_mode) {
    WRAPD_ELEM_LAUNCH(k_mid_candidates, blocks_for(ne, 128), 128, d_x_, d_xfix_, mat_, from_x ? 1 : 0, cand_mode);
}

void SolverGPU::apply_weights() {
    k_apply_weights<<<blocks_for(ne, 256), 256, 0, st_>>>(view());
    WRAPD_LAUNCH_CHECK();
    kernel_launches++;
}

void SolverGPU::factor() {
    chol.factor(d_w2_, d_Di_, ne, st_);
    kernel_launches += chol.launches_factor;
    n_factor++;
}

// Profile slots: 0 = local step, 1 = gradient + gather, 2 = two-loop and
// x-update vector kernels, 3 = triangular solves, 4 unused, 5 = host gaps
// around syncs and the reweight/refactor phase.
void SolverGPU::mark(int slot) {
    if (!profiling) return;
    if (event_next_ == event_pool_.size()) {
        cudaEvent_t e;
        WRAPD_CUDA(cudaEventCreate(&e));
        event_pool_.push_back(e);
    }
    cudaEvent_t e = event_pool_[event_next_++];
    WRAPD_CUDA(cudaEventRecord(e, st_));
    marks_.emplace_back(e, slot);
}

void SolverGPU::profile_flush() {
    if (!profiling || marks_.size() < 2) { marks_.clear(); event_next_ = 0; return; }
    WRAPD_CUDA(cudaEventSynchronize(marks_.back().first));
    for (size_t i = 1; i < marks_.size(); ++i) {
        float ms = 0.f;
        WRAPD_CUDA(cudaEventElapsedTime(&ms, marks_[i - 1].first, marks_[i].first));
        profile_ms[marks_[i].second] += ms;
        profile_n[marks_[i].second]++;
    }
    marks_.clear();
    event_next_ = 0;
}

void SolverGPU::sync_read() {
    WRAPD_CUDA(cudaMemcpyAsync(h_scal_, d_scal_, S_COUNT * sizeof(double), cudaMemcpyDeviceToHost, st_));
    WRAPD_CUDA(cudaStreamSynchronize(st_));
    n_sync++;
    mark(5);
}

void SolverGPU::check_status() {
    int status = 0;
    WRAPD_CUDA(cudaMemcpyAsync(&status, chol.d_status, sizeof(int), cudaMemcpyDeviceToHost, st_));
    WRAPD_CUDA(cudaStreamSynchronize(st_));
    if (status != 0) {
        WRAPD_CUDA(cudaMemsetAsync(chol.d_status, 0, sizeof(int), st_));
        throw CudaError(status, "factorization of D^T W D hit a non-positive pivot");
    }
}

// |x - x_soln| (AlgorithmData::update_per_iter_data, src/AlgorithmData.cpp:66-78;
// x_soln is the rest mesh when no solution mesh is given): q = x - x_soln,
// <q, q> into the scalar block, read at the next sync.
void SolverGPU::x_error_launch() {
    const int n = 3 * nf;
    k_axpy_dot<<<vec_blocks(n), 256, 0, st_>>>(n, d_q_, d_x_, d_xsoln_, d_scal_ + S_ONE, -1.0, nullptr, nullptr,
                                               1.0, d_partials_, d_counter_, d_scal_ + S_XERR);
    k_axpy_dot<<<vec_blocks(n), 256, 0, st_>>>(n, d_q_, nullptr, nullptr, nullptr, 0.0, d_q_, nullptr, 1.0,
                                               d_partials_, d_counter_, d_scal_ + S_XERR);
    WRAPD_LAUNCH_CHECK();
    kernel_launches += 2;
}

double SolverGPU::x_error() {
    x_error_launch();
    sync_read();
    return std::sqrt(h_scal_[S_XERR]);
}

void SolverGPU::begin_solve() {
    if (!initialized_) throw CudaError(WRAPD_E_STATE, "begin_solve before initialize");
    auto t0 = std::chrono::steady_clock::now();
    logs_ = Logs();
    pend_ = PendingTiming{};
    iter = 0;
    converged_ = false;
    fp64_phase_ = false;
    for (double& r : runtime_ms) r = 0.0;
    // setup_solve (src/ADMM.cpp:89-107): X = X_init, defo cache, dual variables
    WRAPD_CUDA(cudaMemcpyAsync(d_x_, d_xinit_, 3 * (size_t)nf * sizeof(double), cudaMemcpyDeviceToDevice, st_));
    grad_at_x(false);
    if (cfg.rot_aware) {
        WRAPD_ELEM_LAUNCH(k_init_dual, blocks_for(ne, 128), 128, d_x_, d_xfix_, mat_, d_partials_, d_counter_,
                          d_scal_ + S_INIT);
    } else {
        WRAPD_ELEM_LAUNCH(k_init_dual_unaware, blocks_for(ne, 128), 128, d_x_, d_xfix_);
    }
    sync_read();
    curr_pe_ = cfg.rot_aware ? h_scal_[S_INIT] : 0.0;
    // log_initial_data (src/AlgorithmData.cpp:50-64)
    logs_.objectives.push_back(h_scal_[S_GRAD + 1]);
    logs_.flips.push_back((int)h_scal_[S_GRAD + 2]);
    logs_.reweighted.push_back(1);
    logs_.acc_time_s.push_back(0.0);
    logs_.x_errors.push_back(1.0);
    init_xerr_ = x_error();
    // initialize_weights (src/GlobalStepBehavior.hpp:223-230)
    if (cfg.reweighting) {
        mid_candidates(false, cand_mode_now());
        count_++;
        apply_weights();
        factor();
        m_k_ = 0;
        check_status();
    }
    solving_ = true;
    marks_.clear();
    event_next_ = 0;
    runtime_ms[0] += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// SplitLBFGS::minimize (deps/mcloptlib/include/MCL/SplitLBFGS.hpp:114-256) with
// LSMethod::None (rate 1).  On entry the gradient at x is in d_gcur_ and the
// |grad - grad_old|^2 early-return test has passed.
// Backtracking::search (deps/mcloptlib/include/MCL/Backtracking.hpp:71-98) as
// SplitLBFGS::minimize calls it for -global_ls 1: p = -q, or -grad with
// alpha0 = min(1, 1 / max|grad|) after a non-descent restart; Armijo decrease
// 1e-4, step factor 0.7; a direction of norm <= machine epsilon returns 1e-4.
// fx0 is the AL value of the last gradient evaluation, which was at x.  Each
// trial value is one gradient-kernel pass (no gradient rows) at x + alpha p
// into a staging vector; the element cache it leaves is refreshed by the
// gradient at the accepted x.  On a non-descent restart the history reset of
// SplitLBFGS.hpp:189-194 is applied here, before the search.
double SolverGPU::line_search() {
    const int n = 3 * nf, vb = vec_blocks(n);
    k_ls_norms<<<vb, 256, 0, st_>>>(n, d_q_, d_gcur_, d_partials_, d_counter_, d_scal_ + S_LSN);
    k_ls_gmax<<<vb, 256, 0, st_>>>(n, d_gcur_, d_partials_, d_counter_, d_scal_ + S_LSM);
    WRAPD_LAUNCH_CHECK();
    kernel_launches += 2;
    sync_read();
    const double dir = h_scal_[S_DIR];
    if (std::isnan(dir)) throw CudaError(WRAPD_E_NAN, "L-BFGS decrement is NaN");
    const bool restart = !(dir > 0.0);
    ls_restart_ = restart;
    const double alpha0 = restart ? std::min(1.0, 1.0 / h_scal_[S_LSM]) : 1.0;
    const double pnorm = std::sqrt(restart ? h_scal_[S_LSN + 1] : h_scal_[S_LSN]);
    const double decrease = 1.e-4, tau = 0.7;
    if (pnorm <= std::numeric_limits<double>::epsilon()) return decrease;
    const double fx0 = h_scal_[S_GRAD];
    const double gtp = restart ? -h_scal_[S_LSN + 1] : -dir;
    const double* step = restart ? d_gcur_ : d_q_;
    double alpha = alpha0;
    for (int it = 0; it < 100000; ++it) {
        k_ls_trial<<<vb, 256, 0, st_>>>(n, d_sstage_, d_x_, step, alpha);
        WRAPD_LAUNCH_CHECK();
        kernel_launches++;
        WRAPD_ELEM_LAUNCH(k_grad, blocks_for(ne, 128), 128, d_sstage_, d_xfix_, mat_, 0, d_partials_, d_counter_,
                          d_scal_ + S_LSV);
        sync_read();
        const double fxa = h_scal_[S_LSV];
        if (fxa <= fx0 + alpha * decrease * gtp) return alpha;
        alpha *= tau;
    }
    return -1.0;
}

int SolverGPU::lbfgs_minimize() {
    const int M = cfg.lbfgs_m, n = 3 * nf, vb = vec_blocks(n);
    int max_iters = cfg.global_iters, global_iter = 1;
    bool breaking = false;
    double* A = d_scal_ + S_ALPHA;
    double* C = d_scal_ + S_C;
    for (; global_iter <= max_iters; ++global_iter) {
        const int it = std::min(M, m_k_);
        const bool small = n <= kTwoLoopMaxN;
        HistPtrs hs{}, hy{};
        HistRho hr{};
        if (small)
            for (int i = 0; i < it; ++i) { hs.p[i] = s_[i]; hy.p[i] = y_[i]; hr.r[i] = rho_[i]; }
        // first loop (newest to oldest): alpha_i = rho_i <s_i, q>, q -= alpha_i y_i
        if (small) {
            k_two_loop_first<<<1, kTwoLoopThreads, 0, st_>>>(n, d_q_, d_gcur_, hs, hy, hr, it, A);
            kernel_launches++;
        } else if (it == 0) {
            k_axpy_dot<<<vb, 256, 0, st_>>>(n, d_q_, d_gcur_, nullptr, nullptr, 0.0, nullptr, nullptr, 1.0,
                                            d_partials_, d_counter_, d_scal_ + S_DUMMY);
            kernel_launches++;
        } else {
            k_axpy_dot<<<vb, 256, 0, st_>>>(n, d_q_, d_gcur_, nullptr, nullptr, 0.0, s_[it - 1], nullptr,
                                            rho_[it - 1], d_partials_, d_counter_, A + (it - 1));
            for (int i = it - 2; i >= 0; --i)
                k_axpy_dot<<<vb, 256, 0, st_>>>(n, d_q_, nullptr, y_[i + 1], A + (i + 1), -1.0, s_[i], nullptr,
                                                rho_[i], d_partials_, d_counter_, A + i);
            k_axpy_dot<<<vb, 256, 0, st_>>>(n, d_q_, nullptr, y_[0], A, -1.0, nullptr, nullptr, 1.0, d_partials_,
                                            d_counter_, d_scal_ + S_DUMMY);
            kernel_launches += it + 1;
        }
        WRAPD_LAUNCH_CHECK();
        // q = A^-1 q, three right-hand sides at once
        mark(2);
        chol.solve(d_q_, st_);
        kernel_launches += chol.launches_solve;
        n_solve++;
        mark(3);
        // second loop (oldest to newest): c_i = alpha_i - rho_i <y_i, q>, q += c_i s_i; then dir = <grad, q>
        if (small) {
            k_two_loop_second<<<1, kTwoLoopThreads, 0, st_>>>(n, d_q_, d_gcur_, hs, hy, hr, it, A, C,
                                                              d_scal_ + S_DIR);
            kernel_launches++;
        } else if (it == 0) {
            k_axpy_dot<<<vb, 256, 0, st_>>>(n, d_q_, nullptr, nullptr, nullptr, 0.0, d_gcur_, nullptr, 1.0,
                                            d_partials_, d_counter_, d_scal_ + S_DIR);
            kernel_launches++;
        } else {
            k_axpy_dot<<<vb, 256, 0, st_>>>(n, d_q_, nullptr, nullptr, nullptr, 0.0, y_[0], A, -rho_[0], d_partials_,
                                            d_counter_, C);
            for (int i = 1; i < it; ++i)
                k_axpy_dot<<<vb, 256, 0, st_>>>(n, d_q_, nullptr, s_[i - 1], C + (i - 1), 1.0, y_[i], A + i, -rho_[i],
                                                d_partials_, d_counter_, C + i);
            k_axpy_dot<<<vb, 256, 0, st_>>>(n, d_q_, nullptr, s_[it - 1], C + (it - 1), 1.0, d_gcur_, nullptr, 1.0,
                                            d_partials_, d_counter_, d_scal_ + S_DIR);
            kernel_launches += it + 1;
        }
        // -global_ls 1: Backtracking::search along p = -q (SplitLBFGS.hpp:196-206)
        double rate = 1.0;
        if (cfg.global_ls && m_tol_ > 1.e-12) {
            rate = line_search();
            if (rate <= 0.0) {   // SplitMinimizer::FAILURE, after the restart's history reset
                if (ls_restart_) m_k_ = 0;
                return -1;
            }
        }
        // x -= rate q (or rate grad on a non-descent direction); s = x_new - x_old
        k_xupdate<<<vb, 256, 0, st_>>>(n, d_x_, d_q_, d_gcur_, d_scal_ + S_DIR, rate, d_sstage_);
        WRAPD_LAUNCH_CHECK();
        kernel_launches++;
        mark(2);
        // gradient at the new x; y = grad_new - grad
        grad_at_x(true);
        gather(d_gnew_, d_gcur_, d_ystage_, d_sstage_, true);
        mark(1);
        sync_read();
        const double dir = h_scal_[S_DIR];
        const double yy = h_scal_[S_GATHER], sy = h_scal_[S_GATHER + 1];
        if (std::isnan(dir)) throw CudaError(WRAPD_E_NAN, "L-BFGS decrement is NaN");
        if (dir <= 0.0) {
            max_iters -= m_k_;
            m_k_ = 0;
        }
        // history push: s[m_k] / y[m_k], or erase(begin) + push_back
        if (m_k_ < M) {
            std::swap(s_[m_k_], d_sstage_);
            std::swap(y_[m_k_], d_ystage_);
            rho_[m_k_] = 1.0 / sy;
        } else {
            double* so = s_[0];
            double* yo = y_[0];
            for (int i = 0; i + 1 < M; ++i) { s_[i] = s_[i + 1]; y_[i] = y_[i + 1]; rho_[i] = rho_[i + 1]; }
            s_[M - 1] = d_sstage_; y_[M - 1] = d_ystage_; rho_[M - 1] = 1.0 / sy;
            d_sstage_ = so; d_ystage_ = yo;
        }
        // grad_old <- grad, grad <- grad_new
        double* t = d_gold_;
        d_gold_ = d_gcur_;
        d_gcur_ = d_gnew_;
        d_gnew_ = t;
        if (dir > 0.0 && (dir < cfg.kappa * m_tol_ || dir < cfg.kappa * 1.e-12)) {
            m_k_ += 1;
            breaking = true;
            break;
        }
        if (std::fabs(yy) <= 0.0) { breaking = true; break; }
        m_k_++;
    }
    m_k_ = std::min(M, m_k_);
    return breaking ? global_iter : global_iter - 1;
}

int SolverGPU::iterate(int n, bool* conv) {
    if (!solving_) throw CudaError(WRAPD_E_STATE, "iterate before begin_solve");
    int done = 0;
    *conv = converged_;
    while (done < n && iter < cfg.max_iters && !converged_) {
        cudaEvent_t* ev_ = evs_[iter & 1];
        WRAPD_CUDA(cudaEventRecord(ev_[0], st_));
        mark(5);
        double dal = 0.0, obj_bef = 0.0, obj_aft = 0.0, prox_it = 0.0;
        int its = 1;
        if (cfg.rot_aware) {
            // ---- local step: polar_update (src/TetElements.cpp:256-356) ----
            local_step(cand_mode_now(), fp32() && !fp64_phase_);
            if (cfg.reweighting) count_++;
            mark(0);
            WRAPD_CUDA(cudaEventRecord(ev_[1], st_));
            // ---- global step: RotAwareGS::global_step (src/GlobalStepBehavior.hpp:246-258) ----
            if (m_k_ == 0) WRAPD_CUDA(cudaMemsetAsync(d_gold_, 0, 3 * (size_t)nf * sizeof(double), st_));
            grad_at_x(true);
            gather(d_gcur_, d_gold_, nullptr, nullptr, true);
            mark(1);
            sync_read();
            settle_timing(false);   // the previous iteration's events are behind this synchronisation
            const double bef = h_scal_[S_LOCAL], aft = h_scal_[S_LOCAL + 1], pe = h_scal_[S_LOCAL + 2];
            prox_it = h_scal_[S_LOCAL + 4];
            if (h_scal_[S_LOCAL + 3] > 0.0) throw CudaError(WRAPD_E_PROX_NEG, "negative singular value in a prox solution");
            dal = aft - bef + pe - curr_pe_;
            curr_pe_ = pe;
            obj_bef = h_scal_[S_GRAD];
            m_tol_ = std::fabs(dal);
            its = 0;
            if (!(h_scal_[S_GATHER] < 1.e-13)) its = lbfgs_minimize();
            obj_aft = h_scal_[S_GRAD];
        } else {
            // ---- local_update: TetElements::update (src/TetElements.cpp:193-254) ----
            local_step_unaware(cand_mode_now(), fp32() && !fp64_phase_);
            if (cfg.reweighting) count_++;
            mark(0);
            WRAPD_CUDA(cudaEventRecord(ev_[1], st_));
            // ---- UnawareGS::global_step (src/GlobalStepBehavior.hpp:162-180): x = A^-1 b ----
            global_step_unaware();
            sync_read();
            prox_it = h_scal_[S_LOCAL + 4];
            if (h_scal_[S_LOCAL + 3] > 0.0) throw CudaError(WRAPD_E_PROX_NEG, "negative singular value in a prox solution");
            obj_aft = 1.e8;   // UnawareGS::last_step_delta_auglag (src/GlobalStepBehavior.hpp:102)
        }
        const double pe_x = h_scal_[S_GRAD + 1];
        const int flips = (int)h_scal_[S_GRAD + 2];
        WRAPD_CUDA(cudaEventRecord(ev_[2], st_));
        // ---- reweighting: possibly_update_weights (src/System.cpp:50-63) ----
        bool rw = false;
        if (cfg.reweighting) {
            if (cfg.rw_every > 0) {
                rw = ((iter + 1) % cfg.rw_every) == 0;
            } else {
                k_ratio<<<blocks_for(ne, 256), 256, 0, st_>>>(view(), d_partials_, d_counter_, d_scal_ + S_RATIO);
                WRAPD_LAUNCH_CHECK();
                kernel_launches++;
                sync_read();
                rw = h_scal_[S_RATIO] > cfg.gamma;
            }
            if (rw) {
                apply_weights();
                factor();
                m_k_ = 0;
            }
        }
        WRAPD_CUDA(cudaEventRecord(ev_[3], st_));
        // The x error of the final x: the rotation-aware step's last gradient
        // gather computed it (outside the timed phases, as the reference logs it);
        // the rotation-unaware step computes it here.
        if (!cfg.rot_aware) {
            x_error_launch();
            sync_read();
        }
        const double xerr2 = cfg.rot_aware ? h_scal_[S_GATHER + 2] : h_scal_[S_XERR];
        if (profiling) {
            sync_read();
            profile_flush();
        }
        if (rw) check_status();
        runtime_ms[5] += its;
        // ---- AlgorithmData::update_per_iter_* (src/AlgorithmData.cpp:66-83) ----
        const int k = iter;
        logs_.reweighted.push_back(rw ? 1 : 0);
        logs_.ls_dal.push_back(std::fabs(dal));
        logs_.gs_dal.push_back(std::fabs(obj_aft - obj_bef));
        logs_.inner.push_back(its);
        logs_.prox_iters.push_back(prox_it / double(ne));
        logs_.objectives.push_back(pe_x);
        logs_.flips.push_back(flips);
        // phase times: read once a later synchronisation has passed the events
        logs_.acc_time_s.push_back(0.0);
        pend_ = PendingTiming{true, k, ev_};
        if (!cfg.rot_aware || profiling || rw) settle_timing(false);
        const double xe = std::sqrt(xerr2) / init_xerr_;
        logs_.x_errors.push_back(xe);
        iter = k + 1;
        done++;
        // ---- ADMM::converged (src/ADMM.cpp:158-169) ----
        const double res = std::fabs(logs_.objectives[k + 1] - logs_.objectives[k]) / (std::fabs(logs_.objectives[k + 1]) + 1.0);
        // Mixed mode refinement: once the energy moves less than FP32 can
        // resolve, finish with FP64 local steps.
        if (fp32() && !fp64_phase_ && res < kMixedSwitch) fp64_phase_ = true;
        if ((logs_.flips[k + 1] == 0 && logs_.flips[k] == 0 && res < cfg.tol) || (have_soln_ && xe < 1.e-4))
            converged_ = true;
    }
    settle_timing(true);
    *conv = converged_;
    return done;
}

// Adds a finished iteration's phase times (CUDA events) to the runtime and its
// accumulated-time log entry.  wait = false: a host synchronisation of the
// stream has already passed the events.
void SolverGPU::settle_timing(bool wait) {
    if (!pend_.on) return;
    if (wait) WRAPD_CUDA(cudaEventSynchronize(pend_.ev[3]));
    float ml = 0.f, mg = 0.f, mr = 0.f;
    WRAPD_CUDA(cudaEventElapsedTime(&ml, pend_.ev[0], pend_.ev[1]));
    WRAPD_CUDA(cudaEventElapsedTime(&mg, pend_.ev[1], pend_.ev[2]));
    WRAPD_CUDA(cudaEventElapsedTime(&mr, pend_.ev[2], pend_.ev[3]));
    runtime_ms[1] += ml; runtime_ms[2] += mg; runtime_ms[3] += mr;
    logs_.acc_time_s[pend_.k + 1] = (runtime_ms[1] + runtime_ms[2] + runtime_ms[3]) / 1000.0;
    pend_.on = false;
}

void SolverGPU::positions(double* out) {
    std::vector<double> xp(3 * (size_t)nf);
    WRAPD_CUDA(cudaMemcpyAsync(xp.data(), d_x_, xp.size() * sizeof(double), cudaMemcpyDeviceToHost, st_));
    WRAPD_CUDA(cudaStreamSynchronize(st_));
    // finish_solve (src/ADMM.cpp:171-182): X = S_free x_free + S_fix x_fix
    for (int i = 0; i < nv; ++i)
        for (int c = 0; c < 3; ++c)
            out[3 * (size_t)i + c] = free_of_vert_[i] >= 0 ? xp[3 * (size_t)iperm_[free_of_vert_[i]] + c]
                                                            : init_[3 * (size_t)i + c];
}

void SolverGPU::solve(double* out) {
    if (!initialized_) throw CudaError(WRAPD_E_STATE, "solve before initialize");
    begin_solve();
    bool conv = false;
    while (iter < cfg.max_iters && !conv) iterate(cfg.max_iters, &conv);
    if (out) positions(out);
}

// ---- components ------------------------------------------------------------------
void SolverGPU::download_elem(const double* d, int comps, std::vector<double>& out) {
    const size_t n = (size_t)comps * ne;
    std::vector<double> soa(n);
    WRAPD_CUDA(cudaMemcpyAsync(soa.data(), d, n * 8, cudaMemcpyDeviceToHost, st_));
    WRAPD_CUDA(cudaStreamSynchronize(st_));
    out.resize(n);
    for (int e = 0; e < ne; ++e)
        for (int k = 0; k < comps; ++k) out[(size_t)e * comps + k] = soa[(size_t)k * ne + e];
}

void SolverGPU::upload_elem(double* d, int comps, const double* in) {
    const size_t n = (size_t)comps * ne;
    std::vector<double> soa(n);
    for (int e = 0; e < ne; ++e)
        for (int k = 0; k < comps; ++k) soa[(size_t)k * ne + e] = in[(size_t)e * comps + k];
    WRAPD_CUDA(cudaMemcpyAsync(d, soa.data(), n * 8, cudaMemcpyHostToDevice, st_));
    WRAPD_CUDA(cudaStreamSynchronize(st_));
}

void SolverGPU::get_state(const std::string& name, std::vector<double>& out) {
    if (!initialized_) throw CudaError(WRAPD_E_STATE, "state before initialize");
    if (name == "Z") download_elem(d_Z_, 9, out);
    else if (name == "U") download_elem(d_U_, 9, out);
    else if (name == "symF") download_elem(d_symF_, 9, out);
    else if (name == "sigma") download_elem(d_sig_, 3, out);
    else if (name == "slast") download_elem(d_slast_, 3, out);
    else if (name == "w2") download_elem(d_w2_, 1, out);
    else if (name == "w2c") download_elem(d_w2c_, 1, out);
    else if (name == "vol") download_elem(d_vol_, 1, out);
    else if (name == "xfree" || name == "grad") {
        std::vector<double> xp(3 * (size_t)nf);
        WRAPD_CUDA(cudaMemcpyAsync(xp.data(), name == "xfree" ? d_x_ : d_gcur_, xp.size() * 8, cudaMemcpyDeviceToHost, st_));
        WRAPD_CUDA(cudaStreamSynchronize(st_));
        out.resize(xp.size());
        for (int i = 0; i < nf; ++i)
            for (int c = 0; c < 3; ++c) out[3 * (size_t)i + c] = xp[3 * (size_t)iperm_[i] + c];
    } else {
        throw CudaError(WRAPD_E_INPUT, "unknown state name " + name);
    }
}

void SolverGPU::set_state(const std::string& name, const double* in, int64_t n) {
    if (!initialized_) throw CudaError(WRAPD_E_STATE, "state before initialize");
    auto need = [&](int64_t m) { if (n != m) throw CudaError(WRAPD_E_INPUT, "wrong length for " + name); };
    if (name == "Z") { need(9LL * ne); upload_elem(d_Z_, 9, in); }
    else if (name == "U") { need(9LL * ne); upload_elem(d_U_, 9, in); }
    else if (name == "slast") { need(3LL * ne); upload_elem(d_slast_, 3, in); }
    else if (name == "w2") { need(ne); upload_elem(d_w2_, 1, in); }
    else if (name == "xfree") {
        need(3LL * nf);
        std::vector<double> xp(3 * (size_t)nf);
        for (int i = 0; i < nf; ++i)
            for (int c = 0; c < 3; ++c) xp[3 * (size_t)iperm_[i] + c] = in[3 * (size_t)i + c];
        WRAPD_CUDA(cudaMemcpyAsync(d_x_, xp.data(), xp.size() * 8, cudaMemcpyHostToDevice, st_));
        WRAPD_CUDA(cudaStreamSynchronize(st_));
    } else {
        throw CudaError(WRAPD_E_INPUT, "state " + name + " is read-only");
    }
}

void SolverGPU::update_defo_cache() {
    grad_at_x(false);
    sync_read();
}

double SolverGPU::polar_update(bool update_candidates) {
    local_step(update_candidates ? cand_mode_now() : CAND_NONE, fp32() && !fp64_phase_);
    if (update_candidates && cfg.reweighting) count_++;
    sync_read();
    if (h_scal_[S_LOCAL + 3] > 0.0) throw CudaError(WRAPD_E_PROX_NEG, "negative singular value in a prox solution");
    const double dal = h_scal_[S_LOCAL + 1] - h_scal_[S_LOCAL] + h_scal_[S_LOCAL + 2] - curr_pe_;
    curr_pe_ = h_scal_[S_LOCAL + 2];
    return dal;
}

double SolverGPU::global_grad(const double* xfree, double* grad) {
    if (xfree) set_state("xfree", xfree, 3LL * nf);
    grad_at_x(true);
    gather(d_gcur_, nullptr, nullptr, nullptr);
    sync_read();
    if (grad) {
        std::vector<double> g;
        get_state("grad", g);
        std::memcpy(grad, g.data(), g.size() * sizeof(double));
    }
    return h_scal_[S_GRAD];
}

void SolverGPU::potential_energy(double* pe, int* flips) {
    grad_at_x(false);
    sync_read();
    if (pe) *pe = h_scal_[S_GRAD + 1];
    if (flips) *flips = (int)h_scal_[S_GRAD + 2];
}

void SolverGPU::solve_A(const double* b, double* x) {
    if (!initialized_) throw CudaError(WRAPD_E_STATE, "solve_A before initialize");
    std::vector<double> xp(3 * (size_t)nf);
    for (int i = 0; i < nf; ++i)
        for (int c = 0; c < 3; ++c) xp[3 * (size_t)iperm_[i] + c] = b[3 * (size_t)i + c];
    WRAPD_CUDA(cudaMemcpyAsync(d_q_, xp.data(), xp.size() * 8, cudaMemcpyHostToDevice, st_));
    chol.solve(d_q_, st_);
    kernel_launches += chol.launches_solve;
    WRAPD_CUDA(cudaMemcpyAsync(xp.data(), d_q_, xp.size() * 8, cudaMemcpyDeviceToHost, st_));
    WRAPD_CUDA(cudaStreamSynchronize(st_));
    for (int i = 0; i < nf; ++i)
        for (int c = 0; c < 3; ++c) x[3 * (size_t)i + c] = xp[3 * (size_t)iperm_[i] + c];
}

}  // namespace wrapd
