// Host orchestration of the ADMM solve loop; see solver.cuh.
#include "solver.cuh"

#include "elements.cuh"

#include <algorithm>
#include <atomic>
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
// Launch masks over the meshes of a batch (one int per mesh each).
enum : int {
    MK_ALL = 0,      // every mesh
    MK_ADMM,         // not yet converged
    MK_LBFGS,        // inside the current SplitLBFGS::minimize iteration
    MK_RW,           // reweights now
    MK_L32, MK_L32N, MK_L64, MK_L64N,   // local step: FP32 / FP64 arithmetic, without / with the prox network
    MK_ZERO,         // grad_old to be zeroed (history empty)
    MK_SMALL,        // MK_LBFGS meshes whose two-loop runs in one CTA
    MK_LARGE,        // the other MK_LBFGS meshes
    MK_COUNT
};
// Dynamic shared memory of k_local<double>: the prox L-BFGS history, 48 doubles
// per thread (kLocalHistBytes for a 128-thread block, the unaware step's).
constexpr int kLocalHistBytes = 48 * 128 * (int)sizeof(double);
constexpr int kLocalTileMax = 512;   // largest local-step tile (elements = threads per CTA)
int local_hist_bytes(int per) { return 48 * per * (int)sizeof(double); }
int local_net_bytes(int per) { return net::IMAGE_BYTES + (per / 32) * net::WARP_SCRATCH; }
// Mixed mode switches its local step to FP64 when the normalized energy
// residual drops below this (the FP32 local step's noise floor is ~1e-7).
constexpr double kMixedSwitch = 1e-7;

int blocks_for(int64_t n, int threads) { return std::max(1, ceil_div(n, threads)); }

// Vector kernels use a fixed grid of 2 CTAs per SM (grid-stride loops).
int vec_blocks(int64_t n) { return std::max(1, std::min(2 * kNumSMs, ceil_div(n, 256))); }

__global__ void k_fill(double* __restrict__ p, int64_t n, double v) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

// (S * Dm^-1)^T and the rest volume of every tet (src/TetElements.cpp:93-118),
// and its weight w^2 = beta_static k vol.  Every operation is an explicitly
// rounded IEEE add, multiply or divide in the order a plain C++ evaluation of
// the same expressions takes (left to right, no fused multiply-add), so the
// values are those of that host computation bit for bit.  An inverted tet
// (negative volume) lowers *first_inverted to its index.
__global__ void k_element_geometry(int ne, const int* __restrict__ tets, const double* __restrict__ rest,
                                   const int* __restrict__ mid, const Material* __restrict__ mats, double wr0,
                                   double beta, double* __restrict__ Di, double* __restrict__ vol,
                                   double* __restrict__ w2, int* first_inverted) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    const double* p0 = rest + 3 * (size_t)tets[4 * (size_t)e];
    const double* p1 = rest + 3 * (size_t)tets[4 * (size_t)e + 1];
    const double* p2 = rest + 3 * (size_t)tets[4 * (size_t)e + 2];
    const double* p3 = rest + 3 * (size_t)tets[4 * (size_t)e + 3];
    double ed[9];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        ed[r + 0] = __dsub_rn(p1[r], p0[r]);
        ed[r + 3] = __dsub_rn(p2[r], p0[r]);
        ed[r + 6] = __dsub_rn(p3[r], p0[r]);
    }
    auto m = [&](int r, int c) { return ed[r + 3 * c]; };
    auto dd = [](double a, double b, double c, double d) { return __dsub_rn(__dmul_rn(a, b), __dmul_rn(c, d)); };
    const double c00 = dd(m(1, 1), m(2, 2), m(1, 2), m(2, 1));
    const double c01 = dd(m(1, 2), m(2, 0), m(1, 0), m(2, 2));
    const double c02 = dd(m(1, 0), m(2, 1), m(1, 1), m(2, 0));
    const double det = __dadd_rn(__dadd_rn(__dmul_rn(m(0, 0), c00), __dmul_rn(m(0, 1), c01)), __dmul_rn(m(0, 2), c02));
    const double id = __ddiv_rn(1.0, det);
    double inv[9];
    inv[0 + 3 * 0] = __dmul_rn(c00, id);
    inv[1 + 3 * 0] = __dmul_rn(c01, id);
    inv[2 + 3 * 0] = __dmul_rn(c02, id);
    inv[0 + 3 * 1] = __dmul_rn(dd(m(0, 2), m(2, 1), m(0, 1), m(2, 2)), id);
    inv[1 + 3 * 1] = __dmul_rn(dd(m(0, 0), m(2, 2), m(0, 2), m(2, 0)), id);
    inv[2 + 3 * 1] = __dmul_rn(dd(m(0, 1), m(2, 0), m(0, 0), m(2, 1)), id);
    inv[0 + 3 * 2] = __dmul_rn(dd(m(0, 1), m(1, 2), m(0, 2), m(1, 1)), id);
    inv[1 + 3 * 2] = __dmul_rn(dd(m(0, 2), m(1, 0), m(0, 0), m(1, 2)), id);
    inv[2 + 3 * 2] = __dmul_rn(dd(m(0, 0), m(1, 1), m(0, 1), m(1, 0)), id);
    const double v = __ddiv_rn(det, 6.0);
    if (v < 0.0) atomicMin(first_inverted, e);
    // Di(r, a): a = 0 -> minus the column sums of Dm^-1 rows; a >= 1 -> row a-1 of Dm^-1
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        Di[(size_t)r * ne + e] = __dsub_rn(__dsub_rn(-inv[0 + 3 * r], inv[1 + 3 * r]), inv[2 + 3 * r]);
#pragma unroll
        for (int a = 1; a < 4; ++a) Di[(size_t)(r + 3 * a) * ne + e] = inv[(a - 1) + 3 * r];
    }
    vol[e] = v;
    const double wr = mid ? mats[mid[e]].wr : wr0;
    w2[e] = __dmul_rn(__dmul_rn(beta, wr), v);
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
    WRAPD_CUDA(cudaFuncSetAttribute(k_local<double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    local_hist_bytes(kLocalTileMax)));
    WRAPD_CUDA(cudaFuncSetAttribute(k_local<double, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    local_net_bytes(kLocalTileMax)));
    WRAPD_CUDA(cudaFuncSetAttribute(k_local<float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    local_net_bytes(kLocalTileMax)));
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
    if (h_status_) cudaFreeHost(h_status_);
    if (h_ctl_block_) cudaFreeHost(h_ctl_block_);
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
    if (meshes_.size() > 1 && (!cfg.rot_aware || cfg.global_ls))
        throw CudaError(WRAPD_E_UNSUPPORTED, "a batch of meshes needs the rotation-aware global step without line search");
    auto t0 = std::chrono::steady_clock::now();
    // host phase timings, printed to stderr with verbose >= 2
    std::vector<std::pair<const char*, double>> laps;
    auto tl = t0;
    auto lap = [&](const char* name) {
        const auto now = std::chrono::steady_clock::now();
        laps.emplace_back(name, std::chrono::duration<double, std::milli>(now - tl).count());
        tl = now;
    };
    // ---- element geometry (TetElements ctor, src/TetElements.cpp:90-142): on
    // the device (k_element_geometry) from the rest positions and the tets,
    // while the host builds the graph and the dissection below ----
    std::vector<int> mid(ne);
    for (const MeshIn& M : meshes_)
        for (int e = M.e_off; e < M.e_off + M.ne; ++e) mid[e] = M.mat;
    if (mats_.size() > 1) {
        d_mid_ = dupload(mid);
        d_mats_ = dupload(mats_);
    } else {
        mat_ = mats_[0];   // one material: the mesh's own when it was given one
    }
    d_Di_ = static_cast<double*>(dalloc(12 * (size_t)ne * sizeof(double)));
    d_vol_ = static_cast<double*>(dalloc((size_t)ne * sizeof(double)));
    d_w2_ = static_cast<double*>(dalloc((size_t)ne * sizeof(double)));
    const size_t geo_tets = 4 * (size_t)ne * sizeof(int), geo_rest = 3 * (size_t)nv * sizeof(double);
    const size_t geo_rest_off = (geo_tets + 15) / 16 * 16, geo_flag_off = (geo_rest_off + geo_rest + 15) / 16 * 16;
    struct GeoBuf {   // freed on every path out of initialize
        char* p = nullptr;
        ~GeoBuf() { if (p) cudaFree(p); }
    } geo;
    char*& d_geo = geo.p;
    if (cudaMalloc(&d_geo, geo_flag_off + 16) != cudaSuccess) {
        cudaGetLastError();
        throw CudaError(WRAPD_E_OOM, "cudaMalloc of the rest mesh failed");
    }
    int* d_first_inverted = reinterpret_cast<int*>(d_geo + geo_flag_off);
    {
        const int none = ne;
        WRAPD_CUDA(cudaMemcpyAsync(d_geo, tets_.data(), geo_tets, cudaMemcpyHostToDevice, st_));
        WRAPD_CUDA(cudaMemcpyAsync(d_geo + geo_rest_off, rest_.data(), geo_rest, cudaMemcpyHostToDevice, st_));
        WRAPD_CUDA(cudaMemcpyAsync(d_first_inverted, &none, sizeof(int), cudaMemcpyHostToDevice, st_));
        k_element_geometry<<<blocks_for(ne, 256), 256, 0, st_>>>(
            ne, reinterpret_cast<const int*>(d_geo), reinterpret_cast<const double*>(d_geo + geo_rest_off),
            mats_.size() > 1 ? d_mid_ : nullptr, d_mats_, mats_[0].wr, cfg.beta_static, d_Di_, d_vol_, d_w2_,
            d_first_inverted);
        WRAPD_LAUNCH_CHECK();
    }
    // the inverted-tet check: read back before the device state is filled in
    auto check_geometry = [&]() {
        int first = ne;
        WRAPD_CUDA(cudaMemcpyAsync(&first, d_first_inverted, sizeof(int), cudaMemcpyDeviceToHost, st_));
        WRAPD_CUDA(cudaStreamSynchronize(st_));
        cudaFree(d_geo);
        d_geo = nullptr;
        if (first < ne) throw CudaError(WRAPD_E_INVERTED_REST, "inverted tet " + std::to_string(first) + " in the rest mesh");
    };
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
    nm = static_cast<int>(meshes_.size());
    runs_.assign(nm, MeshRun{});
    for (int mi = 0; mi < nm; ++mi) {
        const MeshIn& M = meshes_[mi];
        int f0 = -1, f1 = -1;
        for (int i = M.v_off; i < M.v_off + M.nv; ++i)
            if (free_of_vert_[i] >= 0) { if (f0 < 0) f0 = free_of_vert_[i]; f1 = free_of_vert_[i] + 1; }
        if (f0 < 0) throw CudaError(WRAPD_E_INPUT, "a mesh without free vertices");
        // the merged dissection order keeps each mesh's free vertices together,
        // at the same offset as the free numbering
        runs_[mi].e0 = M.e_off;
        runs_[mi].e1 = M.e_off + M.ne;
        runs_[mi].f0 = f0;
        runs_[mi].f1 = f1;
        const int n = f1 - f0;
        std::vector<int> p(n + 1), a(adj.begin() + ptr[f0], adj.begin() + ptr[f1]);
        for (int i = 0; i <= n; ++i) p[i] = ptr[f0 + i] - ptr[f0];
        for (int& v : a) v -= f0;
        std::vector<double> c(coords.begin() + 3 * (size_t)f0, coords.begin() + 3 * (size_t)f1);
        parts.push_back(analyse(n, p, a, c, cfg.leaf_size > 0 ? cfg.leaf_size : 64));
    }
    if (nm > 1)
        for (int m = 0; m < nm; ++m) chol.front_mesh.insert(chol.front_mesh.end(), parts[m].fronts.size(), m);
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
    check_geometry();
    // ---- device state ----
    const size_t TS = sizeof(double);
    d_idx_ = dupload(idx);
    d_w2c_ = static_cast<double*>(dalloc(ne * sizeof(double)));
    // U and V of the last gradient's SVD (single mesh): 18 doubles per element
    d_uv_ = meshes_.size() == 1 ? static_cast<double*>(dalloc((size_t)18 * ne * sizeof(double))) : nullptr;
    uv_valid_ = false;
    d_Z_ = static_cast<double*>(dalloc(9 * (size_t)ne * TS));
    d_U_ = static_cast<double*>(dalloc(9 * (size_t)ne * TS));
    d_symF_ = static_cast<double*>(dalloc(9 * (size_t)ne * TS));
    d_sig_ = static_cast<double*>(dalloc(3 * (size_t)ne * TS));
    d_slast_ = static_cast<double*>(dalloc(3 * (size_t)ne * TS));
    d_gel_ = static_cast<double*>(dalloc(12 * (size_t)ne * TS));
    WRAPD_CUDA(cudaMemsetAsync(d_U_, 0, 9 * (size_t)ne * TS, st_));
    WRAPD_CUDA(cudaMemsetAsync(d_Z_, 0, 9 * (size_t)ne * TS, st_));
    // m_last_sigma = (1, 1, 1)
    k_fill<<<blocks_for(3 * (int64_t)ne, 256), 256, 0, st_>>>(d_slast_, 3 * (int64_t)ne, 1.0);
    WRAPD_LAUNCH_CHECK();
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
    for (double*& g : d_G_) {
        g = static_cast<double*>(dalloc(vb));
        WRAPD_CUDA(cudaMemsetAsync(g, 0, vb, st_));
    }
    d_S_.assign(cfg.lbfgs_m + 1, nullptr);
    d_Y_.assign(cfg.lbfgs_m + 1, nullptr);
    for (int i = 0; i <= cfg.lbfgs_m; ++i) {
        d_S_[i] = static_cast<double*>(dalloc(vb));
        d_Y_[i] = static_cast<double*>(dalloc(vb));
    }
    // launch tilings: element tiles of 128 and 256, vertex tiles of 32 (the
    // gather's eight lanes per vertex), vector tiles of kVecTile doubles; each
    // mesh's tiles start at its first item
    {
        std::vector<std::pair<int, int>> er, vr, qr;
        for (const MeshRun& R : runs_) {
            er.emplace_back(R.e0, R.e1);
            vr.emplace_back(R.f0, R.f1);
            qr.emplace_back(3 * R.f0, 3 * R.f1);
        }
        build_tiles(te128_, 128, er);
        build_tiles(te256_, 256, er);
        build_tiles(te_local_, local_per_, er);
        build_tiles(tv32_, 32, vr);
        build_tiles(tvec_, kVecTile, qr);
    }
    // (partials for the largest tile count: 64-element local tiles are the finest)
    build_tiles(te_local_, 64, [&] {
        std::vector<std::pair<int, int>> er;
        for (const MeshRun& R : runs_) er.emplace_back(R.e0, R.e1);
        return er;
    }());
    const int finest_local = te_local_.count;
    {
        std::vector<std::pair<int, int>> er;
        for (const MeshRun& R : runs_) er.emplace_back(R.e0, R.e1);
        build_tiles(te_local_, local_per_, er);
    }
    const size_t nblk = (size_t)std::max({te128_.count, te256_.count, tv32_.count, tvec_.count, finest_local,
                                          blocks_for(8 * (int64_t)nf, 256), vec_blocks(3 * (int64_t)nf)}) + 8;
    d_partials_ = static_cast<double*>(dalloc(nblk * 5 * sizeof(double)));
    d_counters_ = static_cast<unsigned*>(dalloc(nm * sizeof(unsigned)));
    // the cooperative two-loop recursion (one mesh above the one-CTA size):
    // its grid is what fits on the device at once
    d_bar_ = static_cast<unsigned*>(dalloc(sizeof(unsigned)));
    coop_grid_ = 0;
    {
        int dev = 0, coop = 0, sms = 0;
        WRAPD_CUDA(cudaGetDevice(&dev));
        WRAPD_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
        WRAPD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        auto fits = [&](const void* f) {
            int b = 0;
            WRAPD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, f, kTwoLoopGridThreads, 0));
            return b * sms;
        };
        const int cap = std::min(fits((const void*)k_two_loop_grid<false, false>),
                                 fits((const void*)k_two_loop_grid<true, false>));
        const int cap_reg = std::min(fits((const void*)k_two_loop_grid<false, true>),
                                     fits((const void*)k_two_loop_grid<true, true>));
        // the register form when every vector tile gets its own resident CTA
        coop_reg_ = tvec_.count <= cap_reg;
        if (coop && nm == 1) coop_grid_ = std::min(tvec_.count, coop_reg_ ? cap_reg : cap);
    }
    d_scal_ = static_cast<double*>(dalloc((size_t)nm * kScalStride * sizeof(double)));
    WRAPD_CUDA(cudaMemsetAsync(d_counters_, 0, nm * sizeof(unsigned), st_));
    WRAPD_CUDA(cudaMemsetAsync(d_scal_, 0, (size_t)nm * kScalStride * sizeof(double), st_));
    WRAPD_CUDA(cudaMallocHost(&h_scal_, (size_t)nm * kScalStride * sizeof(double)));
    std::memset(h_scal_, 0, (size_t)nm * kScalStride * sizeof(double));
    WRAPD_CUDA(cudaMallocHost(&h_status_, sizeof(int)));
    *h_status_ = 0;
    {
        static const double one = 1.0;
        WRAPD_CUDA(cudaMemcpyAsync(d_scal_ + S_ONE, &one, sizeof(double), cudaMemcpyHostToDevice, st_));
    }
    // the per-mesh control block: masks, MeshCtl, rho
    {
        const size_t mb = (size_t)MK_COUNT * nm * sizeof(int), cb = (size_t)nm * sizeof(MeshCtl),
                     rb = (size_t)nm * kHistSlots * sizeof(double);
        const size_t mo = 0, co = (mb + 15) / 16 * 16, ro = (co + cb + 15) / 16 * 16;
        ctl_bytes_ = ro + rb;
        d_ctl_block_ = dalloc(ctl_bytes_);
        WRAPD_CUDA(cudaMallocHost(&h_ctl_block_, ctl_bytes_));
        std::memset(h_ctl_block_, 0, ctl_bytes_);
        char* d = static_cast<char*>(d_ctl_block_);
        char* h = static_cast<char*>(h_ctl_block_);
        d_ctl_block_masks_ = reinterpret_cast<int*>(d + mo);
        h_masks_ = reinterpret_cast<int*>(h + mo);
        d_ctl_ = reinterpret_cast<MeshCtl*>(d + co);
        h_ctl_ = reinterpret_cast<MeshCtl*>(h + co);
        d_rho_ = reinterpret_cast<double*>(d + ro);
        h_rho_ = reinterpret_cast<double*>(h + ro);
        for (int m = 0; m < nm; ++m) {
            MeshCtl& c = runs_[m].ctl;
            c.v0 = 3 * runs_[m].f0;
            c.v1 = 3 * runs_[m].f1;
            c.small = (c.v1 - c.v0) <= kTwoLoopMaxN ? 1 : 0;
            set_mask(MK_ALL, m, true);
            set_mask(MK_ADMM, m, true);
        }
        push_ctl();
    }
    lap("element state upload");
    chol.build(S, A_pos, A_ptr, A_con, st_);
    WRAPD_CUDA(cudaStreamSynchronize(st_));
    lap("factor structures upload");
    // ---- GlobalStepBehavior ctor: midupdate_weights(X_init) and the first factorization ----
    if (cfg.reweighting) {
        mid_candidates(true, cand_mode_now());
        count_++;
        apply_weights(MK_ALL);
    }
    if (cfg.autotune) {
        chol.autotune(d_w2_, d_Di_, ne, st_);
        lap("autotune (solve chunks, panel steps)");
    }
    factor();
    for (MeshRun& R : runs_) R.ctl.k = 0;
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

// ---- batch plumbing ------------------------------------------------------------------
// Tiles of `per` items over each [first, end) range, meshes in order.
void SolverGPU::build_tiles(TileSet& t, int per, const std::vector<std::pair<int, int>>& ranges) {
    t.per = per;
    t.n = ranges.empty() ? 0 : ranges.back().second;
    if (ranges.size() == 1) {
        t.count = blocks_for(ranges[0].second - ranges[0].first, per);
        return;
    }
    std::vector<int4> tab;
    std::vector<int> t0;
    for (size_t m = 0; m < ranges.size(); ++m) {
        t0.push_back(static_cast<int>(tab.size()));
        const int a = ranges[m].first, b = ranges[m].second;
        for (int f = a; f < b; f += per) tab.push_back(make_int4((int)m, f, std::min(f + per, b), 0));
        if (a == b) tab.push_back(make_int4((int)m, a, a, 0));
    }
    t0.push_back(static_cast<int>(tab.size()));
    t.count = static_cast<int>(tab.size());
    t.d_t = dupload(tab);
    t.d_tile0 = dupload(t0);
}

bool SolverGPU::any_mask(int which) const {
    for (int m = 0; m < nm; ++m)
        if (h_masks_[(size_t)which * nm + m]) return true;
    return false;
}

// The pinned mirror of the control block is written only after the stream has
// read the last upload from it (normally a synchronisation already passed it).
void SolverGPU::ctl_writable() {
    if (!ctl_pending_) return;
    WRAPD_CUDA(cudaStreamSynchronize(st_));
    ctl_pending_ = false;
}

// Uploads the masks, MeshCtl and rho of every mesh.
void SolverGPU::push_ctl() {
    ctl_writable();
    for (int m = 0; m < nm; ++m) {
        h_ctl_[m] = runs_[m].ctl;
        std::memcpy(h_rho_ + (size_t)m * kHistSlots, runs_[m].rho, sizeof(runs_[m].rho));
    }
    WRAPD_CUDA(cudaMemcpyAsync(d_ctl_block_, h_ctl_block_, ctl_bytes_, cudaMemcpyHostToDevice, st_));
    ctl_pending_ = true;
}

VecPools SolverGPU::pools() const {
    VecPools P{};
    for (int i = 0; i < 3; ++i) P.G[i] = d_G_[i];
    for (int i = 0; i <= cfg.lbfgs_m; ++i) {
        P.S[i] = d_S_[i];
        P.Y[i] = d_Y_[i];
    }
    P.M = cfg.lbfgs_m;
    return P;
}

const Logs& SolverGPU::mesh_logs(int m) const {
    if (m < 0 || m >= nm) throw CudaError(WRAPD_E_INPUT, "mesh index out of range");
    return runs_[m].logs;
}

#define WRAPD_ELEM_LAUNCH(kernel, tiles, block, ...)                                        \
    do {                                                                                    \
        kernel<<<(tiles).count, block, 0, st_>>>(view(), (tiles).view(), __VA_ARGS__);      \
        WRAPD_LAUNCH_CHECK();                                                               \
        kernel_launches++;                                                                  \
    } while (0)

// The global gradient at x.  A single mesh in the rotation-aware global step
// without line search keeps the SVD factors of its last gradient (k_grad
// UV = 1); the first gradient of the next ADMM iteration is taken at the same
// x (the local step changes only Z and U), so it reads them back (UV = 2)
// instead of redoing the per-element SVD.  uv_valid_ is cleared wherever x
// changes.  256-element tiles (786k bar: 1.095 -> 1.077 ms per global step
// against 128; 3.9M bar: 5.09 -> 4.95 ms), in a batch too, so that a mesh's
// sums are added in the same order as when it is solved alone.
void SolverGPU::grad_at_x(bool write_gel, int mk) {
    if (nm > 1) {
        WRAPD_ELEM_LAUNCH(k_grad<true>, te256_, 256, mask(mk), d_x_, d_xfix_, mat_, write_gel ? 1 : 0, d_partials_,
                          d_counters_, ds(S_GRAD), kScalStride);
    } else if (d_uv_ && write_gel && cfg.rot_aware && !cfg.global_ls) {
        if (uv_valid_)
            k_grad<false, 2><<<te256_.count, 256, 0, st_>>>(view(), te256_.view(), mask(mk), d_x_, d_xfix_, mat_, 1,
                                                             d_partials_, d_counters_, ds(S_GRAD), kScalStride, d_uv_);
        else
            k_grad<false, 1><<<te256_.count, 256, 0, st_>>>(view(), te256_.view(), mask(mk), d_x_, d_xfix_, mat_, 1,
                                                             d_partials_, d_counters_, ds(S_GRAD), kScalStride, d_uv_);
        WRAPD_LAUNCH_CHECK();
        kernel_launches++;
        uv_valid_ = true;
        return;
    } else {
        WRAPD_ELEM_LAUNCH(k_grad<false>, te256_, 256, mask(mk), d_x_, d_xfix_, mat_, write_gel ? 1 : 0, d_partials_,
                          d_counters_, ds(S_GRAD), kScalStride);
    }
    uv_valid_ = false;
}

void SolverGPU::gather(int mode, int mk, bool xerr, double* plain) {
    k_gather<<<tv32_.count, 256, 0, st_>>>(tv32_.view(), mask(mk), mode, d_ctl_, pools(), plain, d_inc_ptr_, d_inc_,
                                           d_gel_, ne, xerr ? d_x_ : nullptr, d_xsoln_, d_partials_, d_counters_,
                                           ds(S_GATHER), kScalStride);
    WRAPD_LAUNCH_CHECK();
    kernel_launches++;
}

// The local step over the meshes of MK_ADMM, in the variants the masks
// MK_L32 / MK_L32N / MK_L64 / MK_L64N assign them (set by the caller).
void SolverGPU::local_step(int cand_mode) {
    if (cfg.model == MODEL_ARAP) {
        WRAPD_ELEM_LAUNCH(k_local_arap, te128_, 128, mask(MK_ADMM), d_partials_, d_counters_, ds(S_LOCAL), kScalStride);
        return;
    }
    const int net_smem = local_net_bytes(te_local_.per);
    if ((any_mask(MK_L32N) || any_mask(MK_L64N)) && !d_net_img_)
        throw CudaError(WRAPD_E_STATE, "prox_mode 2 needs a network (wrapd_set_prox_net)");
    const Tiles T = te_local_.view();
    const int nb = te_local_.count, bt = te_local_.per;
    if (any_mask(MK_L32N)) {
        k_local<float, true><<<nb, bt, net_smem, st_>>>(view(), T, mask(MK_L32N), mat_, cfg.prox_iters, cand_mode, 2,
                                                         d_net_img_, d_partials_, d_counters_, ds(S_LOCAL), kScalStride);
        kernel_launches++;
    }
    if (any_mask(MK_L32)) {
        k_local<float, false><<<nb, bt, 0, st_>>>(view(), T, mask(MK_L32), mat_, cfg.prox_iters, cand_mode, 1,
                                                   nullptr, d_partials_, d_counters_, ds(S_LOCAL), kScalStride);
        kernel_launches++;
    }
    if (any_mask(MK_L64N)) {
        k_local<double, true><<<nb, bt, net_smem, st_>>>(view(), T, mask(MK_L64N), mat_, cfg.prox_iters, cand_mode, 2,
                                                          d_net_img_, d_partials_, d_counters_, ds(S_LOCAL), kScalStride);
        kernel_launches++;
    }
    if (any_mask(MK_L64)) {
        k_local<double, false><<<nb, bt, local_hist_bytes(bt), st_>>>(view(), T, mask(MK_L64), mat_, cfg.prox_iters,
                                                                  cand_mode,
                                                                  (fp32() || cfg.prox_mode == 2) ? 1 : cfg.prox_mode,
                                                                  nullptr, d_partials_, d_counters_, ds(S_LOCAL),
                                                                  kScalStride);
        kernel_launches++;
    }
    WRAPD_LAUNCH_CHECK();
}

// Which local-step variant each unconverged mesh runs this iteration:
// FP32 arithmetic in mixed mode until its refinement phase; prox_mode 2 runs
// the network where the last stretches are a stale warm start (the mesh's
// first local step and the one after each of its reweights: the weight
// w^2 / vol, an input of the prox, has just changed).
static void set_local_masks(int nm, int* masks, const std::vector<bool>& act, const std::vector<bool>& f32,
                            const std::vector<bool>& net) {
    for (int m = 0; m < nm; ++m) {
        masks[(size_t)MK_L32 * nm + m] = act[m] && f32[m] && !net[m];
        masks[(size_t)MK_L32N * nm + m] = act[m] && f32[m] && net[m];
        masks[(size_t)MK_L64 * nm + m] = act[m] && !f32[m] && !net[m];
        masks[(size_t)MK_L64N * nm + m] = act[m] && !f32[m] && net[m];
    }
}

void SolverGPU::local_step_unaware(int cand_mode, bool fp32_compute) {
    const int nb = blocks_for(ne, 128);
    if (fp32_compute && cfg.model == MODEL_NH)
        k_local_unaware<float><<<nb, 128, 0, st_>>>(view(), d_x_, d_xfix_, mat_, cfg.prox_iters, cand_mode, 1,
                                                    d_partials_, d_counters_, ds(S_LOCAL));
    else
        k_local_unaware<double><<<nb, 128, kLocalHistBytes, st_>>>(view(), d_x_, d_xfix_, mat_, cfg.prox_iters,
                                                                   cand_mode, (fp32() || cfg.prox_mode != 0) ? 1 : 0,
                                                                   d_partials_, d_counters_, ds(S_LOCAL));
    WRAPD_LAUNCH_CHECK();
    kernel_launches++;
}

void SolverGPU::global_step_unaware() {
    k_rhs_unaware<<<blocks_for(ne, 128), 128, 0, st_>>>(view(), d_xfix_);
    WRAPD_LAUNCH_CHECK();
    kernel_launches++;
    gather(GATHER_PLAIN, MK_ALL, false, d_q_);
    mark(1);
    chol.solve(d_q_, st_);
    kernel_launches += chol.launches_solve;
    n_solve++;
    mark(3);
    uv_valid_ = false;
    WRAPD_CUDA(cudaMemcpyAsync(d_x_, d_q_, 3 * (size_t)nf * sizeof(double), cudaMemcpyDeviceToDevice, st_));
    // update_defo_cache(x, true): singular values for the energy and flips
    grad_at_x(false, MK_ALL);
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
    WRAPD_ELEM_LAUNCH(k_mid_candidates, te128_, 128, mask(MK_ALL), d_x_, d_xfix_, mat_, from_x ? 1 : 0, cand_mode);
}

void SolverGPU::apply_weights(int mk) {
    WRAPD_ELEM_LAUNCH(k_apply_weights, te256_, 256, mask(mk));
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

// The device status word carries a factorization's non-positive pivot and a
// solve's dependency wait that gave up; it is read with every scalar block.
static void throw_status(int status) {
    if (status == WRAPD_E_TIMEOUT)
        throw CudaError(status, "a dependency wait of the triangular solve gave up");
    throw CudaError(status, "factorization of D^T W D hit a non-positive pivot");
}

void SolverGPU::sync_read() {
    WRAPD_CUDA(cudaMemcpyAsync(h_scal_, d_scal_, (size_t)nm * kScalStride * sizeof(double), cudaMemcpyDeviceToHost, st_));
    WRAPD_CUDA(cudaMemcpyAsync(h_status_, chol.d_status, sizeof(int), cudaMemcpyDeviceToHost, st_));
    WRAPD_CUDA(cudaStreamSynchronize(st_));
    ctl_pending_ = false;
    n_sync++;
    mark(5);
    if (*h_status_ != 0) {
        const int status = *h_status_;
        *h_status_ = 0;
        WRAPD_CUDA(cudaMemsetAsync(chol.d_status, 0, sizeof(int), st_));
        throw_status(status);
    }
}

void SolverGPU::check_status() {
    int status = 0;
    WRAPD_CUDA(cudaMemcpyAsync(&status, chol.d_status, sizeof(int), cudaMemcpyDeviceToHost, st_));
    WRAPD_CUDA(cudaStreamSynchronize(st_));
    ctl_pending_ = false;
    if (status != 0) {
        WRAPD_CUDA(cudaMemsetAsync(chol.d_status, 0, sizeof(int), st_));
        throw_status(status);
    }
}

// |x - x_soln|^2 per mesh (AlgorithmData::update_per_iter_data,
// src/AlgorithmData.cpp:66-78; x_soln is the rest mesh when no solution mesh
// is given), into the scalar block, read at the next sync.
void SolverGPU::x_error_launch(int mk) {
    k_xerr<<<tvec_.count, 256, 0, st_>>>(tvec_.view(), mask(mk), d_x_, d_xsoln_, d_partials_, d_counters_, ds(S_XERR),
                                         kScalStride);
    WRAPD_LAUNCH_CHECK();
    kernel_launches++;
}

// The local step's tile (elements per CTA, 64, 128 or 256) timed on this
// system's first local step: every candidate runs the step the solve will run
// (its precision and prox), from the same saved state, which is restored
// afterwards; the fastest is kept.  Called once, from the first begin_solve.
void SolverGPU::autotune_local() {
    const size_t e9 = 9 * (size_t)ne * sizeof(double), e3 = 3 * (size_t)ne * sizeof(double);
    double* saved = static_cast<double*>(dalloc(2 * e9 + e3 + (size_t)ne * sizeof(double)));
    char* sv = reinterpret_cast<char*>(saved);
    auto copy_state = [&](bool save) {
        const std::pair<double*, size_t> parts[] = {{d_Z_, e9}, {d_U_, e9}, {d_slast_, e3}, {d_w2c_, (size_t)ne * 8}};
        size_t off = 0;
        for (const auto& p : parts) {
            if (save) WRAPD_CUDA(cudaMemcpyAsync(sv + off, p.first, p.second, cudaMemcpyDeviceToDevice, st_));
            else WRAPD_CUDA(cudaMemcpyAsync(p.first, sv + off, p.second, cudaMemcpyDeviceToDevice, st_));
            off += p.second;
        }
    };
    std::vector<bool> act(nm, true), f32(nm), net(nm, false);
    for (int m = 0; m < nm; ++m) f32[m] = fp32();
    ctl_writable();
    set_local_masks(nm, h_masks_, act, f32, net);
    push_ctl();
    std::vector<std::pair<int, int>> er;
    for (const MeshRun& R : runs_) er.emplace_back(R.e0, R.e1);
    cudaEvent_t e0, e1;
    WRAPD_CUDA(cudaEventCreate(&e0));
    WRAPD_CUDA(cudaEventCreate(&e1));
    copy_state(true);
    float best = 1e30f;
    int pick = local_per_;
    for (int per : {128, 64, 256, 512}) {
        build_tiles(te_local_, per, er);
        for (int rep = 0; rep < 2; ++rep) {   // the first run warms up
            copy_state(false);
            WRAPD_CUDA(cudaEventRecord(e0, st_));
            local_step(CAND_NONE);
            WRAPD_CUDA(cudaEventRecord(e1, st_));
            WRAPD_CUDA(cudaEventSynchronize(e1));
        }
        float ms = 0.f;
        WRAPD_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (ms < best) { best = ms; pick = per; }
    }
    copy_state(false);
    WRAPD_CUDA(cudaStreamSynchronize(st_));
    ctl_pending_ = false;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    local_per_ = pick;
    build_tiles(te_local_, local_per_, er);
    local_tuned_ = true;
}

void SolverGPU::begin_solve() {
    if (!initialized_) throw CudaError(WRAPD_E_STATE, "begin_solve before initialize");
    auto t0 = std::chrono::steady_clock::now();
    logs_ = Logs();
    pend_ = PendingTiming{};
    iter = 0;
    converged_ = false;
    acc_time_s_.assign(1, 0.0);
    for (double& r : runtime_ms) r = 0.0;
    for (int m = 0; m < nm; ++m) {
        MeshRun& R = runs_[m];
        R.logs = Logs();
        R.converged = false;
        R.fp64_phase = false;
        R.m_tol = 1e-15;
        set_mask(MK_ADMM, m, true);
    }
    push_ctl();
    // setup_solve (src/ADMM.cpp:89-107): X = X_init, defo cache, dual variables
    uv_valid_ = false;
    WRAPD_CUDA(cudaMemcpyAsync(d_x_, d_xinit_, 3 * (size_t)nf * sizeof(double), cudaMemcpyDeviceToDevice, st_));
    grad_at_x(false, MK_ALL);
    if (cfg.rot_aware) {
        WRAPD_ELEM_LAUNCH(k_init_dual, te128_, 128, mask(MK_ALL), d_x_, d_xfix_, mat_, d_partials_, d_counters_,
                          ds(S_INIT), kScalStride);
    } else {
        k_init_dual_unaware<<<blocks_for(ne, 128), 128, 0, st_>>>(view(), d_x_, d_xfix_);
        WRAPD_LAUNCH_CHECK();
        kernel_launches++;
    }
    x_error_launch(MK_ALL);
    sync_read();
    for (int m = 0; m < nm; ++m) {
        MeshRun& R = runs_[m];
        R.curr_pe = cfg.rot_aware ? hs(m, S_INIT) : 0.0;
        // log_initial_data (src/AlgorithmData.cpp:50-64)
        R.logs.objectives.push_back(hs(m, S_GRAD + 1));
        R.logs.flips.push_back((int)hs(m, S_GRAD + 2));
        R.logs.reweighted.push_back(1);
        R.logs.acc_time_s.push_back(0.0);
        R.logs.x_errors.push_back(1.0);
        R.init_xerr = std::sqrt(hs(m, S_XERR));
    }
    if (nm > 1) union_logs(0);
    if (cfg.autotune && !local_tuned_ && cfg.rot_aware && cfg.model == MODEL_NH) autotune_local();
    // initialize_weights (src/GlobalStepBehavior.hpp:223-230)
    if (cfg.reweighting) {
        mid_candidates(false, cand_mode_now());
        count_++;
        apply_weights(MK_ALL);
        factor();
        for (MeshRun& R : runs_) R.ctl.k = 0;
        check_status();
    }
    solving_ = true;
    marks_.clear();
    event_next_ = 0;
    runtime_ms[0] += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// Backtracking::search (deps/mcloptlib/include/MCL/Backtracking.hpp:71-98) as
// SplitLBFGS::minimize calls it for -global_ls 1 (single meshes): p = -q, or
// -grad with alpha0 = min(1, 1 / max|grad|) after a non-descent restart;
// Armijo decrease 1e-4, step factor 0.7; a direction of norm <= machine
// epsilon returns 1e-4.  fx0 is the AL value of the last gradient evaluation,
// which was at x.  Each trial value is one gradient-kernel pass (no gradient
// rows) at x + alpha p into the stage vector; the element cache it leaves is
// refreshed by the gradient at the accepted x.  On a non-descent restart the
// history reset of SplitLBFGS.hpp:189-194 is applied here, before the search.
double SolverGPU::line_search() {
    const int n = 3 * nf, vb = vec_blocks(n);
    const MeshCtl& c = runs_[0].ctl;
    double* gcur = d_G_[c.grot % 3];
    double* trial = d_S_[c.stage];
    k_ls_norms<<<vb, 256, 0, st_>>>(n, d_q_, gcur, d_partials_, d_counters_, ds(S_LSN));
    k_ls_gmax<<<vb, 256, 0, st_>>>(n, gcur, d_partials_, d_counters_, ds(S_LSM));
    WRAPD_LAUNCH_CHECK();
    kernel_launches += 2;
    sync_read();
    const double dir = hs(0, S_DIR);
    if (std::isnan(dir)) throw CudaError(WRAPD_E_NAN, "L-BFGS decrement is NaN");
    const bool restart = !(dir > 0.0);
    ls_restart_ = restart;
    const double alpha0 = restart ? std::min(1.0, 1.0 / hs(0, S_LSM)) : 1.0;
    const double pnorm = std::sqrt(restart ? hs(0, S_LSN + 1) : hs(0, S_LSN));
    const double decrease = 1.e-4, tau = 0.7;
    if (pnorm <= std::numeric_limits<double>::epsilon()) return decrease;
    const double fx0 = hs(0, S_GRAD);
    const double gtp = restart ? -hs(0, S_LSN + 1) : -dir;
    const double* step = restart ? gcur : d_q_;
    double alpha = alpha0;
    for (int it = 0; it < 100000; ++it) {
        k_ls_trial<<<vb, 256, 0, st_>>>(n, trial, d_x_, step, alpha);
        WRAPD_LAUNCH_CHECK();
        kernel_launches++;
        WRAPD_ELEM_LAUNCH(k_grad<false>, te256_, 256, mask(MK_ALL), trial, d_xfix_, mat_, 0, d_partials_,
                          d_counters_, ds(S_LSV), kScalStride);   // one mesh (line search: single meshes only)
        sync_read();
        const double fxa = hs(0, S_LSV);
        if (fxa <= fx0 + alpha * decrease * gtp) return alpha;
        alpha *= tau;
    }
    return -1.0;
}

// One loop of the two-loop recursion of a single mesh as one cooperative
// launch (k_two_loop_grid); its barrier counter starts from 0.
void SolverGPU::two_loop_grid(bool second, const VecPools& P, const TwoLoopSlots& sl) {
    WRAPD_CUDA(cudaMemsetAsync(d_bar_, 0, sizeof(unsigned), st_));
    Tiles T = tvec_.view();
    VecPools Pc = P;
    TwoLoopSlots slc = sl;
    const MeshCtl* ctl = d_ctl_;
    const double* rho = d_rho_;
    double* q = d_q_;
    double* partials = d_partials_;
    unsigned* bar = d_bar_;
    int* status = chol.d_status;
    double* scal = d_scal_;
    void* args[] = {&T, &ctl, &Pc, &rho, &q, &slc, &partials, &bar, &status, &scal};
    const void* fn = coop_reg_ ? (second ? reinterpret_cast<const void*>(&k_two_loop_grid<true, true>)
                                         : reinterpret_cast<const void*>(&k_two_loop_grid<false, true>))
                               : (second ? reinterpret_cast<const void*>(&k_two_loop_grid<true, false>)
                                         : reinterpret_cast<const void*>(&k_two_loop_grid<false, false>));
    WRAPD_CUDA(cudaLaunchCooperativeKernel(fn, dim3(coop_grid_), dim3(kTwoLoopGridThreads), args, 0, st_));
    kernel_launches++;
}

// SplitLBFGS::minimize (deps/mcloptlib/include/MCL/SplitLBFGS.hpp:114-256) with
// LSMethod::None (rate 1), for every mesh R with R.in_loop set: each mesh runs
// its own minimize (its history, decrement, early exit and iteration budget),
// all of them in the same launches; a mesh that exits is masked out of the
// rest.  On entry each such mesh's gradient at x is in its cur buffer and the
// |grad - grad_old|^2 early-return test has passed.  Sets R.its (the
// minimize's return value) and R.obj_aft.
int SolverGPU::lbfgs_minimize() {
    const int M = cfg.lbfgs_m;
    const TwoLoopSlots sl{S_ALPHA, S_C, S_DIR};
    for (MeshRun& R : runs_)
        if (R.in_loop) R.max_iters = cfg.global_iters;
    for (int gi = 1;; ++gi) {
        // the meshes still in their loop (SplitLBFGS.hpp:145: global_iter <= max_iters)
        bool any = false;
        int jmax = 0;
        for (int m = 0; m < nm; ++m) {
            MeshRun& R = runs_[m];
            if (R.in_loop && gi > R.max_iters) {
                R.its = gi - 1;
                R.in_loop = false;
            }
            set_mask(MK_LBFGS, m, R.in_loop);
            set_mask(MK_SMALL, m, R.in_loop && R.ctl.small);
            set_mask(MK_LARGE, m, R.in_loop && !R.ctl.small);
            if (!R.in_loop) continue;
            any = true;
            R.ctl.it = std::min(M, R.ctl.k);
            R.ctl.stage = (R.ctl.head + std::min(R.ctl.k, M)) % (M + 1);
            if (!R.ctl.small) jmax = std::max(jmax, R.ctl.it);
        }
        if (!any) break;
        push_ctl();
        const bool small = any_mask(MK_SMALL), large = any_mask(MK_LARGE);
        const VecPools P = pools();
        // first loop (newest to oldest): alpha_i = rho_i <s_i, q>, q -= alpha_i y_i
        if (small) {
            k_two_loop_first<<<nm, kTwoLoopThreads, 0, st_>>>(mask(MK_SMALL), d_ctl_, P, d_rho_, d_q_, sl, d_scal_,
                                                              kScalStride);
            kernel_launches++;
        }
        if (large && coop_grid_ > 0) {
            two_loop_grid(false, P, sl);
        } else if (large) {
            for (int j = jmax - 1; j >= -1; --j) {
                k_lbfgs_first<<<tvec_.count, 256, 0, st_>>>(tvec_.view(), mask(MK_LARGE), d_ctl_, P, d_rho_, d_q_, j, sl,
                                                            d_partials_, d_counters_, d_scal_, kScalStride);
                kernel_launches++;
            }
        }
        WRAPD_LAUNCH_CHECK();
        // q = A^-1 q, three right-hand sides at once (the block-diagonal system)
        mark(2);
        chol.solve(d_q_, st_, nm > 1 ? mask(MK_LBFGS) : nullptr);   // the meshes out of their loop skip it
        kernel_launches += chol.launches_solve;
        n_solve++;
        mark(3);
        // second loop (oldest to newest): c_i = alpha_i - rho_i <y_i, q>, q += c_i s_i; then dir = <grad, q>
        if (small) {
            k_two_loop_second<<<nm, kTwoLoopThreads, 0, st_>>>(mask(MK_SMALL), d_ctl_, P, d_rho_, d_q_, sl, d_scal_,
                                                               kScalStride);
            kernel_launches++;
        }
        if (large && coop_grid_ > 0) {
            two_loop_grid(true, P, sl);
        } else if (large) {
            for (int j = 0; j <= jmax; ++j) {
                k_lbfgs_second<<<tvec_.count, 256, 0, st_>>>(tvec_.view(), mask(MK_LARGE), d_ctl_, P, d_rho_, d_q_, j,
                                                             sl, d_partials_, d_counters_, d_scal_, kScalStride);
                kernel_launches++;
            }
        }
        WRAPD_LAUNCH_CHECK();
        // -global_ls 1 (single meshes): Backtracking::search along p = -q (SplitLBFGS.hpp:196-206)
        double rate = 1.0;
        if (cfg.global_ls && runs_[0].m_tol > 1.e-12) {
            rate = line_search();
            if (rate <= 0.0) {   // SplitMinimizer::FAILURE, after the restart's history reset
                if (ls_restart_) runs_[0].ctl.k = 0;
                runs_[0].in_loop = false;
                runs_[0].its = -1;
                return -1;
            }
        }
        // x -= rate q (or rate grad on a non-descent direction); s = x_new - x_old
        uv_valid_ = false;   // x moves
        k_xupdate<<<tvec_.count, 256, 0, st_>>>(tvec_.view(), mask(MK_LBFGS), d_ctl_, P, d_x_, d_q_, d_scal_, S_DIR,
                                                kScalStride, rate);
        WRAPD_LAUNCH_CHECK();
        kernel_launches++;
        mark(2);
        // gradient at the new x; y = grad_new - grad
        grad_at_x(true, MK_LBFGS);
        gather(GATHER_LBFGS, MK_LBFGS, true);
        mark(1);
        sync_read();
        for (int m = 0; m < nm; ++m) {
            MeshRun& R = runs_[m];
            if (!R.in_loop) continue;
            MeshCtl& c = R.ctl;
            const double dir = hs(m, S_DIR);
            const double yy = hs(m, S_GATHER), sy = hs(m, S_GATHER + 1);
            if (std::isnan(dir)) throw CudaError(WRAPD_E_NAN, "L-BFGS decrement is NaN");
            const int stage = c.stage;   // where this iteration's s and y were written
            if (dir <= 0.0) {
                R.max_iters -= c.k;
                c.k = 0;
                c.head = stage;          // the new entry becomes the oldest
            } else if (c.k >= M) {
                c.head = (c.head + 1) % (M + 1);   // erase(begin) + push_back
            }
            R.rho[stage] = 1.0 / sy;
            c.grot += 1;                 // grad_old <- grad, grad <- grad_new
            if (dir > 0.0 && (dir < cfg.kappa * R.m_tol || dir < cfg.kappa * 1.e-12)) {
                c.k += 1;
                R.its = gi;
                R.in_loop = false;
            } else if (std::fabs(yy) <= 0.0) {
                R.its = gi;
                R.in_loop = false;
            } else {
                c.k++;
            }
        }
    }
    for (MeshRun& R : runs_) R.ctl.k = std::min(M, R.ctl.k);
    return 0;
}

// A batch's summary log entry k (after iteration k - 1): sums over the
// meshes of each one's latest entry (a converged mesh keeps its last values).
void SolverGPU::union_logs(int k) {
    double obj = 0.0, ls = 0.0, gs = 0.0, xe2 = 0.0, xi2 = 0.0, prox = 0.0;
    int flips = 0, rw = 0, inner = 0;
    for (const MeshRun& R : runs_) {
        const Logs& L = R.logs;
        obj += L.objectives.back();
        flips += L.flips.back();
        const double xe = L.x_errors.back() * R.init_xerr;
        xe2 += xe * xe;
        xi2 += R.init_xerr * R.init_xerr;
        if (k > 0 && (int)L.objectives.size() == k + 1) {
            rw |= L.reweighted.back();
            inner += L.inner.back();
            ls += L.ls_dal.back();
            gs += L.gs_dal.back();
            prox += L.prox_iters.back() * (R.e1 - R.e0);
        }
    }
    logs_.objectives.push_back(obj);
    logs_.flips.push_back(flips);
    logs_.x_errors.push_back(xi2 > 0.0 ? std::sqrt(xe2 / xi2) : 0.0);
    logs_.acc_time_s.push_back(0.0);
    logs_.reweighted.push_back(k == 0 ? 1 : rw);
    if (k > 0) {
        logs_.inner.push_back(inner);
        logs_.ls_dal.push_back(ls);
        logs_.gs_dal.push_back(gs);
        logs_.prox_iters.push_back(prox / double(ne));
    }
}

int SolverGPU::iterate(int n, bool* conv) {
    if (!solving_) throw CudaError(WRAPD_E_STATE, "iterate before begin_solve");
    int done = 0;
    *conv = converged_;
    std::vector<bool> act(nm), f32(nm), net(nm);
    std::vector<double> dal(nm, 0.0), prox_it(nm, 0.0);
    std::vector<int> its(nm, 0);
    std::vector<char> rw(nm, 0);
    while (done < n && iter < cfg.max_iters && !converged_) {
        cudaEvent_t* ev_ = evs_[iter & 1];
        const int k = iter;
        // masks of this iteration: the meshes still iterating and their local-step variant
        for (int m = 0; m < nm; ++m) {
            const MeshRun& R = runs_[m];
            act[m] = !R.converged;
            f32[m] = fp32() && !R.fp64_phase;
            net[m] = cfg.prox_mode == 2 && R.logs.reweighted.back() != 0;
            set_mask(MK_ADMM, m, act[m]);
            set_mask(MK_ZERO, m, act[m] && R.ctl.k == 0);
            set_mask(MK_RW, m, false);
        }
        ctl_writable();
        set_local_masks(nm, h_masks_, act, f32, net);
        push_ctl();
        WRAPD_CUDA(cudaEventRecord(ev_[0], st_));
        mark(5);
        // The candidate weights (w2c) are read only by a reweight: the ratio of
        // the gamma rule every iteration, or with rw_every the reweight every
        // rw_every-th iteration.  On the other iterations of rw_every the local
        // step leaves them alone (the reweight's own local step writes them
        // fresh), which skips the Hessian eigenvalue per element; the results
        // are the same.
        int cand = cand_mode_now();
        if (cfg.rw_every > 0 && ((k + 1) % cfg.rw_every) != 0) cand = CAND_NONE;
        if (cfg.rot_aware) {
            // ---- local step: polar_update (src/TetElements.cpp:256-356) ----
            local_step(cand);
            if (cfg.reweighting) count_++;
            mark(0);
            WRAPD_CUDA(cudaEventRecord(ev_[1], st_));
            // ---- global step: RotAwareGS::global_step (src/GlobalStepBehavior.hpp:246-258) ----
            if (any_mask(MK_ZERO)) {
                k_zero_old<<<tvec_.count, 256, 0, st_>>>(tvec_.view(), mask(MK_ZERO), d_ctl_, pools());
                WRAPD_LAUNCH_CHECK();
                kernel_launches++;
            }
            grad_at_x(true, MK_ADMM);
            gather(GATHER_START, MK_ADMM, true);
            mark(1);
            sync_read();
            settle_timing(false);   // the previous iteration's events are behind this synchronisation
            for (int m = 0; m < nm; ++m) {
                MeshRun& R = runs_[m];
                R.in_loop = false;
                if (!act[m]) continue;
                const double bef = hs(m, S_LOCAL), aft = hs(m, S_LOCAL + 1), pe = hs(m, S_LOCAL + 2);
                prox_it[m] = hs(m, S_LOCAL + 4);
                if (hs(m, S_LOCAL + 3) > 0.0) throw CudaError(WRAPD_E_PROX_NEG, "negative singular value in a prox solution");
                dal[m] = aft - bef + pe - R.curr_pe;
                R.curr_pe = pe;
                R.obj_bef = hs(m, S_GRAD);
                R.m_tol = std::fabs(dal[m]);
                R.its = 0;
                R.in_loop = !(hs(m, S_GATHER) < 1.e-13);
            }
            if (lbfgs_minimize() < 0) {
                // a failed global line search ends the minimize with -1 (single mesh)
            }
            for (int m = 0; m < nm; ++m) its[m] = act[m] ? runs_[m].its : 0;
        } else {
            // ---- local_update: TetElements::update (src/TetElements.cpp:193-254), single mesh ----
            local_step_unaware(cand, fp32() && !runs_[0].fp64_phase);
            if (cfg.reweighting) count_++;
            mark(0);
            WRAPD_CUDA(cudaEventRecord(ev_[1], st_));
            // ---- UnawareGS::global_step (src/GlobalStepBehavior.hpp:162-180): x = A^-1 b ----
            global_step_unaware();
            x_error_launch(MK_ALL);
            sync_read();
            prox_it[0] = hs(0, S_LOCAL + 4);
            if (hs(0, S_LOCAL + 3) > 0.0) throw CudaError(WRAPD_E_PROX_NEG, "negative singular value in a prox solution");
            dal[0] = 0.0;
            its[0] = 1;
        }
        WRAPD_CUDA(cudaEventRecord(ev_[2], st_));
        // ---- reweighting: possibly_update_weights (src/System.cpp:50-63), per mesh ----
        bool any_rw = false;
        for (int m = 0; m < nm; ++m) rw[m] = 0;
        if (cfg.reweighting) {
            if (cfg.rw_every > 0) {
                for (int m = 0; m < nm; ++m) rw[m] = act[m] && ((k + 1) % cfg.rw_every) == 0;
            } else {
                WRAPD_ELEM_LAUNCH(k_ratio, te256_, 256, mask(MK_ADMM), d_partials_, d_counters_, ds(S_RATIO),
                                  kScalStride);
                sync_read();
                for (int m = 0; m < nm; ++m) rw[m] = act[m] && hs(m, S_RATIO) > cfg.gamma;
            }
            for (int m = 0; m < nm; ++m) {
                set_mask(MK_RW, m, rw[m] != 0);
                any_rw = any_rw || rw[m];
            }
            if (any_rw) {
                push_ctl();
                apply_weights(MK_RW);
                factor();
                for (int m = 0; m < nm; ++m)
                    if (rw[m]) runs_[m].ctl.k = 0;
            }
        }
        WRAPD_CUDA(cudaEventRecord(ev_[3], st_));
        if (profiling) {
            sync_read();
            profile_flush();
        }
        if (any_rw) check_status();
        // ---- AlgorithmData::update_per_iter_* (src/AlgorithmData.cpp:66-83), per mesh ----
        acc_time_s_.push_back(0.0);
        int its_sum = 0;
        for (int m = 0; m < nm; ++m) {
            if (!act[m]) continue;
            MeshRun& R = runs_[m];
            Logs& L = R.logs;
            // the energy, flips and x error of the final x: the mesh's last gradient
            // evaluation and gather (or the rotation-unaware step's) computed them,
            // outside the timed phases, as the reference logs them
            const double obj_aft = cfg.rot_aware ? hs(m, S_GRAD) : 1.e8;   // UnawareGS (GlobalStepBehavior.hpp:102)
            const double pe_x = hs(m, S_GRAD + 1);
            const int flips = (int)hs(m, S_GRAD + 2);
            const double xerr2 = cfg.rot_aware ? hs(m, S_GATHER + 2) : hs(m, S_XERR);
            L.reweighted.push_back(rw[m] ? 1 : 0);
            L.ls_dal.push_back(std::fabs(dal[m]));
            L.gs_dal.push_back(cfg.rot_aware ? std::fabs(obj_aft - R.obj_bef) : std::fabs(obj_aft));
            L.inner.push_back(its[m]);
            L.prox_iters.push_back(prox_it[m] / double(R.e1 - R.e0));
            L.objectives.push_back(pe_x);
            L.flips.push_back(flips);
            L.acc_time_s.push_back(0.0);
            L.x_errors.push_back(std::sqrt(xerr2) / R.init_xerr);
            its_sum += its[m];
            // ---- ADMM::converged (src/ADMM.cpp:158-169) ----
            const double res = std::fabs(L.objectives[k + 1] - L.objectives[k]) / (std::fabs(L.objectives[k + 1]) + 1.0);
            // Mixed mode refinement: once the energy moves less than FP32 can
            // resolve, finish with FP64 local steps.
            if (fp32() && !R.fp64_phase && res < kMixedSwitch) R.fp64_phase = true;
            if ((L.flips[k + 1] == 0 && L.flips[k] == 0 && res < cfg.tol) || (have_soln_ && L.x_errors.back() < 1.e-4))
                R.converged = true;
        }
        runtime_ms[5] += its_sum;
        if (nm > 1) union_logs(k + 1);
        // phase times: read once a later synchronisation has passed the events
        pend_ = PendingTiming{true, k, ev_};
        if (profiling || any_rw) settle_timing(false);          // a synchronisation passed ev_[3]
        else if (!cfg.rot_aware) settle_timing(true);          // its last one came before ev_[2]
        iter = k + 1;
        done++;
        converged_ = true;
        for (const MeshRun& R : runs_) converged_ = converged_ && R.converged;
    }
    settle_timing(true);
    *conv = converged_;
    return done;
}

// Adds a finished iteration's phase times (CUDA events) to the runtime and its
// accumulated-time log entries.  wait = false: a host synchronisation of the
// stream has already passed the events.
void SolverGPU::settle_timing(bool wait) {
    if (!pend_.on) return;
    if (wait) WRAPD_CUDA(cudaEventSynchronize(pend_.ev[3]));
    float ml = 0.f, mg = 0.f, mr = 0.f;
    WRAPD_CUDA(cudaEventElapsedTime(&ml, pend_.ev[0], pend_.ev[1]));
    WRAPD_CUDA(cudaEventElapsedTime(&mg, pend_.ev[1], pend_.ev[2]));
    WRAPD_CUDA(cudaEventElapsedTime(&mr, pend_.ev[2], pend_.ev[3]));
    runtime_ms[1] += ml; runtime_ms[2] += mg; runtime_ms[3] += mr;
    const double t = (runtime_ms[1] + runtime_ms[2] + runtime_ms[3]) / 1000.0;
    const size_t j = (size_t)pend_.k + 1;
    acc_time_s_[j] = t;
    for (MeshRun& R : runs_)
        if (R.logs.acc_time_s.size() > j) R.logs.acc_time_s[j] = t;
    if (logs_.acc_time_s.size() > j) logs_.acc_time_s[j] = t;
    pend_.on = false;
}

void SolverGPU::positions(double* out) {
    std::vector<double> xp(3 * (size_t)nf);
    WRAPD_CUDA(cudaMemcpyAsync(xp.data(), d_x_, xp.size() * sizeof(double), cudaMemcpyDeviceToHost, st_));
    WRAPD_CUDA(cudaStreamSynchronize(st_));
    ctl_pending_ = false;
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
// Element-level steps over every mesh; the returned sums are over the batch.
void SolverGPU::download_elem(const double* d, int comps, std::vector<double>& out) {
    const size_t n = (size_t)comps * ne;
    std::vector<double> soa(n);
    WRAPD_CUDA(cudaMemcpyAsync(soa.data(), d, n * 8, cudaMemcpyDeviceToHost, st_));
    WRAPD_CUDA(cudaStreamSynchronize(st_));
    ctl_pending_ = false;
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
    ctl_pending_ = false;
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
        if (name == "xfree") {
            WRAPD_CUDA(cudaMemcpyAsync(xp.data(), d_x_, xp.size() * 8, cudaMemcpyDeviceToHost, st_));
        } else {
            // each mesh's range from its own cur buffer
            for (const MeshRun& R : runs_)
                WRAPD_CUDA(cudaMemcpyAsync(xp.data() + 3 * (size_t)R.f0, d_G_[R.ctl.grot % 3] + 3 * (size_t)R.f0,
                                           3 * (size_t)(R.f1 - R.f0) * 8, cudaMemcpyDeviceToHost, st_));
        }
        WRAPD_CUDA(cudaStreamSynchronize(st_));
        ctl_pending_ = false;
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
        uv_valid_ = false;
        WRAPD_CUDA(cudaMemcpyAsync(d_x_, xp.data(), xp.size() * 8, cudaMemcpyHostToDevice, st_));
        WRAPD_CUDA(cudaStreamSynchronize(st_));
        ctl_pending_ = false;
    } else {
        throw CudaError(WRAPD_E_INPUT, "state " + name + " is read-only");
    }
}

void SolverGPU::update_defo_cache() {
    grad_at_x(false, MK_ALL);
    sync_read();
}

double SolverGPU::polar_update(bool update_candidates) {
    std::vector<bool> act(nm, true), f32(nm), net(nm, false);
    for (int m = 0; m < nm; ++m) {
        f32[m] = fp32() && !runs_[m].fp64_phase;
        set_mask(MK_ADMM, m, true);
    }
    ctl_writable();
    set_local_masks(nm, h_masks_, act, f32, net);
    push_ctl();
    local_step(update_candidates ? cand_mode_now() : CAND_NONE);
    if (update_candidates && cfg.reweighting) count_++;
    sync_read();
    double dal = 0.0;
    for (int m = 0; m < nm; ++m) {
        if (hs(m, S_LOCAL + 3) > 0.0) throw CudaError(WRAPD_E_PROX_NEG, "negative singular value in a prox solution");
        dal += hs(m, S_LOCAL + 1) - hs(m, S_LOCAL) + hs(m, S_LOCAL + 2) - runs_[m].curr_pe;
        runs_[m].curr_pe = hs(m, S_LOCAL + 2);
    }
    return dal;
}

double SolverGPU::global_grad(const double* xfree, double* grad) {
    if (xfree) set_state("xfree", xfree, 3LL * nf);
    grad_at_x(true, MK_ALL);
    gather(GATHER_START, MK_ALL, false);
    sync_read();
    if (grad) {
        std::vector<double> g;
        get_state("grad", g);
        std::memcpy(grad, g.data(), g.size() * sizeof(double));
    }
    double v = 0.0;
    for (int m = 0; m < nm; ++m) v += hs(m, S_GRAD);
    return v;
}

void SolverGPU::potential_energy(double* pe, int* flips) {
    grad_at_x(false, MK_ALL);
    sync_read();
    double p = 0.0;
    int f = 0;
    for (int m = 0; m < nm; ++m) {
        p += hs(m, S_GRAD + 1);
        f += (int)hs(m, S_GRAD + 2);
    }
    if (pe) *pe = p;
    if (flips) *flips = f;
}

void SolverGPU::solve_A(const double* b, double* x, int hold) {
    if (!initialized_) throw CudaError(WRAPD_E_STATE, "solve_A before initialize");
    std::vector<double> xp(3 * (size_t)nf);
    for (int i = 0; i < nf; ++i)
        for (int c = 0; c < 3; ++c) xp[3 * (size_t)iperm_[i] + c] = b[3 * (size_t)i + c];
    WRAPD_CUDA(cudaMemcpyAsync(d_q_, xp.data(), xp.size() * 8, cudaMemcpyHostToDevice, st_));
    if (hold < 0)
        chol.solve(d_q_, st_);
    else
        chol.solve_holding(d_q_, hold, st_);
    kernel_launches += chol.launches_solve;
    WRAPD_CUDA(cudaMemcpyAsync(xp.data(), d_q_, xp.size() * 8, cudaMemcpyDeviceToHost, st_));
    check_status();
    for (int i = 0; i < nf; ++i)
        for (int c = 0; c < 3; ++c) x[3 * (size_t)i + c] = xp[3 * (size_t)iperm_[i] + c];
}

}  // namespace wrapd
