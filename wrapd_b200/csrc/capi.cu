// extern "C" entry points declared in include/wrapd_gpu.h.  Every entry
// catches C++ exceptions and returns a WRAPD_E_* code.
#include <algorithm>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "solver.cuh"

struct wrapd_handle {
    wrapd::SolverGPU* s = nullptr;
    std::string err;
};

struct wrapd_plan {
    wrapd::Symbolic S;
};

namespace {

thread_local std::string g_create_error;

template <typename F>
int guarded(wrapd_handle* h, F&& f) {
    if (!h || !h->s) return WRAPD_E_INPUT;
    try {
        f(*h->s);
        h->err.clear();
        return WRAPD_OK;
    } catch (const wrapd::CudaError& e) {
        h->err = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        h->err = "host allocation failed";
        return WRAPD_E_OOM;
    } catch (const std::exception& e) {
        h->err = e.what();
        return WRAPD_E_INPUT;
    }
}

}  // namespace

extern "C" {

int wrapd_settings_default(wrapd_settings* s) {
    if (!s) return WRAPD_E_INPUT;
    std::memset(s, 0, sizeof *s);
    s->max_iters = 5000;
    s->tol = 1.e-11;
    s->rot_aware = 1;
    s->reweighting = 1;
    s->rw_delay = 50;
    s->gamma = 1.5;
    s->global_iters = 100;
    s->global_ls = 0;
    s->kappa = 1.0;
    s->model = 0;
    s->poisson = 0.45;
    s->beta_static = 1.0;
    s->beta_min = 0.1;
    s->beta_max = 10.0;
    s->prox_iters = 20;
    s->youngs = 1.0e7;
    s->lbfgs_m = 6;
    s->rw_every = 0;
    s->precision = 0;
    s->prox_mode = 0;
    s->leaf_size = 64;
    s->verbose = 0;
    s->device = 0;
    s->autotune = 0;
    return WRAPD_OK;
}

int wrapd_create(const wrapd_settings* s, wrapd_handle** out) {
    if (!s || !out) return WRAPD_E_INPUT;
    *out = nullptr;
    try {
        auto* h = new wrapd_handle();
        try {
            h->s = new wrapd::SolverGPU(*s);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
        g_create_error.clear();
        return WRAPD_OK;
    } catch (const wrapd::CudaError& e) {
        g_create_error = e.what();
        return e.code;
    } catch (const std::exception& e) {
        g_create_error = e.what();
        return WRAPD_E_INPUT;
    }
}

int wrapd_add_tetmesh(wrapd_handle* h, const double* rest_xyz, const double* init_xyz, const double* soln_xyz,
                      int n_verts, const int32_t* tets, int n_tets, const int32_t* pins, int n_pins) {
    return guarded(h, [&](wrapd::SolverGPU& s) {
        s.add_mesh(rest_xyz, init_xyz, soln_xyz, n_verts, tets, n_tets, pins, n_pins);
    });
}

int wrapd_add_tetmesh_material(wrapd_handle* h, const double* rest_xyz, const double* init_xyz,
                               const double* soln_xyz, int n_verts, const int32_t* tets, int n_tets,
                               const int32_t* pins, int n_pins, double youngs, double poisson) {
    if (!(youngs > 0.0) || !(poisson > 0.0)) return WRAPD_E_INPUT;
    return guarded(h, [&](wrapd::SolverGPU& s) {
        s.add_mesh(rest_xyz, init_xyz, soln_xyz, n_verts, tets, n_tets, pins, n_pins, youngs, poisson);
    });
}

int wrapd_initialize(wrapd_handle* h) {
    return guarded(h, [&](wrapd::SolverGPU& s) { s.initialize(); });
}

int wrapd_solve(wrapd_handle* h, double* x_out) {
    return guarded(h, [&](wrapd::SolverGPU& s) { s.solve(x_out); });
}

int wrapd_begin_solve(wrapd_handle* h) {
    return guarded(h, [&](wrapd::SolverGPU& s) { s.begin_solve(); });
}

int wrapd_iterate(wrapd_handle* h, int n, int* iters_done, int* converged) {
    return guarded(h, [&](wrapd::SolverGPU& s) {
        bool c = false;
        const int d = s.iterate(n, &c);
        if (iters_done) *iters_done = d;
        if (converged) *converged = c ? 1 : 0;
    });
}

int wrapd_get_positions(wrapd_handle* h, double* x_out) {
    if (!x_out) return WRAPD_E_INPUT;
    return guarded(h, [&](wrapd::SolverGPU& s) { s.positions(x_out); });
}

int wrapd_set_prox_net(wrapd_handle* h, const float* blob, int n_blob) {
    if (!blob || n_blob != WRAPD_NET_BLOB) return WRAPD_E_INPUT;
    return guarded(h, [&](wrapd::SolverGPU& s) { s.set_prox_net(blob); });
}

namespace {
int copy_log(const wrapd::Logs& L, int which, double* out, int cap, int* len) {
        std::vector<double> v;
        switch (which) {
            case WRAPD_LOG_OBJECTIVES: v = L.objectives; break;
            case WRAPD_LOG_REWEIGHTED: v.assign(L.reweighted.begin(), L.reweighted.end()); break;
            case WRAPD_LOG_FLIPS: v.assign(L.flips.begin(), L.flips.end()); break;
            case WRAPD_LOG_INNER_ITERS: v.assign(L.inner.begin(), L.inner.end()); break;
            case WRAPD_LOG_LS_DELTA_AL: v = L.ls_dal; break;
            case WRAPD_LOG_GS_DELTA_AL: v = L.gs_dal; break;
            case WRAPD_LOG_ACCUMULATED_TIME_S: v = L.acc_time_s; break;
            case WRAPD_LOG_X_ERRORS: v = L.x_errors; break;
            case WRAPD_LOG_PROX_ITERS: v = L.prox_iters; break;
            default: throw wrapd::CudaError(WRAPD_E_INPUT, "unknown log channel");
        }
        if (len) *len = static_cast<int>(v.size());
        if (out)
            for (int i = 0; i < cap && i < (int)v.size(); ++i) out[i] = v[i];
        return 0;
}
}  // namespace

int wrapd_get_log(wrapd_handle* h, int which, double* out, int cap, int* len) {
    return guarded(h, [&](wrapd::SolverGPU& s) { copy_log(s.logs(), which, out, cap, len); });
}

int wrapd_get_mesh_log(wrapd_handle* h, int mesh, int which, double* out, int cap, int* len) {
    return guarded(h, [&](wrapd::SolverGPU& s) {
        if (!s.initialized()) throw wrapd::CudaError(WRAPD_E_STATE, "mesh logs before initialize");
        copy_log(s.mesh_logs(mesh), which, out, cap, len);
    });
}

int wrapd_get_runtime(wrapd_handle* h, double ms[6]) {
    if (!ms) return WRAPD_E_INPUT;
    return guarded(h, [&](wrapd::SolverGPU& s) { std::memcpy(ms, s.runtime_ms, 6 * sizeof(double)); });
}

int wrapd_get_info(wrapd_handle* h, double out[8]) {
    if (!out) return WRAPD_E_INPUT;
    return guarded(h, [&](wrapd::SolverGPU& s) {
        out[0] = s.nv; out[1] = s.ne; out[2] = s.nf; out[3] = s.np;
        out[4] = s.chol.nfronts; out[5] = s.chol.nlevels;
        out[6] = (double)s.chol.nnz_L; out[7] = s.chol.flops;
    });
}

int wrapd_get_counters(wrapd_handle* h, int64_t out[4]) {
    if (!out) return WRAPD_E_INPUT;
    return guarded(h, [&](wrapd::SolverGPU& s) {
        out[0] = s.kernel_launches; out[1] = s.n_factor; out[2] = s.n_solve; out[3] = s.n_sync;
    });
}

int wrapd_set_profiling(wrapd_handle* h, int on) {
    return guarded(h, [&](wrapd::SolverGPU& s) { s.profiling = on != 0; });
}

int wrapd_get_tuning(wrapd_handle* h, int* out, int cap, int* len) {
    if (!len || (cap > 0 && !out)) return WRAPD_E_INPUT;
    return guarded(h, [&](wrapd::SolverGPU& s) {
        std::vector<int> t = s.chol.tuning();
        t.push_back(s.local_tile());
        *len = (int)t.size();
        for (int i = 0; i < (int)t.size() && i < cap; ++i) out[i] = t[i];
    });
}

int wrapd_get_profile(wrapd_handle* h, double ms[6], int64_t counts[6]) {
    if (!ms || !counts) return WRAPD_E_INPUT;
    return guarded(h, [&](wrapd::SolverGPU& s) {
        for (int i = 0; i < 6; ++i) { ms[i] = s.profile_ms[i]; counts[i] = s.profile_n[i]; }
    });
}

int wrapd_plan_create(const double* rest_xyz, int n_verts, const int32_t* tets, int n_tets, const int32_t* pins,
                      int n_pins, int leaf_size, wrapd_plan** out) {
    if (!out) return WRAPD_E_INPUT;
    *out = nullptr;
    try {
        // the argument checks of wrapd_add_tetmesh (SolverGPU::add_mesh)
        if (!rest_xyz || !tets || n_verts <= 0 || n_tets <= 0 || n_pins < 0 || n_pins >= n_verts ||
            (n_pins > 0 && !pins))
            throw wrapd::CudaError(WRAPD_E_INPUT, "bad mesh arguments");
        for (int64_t i = 0; i < 4 * (int64_t)n_tets; ++i)
            if (tets[i] < 0 || tets[i] >= n_verts) throw wrapd::CudaError(WRAPD_E_INPUT, "tet vertex id out of range");
        std::vector<int> p(pins, pins + n_pins);
        std::sort(p.begin(), p.end());
        for (int j = 0; j < n_pins; ++j)
            if (p[j] < 0 || p[j] >= n_verts || (j > 0 && p[j] == p[j - 1]))
                throw wrapd::CudaError(WRAPD_E_INPUT, "pin ids must be distinct vertex ids");
        // free numbering: ascending vertex id, pinned vertices skipped
        std::vector<int> free_of_vert(n_verts, -1);
        for (int i = 0, j = 0, k = 0; i < n_verts; ++i) {
            if (j < n_pins && i == p[j]) ++j;
            else free_of_vert[i] = k++;
        }
        const int nf = n_verts - n_pins;
        std::vector<int> vinc_ptr, vinc, ptr, adj;
        wrapd::free_vertex_graph(nf, n_tets, tets, free_of_vert.data(), vinc_ptr, vinc, ptr, adj);
        std::vector<double> coords(3 * (size_t)nf);
        for (int i = 0; i < n_verts; ++i)
            if (free_of_vert[i] >= 0)
                for (int c = 0; c < 3; ++c) coords[3 * (size_t)free_of_vert[i] + c] = rest_xyz[3 * (size_t)i + c];
        auto* pl = new wrapd_plan();
        try {
            pl->S = wrapd::analyse(nf, ptr, adj, coords, leaf_size > 0 ? leaf_size : 64);
        } catch (...) {
            delete pl;
            throw;
        }
        *out = pl;
        g_create_error.clear();
        return WRAPD_OK;
    } catch (const wrapd::CudaError& e) {
        g_create_error = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        g_create_error = "host allocation failed";
        return WRAPD_E_OOM;
    } catch (const std::exception& e) {
        g_create_error = e.what();
        return WRAPD_E_INPUT;
    }
}

int wrapd_plan_info(const wrapd_plan* p, int64_t out[8]) {
    if (!p || !out) return WRAPD_E_INPUT;
    const wrapd::Symbolic& S = p->S;
    out[0] = S.n;
    out[1] = (int64_t)S.fronts.size();
    out[2] = (int64_t)S.levels.size();
    out[3] = S.nnz_L;
    out[4] = S.f_pool * (int64_t)sizeof(double);
    out[5] = S.y_pool * (int64_t)sizeof(double);
    out[6] = (int64_t)S.relmap.size();
    out[7] = (int64_t)(S.flops + 0.5);
    return WRAPD_OK;
}

int wrapd_plan_fronts(const wrapd_plan* p, int32_t* perm, int32_t* first, int32_t* ncols, int32_t* parent,
                      int32_t* level, int64_t* row_ptr, int32_t* rows, int32_t* relmap) {
    if (!p) return WRAPD_E_INPUT;
    const wrapd::Symbolic& S = p->S;
    if (perm)
        for (int i = 0; i < S.n; ++i) perm[i] = S.perm[i];
    int64_t at = 0;
    for (size_t f = 0; f < S.fronts.size(); ++f) {
        const wrapd::Front& F = S.fronts[f];
        if (first) first[f] = F.first;
        if (ncols) ncols[f] = F.ncols;
        if (parent) parent[f] = F.parent;
        if (level) level[f] = F.level;
        if (row_ptr) row_ptr[f] = at;
        for (int t = 0; t < F.nrows(); ++t) {
            if (rows) rows[at + t] = F.rows[t];
            if (relmap) relmap[at + t] = S.relmap[F.rel_off + t];
        }
        at += F.nrows();
    }
    if (row_ptr) row_ptr[S.fronts.size()] = at;
    return WRAPD_OK;
}

void wrapd_plan_destroy(wrapd_plan* p) { delete p; }

const char* wrapd_last_error(const wrapd_handle* h) {
    if (!h) return g_create_error.c_str();
    return h->err.c_str();
}

void wrapd_destroy(wrapd_handle* h) {
    if (!h) return;
    try {
        delete h->s;
    } catch (...) {
    }
    delete h;
}

int wrapd_get_state(wrapd_handle* h, const char* name, double* out, int64_t cap, int64_t* len) {
    if (!name) return WRAPD_E_INPUT;
    return guarded(h, [&](wrapd::SolverGPU& s) {
        std::vector<double> v;
        s.get_state(name, v);
        if (len) *len = static_cast<int64_t>(v.size());
        if (out) std::memcpy(out, v.data(), sizeof(double) * (size_t)std::min<int64_t>(cap, (int64_t)v.size()));
    });
}

int wrapd_set_state(wrapd_handle* h, const char* name, const double* in, int64_t n) {
    if (!name || !in) return WRAPD_E_INPUT;
    return guarded(h, [&](wrapd::SolverGPU& s) { s.set_state(name, in, n); });
}

int wrapd_update_defo_cache(wrapd_handle* h) {
    return guarded(h, [&](wrapd::SolverGPU& s) { s.update_defo_cache(); });
}

int wrapd_polar_update(wrapd_handle* h, int update_candidates, double* delta_al) {
    return guarded(h, [&](wrapd::SolverGPU& s) {
        const double d = s.polar_update(update_candidates != 0);
        if (delta_al) *delta_al = d;
    });
}

int wrapd_global_grad(wrapd_handle* h, const double* x_free, double* grad, double* value) {
    return guarded(h, [&](wrapd::SolverGPU& s) {
        const double v = s.global_grad(x_free, grad);
        if (value) *value = v;
    });
}

int wrapd_potential_energy(wrapd_handle* h, double* pe, int* flips) {
    return guarded(h, [&](wrapd::SolverGPU& s) { s.potential_energy(pe, flips); });
}

int wrapd_solve_A(wrapd_handle* h, const double* b, double* x) {
    if (!b || !x) return WRAPD_E_INPUT;
    return guarded(h, [&](wrapd::SolverGPU& s) { s.solve_A(b, x); });
}

int wrapd_solve_A_holding(wrapd_handle* h, const double* b, double* x, int front) {
    if (!b || !x) return WRAPD_E_INPUT;
    return guarded(h, [&](wrapd::SolverGPU& s) { s.solve_A(b, x, front); });
}

}  // extern "C"
