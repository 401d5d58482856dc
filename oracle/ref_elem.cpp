// Test infrastructure: C entry points over the reference's own per-element
// code, compiled from the reference sources (see oracle/Makefile), used only
// to generate and check golden vectors.  Each function states the reference
// code it calls.  Matrices are 3x3 column-major (Eigen's default storage).
#include <cstring>
#include <memory>
#include <vector>

// Expose TetElements' protected state to this test harness only (same class
// layout; the reference's own translation units are compiled unchanged).
#define protected public
#include "TetElements.hpp"
#undef protected

using wrapd::math::Mat3x3;
using wrapd::math::Vec3;
using wrapd::math::MatX3;

namespace {
wrapd::Lame make_lame(double mu, double lambda) {
    wrapd::Lame l(1.0, 0.25);
    l.mu(mu);
    l.lambda(lambda);
    return l;
}
}  // namespace

extern "C" {

// math::svd with sign fix (src/Math.hpp:140-161).
void ref_svd3(int n, const double* F, double* sigma, double* U, double* V) {
    for (int e = 0; e < n; ++e) {
        Mat3x3 f = Eigen::Map<const Mat3x3>(F + 9 * e);
        Vec3 s; Mat3x3 u, v;
        wrapd::math::svd(f, s, u, v, true);
        std::memcpy(sigma + 3 * e, s.data(), 3 * sizeof(double));
        std::memcpy(U + 9 * e, u.data(), 9 * sizeof(double));
        std::memcpy(V + 9 * e, v.data(), 9 * sizeof(double));
    }
}

// NHProx + LBFGS<double,3,8> with BacktrackingCubic, max 20 iterations, warm
// started at `start` (src/TetElements.cpp:302-319, src/TetElements.hpp:50-162,
// deps/mcloptlib/include/MCL/LBFGS.hpp:52-152).
void ref_prox(int n, const double* sigma0, const double* wsq_over_vol, const double* start,
              double mu, double lambda, double* out, int* iters) {
    mcl::optlib::LBFGS<double, 3> solver;
    solver.m_settings.ls_method = mcl::optlib::LSMethod::BacktrackingCubic;
    solver.m_settings.max_iters = 20;
    wrapd::NHProx problem;
    problem.set_lame(make_lame(mu, lambda));
    for (int e = 0; e < n; ++e) {
        problem.set_x0(Vec3(sigma0[3 * e], sigma0[3 * e + 1], sigma0[3 * e + 2]));
        problem.set_wsq_over_volume(wsq_over_vol[e]);
        Vec3 s(start[3 * e], start[3 * e + 1], start[3 * e + 2]);
        iters[e] = solver.minimize(problem, s);
        out[3 * e] = s[0]; out[3 * e + 1] = s[1]; out[3 * e + 2] = s[2];
    }
}

// NHProx value and gradient (src/TetElements.hpp:87-107).
void ref_prox_value_grad(int n, const double* x, const double* sigma0, const double* wsq_over_vol,
                         double mu, double lambda, double* value, double* grad) {
    wrapd::NHProx problem;
    problem.set_lame(make_lame(mu, lambda));
    for (int e = 0; e < n; ++e) {
        problem.set_x0(Vec3(sigma0[3 * e], sigma0[3 * e + 1], sigma0[3 * e + 2]));
        problem.set_wsq_over_volume(wsq_over_vol[e]);
        Vec3 xx(x[3 * e], x[3 * e + 1], x[3 * e + 2]), g;
        value[e] = problem.gradient(xx, g);
        grad[3 * e] = g[0]; grad[3 * e + 1] = g[1]; grad[3 * e + 2] = g[2];
    }
}

// Candidate stiffness before the volume factor: max real eigenvalue of the
// PSD-projected NH Hessian density (src/TetElements.cpp:413-417).
void ref_hess_lmax(int n, const double* sigma, double mu, double lambda, double* out) {
    wrapd::NHProx problem;
    problem.set_lame(make_lame(mu, lambda));
    for (int e = 0; e < n; ++e) {
        Mat3x3 K;
        problem.hessian_density(Vec3(sigma[3 * e], sigma[3 * e + 1], sigma[3 * e + 2]), K);
        out[e] = K.eigenvalues().real().maxCoeff();
    }
}

// One setup + local step + gradient of the reference TetElements on a mesh:
// update_fix_cache, update_defo_cache, initialize_dual_vars, polar_update(false)
// (src/TetElements.cpp:145-166, 256-356, 547-596), then the cached gradient and
// AL value (src/TetElements.cpp:678-787).  X is n_verts x 3 row-major; pins
// must be sorted.  Outputs: dal = polar_update's delta-AL, grad (n_free x 3
// row-major, free vertices in ascending id order), value, pe = potential
// energy at x, flips = inversion count, grad2 = full gradient at X2.
void ref_local_and_grad(int nv, const double* rest, const double* X, const double* X2,
                        int ntet, const int* tets, int npins, const int* pins,
                        double youngs, double poisson,
                        double* dal, double* grad, double* value, double* pe, int* flips,
                        double* grad2, double* Zout, double* Uout, double* symFout) {
    static wrapd::Settings settings;
    const_cast<wrapd::Lame&>(settings.m_model_settings.elastic_lame()) = wrapd::Lame(youngs, poisson);
    std::vector<int> free_index(nv), fix_index(nv, -1);
    {
        int j = 0, k = 0;
        for (int i = 0; i < nv; ++i) {
            if (j < npins && i == pins[j]) { free_index[i] = -1; fix_index[i] = j++; }
            else { free_index[i] = k++; }
        }
    }
    const int nfree = nv - npins;
    std::shared_ptr<wrapd::TetElements> te;
    wrapd::create_tets_from_mesh<double, wrapd::TetElements>(te, rest, tets, ntet, settings,
                                                             free_index, fix_index, 0);
    MatX3 Xm(nv, 3), X2m(nv, 3);
    for (int i = 0; i < nv; ++i)
        for (int c = 0; c < 3; ++c) { Xm(i, c) = X[3 * i + c]; X2m(i, c) = X2[3 * i + c]; }
    MatX3 xfree(nfree, 3), xfix(npins, 3), x2free(nfree, 3);
    for (int i = 0; i < nv; ++i) {
        if (free_index[i] >= 0) { xfree.row(free_index[i]) = Xm.row(i); x2free.row(free_index[i]) = X2m.row(i); }
        else xfix.row(fix_index[i]) = Xm.row(i);
    }
    te->update_fix_cache(xfix);
    te->update_defo_cache(xfree);
    te->initialize_dual_vars(Xm);
    *dal = te->polar_update(false);
    te->update_defo_cache(xfree);
    for (int e = 0; e < ntet; ++e) {
        if (Zout) std::memcpy(Zout + 9 * e, te->m_Zi[e].data(), 9 * sizeof(double));
        if (Uout) std::memcpy(Uout + 9 * e, te->m_Ui[e].data(), 9 * sizeof(double));
        if (symFout) std::memcpy(symFout + 9 * e, te->m_cached_symF[e].data(), 9 * sizeof(double));
    }
    MatX3 g = te->global_obj_grad();
    for (int i = 0; i < nfree; ++i)
        for (int c = 0; c < 3; ++c) grad[3 * i + c] = g(i, c);
    *value = te->global_obj_value(xfree);
    *pe = te->potential_energy_x();
    *flips = te->inversion_count();
    MatX3 g2;
    te->global_obj_grad(x2free, g2);
    for (int i = 0; i < nfree; ++i)
        for (int c = 0; c < 3; ++c) grad2[3 * i + c] = g2(i, c);
}

}  // extern "C"
