/* Solver.hpp -- wrapd::Solver (the reference's src/Solver.hpp:37-72,
 * src/Solver.cpp:32-65) on the GPU: the reference's constructor, set_pins,
 * initialize(settings), solve(), algorithm_data(), settings(), and the public
 * m_system and m_settings.  initialize() creates the library handle with the
 * settings it is given, hands it the mesh the System collected (rest = X(),
 * init = X_init(), solution = X_soln(), the element set's tets, the pins) and
 * runs the symbolic analysis and first factorization; solve() runs the ADMM
 * loop on the GPU, then m_system->X() holds the final positions and
 * algorithm_data() the logs.  The reference replaces the element set when a
 * mesh is added twice; so does this class (the C ABI's batches of meshes are
 * reached through ../wrapd_gpu.h).  Errors throw std::runtime_error with the
 * library's message; a failed initialize() leaves no handle behind, so it can
 * be called again.  See Math.hpp for this directory. */
#ifndef WRAPD_COMPAT_SOLVER_HPP
#define WRAPD_COMPAT_SOLVER_HPP

#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../wrapd_gpu.h"
#include "AlgorithmData.hpp"
#include "Math.hpp"
#include "Settings.hpp"
#include "System.hpp"
#include "TetElements.hpp"

namespace wrapd {

class Solver {
public:
    explicit Solver(const Settings& settings) : m_system(std::make_shared<System>(settings)), m_settings(settings) {}
    virtual ~Solver() {
        if (m_system && m_system->tet_elements()) m_system->tet_elements()->attach(nullptr);
        wrapd_destroy(m_h);
    }
    Solver(const Solver&) = delete;
    Solver& operator=(const Solver&) = delete;

    virtual void set_pins(const std::vector<int>& inds, const std::vector<math::Vec3>& points = std::vector<math::Vec3>()) {
        m_system->set_pins(inds, points);
    }

    virtual bool initialize(const Settings& settings_ = Settings()) {
        if (m_h) throw std::runtime_error("Solver: already initialized");
        m_settings = settings_;
        std::shared_ptr<TetElements>& te = m_system->tet_elements();
        if (!te || m_system->num_all_verts() == 0) throw std::runtime_error("Solver: no mesh added");
        const wrapd_settings cs = m_settings.to_c();
        wrapd_handle* h = nullptr;
        if (wrapd_create(&cs, &h) != WRAPD_OK) throw std::runtime_error(wrapd_last_error(nullptr));
        try {
            const int nv = m_system->num_all_verts();
            const std::vector<double> rest = math::to_rows(m_system->X()), init = math::to_rows(m_system->X_init()),
                                      soln = math::to_rows(m_system->X_soln());
            std::vector<int32_t> tets(4 * static_cast<size_t>(te->num_elements()));
            for (int e = 0; e < te->num_elements(); ++e)
                for (int a = 0; a < 4; ++a) tets[4 * static_cast<size_t>(e) + a] = te->inds()[e][a];
            const std::vector<int32_t> pins(m_system->pin_inds().begin(), m_system->pin_inds().end());
            check(h, wrapd_add_tetmesh(h, rest.data(), init.data(), soln.data(), nv, tets.data(), te->num_elements(),
                                       pins.data(), static_cast<int>(pins.size())));
            check(h, wrapd_initialize(h));
        } catch (...) {
            wrapd_destroy(h);
            throw;
        }
        m_h = h;
        te->attach(m_h);
        m_system->set_initial_pose();
        return true;
    }

    virtual void solve() {
        if (!m_h) throw std::runtime_error("Solver: solve before initialize");
        std::vector<double> x(3 * static_cast<size_t>(m_system->num_all_verts()));
        check(m_h, wrapd_solve(m_h, x.data()));
        m_system->X(math::from_rows(x.data(), m_system->num_all_verts()));
        read_logs();
    }

    const Settings& settings() { return m_settings; }
    AlgorithmData* algorithm_data() { return &m_data; }
    /* The library handle (null before initialize), for the C ABI's other entry points. */
    wrapd_handle* handle() const { return m_h; }

    std::shared_ptr<System> m_system;
    Settings m_settings;

private:
    static void check(wrapd_handle* h, int rc) {
        if (rc != WRAPD_OK) throw std::runtime_error(wrapd_last_error(h));
    }
    std::vector<double> log(int which) const {
        int len = 0;
        check(m_h, wrapd_get_log(m_h, which, nullptr, 0, &len));
        std::vector<double> v(static_cast<size_t>(len));
        if (len > 0) check(m_h, wrapd_get_log(m_h, which, v.data(), len, &len));
        return v;
    }
    static std::vector<int> ints(const std::vector<double>& v) { return std::vector<int>(v.begin(), v.end()); }
    void read_logs() {
        m_data.m_objectives = log(WRAPD_LOG_OBJECTIVES);
        m_data.m_reweighted = ints(log(WRAPD_LOG_REWEIGHTED));
        m_data.m_flips_count = ints(log(WRAPD_LOG_FLIPS));
        m_data.m_per_iter_inner_iters = ints(log(WRAPD_LOG_INNER_ITERS));
        m_data.m_per_iter_ls_delta_auglag = log(WRAPD_LOG_LS_DELTA_AL);
        m_data.m_per_iter_gs_delta_auglag = log(WRAPD_LOG_GS_DELTA_AL);
        m_data.m_accumulated_time_s = log(WRAPD_LOG_ACCUMULATED_TIME_S);
        m_data.m_state_x_errors = log(WRAPD_LOG_X_ERRORS);
        m_data.m_per_iter_prox_iters = log(WRAPD_LOG_PROX_ITERS);
        m_data.m_iter = static_cast<int>(m_data.m_per_iter_inner_iters.size());
        m_data.m_norm_obj_residuals.clear();
        const std::vector<double>& o = m_data.m_objectives;
        for (size_t k = 1; k < o.size(); ++k)   // src/AlgorithmData.cpp:75
            m_data.m_norm_obj_residuals.push_back(std::fabs(o[k] - o[k - 1]) / (std::fabs(o[k]) + 1.0));
        double ms[6] = {0, 0, 0, 0, 0, 0};
        check(m_h, wrapd_get_runtime(m_h, ms));
        m_data.m_runtime.setup_solve_ms = ms[0];
        m_data.m_runtime.local_ms = ms[1];
        m_data.m_runtime.global_ms = ms[2];
        m_data.m_runtime.refactor_ms = ms[3];
        m_data.m_runtime.finish_solve_ms = ms[4];
        m_data.m_runtime.inner_iters = static_cast<int>(ms[5]);
    }

    wrapd_handle* m_h = nullptr;
    AlgorithmData m_data;
};

}  // namespace wrapd

#endif  // WRAPD_COMPAT_SOLVER_HPP
