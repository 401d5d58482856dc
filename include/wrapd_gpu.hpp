/* wrapd_gpu.hpp -- C++ classes over the C ABI of wrapd_gpu.h, in the shape of
 * the reference's wrapd::Solver / Settings / AlgorithmData
 * (src/Solver.hpp:37-72, src/Settings.hpp, src/AlgorithmData.hpp:37-146), so
 * that a C++ caller of the reference switches by changing its includes and
 * one namespace.  Header only; link libwrapd_gpu.so.
 *
 * Differences from the reference's classes, all in how meshes come in:
 *   - add_tetmesh takes flat arrays (rest and init positions n x 3
 *     row-major, tets m x 4 0-based) where binding::add_tetmesh
 *     (samples/utils/AddMeshes.hpp:61-132) takes mcl::TetMesh objects;
 *   - meshes and pins are held on the host until initialize(), which
 *     creates the GPU handle with the settings it is given (the reference's
 *     initialize(settings) also takes its settings there, src/Solver.cpp:48-60);
 *   - solve() runs the whole ADMM loop on the GPU and X() returns the
 *     positions of every added mesh in the order added.
 * Errors throw std::runtime_error with the library's message, as the
 * reference throws std::runtime_error; no error code crosses this layer.
 * Callers written against the reference's own headers use include/wrapd/
 * instead: the reference's file and class names (Solver with m_system,
 * System, TetElements, Settings with parse_args, AlgorithmData) with Eigen
 * types, over the same C ABI, so that such a caller builds unchanged. */
#ifndef WRAPD_GPU_HPP
#define WRAPD_GPU_HPP

#include <array>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "wrapd_gpu.h"

namespace wrapd {
namespace gpu {

/* wrapd::Settings + ModelSettings as the flat wrapd_settings struct, starting
 * from the reference's defaults (src/Settings.hpp:154-162,
 * src/ModelSettings.hpp:33-41). */
struct Settings : wrapd_settings {
    Settings() : wrapd_settings() { wrapd_settings_default(this); }
};

/* The per-iteration logs of wrapd::AlgorithmData (src/AlgorithmData.hpp:
 * 43-73), entry 0 being the initial state, with the reference's accessors. */
struct AlgorithmData {
    std::vector<double> objectives, x_errors, accumulated_time_s, ls_delta_al, gs_delta_al, prox_iters;
    std::vector<int> reweighted, flips, inner_iters;

    const std::vector<double>& per_iter_objectives() const { return objectives; }
    const std::vector<int>& per_iter_reweighted() const { return reweighted; }
    const std::vector<double>& per_iter_state_x_errors() const { return x_errors; }
    const std::vector<double>& per_iter_accumulated_time_s() const { return accumulated_time_s; }
    const std::vector<int>& per_iter_inner_iters() const { return inner_iters; }
};

/* wrapd::RuntimeData (src/RuntimeData.hpp:30-44) in milliseconds. */
struct RuntimeData {
    double setup_ms = 0, local_ms = 0, global_ms = 0, refactor_ms = 0, finish_ms = 0, inner_iters = 0;
};

class Solver {
public:
    /* wrapd::Solver::Solver(const Settings&) (src/Solver.cpp:32-35). */
    explicit Solver(const Settings& settings) : m_settings(settings) {}
    ~Solver() { wrapd_destroy(m_h); }
    Solver(const Solver&) = delete;
    Solver& operator=(const Solver&) = delete;

    /* binding::add_tetmesh without set_pins: rest/init are n x 3 row-major,
     * tets m x 4 with 0-based vertex ids, soln (optional) the exact solution
     * for the x-error log.  A second call before initialize() adds another
     * mesh to a batch solved as one block-diagonal system.  Returns the total
     * vertex count so far (as Solver::add_nodes does). */
    int add_tetmesh(std::vector<double> rest, std::vector<double> init, std::vector<int32_t> tets,
                    std::vector<double> soln = {}) {
        if (m_h) throw std::runtime_error("add_tetmesh after initialize");
        if (rest.size() != init.size())
            throw std::runtime_error("Error: Rest mesh and init mesh do not have the same number of vertices.");
        if (rest.size() % 3 || tets.size() % 4 || (!soln.empty() && soln.size() != rest.size()))
            throw std::runtime_error("add_tetmesh: positions must be n x 3 and tets m x 4");
        Mesh m{std::move(rest), std::move(init), std::move(soln), std::move(tets), {}};
        m_verts += static_cast<int>(m.rest.size() / 3);
        m_meshes.push_back(std::move(m));
        return m_verts;
    }

    /* wrapd::Solver::set_pins (src/System.cpp:33-44): pins the listed vertices
     * of the last added mesh where they are; the points, as in the
     * reference's use, are not used. */
    void set_pins(const std::vector<int>& inds, const std::vector<std::array<double, 3>>& points = {}) {
        (void)points;
        if (m_meshes.empty()) throw std::runtime_error("set_pins before add_tetmesh");
        if (m_h) throw std::runtime_error("set_pins after initialize");
        m_meshes.back().pins.assign(inds.begin(), inds.end());
    }

    /* wrapd::Solver::initialize(const Settings&) (src/Solver.cpp:48-60):
     * creates the GPU handle with these settings, hands it the meshes, and
     * runs the symbolic analysis and first factorization. */
    bool initialize(const Settings& settings) {
        m_settings = settings;
        return initialize();
    }
    bool initialize() {
        if (m_h) throw std::runtime_error("already initialized");
        if (m_meshes.empty()) throw std::runtime_error("initialize before add_tetmesh");
        wrapd_handle* h = nullptr;
        if (wrapd_create(&m_settings, &h) != WRAPD_OK) throw std::runtime_error(wrapd_last_error(nullptr));
        // the handle is kept only once it is initialized: a failed call (bad
        // mesh, inverted rest tet, out of memory) leaves none behind, so
        // initialize() can be called again after the input is fixed
        auto fail = [&](int rc) {
            if (rc == WRAPD_OK) return;
            const std::string msg = wrapd_last_error(h);
            wrapd_destroy(h);
            throw std::runtime_error(msg);
        };
        for (const Mesh& m : m_meshes)
            fail(wrapd_add_tetmesh(h, m.rest.data(), m.init.data(), m.soln.empty() ? nullptr : m.soln.data(),
                                   static_cast<int>(m.rest.size() / 3), m.tets.data(),
                                   static_cast<int>(m.tets.size() / 4), m.pins.data(),
                                   static_cast<int>(m.pins.size())));
        fail(wrapd_initialize(h));
        m_h = h;
        return true;
    }

    /* wrapd::Solver::solve (src/Solver.cpp:38-46): the ADMM loop to
     * convergence; then X() and algorithm_data() hold the result. */
    void solve() {
        if (!m_h) throw std::runtime_error("solve before initialize");
        m_x.assign(3 * static_cast<size_t>(m_verts), 0.0);
        check(wrapd_solve(m_h, m_x.data()));
        read_logs();
    }

    /* System::X() after the solve: n x 3 row-major, meshes in the order added. */
    const std::vector<double>& X() const { return m_x; }

    /* wrapd::Solver::algorithm_data(). */
    AlgorithmData* algorithm_data() { return &m_data; }

    RuntimeData runtime() const {
        double ms[6] = {0, 0, 0, 0, 0, 0};
        if (m_h) check(wrapd_get_runtime(m_h, ms));
        return RuntimeData{ms[0], ms[1], ms[2], ms[3], ms[4], ms[5]};
    }

    const Settings& settings() const { return m_settings; }

    /* The underlying C handle (null before initialize()), for the entry
     * points this class does not wrap. */
    wrapd_handle* handle() const { return m_h; }

private:
    struct Mesh {
        std::vector<double> rest, init, soln;
        std::vector<int32_t> tets, pins;
    };

    void check(int rc) const {
        if (rc != WRAPD_OK) throw std::runtime_error(wrapd_last_error(m_h));
    }

    template <typename T>
    std::vector<T> log(int which) const {
        int len = 0;
        check(wrapd_get_log(m_h, which, nullptr, 0, &len));
        std::vector<double> v(static_cast<size_t>(len));
        if (len > 0) check(wrapd_get_log(m_h, which, v.data(), len, &len));
        return std::vector<T>(v.begin(), v.end());
    }

    void read_logs() {
        m_data.objectives = log<double>(WRAPD_LOG_OBJECTIVES);
        m_data.reweighted = log<int>(WRAPD_LOG_REWEIGHTED);
        m_data.flips = log<int>(WRAPD_LOG_FLIPS);
        m_data.inner_iters = log<int>(WRAPD_LOG_INNER_ITERS);
        m_data.ls_delta_al = log<double>(WRAPD_LOG_LS_DELTA_AL);
        m_data.gs_delta_al = log<double>(WRAPD_LOG_GS_DELTA_AL);
        m_data.accumulated_time_s = log<double>(WRAPD_LOG_ACCUMULATED_TIME_S);
        m_data.x_errors = log<double>(WRAPD_LOG_X_ERRORS);
        m_data.prox_iters = log<double>(WRAPD_LOG_PROX_ITERS);
    }

    Settings m_settings;
    std::vector<Mesh> m_meshes;
    int m_verts = 0;
    wrapd_handle* m_h = nullptr;
    std::vector<double> m_x;
    AlgorithmData m_data;
};

}  // namespace gpu
}  // namespace wrapd

#endif /* WRAPD_GPU_HPP */
