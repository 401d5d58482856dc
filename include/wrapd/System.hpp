/* System.hpp -- wrapd::System (the reference's src/System.hpp:41-174): the
 * positions (rest, init, solution), the pins and the element set, reached as
 * Solver::m_system.  Before Solver::initialize it collects the mesh
 * (add_nodes, tet_elements(), set_pins); after it, the element-level steps
 * forward to the GPU state like the reference's delegation to TetElements
 * (src/System.cpp), and X() holds the positions of the last solve.  See
 * Math.hpp for this directory. */
#ifndef WRAPD_COMPAT_SYSTEM_HPP
#define WRAPD_COMPAT_SYSTEM_HPP

#include <algorithm>
#include <memory>
#include <stdexcept>
#include <vector>

#include "Math.hpp"
#include "Settings.hpp"
#include "TetElements.hpp"

namespace wrapd {

class System {
public:
    explicit System(const Settings& settings) : m_settings(settings) {}

    int num_all_verts() const { return static_cast<int>(m_X.rows()); }
    const math::MatX3 X() const { return m_X; }
    const math::MatX3& X_soln() const { return m_X_soln; }
    const math::MatX3& X_init() const { return m_X_init; }
    void X(const math::MatX3& val) { m_X = val; }

    /* System::add_nodes (src/System.hpp:75-92): appends vertices; returns the
     * vertex count after the insert. */
    int add_nodes(const math::MatX3& X, const math::MatX3& X_init, const math::MatX3& X_soln) {
        const Eigen::Index prev = m_X.rows(), n = X.rows();
        m_X.conservativeResize(prev + n, 3);
        m_X_init.conservativeResize(prev + n, 3);
        m_X_soln.conservativeResize(prev + n, 3);
        m_X.bottomRows(n) = X;
        m_X_init.bottomRows(n) = X_init;
        m_X_soln.bottomRows(n) = X_soln;
        return static_cast<int>(prev + n);
    }

    /* System::set_pins (src/System.cpp:33-44): the vertices are held where they
     * are; the points are not used (as in the reference). */
    void set_pins(const std::vector<int>& inds, const std::vector<math::Vec3>& points) {
        (void)points;
        m_pin_inds = inds;
        std::sort(m_pin_inds.begin(), m_pin_inds.end());
    }
    const std::vector<int>& pin_inds() const { return m_pin_inds; }

    int num_tet_elements() const { return m_tet_elements ? m_tet_elements->num_elements() : 0; }
    std::shared_ptr<TetElements>& tet_elements() { return m_tet_elements; }

    void set_initial_pose() { m_X = m_X_init; }

    /* Element-level steps (src/System.cpp forwards each to TetElements). */
    double polar_local_update(bool update_candidate_weights) {
        return elements().polar_update(update_candidate_weights);
    }
    void update_defo_cache(const math::MatX3& x_free, bool update_polar_data = true) {
        elements().update_defo_cache(x_free, update_polar_data);
    }
    double global_obj_grad(const math::MatX3& x_free, math::MatX3& grad, bool positions_have_changed) {
        (void)positions_have_changed;
        return elements().global_obj_grad(x_free, grad);
    }
    double potential_energy() const { return elements().potential_energy_x(); }
    double problem_objective() const { return potential_energy(); }
    int inversion_count() const { return elements().inversion_count(); }

protected:
    const Settings m_settings;
    std::shared_ptr<TetElements> m_tet_elements;

private:
    TetElements& elements() const {
        if (!m_tet_elements) throw std::runtime_error("System: no tet elements");
        return *m_tet_elements;
    }
    math::MatX3 m_X, m_X_init, m_X_soln;
    std::vector<int> m_pin_inds;
};

}  // namespace wrapd

#endif  // WRAPD_COMPAT_SYSTEM_HPP
