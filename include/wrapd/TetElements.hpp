/* TetElements.hpp -- wrapd::TetElements (the reference's
 * src/TetElements.hpp:165-247) and create_tets_from_mesh
 * (src/TetElements.hpp:250-288).  The element set of one mesh: its tets (with
 * the vertex offset applied, as the reference stores them) and, once the
 * owning Solver is initialised, the public element-level steps of the
 * reference on the GPU state through the C ABI: update_defo_cache,
 * polar_update, global_obj_grad, potential_energy_x, inversion_count.
 * Free-vertex blocks (x_free, gradients) are n_free x 3 in ascending vertex id
 * order with the pinned vertices left out, as the reference's x_free.
 * Errors throw std::runtime_error.  See Math.hpp for this directory. */
#ifndef WRAPD_COMPAT_TETELEMENTS_HPP
#define WRAPD_COMPAT_TETELEMENTS_HPP

#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../wrapd_gpu.h"
#include "Math.hpp"
#include "Settings.hpp"

namespace wrapd {

class TetElements {
public:
    TetElements(const std::vector<math::Vec4i>& tet, const std::vector<math::Vec4i>& free_index_tet,
                const std::vector<math::Vec4i>& fix_index_tet, const std::vector<std::vector<math::Vec3>>& verts,
                const Settings& settings)
        : m_tet(tet), m_free_index_tet(free_index_tet), m_fix_index_tet(fix_index_tet) {
        (void)verts;     // the rest geometry comes from System::X() at Solver::initialize
        (void)settings;
    }
    virtual ~TetElements() = default;

    int num_elements() const { return static_cast<int>(m_tet.size()); }
    const std::vector<math::Vec4i>& inds() const { return m_tet; }

    /* TetElements::update_defo_cache (src/TetElements.cpp:564-596): F, its SVD
     * and sym(F) of every element at x_free. */
    void update_defo_cache(const math::MatX3& x_free, bool compute_polar_data = true) {
        (void)compute_polar_data;
        const std::vector<double> x = math::to_rows(x_free);
        check(wrapd_set_state(live(), "xfree", x.data(), static_cast<int64_t>(x_free.rows())));
        check(wrapd_update_defo_cache(m_h));
    }
    /* TetElements::polar_update (src/TetElements.cpp:256-356): the local step
     * on the cache; returns its change of the augmented Lagrangian. */
    double polar_update(bool update_candidate_weights) {
        double dal = 0.0;
        check(wrapd_polar_update(live(), update_candidate_weights ? 1 : 0, &dal));
        return dal;
    }
    /* TetElements::global_obj_grad(x_free, gradient) (src/TetElements.cpp:
     * 691-738): refreshes the cache at x_free; returns the AL value. */
    double global_obj_grad(const math::MatX3& x_free, math::MatX3& gradient) {
        const std::vector<double> x = math::to_rows(x_free);
        std::vector<double> g(x.size());
        double value = 0.0;
        check(wrapd_global_grad(live(), x.data(), g.data(), &value));
        gradient = math::from_rows(g.data(), x_free.rows());
        return value;
    }
    /* TetElements::potential_energy_x and inversion_count on the cache
     * (src/TetElements.cpp:598-635, 444-468). */
    double potential_energy_x() const {
        double pe = 0.0;
        int flips = 0;
        check(wrapd_potential_energy(live(), &pe, &flips));
        return pe;
    }
    int inversion_count() const {
        double pe = 0.0;
        int flips = 0;
        check(wrapd_potential_energy(live(), &pe, &flips));
        return flips;
    }

    /* Set by Solver::initialize: the GPU handle these steps act on. */
    void attach(wrapd_handle* h) { m_h = h; }

protected:
    std::vector<math::Vec4i> m_tet;
    std::vector<math::Vec4i> m_free_index_tet;
    std::vector<math::Vec4i> m_fix_index_tet;

private:
    wrapd_handle* live() const {
        if (!m_h) throw std::runtime_error("TetElements: the Solver is not initialized");
        return m_h;
    }
    void check(int rc) const {
        if (rc != WRAPD_OK) throw std::runtime_error(wrapd_last_error(m_h));
    }
    wrapd_handle* m_h = nullptr;
};

/* create_tets_from_mesh (src/TetElements.hpp:250-288): the element set of a
 * mesh from its flat rest vertices and 0-based tets, with the free and fixed
 * index of every vertex and the offset of the mesh's first vertex. */
template <typename IN_SCALAR, typename TYPE>
inline void create_tets_from_mesh(std::shared_ptr<TetElements>& tet_elements, const IN_SCALAR* verts, const int* inds,
                                  int n_tets, const Settings& settings, const std::vector<int>& free_index_list,
                                  const std::vector<int>& fix_index_list, const int vertex_offset) {
    std::vector<math::Vec4i> tets(n_tets), free_tets(n_tets), fix_tets(n_tets);
    std::vector<std::vector<math::Vec3>> tet_verts(n_tets);
    for (int e = 0; e < n_tets; ++e) {
        const int* t = inds + 4 * e;
        for (int a = 0; a < 4; ++a) {
            free_tets[e][a] = free_index_list[t[a]];
            fix_tets[e][a] = fix_index_list[t[a]];
            tet_verts[e].push_back(math::Vec3(verts[3 * t[a]], verts[3 * t[a] + 1], verts[3 * t[a] + 2]));
            tets[e][a] = t[a] + vertex_offset;
        }
    }
    tet_elements = std::make_shared<TYPE>(tets, free_tets, fix_tets, tet_verts, settings);
}

}  // namespace wrapd

#endif  // WRAPD_COMPAT_TETELEMENTS_HPP
