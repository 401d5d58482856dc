/* AlgorithmData.hpp -- wrapd::AlgorithmData (the reference's
 * src/AlgorithmData.hpp:35-146): the per-iteration logs of a solve, entry 0
 * being the initial state, with the reference's accessors and public members.
 * Filled by Solver::solve from the library's logs.  See Math.hpp for this
 * directory. */
#ifndef WRAPD_COMPAT_ALGORITHMDATA_HPP
#define WRAPD_COMPAT_ALGORITHMDATA_HPP

#include <cmath>
#include <vector>

#include "RuntimeData.hpp"

namespace wrapd {

class AlgorithmData {
public:
    const std::vector<double>& per_iter_objectives() const { return m_objectives; }
    const std::vector<int>& per_iter_reweighted() const { return m_reweighted; }
    const std::vector<double>& per_iter_state_x_errors() const { return m_state_x_errors; }
    const std::vector<double>& per_iter_accumulated_time_s() const { return m_accumulated_time_s; }
    const std::vector<int>& per_iter_inner_iters() const { return m_per_iter_inner_iters; }
    double current_normalized_x_error() const { return m_state_x_errors[m_iter]; }
    double current_normalized_objective_residual() const { return m_norm_obj_residuals[m_iter - 1]; }
    bool no_recent_flips() const { return m_flips_count[m_iter] == 0 && m_flips_count[m_iter - 1] == 0; }

    RuntimeData m_runtime;
    int m_iter = 0;
    std::vector<double> m_norm_obj_residuals;
    std::vector<int> m_per_iter_inner_iters;
    std::vector<double> m_per_iter_ls_delta_auglag;
    std::vector<double> m_per_iter_gs_delta_auglag;
    /* extension: mean prox iterations per element of each local step */
    std::vector<double> m_per_iter_prox_iters;

    std::vector<double> m_objectives;
    std::vector<double> m_state_x_errors;
    std::vector<int> m_reweighted;
    std::vector<double> m_accumulated_time_s;
    std::vector<int> m_flips_count;
};

}  // namespace wrapd

#endif  // WRAPD_COMPAT_ALGORITHMDATA_HPP
