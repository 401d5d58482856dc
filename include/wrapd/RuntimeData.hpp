/* RuntimeData.hpp -- wrapd::RuntimeData (the reference's
 * src/RuntimeData.hpp:28-44): accumulated phase times in milliseconds, here
 * from CUDA events on the solver's stream.  See Math.hpp for this directory. */
#ifndef WRAPD_COMPAT_RUNTIMEDATA_HPP
#define WRAPD_COMPAT_RUNTIMEDATA_HPP

namespace wrapd {

struct RuntimeData {
    double setup_solve_ms = 0;
    double local_ms = 0;
    double global_ms = 0;
    double refactor_ms = 0;
    int inner_iters = 0;
    double finish_solve_ms = 0;
};

}  // namespace wrapd

#endif  // WRAPD_COMPAT_RUNTIMEDATA_HPP
