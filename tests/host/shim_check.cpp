// CPU check of include/wrapd_gpu.hpp, the C++ classes over the C ABI in the
// shape of the reference's wrapd::Solver: settings defaults, the reference's
// error messages and call-order errors as std::runtime_error, and (with the
// argument "nogpu", on a machine without a usable GPU) initialize() failing
// loudly with the library's message instead of running anywhere else.
#include <cstdio>
#include <stdexcept>
#include <string>

#include "wrapd_gpu.hpp"

namespace {

int failures = 0;

void expect(bool ok, const char* what) {
    if (!ok) { std::printf("FAILED: %s\n", what); ++failures; }
}

template <typename F>
std::string thrown(F&& f) {
    try {
        f();
    } catch (const std::runtime_error& e) {
        return e.what()[0] ? e.what() : "(empty message)";
    }
    return "";
}

}  // namespace

int main(int argc, char** argv) {
    const bool no_gpu = argc > 1 && std::string(argv[1]) == "nogpu";
    wrapd::gpu::Settings s;
    expect(s.max_iters == 5000 && s.tol == 1e-11 && s.rot_aware == 1 && s.reweighting == 1, "settings defaults");
    expect(s.lbfgs_m == 6 && s.youngs == 1e7 && s.gamma == 1.5 && s.leaf_size == 64, "settings defaults (extensions)");

    wrapd::gpu::Solver solver(s);
    expect(thrown([&] { solver.set_pins({0}); }) == "set_pins before add_tetmesh", "set_pins before a mesh");
    expect(thrown([&] { solver.add_tetmesh({0, 0, 0}, {0, 0, 0, 1, 1, 1}, {0, 0, 0, 0}); }) ==
               "Error: Rest mesh and init mesh do not have the same number of vertices.",
           "the reference's message for mismatched meshes");
    expect(thrown([&] { solver.solve(); }) == "solve before initialize", "solve before initialize");
    const std::vector<double> rest = {0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0, 1};
    expect(solver.add_tetmesh(rest, rest, {0, 1, 2, 3}) == 4, "vertex count after one tet");
    solver.set_pins({0, 1, 2});
    expect(solver.handle() == nullptr, "no handle before initialize");
    if (no_gpu) {
        const std::string msg = thrown([&] { solver.initialize(s); });
        expect(!msg.empty(), "initialize without a GPU throws");
        expect(solver.handle() == nullptr, "no handle after a failed create");
        std::printf("initialize without a GPU: %s\n", msg.c_str());
    }
    if (failures) return 1;
    std::printf("ok\n");
    return 0;
}
