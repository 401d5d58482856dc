// CPU check of the drop-in headers (include/wrapd): wrapd::Settings parses the
// reference's flags with the reference's defaults and errors
// (src/Settings.cpp:31-176) and hands them to the C ABI unchanged; the
// System/TetElements/Solver classes collect a mesh like the reference's
// binding::add_tetmesh does; and with the argument "nogpu" (a machine without
// a usable GPU) Solver::initialize fails loudly with the library's message and
// leaves no handle behind.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "Solver.hpp"

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

bool parse(wrapd::Settings& s, std::vector<std::string> args) {
    args.insert(args.begin(), "prog");
    std::vector<char*> argv;
    for (auto& a : args) argv.push_back(&a[0]);
    return s.parse_args(static_cast<int>(argv.size()), argv.data());
}

}  // namespace

int main(int argc, char** argv) {
    {   // defaults: src/Settings.hpp:154-162, src/ModelSettings.hpp:33-41, GStep
        wrapd::Settings s;
        const wrapd_settings c = s.to_c();
        expect(c.max_iters == 5000 && c.tol == 1e-11 && c.rot_aware == 1 && c.reweighting == 1, "defaults 1");
        expect(c.rw_delay == 50 && c.gamma == 1.5 && c.global_iters == 100 && c.global_ls == 0, "defaults 2");
        expect(c.kappa == 1.0 && c.model == 0 && c.beta_static == 1.0 && c.beta_min == 0.1 && c.beta_max == 10.0,
               "defaults 3");
        expect(std::fabs(c.youngs - 1e7) < 1e-6 && std::fabs(c.poisson - 0.45) < 1e-15, "1e7 Pa preset");
        expect(s.m_io.verbose() == 1 && !s.m_io.soln_provided(), "io defaults");
    }
    {   // the reference's flags
        wrapd::Settings s;
        const bool help = parse(s, {"-rest", "dir/bar.node", "-init", "bar_init", "-handles", "h.txt", "-it", "20",
                                    "-tol", "1e-9", "-ra", "0", "-rw", "0", "-rw_delay", "5", "-gamma", "2",
                                    "-global_it", "7", "-global_ls", "1", "-kappa", "0.5", "-model", "arap",
                                    "-poisson", "0.3", "-beta_min", "0.2", "-p", "0", "-s", "1", "-youngs", "1e5",
                                    "-lbfgs_m", "5", "-rw_every", "10", "-precision", "mixed"});
        const wrapd_settings c = s.to_c();
        expect(!help, "no help");
        expect(s.m_io.rest_mesh() == "dir/bar" && s.m_io.init_mesh() == "bar_init", "extension stripped");
        expect(c.max_iters == 20 && c.tol == 1e-9 && c.rot_aware == 0 && c.reweighting == 0, "flags 1");
        expect(c.rw_delay == 5 && c.gamma == 2.0 && c.global_iters == 7 && c.global_ls == 1 && c.kappa == 0.5,
               "flags 2");
        expect(c.model == 1 && c.beta_min == 0.2 && c.verbose == 0, "flags 3");
        expect(std::fabs(c.youngs - 1e5) < 1e-9 && std::fabs(c.poisson - 0.3) < 1e-14, "material (any order)");
        expect(c.lbfgs_m == 5 && c.rw_every == 10 && c.precision == 1, "extensions");
        wrapd::Settings t;
        parse(t, {"-poisson", "0.3", "-youngs", "1e5"});
        expect(std::fabs(t.to_c().youngs - 1e5) < 1e-9 && std::fabs(t.to_c().poisson - 0.3) < 1e-14, "order");
    }
    {   // the reference's errors
        wrapd::Settings s;
        expect(thrown([&] { parse(s, {"-ra", "2"}); }) == "Error: Invalid value provided for argument -rotaware (or -ra)",
               "-ra message");
        expect(thrown([&] { parse(s, {"-rw", "3"}); }) ==
                   "Error: Invalid value provided for argument -reweighting (or -rw)", "-rw message");
        expect(thrown([&] { parse(s, {"-model", "stvk"}); }) == "Error: Invalid input for -elastic_model",
               "-model message");
        expect(thrown([&] { parse(s, {"-bogus", "1"}); }) == "Error: Unrecognized command-line argument: -bogus",
               "unknown flag");
        expect(parse(s, {"-help"}), "help returns true");
    }
    {   // collecting a mesh as binding::add_tetmesh does, then initialize
        wrapd::Settings s;
        auto solver = std::make_shared<wrapd::Solver>(s);
        const int n = 5;
        wrapd::math::MatX3 X(n, 3);
        X << 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0, 1, 1, 1, 1;
        expect(solver->m_system->add_nodes(X, X, X) == n, "add_nodes count");
        const int tets[8] = {0, 1, 2, 3, 1, 2, 3, 4};
        const std::vector<int> free_idx = {-1, 0, 1, 2, 3}, fix_idx = {0, -1, -1, -1, -1};
        wrapd::create_tets_from_mesh<double, wrapd::TetElements>(solver->m_system->tet_elements(), X.data(), tets, 2,
                                                                 s, free_idx, fix_idx, 0);
        expect(solver->m_system->num_tet_elements() == 2, "element count");
        expect(solver->m_system->tet_elements()->inds()[1][3] == 4, "tets kept");
        solver->set_pins({0});
        expect(!thrown([&] { solver->m_system->potential_energy(); }).empty(), "energy needs an initialized solver");
        expect(thrown([&] { solver->solve(); }) == "Solver: solve before initialize", "solve before initialize");
        if (argc > 1 && std::strcmp(argv[1], "nogpu") == 0) {
            const std::string m = thrown([&] { solver->initialize(s); });
            expect(!m.empty(), "initialize without a GPU throws");
            expect(solver->handle() == nullptr, "no handle left after a failed initialize");
            expect(!thrown([&] { solver->initialize(s); }).empty() &&
                       thrown([&] { solver->initialize(s); }) != "Solver: already initialized",
                   "initialize can be called again");
        }
    }
    if (failures == 0) std::printf("ok\n");
    return failures == 0 ? 0 : 1;
}
